"""ctypes binding of ``libwcb200.so`` (the C ABI in ``include/witwin_channel_b200.h``).

The library is built in-tree (``witwin_channel_b200/csrc/libwcb200.so``).  There
is no fallback: if it is missing or fails to load, every solve raises.
"""

from __future__ import annotations

import ctypes
import os
from pathlib import Path

import torch

_LIB_PATH = Path(__file__).resolve().parent / "csrc" / "libwcb200.so"

WCB_OK = 0
WCB_ERR_INVALID_ARGUMENT = 1
WCB_ERR_CUDA = 2
WCB_ERR_CAPACITY = 3
WCB_ERR_BVH_DEPTH = 4
WCB_ERR_NOT_SUPPORTED = 5
WCB_ERR_DEVICE_STATUS = 6

COMPONENT_LOS = 1
COMPONENT_REFLECTION = 2
COMPONENT_DIFFRACTION = 4
COMPONENT_TRANSMISSION = 8

PRECISION_MIXED = 0
PRECISION_FP64 = 1

DTYPE_F32 = 0
DTYPE_F64 = 1

_f32p = ctypes.POINTER(ctypes.c_float)
_i32p = ctypes.POINTER(ctypes.c_int32)
_i64p = ctypes.POINTER(ctypes.c_int64)
_vp = ctypes.c_void_p


class Materials(ctypes.Structure):
    _fields_ = [
        ("num_materials", ctypes.c_int32),
        ("eps_r", _vp),
        ("sigma_e", _vp),
        ("mu_r", _vp),
        ("gain", _vp),
        ("thickness", _vp),
        ("volumetric", _vp),
        ("num_layers", ctypes.c_int32),
        ("layer_offset", _vp),
        ("layer_count", _vp),
        ("layer_thickness", _vp),
        ("layer_eps_r", _vp),
        ("layer_sigma_e", _vp),
        ("layer_mu_r", _vp),
    ]


class SolveDesc(ctypes.Structure):
    _fields_ = [
        ("num_tx", ctypes.c_int32),
        ("tx_pos", _vp),
        ("tx_power", _vp),
        ("tx_pol", _vp),
        ("rx_kind", ctypes.c_int32),
        ("num_rx", ctypes.c_int32),
        ("rx_pos", _vp),
        ("grid_origin", ctypes.c_float * 3),
        ("grid_x_axis", ctypes.c_float * 3),
        ("grid_y_axis", ctypes.c_float * 3),
        ("grid_rows", ctypes.c_int32),
        ("grid_cols", ctypes.c_int32),
        ("grid_spacing", ctypes.c_float * 2),
        ("rx_pol", _vp),
        ("rx_pol_stride", ctypes.c_int32),
        ("num_freq", ctypes.c_int32),
        ("frequency_hz", ctypes.POINTER(ctypes.c_double)),
        ("components", ctypes.c_int32),
        ("max_depth", ctypes.c_int32),
        ("coherent", ctypes.c_int32),
        ("precision", ctypes.c_int32),
        ("discovery_rays", ctypes.c_int32),
        ("stack_entries", ctypes.c_int32),
    ]


class Outputs(ctypes.Structure):
    _fields_ = [
        ("path_gain", _vp),
        ("field", _vp),
        ("comp_power", _vp),
        ("comp_field", _vp),
        ("diff_vec_power", _vp),
        ("rows", _vp),
        ("row_capacity", ctypes.c_int64),
        ("row_count", _vp),
        ("status", _vp),
        ("transmission_overflow", _vp),
    ]


class RowFields(ctypes.Structure):
    _fields_ = [
        ("path_length_m", _vp),
        ("delay_s", _vp),
        ("path_gain", _vp),
        ("path_field", _vp),
        ("coefficient", _vp),
        ("field_xyz", _vp),
        ("field_direction", _vp),
        ("interaction_positions", _vp),
        ("interaction_normals", _vp),
        ("phase_rad", _vp),
    ]


class AccumulateOutputs(ctypes.Structure):
    _fields_ = [
        ("power_total", _vp),
        ("field_total_real", _vp),
        ("field_total_imag", _vp),
        ("component_power", _vp),
        ("component_field_real", _vp),
        ("component_field_imag", _vp),
    ]


class FrozenRows(ctypes.Structure):
    _fields_ = [
        ("num_rows", ctypes.c_int64),
        ("width", ctypes.c_int32),
        ("component_id", _vp),
        ("depth", _vp),
        ("primitive_sequence", _vp),
        ("source_index", _vp),
        ("sink_index", _vp),
        ("source_id", _vp),
        ("sink_id", _vp),
        ("order", _vp),
    ]


class EndpointBatch(ctypes.Structure):
    _fields_ = [
        ("count", ctypes.c_int64),
        ("positions", _vp),
        ("polarizations", _vp),
        ("stable_ids", _vp),
        ("powers", _vp),
        ("polarization_basis", _vp),
    ]


class ReplayOutputs(ctypes.Structure):
    _fields_ = [
        ("coefficient", _vp),
        ("coefficient_offsets", _vp),
        ("field", _vp),
        ("field_offsets", _vp),
        ("path_length_m", _vp),
        ("delay_s", _vp),
        ("direction", _vp),
        ("interaction_positions", _vp),
        ("interaction_normals", _vp),
        ("row_valid", _vp),
        ("jones", _vp),
        ("source_basis", _vp),
        ("sink_basis", _vp),
        ("pair_index", _vp),
        ("pair_offsets", _vp),
    ]


ROW_BYTES = 48
# wcb_row as int32 words: tx, rx, (component | depth << 16), seq[5], edge, length(f32 bits), reserved[2]
ROW_WORDS = 12

EXPORTED_SYMBOLS = (
    "wcb_scene_create",
    "wcb_scene_destroy",
    "wcb_scene_refit",
    "wcb_scene_rebuild_bvh",
    "wcb_scene_info",
    "wcb_scene_groups",
    "wcb_scene_edges",
    "wcb_solve_workspace_size",
    "wcb_solve",
    "wcb_rows_select_workspace_size",
    "wcb_rows_select",
    "wcb_rows_select_noalloc",
    "wcb_rows_evaluate",
    "wcb_rows_accumulate",
    "wcb_accumulate_flat_workspace_size",
    "wcb_accumulate_flat",
    "wcb_accumulate_flat_backward",
    "wcb_accumulate_flat_jvp_workspace_size",
    "wcb_accumulate_flat_jvp",
    "wcb_rows_vjp_layout",
    "wcb_rows_vjp_workspace_size",
    "wcb_rows_vjp",
    "wcb_rows_jvp",
    "wcb_rows_order_workspace_size",
    "wcb_rows_order",
    "wcb_rows_decode",
    "wcb_cfr_workspace_size",
    "wcb_cfr",
    "wcb_field_free_space",
    "wcb_field_reflection_sequence",
    "wcb_field_transmission_sequence",
    "wcb_field_project_complex3",
    "wcb_los_jones",
    "wcb_rows_replay",
    "wcb_profile_enable",
    "wcb_profile_read",
    "wcb_build_info",
    "wcb_launch_count",
)

_lib: ctypes.CDLL | None = None


def library_path() -> Path:
    return Path(os.environ.get("WITWIN_CHANNEL_B200_LIB", str(_LIB_PATH)))


def load() -> ctypes.CDLL:
    """Load the native library (once).  Raises if it is missing."""

    global _lib
    if _lib is not None:
        return _lib
    path = library_path()
    if not path.exists():
        raise RuntimeError(
            f"witwin_channel_b200 native library not found at {path}; "
            "build it with `python -c 'import __graft_entry__ as g; g.build()'` or `make -C witwin_channel_b200/csrc`"
        )
    lib = ctypes.CDLL(str(path))
    lib.wcb_scene_create.argtypes = [_vp, ctypes.c_int64, _vp, ctypes.c_int64, _vp, _vp, _vp, ctypes.c_int32,
                                     ctypes.c_int32, ctypes.c_double, _vp, ctypes.POINTER(_vp)]
    lib.wcb_scene_destroy.argtypes = [_vp]
    lib.wcb_scene_refit.argtypes = [_vp, _vp, ctypes.c_int64, ctypes.POINTER(ctypes.c_int32), _vp]
    lib.wcb_scene_rebuild_bvh.argtypes = [_vp, ctypes.POINTER(ctypes.c_int32), _vp]
    lib.wcb_scene_info.argtypes = [_vp, _i64p]
    lib.wcb_scene_groups.argtypes = [_vp, _vp, _vp, _vp]
    lib.wcb_scene_edges.argtypes = [_vp, _vp, _vp]
    lib.wcb_solve_workspace_size.argtypes = [_vp, ctypes.POINTER(SolveDesc), _i64p]
    lib.wcb_solve.argtypes = [_vp, ctypes.POINTER(SolveDesc), ctypes.POINTER(Materials), ctypes.POINTER(Outputs), _vp,
                              ctypes.c_int64, _vp]
    lib.wcb_rows_select_workspace_size.argtypes = [ctypes.c_int64, _i64p]
    lib.wcb_rows_select.argtypes = [_vp, ctypes.c_int64, ctypes.c_int32, ctypes.c_int64, ctypes.c_int32, _vp, _i64p, _vp,
                                    ctypes.c_int64, _vp]
    lib.wcb_rows_select_noalloc.argtypes = [_vp, ctypes.c_int64, ctypes.c_int32, ctypes.c_int64, ctypes.c_int32, _vp,
                                            _i64p, _vp]
    lib.wcb_rows_evaluate.argtypes = [_vp, ctypes.POINTER(SolveDesc), ctypes.POINTER(Materials), ctypes.c_int32, _vp, _vp,
                                      ctypes.c_int64, ctypes.c_int32, ctypes.POINTER(RowFields), _vp]
    lib.wcb_rows_accumulate.argtypes = [_vp, _vp, ctypes.c_int64, _vp, _vp, _vp, _vp, ctypes.c_int32, ctypes.c_int32,
                                        ctypes.c_int32, ctypes.POINTER(Outputs), _vp]
    lib.wcb_accumulate_flat_workspace_size.argtypes = [ctypes.c_int64, _i64p]
    lib.wcb_accumulate_flat.argtypes = [_vp, _vp, _vp, _vp, _vp, _vp, _vp, ctypes.c_int64, ctypes.c_int32,
                                        ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32,
                                        ctypes.POINTER(AccumulateOutputs), _vp, ctypes.c_int64, _vp]
    lib.wcb_accumulate_flat_backward.argtypes = [_vp, _vp, _vp, _vp, ctypes.c_int64, ctypes.c_int32, ctypes.c_int32,
                                                 ctypes.c_int32, ctypes.c_int32, ctypes.c_int32,
                                                 ctypes.POINTER(AccumulateOutputs), ctypes.POINTER(AccumulateOutputs),
                                                 _vp, _vp, _vp, _vp]
    lib.wcb_accumulate_flat_jvp_workspace_size.argtypes = [ctypes.c_int64, ctypes.c_int32, _i64p]
    lib.wcb_accumulate_flat_jvp.argtypes = [_vp, _vp, _vp, _vp, _vp, _vp, _vp, ctypes.c_int64, ctypes.c_int32,
                                            ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32,
                                            ctypes.POINTER(AccumulateOutputs), ctypes.POINTER(AccumulateOutputs), _vp,
                                            ctypes.c_int64, _vp]
    lib.wcb_rows_vjp_layout.argtypes = [_vp, ctypes.POINTER(SolveDesc), ctypes.POINTER(Materials), _i64p]
    lib.wcb_rows_vjp_workspace_size.argtypes = [ctypes.c_int64, ctypes.c_int32, ctypes.c_int32, _i64p]
    lib.wcb_rows_vjp.argtypes = [_vp, ctypes.POINTER(SolveDesc), ctypes.POINTER(Materials), ctypes.c_int32, _vp, _vp,
                                 ctypes.c_int64, _vp, _vp, _vp, ctypes.c_int32, _vp, _vp, ctypes.c_int64, _vp, _vp,
                                 ctypes.POINTER(ctypes.c_int64), _vp, ctypes.c_int64, _vp]
    lib.wcb_rows_jvp.argtypes = [_vp, ctypes.POINTER(SolveDesc), ctypes.POINTER(Materials), ctypes.c_int32, _vp, _vp,
                                 ctypes.c_int64, _vp, ctypes.c_int64, _vp, _vp, _vp, ctypes.POINTER(ctypes.c_int64),
                                 _vp]
    lib.wcb_rows_order_workspace_size.argtypes = [ctypes.c_int64, ctypes.POINTER(ctypes.c_int64)]
    lib.wcb_rows_decode.argtypes = [_vp, _vp, ctypes.c_int64, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp]
    lib.wcb_rows_order.argtypes = [_vp, _vp, _vp, ctypes.c_int64, _vp, ctypes.POINTER(ctypes.c_int64), _vp,
                                   ctypes.c_int64, _vp]
    lib.wcb_cfr_workspace_size.argtypes = [ctypes.c_int32, ctypes.c_int32, _i64p]
    lib.wcb_cfr.argtypes = [_vp, _vp, _vp, _vp, ctypes.c_int64, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32,
                            ctypes.c_double, ctypes.c_double, _vp, ctypes.c_int32, _vp, _vp, ctypes.c_int64, _vp]
    lib.wcb_field_free_space.argtypes = [ctypes.c_int64] + [_vp] * 5 + [ctypes.c_double] + [_vp] * 7 + [_vp]
    lib.wcb_field_reflection_sequence.argtypes = [ctypes.c_int64, ctypes.c_int32] + [_vp] * 12 + [ctypes.c_double] + [_vp] * 7 + [_vp]
    lib.wcb_field_transmission_sequence.argtypes = [ctypes.c_int64, ctypes.c_int32] + [_vp] * 8 + [
        ctypes.POINTER(Materials), ctypes.c_double] + [_vp] * 7 + [_vp]
    lib.wcb_field_project_complex3.argtypes = [ctypes.c_int64] + [_vp] * 5 + [_vp]
    lib.wcb_los_jones.argtypes = [_vp, ctypes.c_int64, _vp, ctypes.c_int64, _vp, ctypes.c_int64, _vp, _vp,
                                  ctypes.c_double, _vp, _vp, _vp, _vp, _vp]
    lib.wcb_rows_replay.argtypes = [_vp, ctypes.POINTER(FrozenRows), ctypes.POINTER(EndpointBatch),
                                    ctypes.POINTER(EndpointBatch), ctypes.c_int64, ctypes.POINTER(Materials), _vp,
                                    ctypes.c_int32, ctypes.c_int32, ctypes.POINTER(ReplayOutputs), _vp, _vp]
    lib.wcb_profile_enable.argtypes = [ctypes.c_int32]
    lib.wcb_profile_read.argtypes = [ctypes.POINTER(ctypes.c_double)]
    lib.wcb_build_info.argtypes = [ctypes.c_char_p, ctypes.c_int64]
    lib.wcb_launch_count.restype = ctypes.c_int64
    for name in EXPORTED_SYMBOLS:
        if name != "wcb_launch_count":
            getattr(lib, name).restype = ctypes.c_int
    _lib = lib
    return lib


_STATUS_TEXT = {
    WCB_ERR_INVALID_ARGUMENT: "invalid argument",
    WCB_ERR_CUDA: "CUDA error",
    WCB_ERR_CAPACITY: "buffer capacity exceeded",
    WCB_ERR_BVH_DEPTH: "BVH deeper than the traversal stack",
    WCB_ERR_NOT_SUPPORTED: "not supported",
    WCB_ERR_DEVICE_STATUS: "device reported a failure",
}


class NativeError(RuntimeError):
    def __init__(self, status: int, where: str):
        super().__init__(f"{where} failed: {_STATUS_TEXT.get(status, 'status ' + str(status))}")
        self.status = status


def check(status: int, where: str) -> None:
    if status != WCB_OK:
        raise NativeError(status, where)


def ptr(t: torch.Tensor | None) -> int | None:
    if t is None:
        return None
    return t.data_ptr()


def stream_handle(device: torch.device | None = None) -> int:
    return torch.cuda.current_stream(device).cuda_stream


def launch_count() -> int:
    return int(load().wcb_launch_count())


def profile_enable(enabled: bool) -> None:
    check(load().wcb_profile_enable(int(bool(enabled))), "wcb_profile_enable")


def profile_read() -> dict:
    vals = (ctypes.c_double * 23)()
    check(load().wcb_profile_read(vals), "wcb_profile_read")
    return {"main_ms": vals[0], "prep_ms": vals[1], "rays": int(vals[2]), "main_launches": int(vals[3]),
            "prep_rays": int(vals[4]),
            "kernel_ms": {"k_los_trans": vals[5], "k_reflect": vals[6], "k_diffract": vals[7], "k_finalize": vals[8],
                          "k_diffract_vis": vals[18], "k_diffract_utd": vals[7] - vals[18]},
            "kernel_rays": {"k_los_trans": int(vals[9]), "k_reflect": int(vals[10]), "k_diffract": int(vals[11])},
            "chains": [int(v) for v in vals[12:17]], "edges": int(vals[17]),
            "acc_rays": int(vals[19]), "acc_vjp_diffraction_ms": vals[20],
            "acc_vjp_diffraction_records": int(vals[21]), "acc_vjp_diffraction_launches": int(vals[22])}


def build_info() -> str:
    buf = ctypes.create_string_buffer(256)
    check(load().wcb_build_info(buf, 256), "wcb_build_info")
    return buf.value.decode()
