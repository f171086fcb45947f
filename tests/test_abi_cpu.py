"""CPU: the C-ABI library loads, exports every declared entry point, rejects
bad arguments before touching the device, and the product path has no CPU
fallback.  No compute call is made here (there is no GPU)."""

from __future__ import annotations

import ctypes
import re
import subprocess
import sys
from pathlib import Path

import pytest

from witwin_channel_b200 import Config, _native

ROOT = Path(__file__).resolve().parents[1]
HEADER = ROOT / "include" / "witwin_channel_b200.h"


def _declared() -> set[str]:
    text = re.sub(r"/\*.*?\*/", "", HEADER.read_text(), flags=re.S)
    return set(re.findall(r"^\s*(?:int|int64_t|void)\s+(wcb_\w+)\s*\(", text, flags=re.M))


def test_library_exports_every_declared_symbol():
    lib = _native.load()
    declared = _declared()
    assert len(declared) >= 20
    missing = sorted(s for s in declared if not hasattr(lib, s))
    assert not missing, missing
    assert declared == set(_native.EXPORTED_SYMBOLS)


def test_host_only_entry_points():
    lib = _native.load()
    assert "sm_100a" in _native.build_info()
    assert isinstance(_native.launch_count(), int)
    _native.profile_enable(False)
    assert set(_native.profile_read()) >= {"main_ms", "rays", "kernel_ms", "chains"}


def test_invalid_arguments_are_rejected_before_device_work():
    lib = _native.load()
    bad = _native.WCB_ERR_INVALID_ARGUMENT
    assert lib.wcb_scene_create(None, 0, None, 0, None, None, None, 1, 0, 0.7, None, None) == bad
    count = ctypes.c_int64()
    assert lib.wcb_rows_select(None, 4, 3, -1, 0, None, ctypes.byref(count), None, 0, None) == bad
    assert lib.wcb_rows_select(None, 0, 9, -1, 0, None, ctypes.byref(count), None, 0, None) == bad
    assert lib.wcb_rows_select_noalloc(None, 4, 3, -1, 0, None, ctypes.byref(count), None) == bad
    assert lib.wcb_rows_select_noalloc(None, 0, 3, -1, 7, None, ctypes.byref(count), None) == bad
    out = _native.AccumulateOutputs()
    assert lib.wcb_accumulate_flat(None, None, None, None, None, None, None, 0, 1, 1, 1, 0, 7, ctypes.byref(out),
                                   None, 0, None) == bad
    assert lib.wcb_accumulate_flat(None, None, None, None, None, None, None, 3, 1, 1, 1, 0, 0, ctypes.byref(out),
                                   None, 0, None) == bad
    assert lib.wcb_accumulate_flat_backward(None, None, None, None, -1, 1, 1, 1, 0, 0, ctypes.byref(out),
                                            ctypes.byref(out), None, None, None, None) == bad
    assert lib.wcb_profile_read(None) == bad
    assert lib.wcb_build_info(None, 0) == bad


def test_missing_library_fails_loudly():
    code = ("import os; os.environ['WITWIN_CHANNEL_B200_LIB'] = '/nonexistent/libwcb200.so'\n"
            "from witwin_channel_b200 import _native\n"
            "try:\n    _native.load()\nexcept RuntimeError as e:\n    print('raised', e)\n")
    out = subprocess.run([sys.executable, "-c", code], cwd=ROOT, capture_output=True, text=True, timeout=120)
    assert "raised" in out.stdout and "not found" in out.stdout


def test_solve_without_cuda_raises():
    import torch

    from tests import scenes
    from witwin_channel_b200 import solve

    if torch.cuda.is_available():
        pytest.skip("CUDA present")
    with pytest.raises(RuntimeError, match="CUDA"):
        solve(scenes.two_wall_scene(), Config(components={"reflection"}, max_depth=2), reference_frequency_hz=3e9)


def test_package_never_imports_the_oracle():
    pkg = ROOT / "witwin_channel_b200"
    for path in pkg.rglob("*.py"):
        src = path.read_text()
        assert not re.search(r"^\s*(from|import)\s+oracle", src, flags=re.M), path
        assert "tests.golden" not in src, path
