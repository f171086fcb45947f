"""wcb_rows_select against the oracle's canonical selection at large ids.

The sort key keeps every field at full width: sources past 2048, sinks past
2^21 and face/edge ids past 2^18 must sort and deduplicate exactly like the
reference's selection (full int tx_id/rx_id/object ids,
``native/channel/kernels/evaluated_paths.cu:56-57,182``).  The records include
identities that differ only above those bit positions (tx 5 and 2053, rx r and
r + 2^21, face f and f + 2^18), which a truncated key would merge.
"""

from __future__ import annotations

import ctypes

import numpy as np
import pytest
import torch

from oracle import solve as osolve
from witwin_channel_b200 import _native

pytestmark = pytest.mark.gpu


def _records(n: int, seed: int) -> dict:
    rng = np.random.default_rng(seed)
    tx_pool = np.array([5, 2053, 2047, 3000, 4101])
    rx_pool = np.array([7, 7 + (1 << 21), 1 << 20, 3_000_000, 4_194_303 + 17])
    face_pool = np.array([3, 3 + (1 << 18), 262_143, 262_144, 300_001, 9])
    edge_pool = np.array([1, 1 + (1 << 18), 270_000])
    tx = rng.choice(tx_pool, n)
    rx = rng.choice(rx_pool, n)
    cid = rng.choice(np.array([0, 1, 2, 5]), n)
    depth = np.where(cid == 1, rng.integers(1, 4, n), np.where(cid == 5, rng.integers(1, 3, n),
                                                               np.where(cid == 2, 1, 0)))
    width = 3
    seq = np.full((n, width), -1, dtype=np.int64)
    faces = rng.choice(face_pool, (n, width))
    slot = np.arange(width)[None, :]
    use = ((cid == 1) | (cid == 5))[:, None] & (slot < depth[:, None])
    seq[use] = faces[use]
    edge = np.where(cid == 2, rng.choice(edge_pool, n), -1)
    length = (rng.random(n) * 100.0 + 1.0).astype(np.float32)
    length[rng.random(n) < 0.003] = np.nan
    # exact length ties inside some identities (first in canonical order wins)
    length[rng.random(n) < 0.2] = np.float32(50.0)
    return dict(tx=tx.astype(np.int64), rx=rx.astype(np.int64), cid=cid.astype(np.int64), depth=depth.astype(np.int64),
                edge=edge.astype(np.int64), seq=seq, length=length, width=width)


def _pack(r: dict) -> torch.Tensor:
    n = len(r["tx"])
    words = np.full((n, _native.ROW_WORDS), -1, dtype=np.int32)
    words[:, 0] = r["tx"]
    words[:, 1] = r["rx"]
    words[:, 2] = r["cid"] | (r["depth"] << 16)
    words[:, 3:3 + r["width"]] = r["seq"]
    words[:, 8] = r["edge"]
    words[:, 9] = r["length"].view(np.int32)
    words[:, 10:] = 0
    return torch.from_numpy(words).cuda()


def _select(rows: torch.Tensor, width: int, max_paths: int, scope: int) -> np.ndarray:
    lib = _native.load()
    n = int(rows.shape[0])
    nbytes = ctypes.c_int64()
    assert lib.wcb_rows_select_workspace_size(n, ctypes.byref(nbytes)) == _native.WCB_OK
    ws = torch.empty(max(nbytes.value, 1), dtype=torch.uint8, device="cuda")
    selected = torch.full((max(n, 1),), -7, dtype=torch.int64, device="cuda")
    count = ctypes.c_int64(-1)
    rc = lib.wcb_rows_select(ctypes.c_void_p(rows.data_ptr()), n, width, max_paths, scope,
                             ctypes.c_void_p(selected.data_ptr()), ctypes.byref(count),
                             ctypes.c_void_p(ws.data_ptr()), nbytes.value,
                             ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))
    assert rc == _native.WCB_OK
    return selected[: count.value].cpu().numpy()


@pytest.mark.parametrize("max_paths,scope", [(None, "global"), (400, "global"), (2, "pair")])
def test_full_width_key_matches_oracle(max_paths, scope):
    r = _records(30000, seed=3)
    rows = _pack(r)
    got = _select(rows, r["width"], -1 if max_paths is None else max_paths, 0 if scope == "global" else 1)
    want = osolve.select_records(r["tx"], r["rx"], r["cid"], r["depth"], r["edge"], r["seq"],
                                 r["length"].astype(np.float64), max_paths=max_paths, scope=scope)
    assert got.shape == want.shape
    assert np.array_equal(got, want)
    if max_paths is not None:
        return
    # the truncation-sensitive identities survive as distinct rows
    kept_tx = set(r["tx"][got].tolist())
    assert {5, 2053} <= kept_tx
    kept_rx = set(r["rx"][got].tolist())
    assert {7, 7 + (1 << 21)} <= kept_rx
