"""wcb_rows_select_noalloc against wcb_rows_select, through the C ABI.

The allocation-free entry point must return the same selected record indices
as the workspace entry point (canonical order, identity dedup, max_paths) on
every call, including calls made back to back on the shared scratch array and
a small call after a large one.  Kept in its own file, collected last, so it
runs both alone in a fresh process and after the rest of the GPU suite.
"""

from __future__ import annotations

import ctypes

import pytest
import torch

from witwin_channel_b200 import _native

pytestmark = pytest.mark.gpu

SCRATCH_BYTES = 32 << 20  # WCB_ROWS_SELECT_NOALLOC_SCRATCH_BYTES


def _rows(n: int, seed: int, num_tx: int = 3, num_rx: int = 40) -> torch.Tensor:
    """Random wcb_row records with repeated identities and a few NaN lengths."""
    g = torch.Generator().manual_seed(seed)
    words = torch.full((n, _native.ROW_WORDS), -1, dtype=torch.int32)
    words[:, 0] = torch.randint(0, num_tx, (n,), generator=g)
    words[:, 1] = torch.randint(0, num_rx, (n,), generator=g)
    component = torch.randint(0, 4, (n,), generator=g)  # los, reflection, diffraction, transmission
    depth = torch.where(component == 1, torch.randint(1, 4, (n,), generator=g),
                        torch.where(component == 2, torch.ones_like(component), torch.zeros_like(component)))
    words[:, 2] = (component | (depth << 16)).to(torch.int32)
    faces = torch.randint(0, 6, (n, 5), generator=g).to(torch.int32)
    slot = torch.arange(5).expand(n, 5)
    words[:, 3:8] = torch.where((component == 1).unsqueeze(1) & (slot < depth.unsqueeze(1)), faces, -1)
    edge = torch.randint(0, 4, (n,), generator=g).to(torch.int32)
    words[:, 8] = torch.where(component == 2, edge, -1)
    length = torch.rand(n, generator=g) * 100.0 + 1.0
    length = torch.where(torch.rand(n, generator=g) < 0.002, torch.full_like(length, float("nan")), length)
    words[:, 9] = length.view(torch.int32)
    words[:, 10:12] = 0
    return words.cuda()


def _stream() -> ctypes.c_void_p:
    return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)


def _select_workspace(rows: torch.Tensor, width: int, max_paths: int, scope: int) -> torch.Tensor:
    lib = _native.load()
    n = int(rows.shape[0])
    nbytes = ctypes.c_int64()
    assert lib.wcb_rows_select_workspace_size(n, ctypes.byref(nbytes)) == _native.WCB_OK
    ws = torch.empty(max(nbytes.value, 1), dtype=torch.uint8, device="cuda")
    selected = torch.full((max(n, 1),), -7, dtype=torch.int64, device="cuda")
    count = ctypes.c_int64(-1)
    rc = lib.wcb_rows_select(ctypes.c_void_p(rows.data_ptr()), n, width, max_paths, scope,
                             ctypes.c_void_p(selected.data_ptr()), ctypes.byref(count),
                             ctypes.c_void_p(ws.data_ptr()), nbytes.value, _stream())
    assert rc == _native.WCB_OK
    return selected[: count.value].cpu()


def _select_noalloc(rows: torch.Tensor, width: int, max_paths: int, scope: int,
                    selected: torch.Tensor | None = None) -> tuple[int, torch.Tensor]:
    lib = _native.load()
    n = int(rows.shape[0])
    if selected is None:
        selected = torch.full((max(n, 1),), -7, dtype=torch.int64, device="cuda")
    count = ctypes.c_int64(-1)
    rc = lib.wcb_rows_select_noalloc(ctypes.c_void_p(rows.data_ptr()), n, width, max_paths, scope,
                                     ctypes.c_void_p(selected.data_ptr()), ctypes.byref(count), _stream())
    return rc, selected[: max(count.value, 0)].cpu()


def _max_rows() -> int:
    """Largest record count whose selection workspace fits the fixed scratch."""
    lib = _native.load()
    nbytes = ctypes.c_int64()
    lo, hi = 1, 1 << 24
    while lo < hi:
        mid = (lo + hi + 1) // 2
        assert lib.wcb_rows_select_workspace_size(mid, ctypes.byref(nbytes)) == _native.WCB_OK
        if nbytes.value <= SCRATCH_BYTES:
            lo = mid
        else:
            hi = mid - 1
    return lo


@pytest.mark.parametrize("max_paths,scope", [(-1, 0), (500, 0), (3, 1)])
def test_matches_workspace_entry_two_calls(max_paths, scope):
    rows = _rows(20000, seed=11)
    expected = _select_workspace(rows, 3, max_paths, scope)
    assert expected.numel() > 0
    for _ in range(2):  # back to back on the shared scratch
        rc, got = _select_noalloc(rows, 3, max_paths, scope)
        assert rc == _native.WCB_OK
        assert torch.equal(got, expected)


def test_call_allocates_nothing():
    """After a warm-up call, a second call on a stream the caller already owns
    leaves the device's free memory and torch's allocation counters as they
    were: the selection's scratch all comes from the fixed array."""
    rows = _rows(50000, seed=21)
    selected = torch.full((50000,), -7, dtype=torch.int64, device="cuda")
    rc, first = _select_noalloc(rows, 3, -1, 0, selected)
    assert rc == _native.WCB_OK
    torch.cuda.synchronize()
    free_before, _ = torch.cuda.mem_get_info()
    stats_before = torch.cuda.memory_stats()
    rc, second = _select_noalloc(rows, 3, -1, 0, selected)
    assert rc == _native.WCB_OK
    torch.cuda.synchronize()
    free_after, _ = torch.cuda.mem_get_info()
    stats_after = torch.cuda.memory_stats()
    assert free_after == free_before
    for key in ("allocation.all.allocated", "segment.all.allocated"):
        assert stats_after.get(key, 0) == stats_before.get(key, 0), key
    assert torch.equal(first, second)


def test_small_after_large_and_empty():
    big = _rows(150000, seed=5)
    small = _rows(700, seed=6)
    rc, got_big = _select_noalloc(big, 3, -1, 0)
    assert rc == _native.WCB_OK
    assert torch.equal(got_big, _select_workspace(big, 3, -1, 0))
    for _ in range(2):
        rc, got_small = _select_noalloc(small, 3, 2, 1)
        assert rc == _native.WCB_OK
        assert torch.equal(got_small, _select_workspace(small, 3, 2, 1))
    empty = torch.empty((0, _native.ROW_WORDS), dtype=torch.int32, device="cuda")
    rc, got = _select_noalloc(empty, 3, -1, 0)
    assert rc == _native.WCB_OK and got.numel() == 0


def test_capacity_boundary():
    n_max = _max_rows()
    rows = _rows(n_max + 1, seed=9, num_tx=8, num_rx=4000)
    selected = torch.full((n_max + 1,), -7, dtype=torch.int64, device="cuda")
    # one record over the limit: rejected before any work, output untouched
    rc, _ = _select_noalloc(rows, 3, -1, 0, selected)
    assert rc == _native.WCB_ERR_CAPACITY
    torch.cuda.synchronize()
    assert bool((selected == -7).all())
    # exactly at the limit: accepted and equal to the workspace entry point
    at_limit = rows[:n_max]
    expected = _select_workspace(at_limit, 3, 5, 1)
    for _ in range(2):
        rc, got = _select_noalloc(at_limit, 3, 5, 1, selected)
        assert rc == _native.WCB_OK
        assert torch.equal(got, expected)


def test_invalid_arguments():
    lib = _native.load()
    rows = _rows(10, seed=1)
    count = ctypes.c_int64()
    out = torch.empty(10, dtype=torch.int64, device="cuda")
    assert lib.wcb_rows_select_noalloc(ctypes.c_void_p(rows.data_ptr()), 10, 6, -1, 0,
                                       ctypes.c_void_p(out.data_ptr()), ctypes.byref(count),
                                       _stream()) == _native.WCB_ERR_INVALID_ARGUMENT
    assert lib.wcb_rows_select_noalloc(ctypes.c_void_p(rows.data_ptr()), 10, 3, -1, 2,
                                       ctypes.c_void_p(out.data_ptr()), ctypes.byref(count),
                                       _stream()) == _native.WCB_ERR_INVALID_ARGUMENT
    assert lib.wcb_rows_select_noalloc(None, 10, 3, -1, 0, ctypes.c_void_p(out.data_ptr()), ctypes.byref(count),
                                       _stream()) == _native.WCB_ERR_INVALID_ARGUMENT
