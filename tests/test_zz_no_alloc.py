"""The allocation-free scan entry point (rm_scan_tiles_noalloc) against the
regular one (rm_scan_tiles with a workspace), through the C ABI.

Some callers cannot allocate device memory (a host runtime that gives the
library only its inputs and outputs); for them the scan keeps its look-back
scratch in a fixed array inside the library.  The offsets and the pair total
are integers and must match exactly, on two calls in a row with different
inputs (the second call must not see the first call's scratch contents).
"""
import ctypes

import numpy as np
import pytest
import torch

from radiance_meshes_b200 import _capi as C

pytestmark = pytest.mark.gpu


def _scan_with_workspace(tiles):
    L = C.lib()
    T = tiles.numel()
    off = torch.empty_like(tiles)
    tot = torch.zeros(1, dtype=torch.int64, device=tiles.device)
    ws_n = L.rm_scan_workspace_size(T)
    ws = torch.empty(ws_n, dtype=torch.uint8, device=tiles.device)
    C.check(L.rm_scan_tiles(C.ptr(tiles), T, C.ptr(off), C.ptr(tot), C.ptr(ws), ws_n, C.stream_handle()), "scan")
    return off, tot


def _scan_no_alloc(tiles):
    L = C.lib()
    T = tiles.numel()
    off = torch.empty_like(tiles)
    tot = torch.full((1,), -1, dtype=torch.int64, device=tiles.device)
    C.check(L.rm_scan_tiles_noalloc(C.ptr(tiles), T, C.ptr(off), C.ptr(tot), C.stream_handle()), "scan noalloc")
    return off, tot


def test_no_alloc_scan_matches_workspace_scan(cuda):
    rng = np.random.default_rng(7)
    for T in (1_317_313, 70_001):  # two calls in a row, different sizes and values
        tiles = torch.from_numpy(rng.integers(0, 9, size=T).astype(np.int32)).cuda()
        ref_off, ref_tot = _scan_with_workspace(tiles)
        off, tot = _scan_no_alloc(tiles)
        torch.cuda.synchronize()
        assert torch.equal(off, ref_off)
        assert int(tot.item()) == int(ref_tot.item()) == int(tiles.sum().item())


def _noalloc_status():
    st = ctypes.c_uint32(0)
    C.check(C.lib().rm_scan_noalloc_read_status(ctypes.byref(st), C.stream_handle()), "noalloc status")
    return st.value


def test_no_alloc_scan_reports_through_its_status_word(cuda):
    """The fixed scratch has its own status word, read (and cleared) with
    rm_scan_noalloc_read_status: a total beyond int32 and a look-back that
    gives up (a wait limit of one poll) are reported there, and a clean call
    leaves it zero."""
    rng = np.random.default_rng(11)
    tiles = torch.from_numpy(rng.integers(0, 9, size=3_000_000).astype(np.int32)).cuda()
    _scan_no_alloc(tiles)
    assert _noalloc_status() == 0
    big = torch.full((600_000,), 4096, dtype=torch.int32, device="cuda")
    _scan_no_alloc(big)
    assert _noalloc_status() & C.RM_STATUS_OVERFLOW
    assert _noalloc_status() == 0  # cleared by the read
    seen = False
    try:
        C.set_wait_limit(1)
        for _ in range(5):
            _scan_no_alloc(tiles)
            if _noalloc_status() & C.RM_STATUS_SCAN_TIMEOUT:
                seen = True
                break
    finally:
        C.set_wait_limit(0)
    assert seen
    off, tot = _scan_no_alloc(tiles)
    ref_off, ref_tot = _scan_with_workspace(tiles)
    torch.cuda.synchronize()
    assert _noalloc_status() == 0 and torch.equal(off, ref_off) and int(tot.item()) == int(ref_tot.item())


def test_no_alloc_scan_rejects_oversize():
    L = C.lib()
    rc = L.rm_scan_tiles_noalloc(None, (1 << 26) + 1, None, None, None)
    assert rc == C.RM_EINVAL and "limit" in C.last_error()
