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


def test_no_alloc_scan_rejects_oversize():
    L = C.lib()
    rc = L.rm_scan_tiles_noalloc(None, (1 << 26) + 1, None, None, None)
    assert rc == C.RM_EINVAL and "limit" in C.last_error()
