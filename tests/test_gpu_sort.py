"""Onesweep radix sort (stage c) against numpy's stable argsort on the masked
keys: sizes around the 4096-pair tile, heavy duplicates (stability), every
digit-boundary end bit, and the device-side pair count used under graph
capture."""
import ctypes

import numpy as np
import pytest
import torch

from radiance_meshes_b200 import _capi as C

pytestmark = pytest.mark.gpu


def gpu_sort(keys, vals, end_bit, n_dev=None):
    L = C.lib()
    n = len(keys)
    k = torch.from_numpy(keys).cuda()
    v = torch.from_numpy(vals).cuda()
    ko = torch.empty_like(k)
    vo = torch.empty_like(v)
    ws_n = L.rm_sort_workspace_size(n)
    ws = torch.zeros(ws_n, dtype=torch.uint8, device="cuda")
    nd = None
    if n_dev is not None:
        nd = torch.tensor([n_dev], dtype=torch.int64, device="cuda")
    C.check(L.rm_sort_pairs(C.ptr(k), C.ptr(v), n, C.ptr(nd), end_bit, C.ptr(ko), C.ptr(vo), C.ptr(ws), ws_n,
                            None, C.stream_handle()), "sort")
    st = ctypes.c_uint32(0)
    C.check(L.rm_read_status(C.ptr(ws), ctypes.byref(st), C.stream_handle()))
    assert st.value == 0
    return ko.cpu().numpy(), vo.cpu().numpy()


def ref_sort(keys, vals, end_bit):
    mask = np.uint64((1 << end_bit) - 1) if end_bit < 64 else np.uint64(0xFFFFFFFFFFFFFFFF)
    mk = keys.view(np.uint64) & mask
    order = np.argsort(mk, kind="stable")
    return keys[order], vals[order]


@pytest.mark.parametrize("n", [1, 2, 31, 4095, 4096, 4097, 65537, 1_000_003])
@pytest.mark.parametrize("end_bit", [8, 13, 33, 45])
def test_sort_random(cuda, n, end_bit):
    rng = np.random.default_rng(n * 100 + end_bit)
    keys = rng.integers(0, 2 ** 62, size=n, dtype=np.int64)
    vals = np.arange(n, dtype=np.int32)
    ko, vo = gpu_sort(keys, vals, end_bit)
    rk, rv = ref_sort(keys, vals, end_bit)
    assert np.array_equal(ko, rk) and np.array_equal(vo, rv)


@pytest.mark.parametrize("end_bit", [1, 7, 40, 64])
def test_sort_duplicates_stable(cuda, end_bit):
    rng = np.random.default_rng(end_bit)
    n = 300_000
    keys = rng.integers(0, 5, size=n, dtype=np.int64) << np.int64(max(0, min(end_bit, 62) - 3))
    keys |= rng.integers(0, 3, size=n, dtype=np.int64)
    vals = np.arange(n, dtype=np.int32)
    ko, vo = gpu_sort(keys, vals, end_bit)
    rk, rv = ref_sort(keys, vals, end_bit)
    assert np.array_equal(ko, rk) and np.array_equal(vo, rv)


def test_sort_tile_shaped_keys(cuda):
    """Keys shaped like the rasterizer's: (tile << 32) | sortable(depth), with
    many equal depths so ordering falls back to emission (tet id) order."""
    rng = np.random.default_rng(11)
    n = 2_000_000
    G = 82 * 53
    tile = rng.integers(0, G, size=n).astype(np.uint64)
    depth = rng.integers(0, 1000, size=n).astype(np.uint64) | np.uint64(0x80000000)
    keys = ((tile << np.uint64(32)) | depth).view(np.int64)
    vals = rng.integers(0, 1_300_000, size=n).astype(np.int32)
    end_bit = 32 + G.bit_length()
    ko, vo = gpu_sort(keys, vals, end_bit)
    rk, rv = ref_sort(keys, vals, end_bit)
    assert np.array_equal(ko, rk) and np.array_equal(vo, rv)


def test_sort_device_count(cuda):
    rng = np.random.default_rng(5)
    cap, n = 50_000, 37_123
    keys = rng.integers(0, 2 ** 40, size=cap, dtype=np.int64)
    vals = np.arange(cap, dtype=np.int32)
    ko, vo = gpu_sort(keys, vals, 40, n_dev=n)
    rk, rv = ref_sort(keys[:n], vals[:n], 40)
    assert np.array_equal(ko[:n], rk) and np.array_equal(vo[:n], rv)
