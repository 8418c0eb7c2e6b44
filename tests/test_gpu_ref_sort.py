"""Stage (c) pinned to the reference's own code: rm_sort_pairs against the
reference's CUB sort wrapper (delaunay_rasterization/internal/sort_by_keys/
sort_by_keys.cu:10-53, compiled unchanged into oracle/_ref by
oracle/build_ref.py), bit for bit, on the coarse pair lists of the plain-forward,
gradient-check and 1.32M-tet training workloads and on synthetic key sets
(duplicate keys, every end_bit, bits above end_bit set)."""
import os
import sys

import numpy as np
import pytest
import torch

from gpu_util import to_dev
from radiance_meshes_b200 import _capi as C
from radiance_meshes_b200 import rasterizer as R
from radiance_meshes_b200 import scenes
from radiance_meshes_b200.camera import tcam_to_struct

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module")
def ref_sort(cuda):
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    try:
        import build_ref
    finally:
        sys.path.pop(0)
    mod = build_ref.load_sort()
    assert mod is not None, "oracle/_ref/sort_by_keys is not built (python oracle/build_ref.py)"
    return mod.sort_by_keys


def _ours(keys, vals, end_bit):
    L = C.lib()
    n = keys.numel()
    ko, vo = torch.empty_like(keys), torch.empty_like(vals)
    if n == 0:
        return ko, vo
    ws_n = L.rm_sort_workspace_size(n)
    ws = torch.empty(ws_n, dtype=torch.uint8, device=keys.device)
    status = torch.zeros(1, dtype=torch.int32, device=keys.device)
    C.check(L.rm_sort_pairs(C.ptr(keys), C.ptr(vals), n, None, end_bit, C.ptr(ko), C.ptr(vo), C.ptr(ws), ws_n,
                            C.ptr(status), C.stream_handle()), "rm_sort_pairs")
    torch.cuda.synchronize()
    assert int(status.item()) == 0
    return ko, vo


def _compare(ref_sort, keys, vals, msb):
    rk, rv = ref_sort(keys, vals, msb)
    ok, ov = _ours(keys, vals, 32 + msb)
    torch.cuda.synchronize()
    assert torch.equal(ok, rk), "sorted keys differ from the reference's CUB sort"
    assert torch.equal(ov, rv), "sorted values differ from the reference's CUB sort (stability)"


def _coarse_pairs(mesh, view, tile=16):
    tcam = view.tcam(tile_size=tile)
    cam = tcam_to_struct(tcam)
    i, v = to_dev(mesh.indices), to_dev(mesh.vertices)
    tiles, rect, vs, cc = R.project_fwd(i, v, cam)
    lists = R.build_tile_lists(tiles, rect, vs, cam, keep_debug=True)
    msb = int(cam.grid_width * cam.grid_height).bit_length()
    return lists.keys.contiguous(), lists.values.contiguous(), msb, lists


@pytest.mark.parametrize("workload", ["plain_forward", "gradient_check", "training_step"])
def test_sort_matches_reference_on_workload_pairs(ref_sort, workload):
    if workload == "plain_forward":
        mesh, view = scenes.workload_plain_forward(16)
    elif workload == "gradient_check":
        mesh, view = scenes.workload_gradient_check()
    else:
        mesh, view = scenes.workload_training_step(n_points=200_000, seed=2, tile_size=16, height=840, width=1297)
    keys, vals, msb, lists = _coarse_pairs(mesh, view)
    assert keys.numel() > 0
    _compare(ref_sort, keys, vals, msb)
    # and the sorted lists the drop-in returns are the reference's
    rk, rv = ref_sort(keys, vals, msb)
    assert torch.equal(lists.sorted_ids, rv) and torch.equal(lists.sorted_keys, rk)


@pytest.mark.parametrize("msb", [1, 5, 8, 13, 16, 24, 31])
def test_sort_matches_reference_every_end_bit(ref_sort, msb):
    rng = np.random.default_rng(msb)
    n = 300_001
    tile = rng.integers(0, 1 << msb, size=n, dtype=np.int64)
    depth = rng.integers(0, 1 << 32, size=n, dtype=np.int64)
    keys = to_dev((tile << 32) | depth)
    vals = to_dev(rng.permutation(n).astype(np.int32))
    _compare(ref_sort, keys, vals, msb)


def test_sort_matches_reference_duplicates_and_high_bits(ref_sort):
    rng = np.random.default_rng(5)
    n = 1_000_003
    # few distinct keys: long runs of ties whose order must stay the emission order
    base = rng.integers(0, 37, size=n, dtype=np.int64)
    keys = to_dev((base << 32) | (base * 7 % 5))
    vals = to_dev(np.arange(n, dtype=np.int32))
    _compare(ref_sort, keys, vals, 6)
    # bits above end_bit are carried along but do not take part in the order
    hi = rng.integers(0, 1 << 20, size=n, dtype=np.int64) << 43
    keys2 = to_dev(hi | (rng.integers(0, 1 << 11, size=n, dtype=np.int64) << 32) |
                   rng.integers(0, 1 << 32, size=n, dtype=np.int64))
    _compare(ref_sort, keys2, vals, 11)


@pytest.mark.parametrize("n", [1, 2, 31, 4095, 4096, 4097])
def test_sort_matches_reference_small(ref_sort, n):
    rng = np.random.default_rng(n)
    keys = to_dev(rng.integers(0, 1 << 40, size=n, dtype=np.int64))
    vals = to_dev(rng.integers(-(1 << 31), (1 << 31) - 1, size=n, dtype=np.int64).astype(np.int32))
    _compare(ref_sort, keys, vals, 8)
