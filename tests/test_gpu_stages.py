"""Stages (a)-(c) on the GPU against the oracle: bit-exact integer outputs.

Covers the reference's scenario families (camera inside a tet, on a face,
outside, inside a point cloud, empty lists) from the golden fixtures and the
plain-forward workload (4,096 points, 256x256) computed by the oracle on the fly.
"""
import numpy as np
import pytest
import torch

import golden_util as G
from gpu_util import bits, run_gpu_forward

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name", G.names())
def test_integer_stages_match_golden(cuda, name):
    z, tcam = G.load(name)
    r = run_gpu_forward(z["vertices"], z["indices"], z["cell_values"], tcam, z["jitter"])
    L = r["lists"]
    assert np.array_equal(r["tiles"].cpu().numpy(), z["tiles_touched"])
    assert np.array_equal(r["rect"].cpu().numpy(), z["rect"])
    assert np.array_equal(bits(r["vs"].cpu().numpy()), bits(z["vs"]))
    assert np.array_equal(bits(r["cc"].cpu().numpy()), bits(z["circumcenter"]))
    assert L.n_pairs == len(z["sorted_ids"])
    assert np.array_equal(L.offsets.cpu().numpy(), z["offsets"])
    assert np.array_equal(L.keys.cpu().numpy(), z["keys"])
    assert np.array_equal(L.values.cpu().numpy(), z["values"])
    assert np.array_equal(L.sorted_keys.cpu().numpy(), z["sorted_keys"])
    assert np.array_equal(L.sorted_ids.cpu().numpy(), z["sorted_ids"])
    assert np.array_equal(L.ranges.cpu().numpy(), z["ranges"])


@pytest.mark.parametrize("tile", [4, 8, 16, 32])
def test_integer_stages_plain_forward_workload(cuda, plain_forward_oracle, tile):
    mesh, view, lists, _ = plain_forward_oracle(tile)
    tcam = view.tcam(tile_size=tile)
    jitter = np.full((view.height, view.width, 2), 0.5, np.float32)
    r = run_gpu_forward(mesh.vertices, mesh.indices, mesh.cell_values, tcam, jitter)
    L = r["lists"]
    assert np.array_equal(r["tiles"].cpu().numpy(), lists["tiles_touched"])
    assert np.array_equal(r["rect"].cpu().numpy(), lists["rect"])
    assert np.array_equal(bits(r["vs"].cpu().numpy()), bits(lists["vs"]))
    assert np.array_equal(L.sorted_ids.cpu().numpy(), lists["sorted_ids"])
    assert np.array_equal(L.ranges.cpu().numpy(), lists["ranges"])


def _fine_rects(box, rect, jb, tile, f, gw, gh):
    """Rectangles on the fine grid of the fine tiles whose pixel rays a tet can
    reach: the fine tiles of the tet's coarse rectangle passing the test of
    rm_fine_lists (box grown by 1/64 pixel against the jittered footprint),
    restated in float32 (the set is an interval in each axis)."""
    w = tile // f
    m = np.float32(1.0 / 64.0)
    b = box.astype(np.float32)
    jb = jb.astype(np.float32)
    out = np.zeros_like(rect)

    def axis(lo_b, hi_b, r0, r1, jmin, jmax, n):
        lo = np.full(len(b), n, np.int64)
        hi = np.full(len(b), -1, np.int64)
        for t in range(n):
            ok = (lo_b - m <= np.float32(t * w + w - 1) + jmax) & (hi_b + m >= np.float32(t * w) + jmin)
            ok &= (r0 * f <= t) & (t < r1 * f)
            lo = np.where(ok & (t < lo), t, lo)
            hi = np.where(ok, t, hi)
        return lo, hi + 1

    x0, x1 = axis(b[:, 0], b[:, 2], rect[:, 0], rect[:, 2], jb[0], jb[2], gw * f)
    y0, y1 = axis(b[:, 1], b[:, 3], rect[:, 1], rect[:, 3], jb[1], jb[3], gh * f)
    ok = (x1 > x0) & (y1 > y0)
    out[:, 0], out[:, 1], out[:, 2], out[:, 3] = x0, y0, x1, y1
    out[~ok] = 0
    return out


@pytest.mark.parametrize("tile,jit", [(16, "unit"), (32, "unit"), (16, "half"), (16, "wide")])
def test_fine_lists_split_equals_fine_sort(cuda, tile, jit):
    """Splitting the sorted coarse lists (rm_fine_lists) gives exactly the
    lists that emitting and sorting the pairs of the fine tiles each tet can
    reach gives."""
    import torch

    from radiance_meshes_b200 import rasterizer as R
    from radiance_meshes_b200 import scenes
    from radiance_meshes_b200.camera import tcam_to_struct

    mesh, view = scenes.workload_training_step(n_points=20000, seed=2, tile_size=tile, height=420, width=649)
    cam = tcam_to_struct(view.tcam())
    fs = R.fine_shift_for(cam)
    assert fs == (1 if tile == 16 else 2)
    i = torch.from_numpy(mesh.indices).cuda()
    v = torch.from_numpy(mesh.vertices).cuda()
    tiles, rect, vs, cc, box = R.project_fwd_fine(i, v, cam)
    t0, r0, vs0, cc0 = R.project_fwd(i, v, cam)
    assert torch.equal(tiles, t0) and torch.equal(rect, r0) and torch.equal(vs, vs0) and torch.equal(cc, cc0)
    rng = np.random.default_rng(7)
    shape = (view.height, view.width, 2)
    j = {"unit": rng.uniform(0, 1, shape), "half": np.full(shape, 0.5), "wide": rng.uniform(-1.5, 2.5, shape)}[jit]
    jitter = torch.from_numpy(j.astype(np.float32)).cuda()
    jb = R.jitter_bounds(jitter)
    jj = j.astype(np.float32).reshape(-1, 2)
    assert np.array_equal(jb.cpu().numpy(), np.array([jj[:, 0].min(), jj[:, 1].min(), jj[:, 0].max(),
                                                      jj[:, 1].max()], np.float32))
    coarse = R.build_tile_lists(tiles, rect, vs, cam)
    fine = R.split_fine_lists(coarse.sorted_ids, coarse.ranges, cam, fs, box, jb)
    rf_np = _fine_rects(box.cpu().numpy(), rect.cpu().numpy(), jb.cpu().numpy(), tile, 1 << fs, cam.grid_width,
                        cam.grid_height)
    rf = torch.from_numpy(rf_np).cuda()
    tf = ((rf[:, 2] - rf[:, 0]) * (rf[:, 3] - rf[:, 1])).to(torch.int32).contiguous()
    assert bool(((tf > 0) <= (tiles > 0)).all())
    ref = R.build_tile_lists(tf, rf, vs, R.fine_camera(cam, fs))
    n = fine.n_pairs
    assert n == ref.n_pairs == int(tf.sum())
    assert torch.equal(fine.sorted_ids[:n], ref.sorted_ids)
    lf = fine.ranges[:, 1] - fine.ranges[:, 0]
    lr = ref.ranges[:, 1] - ref.ranges[:, 0]
    assert torch.equal(lf, lr)
    ne = lr > 0
    assert torch.equal(fine.ranges[ne], ref.ranges[ne])
