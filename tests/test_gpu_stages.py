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


@pytest.mark.parametrize("tile", [16, 32])
def test_fine_lists_split_equals_fine_sort(cuda, tile):
    """Splitting the sorted coarse lists (rm_fine_lists) gives exactly the
    lists that emitting and sorting the fine pairs gives."""
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
    tiles, rect, vs, cc, tf, rf = R.project_fwd_fine(i, v, cam, fs)
    t0, r0, vs0, cc0 = R.project_fwd(i, v, cam)
    assert torch.equal(tiles, t0) and torch.equal(rect, r0) and torch.equal(vs, vs0) and torch.equal(cc, cc0)
    assert bool(((tf > 0) <= (tiles > 0)).all())
    coarse = R.build_tile_lists(tiles, rect, vs, cam)
    fine = R.attach_fine_lists(coarse.sorted_ids, coarse.ranges, cam, fs, rf)
    ref = R.build_tile_lists(tf, rf, vs, R.fine_camera(cam, fs))
    n = fine.n_pairs
    assert n == ref.n_pairs == int(tf.sum())
    assert torch.equal(fine.sorted_ids[:n], ref.sorted_ids)
    lf = fine.ranges[:, 1] - fine.ranges[:, 0]
    lr = ref.ranges[:, 1] - ref.ranges[:, 0]
    assert torch.equal(lf, lr)
    ne = lr > 0
    assert torch.equal(fine.ranges[ne], ref.ranges[ne])
