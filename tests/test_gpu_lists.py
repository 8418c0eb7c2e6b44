"""The depth-first list build (visible tets sorted by depth once, pairs
emitted in that order, then sorted on the tile bits only) gives the same
sorted keys, tet ids and tile ranges as the reference's order of work
(emission in tet order, one sort on 32 + msb bits; keep_debug builds them that
way), on the workloads and on synthetic tets with many equal depths (ties
must stay in tet order)."""
import numpy as np
import pytest
import torch

from gpu_util import to_dev
from radiance_meshes_b200 import _capi as C
from radiance_meshes_b200 import rasterizer as R
from radiance_meshes_b200 import scenes
from radiance_meshes_b200.camera import tcam_to_struct

pytestmark = pytest.mark.gpu


def _both(tiles, rect, vs, cam):
    ref = R.build_tile_lists(tiles, rect, vs, cam, keep_debug=True)
    R._PAIR_GUESS.clear()  # the first-frame path: the count read, then buffers of exactly P
    a = R.build_tile_lists(tiles, rect, vs, cam)
    b = R.build_tile_lists(tiles, rect, vs, cam)  # capacity from the previous frame, all queued before the read
    torch.cuda.synchronize()
    R.check_status(tiles.shape[0], tiles.device)  # what the kernels after the count read reported
    for got in (a, b):
        assert got.n_pairs == ref.n_pairs
        assert torch.equal(got.sorted_ids, ref.sorted_ids)
        assert torch.equal(got.sorted_keys, ref.sorted_keys)
        assert torch.equal(got.ranges, ref.ranges)
    return ref


@pytest.mark.parametrize("workload,tile", [("gradient_check", 16), ("plain_forward", 4), ("plain_forward", 8),
                                           ("plain_forward", 32), ("mixture", 16)])
def test_depth_first_lists_equal_reference_order(cuda, workload, tile):
    if workload == "gradient_check":
        mesh, view = scenes.workload_gradient_check()
    elif workload == "plain_forward":
        mesh, view = scenes.workload_plain_forward(tile)
    else:
        mesh, view = scenes.workload_training_step(n_points=60_000, seed=2, tile_size=16, height=420, width=648)
    cam = tcam_to_struct(view.tcam(tile_size=tile))
    tiles, rect, vs, cc = R.project_fwd(to_dev(mesh.indices), to_dev(mesh.vertices), cam)
    ref = _both(tiles, rect, vs, cam)
    assert ref.n_pairs > 0


def test_depth_first_lists_keep_ties_in_tet_order(cuda):
    rng = np.random.default_rng(11)
    T, gw, gh = 200_000, 37, 23
    x0 = rng.integers(0, gw, T)
    y0 = rng.integers(0, gh, T)
    x1 = np.minimum(gw, x0 + rng.integers(1, 4, T))
    y1 = np.minimum(gh, y0 + rng.integers(1, 4, T))
    visible = rng.uniform(size=T) < 0.6
    rect = np.stack([x0, y0, x1, y1], 1).astype(np.int32)
    rect[~visible] = 0
    tiles = ((x1 - x0) * (y1 - y0)).astype(np.int32)
    tiles[~visible] = 0
    vs = np.zeros((T, 3), np.float32)
    vs[:, 2] = rng.choice(np.array([-3.5, -0.0, 0.0, 1.25, 7.0, 1e20], np.float32), T)  # heavy ties, both zeros
    cam = tcam_to_struct(scenes.workload_gradient_check()[1].tcam())
    cam.grid_width, cam.grid_height = gw, gh
    cam.image_width, cam.image_height = gw * cam.tile_width, gh * cam.tile_height
    _both(to_dev(tiles), to_dev(rect), to_dev(vs), cam)


def test_depth_first_lists_nothing_visible(cuda):
    mesh, view = scenes.workload_gradient_check()
    cam = tcam_to_struct(view.tcam())
    T = len(mesh.indices)
    zeros = torch.zeros(T, dtype=torch.int32, device="cuda")
    ref = _both(zeros, torch.zeros((T, 4), dtype=torch.int32, device="cuda"),
                torch.zeros((T, 3), device="cuda"), cam)
    assert ref.n_pairs == 0 and int(ref.ranges.abs().sum()) == 0
