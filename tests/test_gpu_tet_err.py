"""Densification statistics (calc_tet_err) against the oracle's FP32
restatement: hit counts exact, int(65535 T) maxima within one unit (exp
rounding), float sums within summation-order tolerance; the same with the
8x8-pixel fine lists; and the render_err drop-in end to end."""
import numpy as np
import pytest
import torch

import radiance_meshes_b200 as RMB
from gpu_util import to_dev
from oracle import oracle as O
from radiance_meshes_b200 import rasterizer as R
from radiance_meshes_b200 import scenes
from radiance_meshes_b200.camera import tcam_to_struct

pytestmark = pytest.mark.gpu

COLS = [0, 1, 2, 5, 6, 7, 8, 9, 10, 11, 12, 13, 14, 15]


def _errs(view, seed):
    rng = np.random.default_rng(seed)
    pe = rng.normal(0, 0.2, (view.height, view.width)).astype(np.float32)
    se = rng.uniform(0, 1, (view.height, view.width)).astype(np.float32)
    return pe, se


def _check(err, cnt, ref_err, ref_cnt, ref_max):
    err, cnt = err.cpu().numpy(), cnt.cpu().numpy()
    assert np.array_equal(cnt[:, 0], ref_cnt)
    assert np.abs(cnt[:, 1].astype(np.int64) - ref_max).max() <= 1
    assert np.all(err[:, 3] == 0) and np.all(err[:, 4] == 0)
    for k in COLS:
        a, b = err[:, k].astype(np.float64), ref_err[:, k]
        scale = np.abs(b).max() + 1e-30
        assert np.abs(a - b).max() <= 1e-4 * scale + 1e-5 * np.abs(b).max(), k
        assert np.linalg.norm(a - b) <= 1e-5 * np.linalg.norm(b) + 1e-12, k


@pytest.mark.parametrize("scene", ["ball", "cube"])
def test_calc_tet_err_matches_oracle(cuda, scene):
    mesh, view = scenes.workload_gradient_check() if scene == "ball" else scenes.workload_plain_forward()
    cam = tcam_to_struct(view.tcam())
    pe, se = _errs(view, 3)
    i, v, c = to_dev(mesh.indices), to_dev(mesh.vertices), to_dev(mesh.cell_values)
    tiles, rect, vs, cc = R.project_fwd(i, v, cam)
    L = R.build_tile_lists(tiles, rect, vs, cam)
    err, cnt = R.calc_tet_err(L.sorted_ids, L.ranges, i, v, c, cam, to_dev(pe), to_dev(se), tiles_touched=tiles)
    lists = dict(cam=cam, sorted_ids=L.sorted_ids.cpu().numpy(), ranges=L.ranges.cpu().numpy())
    ref_err, ref_cnt, ref_max = O.calc_tet_err(lists, mesh.indices, mesh.vertices, mesh.cell_values, pe, se)
    assert ref_cnt.sum() > 1000
    _check(err, cnt, ref_err, ref_cnt, ref_max)
    # the fine lists visit the same hits in the same order
    fs = R.fine_shift_for(cam)
    t2, r2, vs2, cc2, fp = R.project_fwd_fine(i, v, cam)
    L2 = R.build_tile_lists(t2, r2, vs2, cam)
    half = torch.full((view.height, view.width, 2), 0.5, device="cuda")
    F = R.split_fine_lists(L2.sorted_ids, L2.ranges, cam, fs, fp, R.jitter_bounds(half), L2.sorted_keys)
    err2, cnt2 = R.calc_tet_err(F.sorted_ids, F.ranges, i, v, c, F.cam, to_dev(pe), to_dev(se), tiles_touched=t2)
    _check(err2, cnt2, ref_err, ref_cnt, ref_max)


class _Cam:
    def __init__(self, view):
        self.view = view
        self.image_height, self.image_width = view.height, view.width
        self.gt_alpha_mask = torch.ones((1, view.height, view.width))

    def to_dict(self, device):
        t = self.view.tcam(device=device)
        keep = ("world_view_transform", "cam_pos", "K", "image_height", "image_width", "fovy", "fovx",
                "distortion_params", "camera_type")
        return {k: t[k] for k in keep}


class _Model:
    feature_dim = 7

    def __init__(self, mesh):
        self.vertices = to_dev(mesh.vertices)
        self.indices = to_dev(mesh.indices)
        self.cv = to_dev(mesh.cell_values)
        self.device = "cuda"

    def get_cell_values(self, camera, mask):
        return None, self.cv[mask]


def test_render_err_dropin(cuda):
    RMB.install_dropin()
    from delaunay_rasterization.internal.render_err import render_err

    mesh, view = scenes.workload_plain_forward()
    gt = torch.rand(3, view.height, view.width, device="cuda", generator=torch.Generator("cuda").manual_seed(1))
    tet_err, extras = render_err(gt, _Cam(view), _Model(mesh), tile_size=16)
    assert tet_err.shape == (len(mesh.indices), 16) and extras["tet_count"].shape == (len(mesh.indices), 2)
    assert extras["pixel_err"].shape == (view.height, view.width)
    cam = tcam_to_struct(view.tcam())
    lists = O.rasterize_lists(mesh.indices, mesh.vertices, view.tcam())
    ref_err, ref_cnt, ref_max = O.calc_tet_err(lists, mesh.indices, mesh.vertices, mesh.cell_values,
                                               extras["pixel_err"].cpu().numpy(), extras["ssim_err"].cpu().numpy())
    _check(tet_err, extras["tet_count"], ref_err, ref_cnt, ref_max)
