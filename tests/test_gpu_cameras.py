"""Non-pinhole cameras (camera.slang:241-508): radial/tangential distortion
and the fisheye model, projection and blend against the oracle.  Distortion
is polynomial arithmetic, so the integer stages stay bit-exact; the fisheye
model goes through sin/cos/acos, whose last bits differ between CUDA and the
host libm, so there the rectangles may differ for a few tets whose box edge
lies on a tile boundary, and images are compared on the GPU's own lists."""
import numpy as np
import pytest
import torch

from gpu_util import to_dev
from oracle import oracle as O
from radiance_meshes_b200 import rasterizer as R
from radiance_meshes_b200 import scenes
from radiance_meshes_b200.camera import tcam_to_struct

pytestmark = pytest.mark.gpu

CASES = {
    "distorted": dict(camera_type=0, distortion_params=[0.05, -0.01, 0.001, -0.002]),
    "fisheye": dict(camera_type=1, distortion_params=[0.0, 0.0, 0.0, 0.0]),
    "fisheye_distorted": dict(camera_type=1, distortion_params=[0.02, 0.003, -0.001, 0.0005]),
}


def _scene(case):
    mesh, view = scenes.workload_plain_forward()
    t = view.tcam()
    for k, v in CASES[case].items():
        t[k] = np.asarray(v, np.float32) if k == "distortion_params" else v
    return mesh, view, t


@pytest.mark.parametrize("case", list(CASES))
def test_projection_and_blend_vs_oracle(cuda, case):
    mesh, view, tcam = _scene(case)
    cam = tcam_to_struct(tcam)
    i, v, c = to_dev(mesh.indices), to_dev(mesh.vertices), to_dev(mesh.cell_values)
    tiles, rect, vs, cc = R.project_fwd(i, v, cam)
    cs = O.camstruct(tcam)
    ot, orect, ovs, occ = O.project(mesh.indices, mesh.vertices, cs)
    gt, grect = tiles.cpu().numpy(), rect.cpu().numpy()
    same = (gt == ot) & (grect == orect).all(1)
    if case == "distorted":
        assert same.all()
        assert np.array_equal(vs.cpu().numpy(), ovs)
    else:
        assert same.mean() > 0.995, same.mean()
    assert (gt > 0).sum() > 1000
    L = R.build_tile_lists(tiles, rect, vs, cam)
    jitter = np.random.default_rng(2).uniform(0, 1, (view.height, view.width, 2)).astype(np.float32)
    img, dist, nc, _ = R.blend_fwd(L.sorted_ids, L.ranges, i, v, c, to_dev(jitter), cam, tiles_touched=tiles)
    lists = dict(cam=cs, sorted_ids=L.sorted_ids.cpu().numpy(), ranges=L.ranges.cpu().numpy())
    img32, dist32, nc32 = O.blend_fwd_f32(lists, mesh.indices, mesh.vertices, mesh.cell_values, jitter)
    g = img.cpu().numpy()
    err = np.abs(g[..., :3] - img32[..., :3])
    if case == "distorted":
        assert np.array_equal(nc.cpu().numpy()[..., 0], nc32)
        assert err.max() <= 1e-4
    else:
        assert np.mean(nc.cpu().numpy()[..., 0] == nc32) > 0.99
        assert np.quantile(err, 0.999) <= 1e-4 and err.max() <= 5e-2
    assert float(np.abs(g[..., :3]).sum()) > 0


def test_fisheye_sees_wider_than_perspective(cuda):
    """A fisheye camera with the same focal length covers a wider field: more
    tets reach its image than the pinhole's."""
    mesh, view, t_fish = _scene("fisheye")
    t_pin = view.tcam()
    i, v = to_dev(mesh.indices), to_dev(mesh.vertices)
    n_fish = int((R.project_fwd(i, v, tcam_to_struct(t_fish))[0] > 0).sum())
    n_pin = int((R.project_fwd(i, v, tcam_to_struct(t_pin))[0] > 0).sum())
    assert n_fish >= n_pin
