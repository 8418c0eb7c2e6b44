"""Parity against outputs of the reference's own Python code
(tests/golden/make_ref_golden.py imported it to make these fixtures):

  * the fused feature kernel against the reference's activate_output
    (utils/model_util.py:93-105), values and gradients, SH degrees 0-3;
  * this package's render() with the CUDA drop-in and the fused feature
    kernel against the reference's render() (utils/train_util.py:15-77) fed
    by the reference's Camera.to_dict and activate_output, with the oracle's
    FP32 restatement standing in for the Slang kernels: render_pkg (render,
    alpha, distortion_loss, mask, sh_reg) and the gradients of
    L1 + 0.01 distortion + 0.001 sh_reg.

Tolerances: features 1e-5 (abs + rel); gradients relative L2 <= 1e-4 for the
feature kernel; for render(): image and alpha <= 1e-4 max-abs, losses 1e-5
relative, gradients relative L2 <= 1e-3 per group (the blend adjoint against
the FP32 restatement is within 1e-4; the rest is summation order)."""
import os

import numpy as np
import pytest
import torch

import radiance_meshes_b200 as RMB
from radiance_meshes_b200 import features as FT
from radiance_meshes_b200 import render as RR

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def _rel(a, b):
    a, b = a.double(), b.double()
    den = float(b.norm())
    return float((a - b).norm()) / den if den > 0 else float(a.norm())


@pytest.mark.parametrize("deg", [0, 1, 2, 3])
def test_features_match_reference_activate_output(cuda, deg):
    g = np.load(os.path.join(GOLDEN, "ref_activate_output.npz"))
    t = lambda k: torch.tensor(g[k], device="cuda", requires_grad=True)
    density, rgb, grd, sh, cc, verts = (t(k) for k in ("density", "rgb", "grd", "sh", "circumcenters", "vertices"))
    idx = torch.tensor(g["indices"], device="cuda")
    cam = torch.tensor(g["camera_center"])
    out = FT.activate_output(cam, density, rgb, grd, sh, idx, cc, verts, deg, 3)
    ref = torch.tensor(g[f"features_{deg}"], device="cuda")
    assert torch.allclose(out, ref, rtol=1e-5, atol=1e-5), float((out - ref).abs().max())
    (out * torch.tensor(g["w"], device="cuda")).sum().backward()
    for name, p in zip(("density", "rgb", "grd", "sh", "circumcenters", "vertices"),
                       (density, rgb, grd, sh, cc, verts)):
        want = torch.tensor(g[f"grad_{name}_{deg}"], device="cuda")
        got = p.grad if p.grad is not None else torch.zeros_like(p)
        if float(want.norm()) == 0.0:
            assert float(got.norm()) == 0.0, name
        else:
            assert _rel(got, want) <= 1e-4, (name, _rel(got, want))


class _Camera:
    """The camera record the reference's Camera.to_dict produced
    (data/camera.py:72-91), replayed on the device."""

    def __init__(self, g, device):
        self.g = g
        self.image_height = int(g["tcam_image_height"])
        self.image_width = int(g["tcam_image_width"])
        self.gt_alpha_mask = torch.tensor(g["gt_alpha_mask"])
        self.camera_center = torch.tensor(g["camera_center"])

    def to_dict(self, device):
        g = self.g
        return dict(world_view_transform=torch.tensor(g["tcam_world_view_transform"], device=device),
                    cam_pos=torch.tensor(g["tcam_cam_pos"], device=device),
                    K=torch.tensor(g["tcam_K"], device=device), image_height=self.image_height,
                    image_width=self.image_width, fovy=float(g["tcam_fovy"]), fovx=float(g["tcam_fovx"]),
                    distortion_params=torch.tensor(g["tcam_distortion_params"], device=device),
                    camera_type=int(g["tcam_camera_type"]))


class _Model:
    """get_cell_values of the reference model (models/ingp_color.py:361-387)
    over fixed raw per-tet outputs, with this package's fused feature kernel."""
    feature_dim = 7
    mask_values = True
    max_sh_deg = 1
    current_sh_deg = 1

    def __init__(self, g):
        self.device = torch.device("cuda")
        self.vertices = torch.tensor(g["vertices"], device="cuda", requires_grad=True)
        self.indices = torch.tensor(g["indices"], device="cuda")
        self.leaves = [torch.tensor(g[k], device="cuda", requires_grad=True) for k in ("density", "rgb", "grd", "sh")]

    def get_cell_values(self, camera, mask=None, all_circumcenters=None):
        m = mask if mask is not None else torch.ones(self.indices.shape[0], dtype=torch.bool, device="cuda")
        d, c, gr, s = (x[m] for x in self.leaves)
        indices = self.indices[m]
        centroids = self.vertices[indices.long()].mean(dim=1)
        feats = FT.activate_output(camera.camera_center, d, c, gr, s, indices, centroids, self.vertices.detach(),
                                   self.current_sh_deg, self.max_sh_deg)
        return s, feats


def test_render_matches_reference_render(cuda):
    RMB.install_dropin()
    g = np.load(os.path.join(GOLDEN, "ref_render.npz"))
    cam = _Camera(g, "cuda")
    model = _Model(g)
    jitter = torch.tensor(g["jitter"], device="cuda")
    target = torch.tensor(g["target"], device="cuda")
    pkg = RR.render(cam, model, tile_size=16, min_t=0.1, ray_jitter=jitter)
    assert torch.equal(pkg["mask"].cpu(), torch.tensor(g["mask"]))
    err_img = float((pkg["render"].detach().cpu() - torch.tensor(g["render"])).abs().max())
    err_alpha = float((pkg["alpha"].detach().cpu() - torch.tensor(g["alpha"])).abs().max())
    assert err_img <= 1e-4 and err_alpha <= 1e-4, (err_img, err_alpha)
    assert abs(float(pkg["distortion_loss"]) - float(g["distortion_loss"])) <= 1e-5 * abs(float(g["distortion_loss"]))
    assert abs(float(pkg["sh_reg"]) - float(g["sh_reg"])) <= 1e-6 * abs(float(g["sh_reg"]))
    loss = (pkg["render"] - target).abs().mean() + 0.01 * pkg["distortion_loss"] + 0.001 * pkg["sh_reg"]
    assert abs(float(loss) - float(g["loss"])) <= 1e-5 * float(g["loss"])
    loss.backward()
    grads = dict(vertices=model.vertices.grad, density=model.leaves[0].grad, rgb=model.leaves[1].grad,
                 grd=model.leaves[2].grad, sh=model.leaves[3].grad)
    for name, got in grads.items():
        want = torch.tensor(g[f"grad_{name}"], device="cuda")
        assert got is not None, name
        assert _rel(got, want) <= 1e-3, (name, _rel(got, want))
