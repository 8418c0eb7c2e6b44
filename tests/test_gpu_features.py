"""The fused per-tet feature producer against a plain PyTorch fp32
restatement of the reference's activate_output (offset_normalize, the SH
evaluation, softplus), values and gradients."""
import math

import numpy as np
import pytest
import torch

from radiance_meshes_b200 import features as FT
from radiance_meshes_b200 import scenes

pytestmark = pytest.mark.gpu

C0 = 0.28209479177387814


def _sh_basis(d, deg):
    x, y, z = d[:, 0:1], d[:, 1:2], d[:, 2:3]
    out = [-0.4886025119029199 * y, 0.4886025119029199 * z, -0.4886025119029199 * x]
    if deg > 1:
        xx, yy, zz, xy, yz, xz = x * x, y * y, z * z, x * y, y * z, x * z
        out += [1.0925484305920792 * xy, -1.0925484305920792 * yz, 0.31539156525252005 * (2.0 * zz - xx - yy),
                -1.0925484305920792 * xz, 0.5462742152960396 * (xx - yy)]
        if deg > 2:
            out += [-0.5900435899266435 * y * (3 * xx - yy), 2.890611442640554 * xy * z,
                    -0.4570457994644658 * y * (4 * zz - xx - yy), 0.3731763325901154 * z * (2 * zz - 3 * xx - 3 * yy),
                    -0.4570457994644658 * x * (4 * zz - xx - yy), 1.445305721320277 * z * (xx - yy),
                    -0.5900435899266435 * x * (xx - 3 * yy)]
            if deg > 3:
                out += [2.5033429417967046 * xy * (xx - yy), -1.7701307697799304 * yz * (3 * xx - yy),
                        0.9461746957575601 * xy * (7 * zz - 1), -0.6690465435572892 * yz * (7 * zz - 3),
                        0.10578554691520431 * (zz * (35 * zz - 30) + 3), -0.6690465435572892 * xz * (7 * zz - 3),
                        0.47308734787878004 * (xx - yy) * (7 * zz - 1), -1.7701307697799304 * xz * (xx - 3 * yy),
                        0.6258357354491761 * (xx * (xx - 3 * yy) - yy * (3 * xx - yy))]
    return out


def _reference(cam, density, rgb, grd, sh, indices, cc, vertices, deg):
    tets = vertices[indices.long()]
    m = rgb.reshape(-1, 3, 1).min(dim=1, keepdim=True).values  # [T,1,1]
    g = grd.reshape(-1, 1, 3) * m
    r = torch.linalg.norm(tets[:, 0] - cc, dim=-1, keepdim=True).reshape(-1, 1, 1)
    ng = g / r
    off = ((tets.detach()[:, 0] - cc.detach()) * ng.reshape(-1, 3)).sum(-1, keepdim=True)
    c0 = rgb.reshape(-1, 3) + off
    dirs = torch.nn.functional.normalize(tets.mean(dim=1) - cam.reshape(1, 3), dim=1, eps=1e-8)
    col = C0 * ((c0 - 0.5) / C0) + 0.5
    if deg > 0:
        for k, b in enumerate(_sh_basis(dirs, deg)):
            col = col + b * sh[:, k, :]
    base = torch.nn.functional.softplus(col, beta=10)
    return torch.cat([density, base, ng.reshape(-1, 3)], dim=1)


@pytest.mark.parametrize("deg", [0, 1, 3, 4])
def test_activate_output_matches_torch(cuda, deg):
    mesh, view = scenes.workload_gradient_check()
    rng = np.random.default_rng(deg)
    T = len(mesh.indices)
    n_rest = (4 + 1) ** 2 - 1
    dev = "cuda"
    idx = torch.from_numpy(mesh.indices).to(dev)
    t = lambda a: torch.tensor(a, dtype=torch.float32, device=dev, requires_grad=True)
    vertices = t(mesh.vertices)
    density = t(rng.lognormal(0, 1, (T, 1)))
    rgb = t(rng.uniform(0, 1, (T, 3)))
    grd = t(rng.normal(0, 0.1, (T, 3)))
    sh = t(rng.normal(0, 0.2, (T, n_rest, 3)))
    tv = mesh.vertices[mesh.indices].astype(np.float64)
    cc = t((tv.mean(1) + rng.normal(0, 0.05, (T, 3))).astype(np.float32))
    cam = torch.tensor([0.3, 0.4, -2.9], device=dev)
    ref = _reference(cam, density, rgb, grd, sh, idx, cc, vertices, deg)
    out = FT.activate_output(cam, density, rgb, grd, sh, idx, cc, vertices, deg, 4)
    assert out.shape == (T, 7)
    assert torch.allclose(out, ref, rtol=1e-5, atol=1e-5)
    w = torch.randn(T, 7, device=dev, generator=torch.Generator(dev).manual_seed(deg))
    params = [density, rgb, grd, sh, cc, vertices]
    gr = torch.autograd.grad((ref * w).sum(), params, allow_unused=True)
    go = torch.autograd.grad((out * w).sum(), params, allow_unused=True)
    gr = [torch.zeros_like(p) if g is None else g for p, g in zip(params, gr)]  # SH rows unused at degree 0
    go = [torch.zeros_like(p) if g is None else g for p, g in zip(params, go)]
    for name, a, b in zip(["density", "rgb", "grd", "sh", "cc", "vertices"], go, gr):
        if float(b.norm()) == 0.0:
            assert float(a.norm()) == 0.0, name
            continue
        rel = float((a - b).norm() / (b.norm() + 1e-30))
        assert rel < 1e-4, (name, rel)
