"""Golden vectors computed by the reference's own Python code.

Run in a container that holds the reference tree (it is read here and
nowhere else; the fixtures travel with the tests):

    python tests/golden/make_ref_golden.py [--reference /path/to/reference]

Writes, next to this script:

  ref_activate_output.npz  the reference's activate_output
      (utils/model_util.py:93-105, with offset_normalize :82-91 and eval_sh
      utils/eval_sh_py.py:138-200), imported unchanged and run in fp32 on the
      CPU, at SH degrees 0, 1, 2, 3 (max degree 3): inputs, features and the
      gradients of sum(features * w) for a fixed random w.
  ref_render.npz  the reference's render() (utils/train_util.py:15-77) with its
      own Camera (data/camera.py:16-91), weigh_degree and activate_output, on
      the 2,000-point gradient-check mesh (128x128, SH degree 1, random jitter
      and alpha mask), then L1 + distortion + SH losses and backward.  The
      Slang rasterizer it calls cannot run here, so the two drop-in modules
      are stood in by the oracle's FP32 restatement (oracle/, forward and
      adjoint); everything else is the reference's code.  Saved: the camera
      record to_dict() produced, the model's raw outputs, render_pkg and the
      gradients of the loss.

Modules the imported files name but this container lacks are stubbed:
icecream (a debug printer) and matplotlib (a colour map at import time).
"""
from __future__ import annotations

import argparse
import os
import sys
import types

import numpy as np
import torch

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def _stub_modules():
    ic = types.ModuleType("icecream")
    ic.ic = lambda *a, **k: (a[0] if len(a) == 1 else a)
    sys.modules.setdefault("icecream", ic)
    mpl = types.ModuleType("matplotlib")
    plt = types.ModuleType("matplotlib.pyplot")
    plt.get_cmap = lambda name: None
    mpl.pyplot = plt
    sys.modules.setdefault("matplotlib", mpl)
    sys.modules.setdefault("matplotlib.pyplot", plt)


def _install_oracle_rasterizer(reference):
    """delaunay_rasterization.internal.{tile_shader_slang,
    alphablend_tiled_slang_interp} as CPU modules over the oracle, so that the
    reference's render() imports and runs here; render_grid and util are the
    reference's own files."""
    from oracle import oracle as O

    sys.path.insert(0, reference)
    import delaunay_rasterization.internal.render_grid  # noqa: F401  (the reference's file)

    def vertex_and_tile_shader(indices, vertices, tcam, render_grid):
        L = O.rasterize_lists(indices.numpy(), vertices.detach().numpy(), tcam)
        return (torch.from_numpy(L["sorted_ids"]), torch.from_numpy(L["ranges"]), torch.from_numpy(L["vs"]),
                torch.from_numpy(L["circumcenter"]), torch.from_numpy(L["tiles_touched"] > 0),
                torch.from_numpy(L["rect"]))

    class AlphaBlendTiledRender(torch.autograd.Function):
        @staticmethod
        def forward(ctx, sorted_tetra_idx, tile_ranges, indices, vertices, tet_density, render_grid, tcam,
                    ray_jitter, device="cuda"):
            L = dict(cam=O.camstruct(tcam), sorted_ids=sorted_tetra_idx.numpy(), ranges=tile_ranges.numpy())
            args = (L, indices.numpy(), vertices.detach().numpy(), tet_density.detach().numpy(),
                    ray_jitter.numpy())
            img, dist, nc = O.blend_fwd_f32(*args)
            ctx.args, ctx.out = args, (img, dist, nc)
            return (torch.from_numpy(img), torch.from_numpy(dist),
                    torch.zeros(indices.shape[0], dtype=torch.bool))

        @staticmethod
        def backward(ctx, g_img, g_dist, _):
            img, dist, nc = ctx.out
            gv, gc = O.blend_bwd(*ctx.args, img, dist, nc, g_img.numpy(), g_dist.numpy(), precision="f32")
            return (None, None, None, torch.from_numpy(gv).float(), torch.from_numpy(gc).float(), None, None,
                    None, None)

    ts = types.ModuleType("delaunay_rasterization.internal.tile_shader_slang")
    ts.vertex_and_tile_shader = vertex_and_tile_shader
    ab = types.ModuleType("delaunay_rasterization.internal.alphablend_tiled_slang_interp")
    ab.AlphaBlendTiledRender = AlphaBlendTiledRender
    sys.modules[ts.__name__] = ts
    sys.modules[ab.__name__] = ab


def _leaves(T, rng, sh_rows=15):
    density = np.exp(rng.normal(0.0, 2.0, size=(T, 1))).astype(np.float32)
    rgb = rng.uniform(-1.0, 1.0, size=(T, 3)).astype(np.float32)
    grd = rng.normal(0.0, 0.1, size=(T, 3)).astype(np.float32)
    sh = rng.normal(0.0, 0.3, size=(T, sh_rows, 3)).astype(np.float32)
    return density, rgb, grd, sh


def make_activate_output(activate_output, out_path):
    from radiance_meshes_b200 import scenes

    mesh, view = scenes.workload_gradient_check()
    rng = np.random.default_rng(21)
    T = 3000
    idx = mesh.indices[rng.choice(len(mesh.indices), T, replace=False)]
    verts = mesh.vertices
    tets = verts[idx]
    cc = (tets.mean(axis=1) + rng.normal(0.0, 0.02, size=(T, 3))).astype(np.float32)
    density, rgb, grd, sh = _leaves(T, rng)
    cam = np.asarray(view.cam_pos, np.float32)
    w = rng.normal(size=(T, 7)).astype(np.float32)
    out = dict(indices=idx.astype(np.int32), vertices=verts.astype(np.float32), circumcenters=cc,
               density=density, rgb=rgb, grd=grd, sh=sh, camera_center=cam, w=w)
    for deg in (0, 1, 2, 3):
        ts = [torch.from_numpy(x.copy()).requires_grad_(True) for x in (density, rgb, grd, sh, cc, verts)]
        feats = activate_output(torch.from_numpy(cam), ts[0], ts[1], ts[2], ts[3], torch.from_numpy(idx).long(),
                                ts[4], ts[5], deg, 3)
        (feats * torch.from_numpy(w)).sum().backward()
        out[f"features_{deg}"] = feats.detach().numpy()
        for name, t in zip(("density", "rgb", "grd", "sh", "circumcenters", "vertices"), ts):
            out[f"grad_{name}_{deg}"] = (t.grad if t.grad is not None else torch.zeros_like(t)).numpy()
    np.savez_compressed(out_path, **out)
    print("wrote", out_path)


def make_render(reference, out_path):
    from data.camera import Camera
    from utils.eval_sh_py import weigh_degree  # noqa: F401  (render() imports it)
    from utils.model_util import activate_output
    from utils.train_util import render

    from radiance_meshes_b200 import scenes

    mesh, view = scenes.workload_gradient_check()
    H, W = view.height, view.width
    M = np.asarray(view.world_view, np.float64).reshape(4, 4)
    rng = np.random.default_rng(31)
    image = torch.from_numpy(rng.uniform(size=(3, H, W)).astype(np.float32))
    alpha_mask = torch.from_numpy((rng.uniform(size=(1, H, W)) > 0.1).astype(np.float32))
    cam = Camera(0, M[:3, :3].T.copy(), M[:3, 3].copy(), float(view.fovx), float(view.fovy), image,
                 gt_alpha_mask=alpha_mask, data_device="cpu")
    tcam_dict = cam.to_dict("cpu")
    T = len(mesh.indices)
    density, rgb, grd, sh = _leaves(T, rng, sh_rows=3)
    density[rng.uniform(size=T) < 0.3] = 1e-4

    class Model:
        """The reference model's get_cell_values (models/ingp_color.py:361-387)
        with the hashgrid backbone (out of scope) replaced by fixed raw
        per-tet outputs."""
        device = torch.device("cpu")
        feature_dim = 7
        mask_values = True
        max_sh_deg = 1
        current_sh_deg = 1

        def __init__(self):
            self.vertices = torch.from_numpy(mesh.vertices.copy()).requires_grad_(True)
            self.indices = torch.from_numpy(mesh.indices.copy())
            self.leaves = [torch.from_numpy(x.copy()).requires_grad_(True) for x in (density, rgb, grd, sh)]

        def get_cell_values(self, camera, mask=None, all_circumcenters=None):
            m = mask if mask is not None else torch.ones(T, dtype=torch.bool)
            d, c, g, s = (x[m] for x in self.leaves)
            indices = self.indices[m]
            centroids = self.vertices[indices].mean(dim=1)
            feats = activate_output(camera.camera_center, d, c, g, s, indices, centroids, self.vertices.detach(),
                                    self.current_sh_deg, self.max_sh_deg)
            return s, feats

    model = Model()
    jitter = torch.from_numpy(rng.uniform(size=(H, W, 2)).astype(np.float32))
    target = torch.from_numpy(rng.uniform(size=(3, H, W)).astype(np.float32))
    pkg = render(cam, model, tile_size=16, min_t=0.1, ray_jitter=jitter)
    loss = (pkg["render"] - target).abs().mean() + 0.01 * pkg["distortion_loss"] + 0.001 * pkg["sh_reg"]
    loss.backward()
    out = dict(indices=mesh.indices.astype(np.int32), vertices=mesh.vertices.astype(np.float32),
               density=density, rgb=rgb, grd=grd, sh=sh, jitter=jitter.numpy(), target=target.numpy(),
               gt_alpha_mask=alpha_mask.numpy(), camera_center=cam.camera_center.numpy(),
               render=pkg["render"].detach().numpy(), alpha=pkg["alpha"].detach().numpy(),
               distortion_loss=float(pkg["distortion_loss"]), mask=pkg["mask"].numpy(),
               sh_reg=float(pkg["sh_reg"]), loss=float(loss),
               grad_vertices=model.vertices.grad.numpy(),
               **{f"grad_{n}": t.grad.numpy() for n, t in zip(("density", "rgb", "grd", "sh"), model.leaves)})
    for k, v in tcam_dict.items():
        out[f"tcam_{k}"] = v.numpy() if isinstance(v, torch.Tensor) else np.asarray(v)
    np.savez_compressed(out_path, **out)
    print("wrote", out_path, "loss", float(loss))


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", default=os.environ.get("RM_REFERENCE_TREE", "/root/reference"))
    a = ap.parse_args(argv)
    torch.manual_seed(0)
    _stub_modules()
    _install_oracle_rasterizer(a.reference)
    from utils.model_util import activate_output

    make_activate_output(activate_output, os.path.join(HERE, "ref_activate_output.npz"))
    make_render(a.reference, os.path.join(HERE, "ref_render.npz"))


if __name__ == "__main__":
    main()
