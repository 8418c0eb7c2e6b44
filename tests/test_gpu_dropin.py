"""The reference-facing API: delaunay_rasterization.internal.* drop-in modules
and render(), with autograd, on the GPU."""
import numpy as np
import pytest
import torch

import radiance_meshes_b200 as RMB
from gpu_util import run_gpu_forward, to_dev
from oracle import oracle as O
from radiance_meshes_b200 import render as RR
from radiance_meshes_b200 import scenes

pytestmark = pytest.mark.gpu


def test_dropin_forward_backward(cuda):
    RMB.install_dropin()
    from delaunay_rasterization.internal.alphablend_tiled_slang_interp import AlphaBlendTiledRender
    from delaunay_rasterization.internal.render_grid import RenderGrid
    from delaunay_rasterization.internal.tile_shader_slang import vertex_and_tile_shader

    mesh, view = scenes.workload_gradient_check()
    tcam = view.tcam(device="cuda")
    grid = RenderGrid(view.height, view.width, tile_width=16, tile_height=16)
    verts = to_dev(mesh.vertices).requires_grad_(True)
    cv = to_dev(mesh.cell_values).requires_grad_(True)
    idx = to_dev(mesh.indices)
    jitter = torch.full((view.height, view.width, 2), 0.5, device="cuda")
    sorted_ids, ranges, vs, cc, mask, rect = vertex_and_tile_shader(idx, verts, tcam, grid)
    assert sorted_ids.dtype == torch.int32 and ranges.shape == (grid.grid_height * grid.grid_width, 2)
    assert vs.shape == (len(mesh.indices), 3) and mask.dtype == torch.bool and rect.shape[1] == 4
    img, dist, alive = AlphaBlendTiledRender.apply(sorted_ids, ranges, idx, verts, cv, grid, tcam, jitter)
    assert img.shape == (view.height, view.width, 4) and dist.shape == (view.height, view.width, 5)
    assert alive.dtype == torch.bool and not alive.any()
    # same result as the stage-level path
    ref = run_gpu_forward(mesh.vertices, mesh.indices, mesh.cell_values, view.tcam(),
                          np.full((view.height, view.width, 2), 0.5, np.float32))
    assert torch.equal(img, ref["img"]) and torch.equal(dist, ref["dist"])
    # gradients flow into vertices (blend + circumcenter path) and cell values
    loss = img[..., :3].sum() + 0.1 * cc.sum() + 1e-3 * vs[:, 2].sum()
    loss.backward()
    assert verts.grad is not None and torch.isfinite(verts.grad).all() and verts.grad.abs().sum() > 0
    assert cv.grad is not None and torch.isfinite(cv.grad).all() and cv.grad.abs().sum() > 0


class _Cam:
    def __init__(self, view):
        self.view = view
        self.image_height = view.height
        self.image_width = view.width
        self.gt_alpha_mask = torch.ones((1, view.height, view.width))

    def to_dict(self, device):
        t = self.view.tcam(device=device)
        keep = ("world_view_transform", "cam_pos", "K", "image_height", "image_width", "fovy", "fovx",
                "distortion_params", "camera_type")
        return {k: t[k] for k in keep}


class _Model:
    def __init__(self, mesh):
        self.vertices = to_dev(mesh.vertices).requires_grad_(True)
        self.indices = to_dev(mesh.indices)
        self.device = "cuda"


def test_render_api(cuda):
    mesh, view = scenes.workload_plain_forward()
    model = _Model(mesh)
    cv = to_dev(mesh.cell_values).requires_grad_(True)
    pkg = RR.render(_Cam(view), model, cell_values=cv, tile_size=16, min_t=0.1)
    assert pkg["render"].shape == (3, view.height, view.width)
    assert pkg["alpha"].shape == (view.height, view.width)
    L = O.rasterize_lists(mesh.indices, mesh.vertices, view.tcam())
    img, _, _ = O.blend_fwd_f32(L, mesh.indices, mesh.vertices, mesh.cell_values,
                                np.full((view.height, view.width, 2), 0.5, np.float32))
    assert np.abs(pkg["render"].detach().permute(1, 2, 0).cpu().numpy() - img[..., :3]).max() <= 1e-4
    (pkg["render"].mean() + pkg["distortion_loss"]).backward()
    assert torch.isfinite(cv.grad).all() and torch.isfinite(model.vertices.grad).all()


def test_bad_camera_raises(cuda):
    RMB.install_dropin()
    from delaunay_rasterization.internal.render_grid import RenderGrid
    from delaunay_rasterization.internal.tile_shader_slang import vertex_and_tile_shader

    mesh, view = scenes.workload_gradient_check()
    tcam = view.tcam(device="cuda")
    tcam["camera_type"] = 2  # neither perspective nor fisheye
    with pytest.raises(ValueError):
        vertex_and_tile_shader(to_dev(mesh.indices), to_dev(mesh.vertices), tcam,
                               RenderGrid(view.height, view.width, 16, 16))


def _dropin_step(mesh, view, jitter, fine, tile=16, cam_shift=None):
    RMB.install_dropin()
    from delaunay_rasterization.internal.alphablend_tiled_slang_interp import AlphaBlendTiledRender
    from delaunay_rasterization.internal.render_grid import RenderGrid
    from delaunay_rasterization.internal.tile_shader_slang import vertex_and_tile_shader
    from radiance_meshes_b200 import rasterizer as R

    R.use_fine_lists(fine)
    try:
        tcam = view.tcam(device="cuda", tile_size=tile)
        if cam_shift is not None:  # rays from a point off the projection centre
            tcam["cam_pos"] = tcam["cam_pos"] + torch.tensor(cam_shift, device="cuda")
        grid = RenderGrid(view.height, view.width, tile_width=tile, tile_height=tile)
        verts = to_dev(mesh.vertices).requires_grad_(True)
        cv = to_dev(mesh.cell_values).requires_grad_(True)
        idx = to_dev(mesh.indices)
        sorted_ids, ranges, vs, cc, mask, rect = vertex_and_tile_shader(idx, verts, tcam, grid)
        assert (getattr(sorted_ids, "rm_fine", None) is not None) == fine
        img, dist, _ = AlphaBlendTiledRender.apply(sorted_ids, ranges, idx, verts, cv, grid, tcam, jitter)
        g = torch.Generator(device="cuda").manual_seed(2)
        w = torch.randn(img.shape, device="cuda", generator=g)
        wd = torch.randn(dist.shape, device="cuda", generator=g) * 0.01
        ((img * w).sum() + (dist * wd).sum()).backward()
        torch.cuda.synchronize()
        return sorted_ids, ranges, img.detach(), dist.detach(), verts.grad, cv.grad
    finally:
        R.use_fine_lists(True)


@pytest.mark.parametrize("scene,tile,jit", [("plain", 16, "unit"), ("mixture", 16, "unit"), ("mixture", 32, "unit"),
                                            ("mixture", 16, "half"), ("mixture", 16, "wide"),
                                            ("plain", 32, "wide"), ("mixture", 16, "offcentre")])
def test_fine_lists_give_the_coarse_frame(cuda, scene, tile, jit):
    """Blending over the 8x8-pixel lists reproduces the blend over the
    caller's 16x16 / 32x32 lists for any ray jitter (uniform in [0, 1) as in
    training, the constant 0.5 of render(), and a jitter that reaches up to
    1.5 pixels past the pixel): image and distortion bit for bit, gradients up
    to FP32 summation order; the lists returned to the caller are the coarse
    ones."""
    if scene == "plain":
        mesh, view = scenes.workload_plain_forward()
    else:
        mesh, view = scenes.workload_training_step(n_points=20000, seed=2, height=420, width=649)
    rng = np.random.default_rng(4)
    shape = (view.height, view.width, 2)
    cam_shift = None
    if jit == "offcentre":  # rays start 2.3e-5 away from the projection centre
        j = rng.uniform(0, 1, shape)
        cam_shift = [2e-5, -1e-5, 5e-6]
    elif jit == "unit":
        j = rng.uniform(0, 1, shape)
    elif jit == "half":
        j = np.full(shape, 0.5)
    else:
        j = rng.uniform(-1.5, 2.5, shape)
    jitter = torch.from_numpy(j.astype(np.float32)).cuda()
    ids_c, rg_c, img_c, dist_c, gv_c, gc_c = _dropin_step(mesh, view, jitter, False, tile, cam_shift)
    ids_f, rg_f, img_f, dist_f, gv_f, gc_f = _dropin_step(mesh, view, jitter, True, tile, cam_shift)
    assert torch.equal(ids_c, ids_f) and torch.equal(rg_c, rg_f)
    assert torch.equal(img_c.view(torch.int32), img_f.view(torch.int32))
    assert torch.equal(dist_c.view(torch.int32), dist_f.view(torch.int32))
    fine = ids_f.rm_fine.lists
    assert fine.n_pairs > ids_c.shape[0]
    assert fine.sorted_ids.shape[0] >= fine.n_pairs
    for a, b in ((gv_f, gv_c), (gc_f, gc_c)):
        assert float((a - b).norm() / b.norm()) < 1e-5


def test_dropin_frames_of_changing_size(cuda):
    """Frames whose pair counts grow and shrink: the lists are built on
    buffers sized from the previous frame (all queued before the count is
    read), a frame that outgrows them is built again at its exact size, and
    every frame's lists, image and distortion equal those of a first frame
    (buffers of exactly P); no capacity bit is left for the next readback."""
    from radiance_meshes_b200 import rasterizer as R

    small = scenes.workload_plain_forward()
    big = scenes.workload_training_step(n_points=20000, seed=2, height=420, width=649)
    refs = {}
    for name, (mesh, view) in (("small", small), ("big", big)):
        R._PAIR_GUESS.clear()  # a first frame: the count read, then exactly P
        jitter = torch.full((view.height, view.width, 2), 0.5, device="cuda")
        refs[name] = _dropin_step(mesh, view, jitter, True)[:4]
    for name in ("small", "big", "big", "small", "big"):
        mesh, view = small if name == "small" else big
        jitter = torch.full((view.height, view.width, 2), 0.5, device="cuda")
        got = _dropin_step(mesh, view, jitter, True)[:4]
        ids, rg, img, dist = refs[name]
        assert torch.equal(got[0], ids) and torch.equal(got[1], rg)
        assert torch.equal(got[2].view(torch.int32), img.view(torch.int32))
        assert torch.equal(got[3].view(torch.int32), dist.view(torch.int32))
    n_small = refs["small"][0].shape[0]
    assert refs["big"][0].shape[0] > n_small + n_small // 4 + 4096  # big after small takes the rebuild
    R.check_status(len(big[0].indices), torch.device("cuda"))
