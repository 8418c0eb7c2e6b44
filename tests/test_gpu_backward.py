"""Stage (d) backward and the projection adjoint on the GPU against the
oracle's hand-derived adjoint (checked against FP64 central differences in
tests/test_oracle_grad.py).

Two references, per parameter group (vertex positions, density, base RGB,
colour gradient), with the relative L2 error ||g_gpu - g_ref|| / ||g_ref||:
  * the adjoint evaluated in FP32 with the reference's rounding (the
    reference's own backward, restated): <= 1e-4, and every entry within
    1e-3 |g_ref| + 1e-4 max|g_ref|;
  * the adjoint evaluated in FP64 (the exact reference): <= 1e-3, the stated
    gradient tolerance, over every entry (the FP32 restatement itself is within
    6.2e-5 of FP64 on these cases).  Rays are jittered randomly.  At pixel
    centres a ray can graze a tet edge, where the segment length is not
    differentiable and FP32 and FP64 resolve the kink differently (for the
    reference algorithm in FP32 as much as for this kernel), so that case is
    compared with the FP32 restatement only.  Distortion
    gradients are compared with the FP32 restatement only: the reference's
    distortion moments add the full density of every hit tet, however short
    the segment (moment_0_int returns the density,
    alphablend_shader_interp.slang:84-86), so a grazing hit that FP32 counts
    and FP64 does not (or the reverse) changes them by a finite step.
"""
import numpy as np
import pytest
import torch

import golden_util as G
from gpu_util import run_gpu_forward, to_dev
from oracle import oracle as O
from radiance_meshes_b200 import rasterizer as R
from radiance_meshes_b200 import scenes

pytestmark = pytest.mark.gpu

GRAD_TOL = 1e-3


def _groups(gv, gc):
    return {"vertices": gv.ravel(), "density": gc[:, 0], "rgb": gc[:, 1:4].ravel(), "grd": gc[:, 4:7].ravel()}


def _compare(gpu, ref, rel_tol, entry_rtol=None, entry_atol=None, what=""):
    out = {}
    for k in ref:
        a, b = gpu[k].astype(np.float64), ref[k]
        nb = np.linalg.norm(b)
        if nb == 0:
            assert np.abs(a).max() == 0, k
            continue
        rel = np.linalg.norm(a - b) / nb
        out[k] = rel
        assert rel <= rel_tol, f"{what} {k}: relative L2 error {rel:.3e}"
        if entry_rtol is not None:
            bound = entry_rtol * np.abs(b) + entry_atol * np.abs(b).max()
            bad = np.abs(a - b) > bound
            assert not bad.any(), f"{what} {k}: {bad.sum()} entries out of tolerance, worst {np.abs(a - b)[bad].max():.3e}"
    return out


def _run(verts, idx, cv, tcam, jitter, loss, seed=0, check_f64=True, hit_masks=False):
    r = run_gpu_forward(verts, idx, cv, tcam, jitter, hit_masks=hit_masks)
    img = r["img"].cpu().numpy()
    H, W = img.shape[:2]
    rng = np.random.default_rng(seed)
    if loss == "l1":
        target = rng.uniform(size=(H, W, 3)).astype(np.float32)
        gimg = np.zeros((H, W, 4), np.float32)
        gimg[..., :3] = np.sign(img[..., :3] - target) / (H * W * 3)
        gdist = np.zeros((H, W, 5), np.float32)
    else:
        gimg = rng.normal(size=(H, W, 4)).astype(np.float32)
        gdist = (rng.normal(size=(H, W, 5)) * 1e-3).astype(np.float32)
        if loss == "linear_nodist":
            gdist[:] = 0.0
    L = r["lists"]
    gv, gc = R.blend_bwd(L.sorted_ids, L.ranges, r["i"], r["v"], r["c"], r["j"], r["cam"], r["img"], r["dist"],
                         r["nc"], to_dev(gimg), to_dev(gdist), r["records"], reuse_records=True,
                         hit_masks=hit_masks)
    torch.cuda.synchronize()
    lists = dict(cam=r["cam"], sorted_ids=L.sorted_ids.cpu().numpy(), ranges=L.ranges.cpu().numpy())
    nc = r["nc"].cpu().numpy()[..., 0]
    gpu = _groups(gv.cpu().numpy(), gc.cpu().numpy())
    img32, dist32, nc32 = O.blend_fwd_f32(lists, idx, verts, cv, jitter)
    assert np.array_equal(nc32, nc)
    fgv, fgc = O.blend_bwd(lists, idx, verts, cv, jitter, img32, dist32, nc, gimg, gdist, "f32")
    out = {"f32": _compare(gpu, _groups(fgv, fgc), 1e-4, 1e-3, 1e-4, "vs fp32 restatement")}
    if check_f64:
        v64, c64 = verts.astype(np.float64), cv.astype(np.float64)
        img64, dist64, _, _, _ = O.blend_fwd_f64(lists, idx, v64, c64, jitter, cut=nc)
        rgv, rgc = O.blend_bwd(lists, idx, v64, c64, jitter, img64, dist64, nc, gimg.astype(np.float64),
                               gdist.astype(np.float64), "f64")
        out["f64"] = _compare(gpu, _groups(rgv, rgc), GRAD_TOL, what="vs fp64")
    return out


@pytest.mark.parametrize("loss", ["l1", "linear_nodist", "linear"])
def test_backward_gradient_check_workload(cuda, loss):
    mesh, view = scenes.workload_gradient_check()
    jitter = np.random.default_rng(1).uniform(0, 1, (view.height, view.width, 2)).astype(np.float32)
    rel = _run(mesh.vertices, mesh.indices, mesh.cell_values, view.tcam(), jitter, loss,
               check_f64=(loss != "linear"))
    print("relative L2 errors", rel)


@pytest.mark.parametrize("name", [n for n in G.names() if not n.startswith("ball")])
def test_backward_golden_scenes(cuda, name):
    z, tcam = G.load(name)
    _run(z["vertices"], z["indices"], z["cell_values"], tcam, z["jitter"], "linear", seed=3, check_f64=False)
    _run(z["vertices"], z["indices"], z["cell_values"], tcam, z["jitter"], "linear_nodist", seed=3)


@pytest.mark.parametrize("tile", [4, 8, 32])
def test_backward_tile_sizes(cuda, tile):
    mesh, view = scenes.workload_gradient_check(tile)
    jitter = np.random.default_rng(tile).uniform(0, 1, (view.height, view.width, 2)).astype(np.float32)
    _run(mesh.vertices, mesh.indices, mesh.cell_values, view.tcam(tile_size=tile), jitter, "linear", seed=tile,
         check_f64=False)
    _run(mesh.vertices, mesh.indices, mesh.cell_values, view.tcam(tile_size=tile), jitter, "linear_nodist",
         seed=tile)


def test_backward_pixel_centres_vs_fp32_restatement(cuda):
    """Pixel-centre rays (jitter 0.5) include edge-grazing rays: compared with
    the FP32 restatement only (see the module docstring)."""
    mesh, view = scenes.workload_gradient_check(4)
    jitter = np.full((view.height, view.width, 2), 0.5, np.float32)
    _run(mesh.vertices, mesh.indices, mesh.cell_values, view.tcam(tile_size=4), jitter, "linear", seed=4,
         check_f64=False)


def test_project_backward(cuda):
    mesh, view = scenes.workload_gradient_check()
    tcam = view.tcam()
    cam = R.camera(tcam)
    v, i = to_dev(mesh.vertices), to_dev(mesh.indices)
    tiles, rect, vs, cc = R.project_fwd(i, v, cam)
    rng = np.random.default_rng(9)
    T = len(mesh.indices)
    gvs = rng.normal(size=(T, 3)).astype(np.float32)
    gcc = rng.normal(size=(T, 3)).astype(np.float32)
    gv = R.project_bwd(i, v, cam, tiles, to_dev(gvs), to_dev(gcc)).cpu().numpy()
    ref = O.project_bwd(mesh.indices, mesh.vertices, cam, tiles.cpu().numpy(), gvs, gcc)
    rel = np.linalg.norm(gv - ref) / np.linalg.norm(ref)
    assert rel <= 1e-5, rel


@pytest.mark.parametrize("route", ["all_dense", "all_pair"])
@pytest.mark.parametrize("tile", [4, 16])
def test_backward_each_kernel_path(cuda, route, tile):
    """Every tile through the one-thread-per-pixel backward, or every tile
    through the pair-parallel backward (packed hits)."""
    from radiance_meshes_b200 import _capi as C

    shift = 15 if route == "all_dense" else 1
    flags = (shift << C.RM_BLEND_HEAVY_SHIFT) | (2 << C.RM_BLEND_PAIR_CTAS_SHIFT)
    old = R.blend_tuning()
    R.set_blend_tuning(flags, flags)
    try:
        mesh, view = scenes.workload_gradient_check(tile)
        jitter = np.random.default_rng(tile + 7).uniform(0, 1, (view.height, view.width, 2)).astype(np.float32)
        _run(mesh.vertices, mesh.indices, mesh.cell_values, view.tcam(tile_size=tile), jitter, "linear",
             seed=tile, check_f64=False)
        _run(mesh.vertices, mesh.indices, mesh.cell_values, view.tcam(tile_size=tile), jitter, "linear_nodist",
             seed=tile)
    finally:
        R.set_blend_tuning(*old)


@pytest.mark.parametrize("fwd_route", ["all_pair", "split"])
@pytest.mark.parametrize("tile", [8, 16, 32])
def test_backward_with_hit_masks(cuda, fwd_route, tile):
    """The backward that revisits only the forward's hits (RM_BLEND_HIT_MASKS)
    matches the FP32 restatement like the full backward, whichever forward
    kernel recorded the masks; the forward's outputs do not change."""
    from radiance_meshes_b200 import _capi as C

    fwd_flags = 0 if fwd_route == "all_pair" else (2 << C.RM_BLEND_HEAVY_SHIFT) | (2 << C.RM_BLEND_PAIR_CTAS_SHIFT)
    old = R.blend_tuning()
    R.set_blend_tuning(fwd_flags, 0)
    try:
        mesh, view = scenes.workload_gradient_check(tile)
        jitter = np.random.default_rng(tile + 3).uniform(0, 1, (view.height, view.width, 2)).astype(np.float32)
        a = run_gpu_forward(mesh.vertices, mesh.indices, mesh.cell_values, view.tcam(tile_size=tile), jitter)
        b = run_gpu_forward(mesh.vertices, mesh.indices, mesh.cell_values, view.tcam(tile_size=tile), jitter,
                            hit_masks=True)
        assert torch.equal(a["img"], b["img"]) and torch.equal(a["nc"], b["nc"])
        for loss in ("linear", "l1"):
            _run(mesh.vertices, mesh.indices, mesh.cell_values, view.tcam(tile_size=tile), jitter, loss,
                 seed=tile, check_f64=False, hit_masks=True)
    finally:
        R.set_blend_tuning(*old)


def test_hit_masks_invalidated_by_a_forward_without_them(cuda):
    """A forward without RM_BLEND_HIT_MASKS on a workspace that holds masks
    from an earlier frame marks them invalid: a masked backward then tests
    every entry and still matches."""
    mesh, view = scenes.workload_gradient_check(8)
    tcam = view.tcam(tile_size=8)
    jitter = np.full((view.height, view.width, 2), 0.5, np.float32)
    r = run_gpu_forward(mesh.vertices, mesh.indices, mesh.cell_values, tcam, jitter, hit_masks=True)
    L = r["lists"]
    cv2 = r["c"] * 0.5  # another frame: different densities, same lists
    img2, dist2, nc2, _ = R.blend_fwd(L.sorted_ids, L.ranges, r["i"], r["v"], cv2, r["j"], r["cam"],
                                      tiles_touched=r["tiles"], records=r["records"], hit_masks=False)
    g = torch.randn_like(img2)
    gv_m, gc_m = R.blend_bwd(L.sorted_ids, L.ranges, r["i"], r["v"], cv2, r["j"], r["cam"], img2, dist2, nc2, g,
                             None, r["records"], reuse_records=True, hit_masks=True)
    gv, gc = R.blend_bwd(L.sorted_ids, L.ranges, r["i"], r["v"], cv2, r["j"], r["cam"], img2, dist2, nc2, g, None,
                         r["records"], reuse_records=True, hit_masks=False)
    torch.cuda.synchronize()
    assert float((gv_m - gv).norm() / gv.norm()) < 1e-5
    assert float((gc_m - gc).norm() / gc.norm()) < 1e-5
