"""Batched multi-view path against the single-camera path, view by view.

Every stage of a batch must reproduce the single-camera calls: projection
outputs, the per-tile sorted lists, and the forward image / log T /
distortion / n_contributors bit for bit; the backward gradients equal the
sum over views of the single-camera gradients up to FP32 summation order.
"""
import numpy as np
import pytest
import torch

from radiance_meshes_b200 import batch as B
from radiance_meshes_b200 import rasterizer as R
from radiance_meshes_b200 import scenes
from radiance_meshes_b200.camera import tcam_to_struct

pytestmark = pytest.mark.gpu


def _scene(tile=16):
    mesh, _ = scenes.workload_gradient_check()
    res = [(128, 128), (96, 160), (48, 64), (77, 131)]
    views = scenes.ring_views(len(res), res, radius=2.9, height_offset=0.4, tile_size=tile)
    cams = [tcam_to_struct(v.tcam()) for v in views]
    return mesh, views, cams


def _dev(mesh):
    return (torch.from_numpy(mesh.indices).cuda(), torch.from_numpy(mesh.vertices).cuda(),
            torch.from_numpy(mesh.cell_values).cuda())


def _jitter(vb, seed=5):
    rng = np.random.default_rng(seed)
    return torch.from_numpy(rng.uniform(0, 1, (vb.n_pixels, 2)).astype(np.float32)).cuda()


def _single(i, v, c, cam, jit):
    tiles, rect, vs, cc = R.project_fwd(i, v, cam)
    lists = R.build_tile_lists(tiles, rect, vs, cam, keep_debug=True)
    img, dist, nc, recs = R.blend_fwd(lists.sorted_ids, lists.ranges, i, v, c, jit, cam, tiles_touched=tiles)
    return dict(tiles=tiles, rect=rect, vs=vs, cc=cc, lists=lists, img=img, dist=dist, nc=nc, recs=recs)


@pytest.mark.parametrize("tile", [8, 16])
def test_batch_forward_matches_single_views(cuda, tile):
    mesh, views, cams = _scene(tile)
    i, v, c = _dev(mesh)
    vb = B.ViewBatch(cams)
    jit = _jitter(vb)
    br = B.BatchedRasterizer(i, v, c, vb, jitter=jit)
    br.forward()
    br.check()
    torch.cuda.synchronize()
    T = len(mesh.indices)
    any_ref = torch.zeros(T, dtype=torch.int32, device="cuda")
    per = vb.split(jit)
    for k, cam in enumerate(cams):
        ref = _single(i, v, c, cam, per[k].contiguous())
        sl = slice(k * T, (k + 1) * T)
        assert torch.equal(br.tiles[sl], ref["tiles"])
        vis = ref["tiles"] > 0  # rows without tiles are not written by the batched projection
        assert torch.equal(br.rect[sl][vis], ref["rect"][vis])
        assert torch.equal(br.depth[sl][vis].view(torch.int32), ref["vs"][vis, 2].contiguous().view(torch.int32))
        any_ref += ref["tiles"]
        # per-tile lists: the batch's global tile tb + t holds the single view's tile t
        G = cam.grid_width * cam.grid_height
        tb = vb.tile_base[k]
        rg_b = br.ranges[tb:tb + G].cpu().numpy()
        rg_s = ref["lists"].ranges.cpu().numpy()
        ids_b = br.sorted_ids.cpu().numpy()
        ids_s = ref["lists"].sorted_ids.cpu().numpy()
        assert np.array_equal(rg_b[:, 1] - rg_b[:, 0], rg_s[:, 1] - rg_s[:, 0])
        for t in np.nonzero(rg_s[:, 1] > rg_s[:, 0])[0]:
            assert np.array_equal(ids_b[rg_b[t, 0]:rg_b[t, 1]], ids_s[rg_s[t, 0]:rg_s[t, 1]])
        img_b, dist_b, nc_b = br.images()[k]
        assert torch.equal(img_b.view(torch.int32), ref["img"].view(torch.int32))
        assert torch.equal(dist_b.view(torch.int32), ref["dist"].view(torch.int32))
        assert torch.equal(nc_b, ref["nc"])
    assert torch.equal(br.tiles_any, any_ref)
    assert int(br.total.item()) == int(br.tiles.sum().item())


def test_batch_backward_is_sum_of_single_views(cuda):
    mesh, views, cams = _scene(16)
    i, v, c = _dev(mesh)
    vb = B.ViewBatch(cams)
    jit = _jitter(vb)
    rng = np.random.default_rng(9)
    gimg = torch.from_numpy(rng.normal(size=(vb.n_pixels, 4)).astype(np.float32)).cuda()
    gdist = torch.from_numpy(rng.normal(size=(vb.n_pixels, 5)).astype(np.float32) * 0.1).cuda()
    br = B.BatchedRasterizer(i, v, c, vb, jitter=jit)
    br.forward()
    gv_b, gc_b = br.backward(gimg, gdist)
    gv_s = torch.zeros_like(v)
    gc_s = torch.zeros_like(c)
    pj, pg, pd = vb.split(jit), vb.split(gimg), vb.split(gdist)
    for k, cam in enumerate(cams):
        ref = _single(i, v, c, cam, pj[k].contiguous())
        R.blend_bwd(ref["lists"].sorted_ids, ref["lists"].ranges, i, v, c, pj[k].contiguous(), cam, ref["img"],
                    ref["dist"], ref["nc"], pg[k].contiguous(), pd[k].contiguous(), ref["recs"],
                    tiles_touched=ref["tiles"], grad_vertices=gv_s, grad_cell_values=gc_s)
    torch.cuda.synchronize()
    for a, b in ((gv_b, gv_s), (gc_b, gc_s)):
        rel = float((a - b).norm() / b.norm())
        assert rel < 1e-5, rel
        assert torch.allclose(a, b, rtol=1e-4, atol=1e-5 * float(b.abs().max()))


def test_graph_replay_matches_eager(cuda):
    mesh, views, cams = _scene(16)
    i, v, c = _dev(mesh)
    vb = B.ViewBatch(cams)
    br = B.BatchedRasterizer(i, v, c, vb)
    target = torch.rand(vb.n_pixels, 3, device="cuda", generator=torch.Generator("cuda").manual_seed(3))
    step = B.L1Step(br, target)
    loss_e = float(step.run())
    img_e = br.img.clone()
    gv_e, gc_e = br.grad_vertices.clone(), br.grad_cell_values.clone()
    step.capture()
    for _ in range(2):
        br.img.zero_()
        loss_g = float(step.run())
        torch.cuda.synchronize()
        assert torch.equal(br.img.view(torch.int32), img_e.view(torch.int32))
        assert abs(loss_g - loss_e) <= 1e-6 * abs(loss_e)
        assert float((br.grad_vertices - gv_e).norm() / gv_e.norm()) < 1e-5
        assert float((br.grad_cell_values - gc_e).norm() / gc_e.norm()) < 1e-5
    # the graph reads the parameters in place: a new cell-value tensor content renders anew
    c.mul_(0.5)
    step.run()
    torch.cuda.synchronize()
    br2 = B.BatchedRasterizer(i, v, c, vb)
    br2.forward()
    torch.cuda.synchronize()
    assert torch.equal(br.img.view(torch.int32), br2.img.view(torch.int32))


def test_capacity_overflow_is_reported_and_recovers(cuda):
    mesh, views, cams = _scene(16)
    i, v, c = _dev(mesh)
    vb = B.ViewBatch(cams)
    full = B.BatchedRasterizer(i, v, c, vb)
    full.forward()
    P = int(full.total.item())
    small = B.BatchedRasterizer(i, v, c, vb, capacity=P // 3)
    small.forward()
    with pytest.raises(RuntimeError, match="capacity"):
        small.check()
    assert small.ensure_capacity()
    small.forward()
    small.check()
    torch.cuda.synchronize()
    assert torch.equal(small.img.view(torch.int32), full.img.view(torch.int32))
    assert torch.equal(small.nc, full.nc)


def test_every_tuning_gives_the_same_frame(cuda):
    """The autotuner's candidates change only the work decomposition: the
    forward is bit-identical and the gradients agree to summation order."""
    from radiance_meshes_b200 import autotune as AT

    mesh, views, cams = _scene(16)
    i, v, c = _dev(mesh)
    vb = B.ViewBatch(cams)
    br = B.BatchedRasterizer(i, v, c, vb)
    br.forward()
    img0, nc0 = br.img.clone(), br.nc.clone()
    br.grad_img.normal_(generator=torch.Generator("cuda").manual_seed(4))
    gv0, gc0 = [t.clone() for t in br.backward()]
    for cand in AT.candidates_fwd(16):
        br.fwd_flags = AT.flags(**cand)
        br._blend_fwd()
        torch.cuda.synchronize()
        assert torch.equal(br.img.view(torch.int32), img0.view(torch.int32)), cand
        assert torch.equal(br.nc, nc0), cand
    for cand in AT.candidates_bwd(16):
        br.bwd_flags = AT.flags(**cand)
        gv, gc = br.backward()
        torch.cuda.synchronize()
        assert float((gv - gv0).norm() / gv0.norm()) < 1e-5, cand
        assert float((gc - gc0).norm() / gc0.norm()) < 1e-5, cand


def test_autotuner_returns_a_valid_choice(cuda, tmp_path, monkeypatch):
    from radiance_meshes_b200 import autotune as AT

    monkeypatch.setenv("RM_AUTOTUNE_CACHE", str(tmp_path / "cache.json"))
    mesh, views, cams = _scene(16)
    i, v, c = _dev(mesh)
    out = AT.tune_batch(i, v, c, views, tiles=(8, 16))
    assert out["tile"] in (8, 16) and not out["cached"]
    assert set(out["ms"]) == {"8/8", "16/16", "16/8"}
    again = AT.tune_batch(i, v, c, views, tiles=(8, 16))
    assert again["cached"] and again["tile"] == out["tile"] and again["fwd_flags"] == out["fwd_flags"]
    assert again["fine_shift"] == out["fine_shift"]
    cams_t = [tcam_to_struct(x.tcam(tile_size=out["tile"])) for x in views]
    br = B.BatchedRasterizer(i, v, c, B.ViewBatch(cams_t), fwd_flags=out["fwd_flags"], bwd_flags=out["bwd_flags"],
                             fine_shift=out["fine_shift"])
    br.forward()
    br.check()


@pytest.mark.parametrize("tile,shift,offcentre", [(16, 1, False), (32, 1, False), (32, 2, False), (16, 1, True),
                                                  (32, 2, True)])
def test_batch_fine_split_gives_the_coarse_frames(cuda, tile, shift, offcentre):
    """Lists sorted on the cameras' tiles and split into tiles 2^shift times
    smaller (rm_fine_lists_multi) render every view exactly as the
    single-camera blend over the coarse lists; the gradients are the sum of
    the single-camera gradients.  Also with cameras whose rays start a little
    off their projection centre (the split widens its test per view)."""
    mesh, views, cams = _scene(tile)
    if offcentre:
        for k, cam in enumerate(cams):
            cam.cam_pos[k % 3] += 3e-5 * (k + 1)
    i, v, c = _dev(mesh)
    vb = B.ViewBatch(cams)
    jit = _jitter(vb, seed=6)
    br = B.BatchedRasterizer(i, v, c, vb, jitter=jit, fine_shift=shift)
    br.forward()
    br.check()
    g = torch.Generator("cuda").manual_seed(8)
    gimg = torch.randn(vb.n_pixels, 4, device="cuda", generator=g)
    gv_b, gc_b = br.backward(gimg, None)
    torch.cuda.synchronize()
    assert int(br.fine_total.item()) > int(br.total.item())
    gv_s, gc_s = torch.zeros_like(v), torch.zeros_like(c)
    pj, pg = vb.split(jit), vb.split(gimg)
    for k, cam in enumerate(cams):
        ref = _single(i, v, c, cam, pj[k].contiguous())
        img_b, dist_b, _ = br.images()[k]
        assert torch.equal(img_b.view(torch.int32), ref["img"].view(torch.int32))
        assert torch.equal(dist_b.view(torch.int32), ref["dist"].view(torch.int32))
        R.blend_bwd(ref["lists"].sorted_ids, ref["lists"].ranges, i, v, c, pj[k].contiguous(), cam, ref["img"],
                    ref["dist"], ref["nc"], pg[k].contiguous(), None, ref["recs"], tiles_touched=ref["tiles"],
                    grad_vertices=gv_s, grad_cell_values=gc_s)
    torch.cuda.synchronize()
    for a, b in ((gv_b, gv_s), (gc_b, gc_s)):
        assert float((a - b).norm() / b.norm()) < 1e-5
