"""Errors found on the device are reported, not hidden: a tet index outside
[0, n_verts), a NaN or infinite vertex, a pair count beyond int32 and a
bounded wait that gives up set RM_STATUS_* bits, and the drop-in raises
``DeviceStatusError`` at its one readback, where the reference asserts on the
host (delaunay_rasterization/internal/tile_shader_slang.py:78).

Nothing here faults or hangs the GPU: bad indices are rejected before any
load, and the waits are made to give up by a small iteration limit
(rm_set_wait_limit), after which the kernels go on with every store in
bounds."""
import ctypes

import numpy as np
import pytest
import torch

import radiance_meshes_b200 as RMB
from gpu_util import to_dev
from radiance_meshes_b200 import _capi as C
from radiance_meshes_b200 import rasterizer as R
from radiance_meshes_b200 import scenes
from radiance_meshes_b200.camera import tcam_to_struct

pytestmark = pytest.mark.gpu


def _dropin():
    RMB.install_dropin()
    from delaunay_rasterization.internal.alphablend_tiled_slang_interp import AlphaBlendTiledRender
    from delaunay_rasterization.internal.render_grid import RenderGrid
    from delaunay_rasterization.internal.tile_shader_slang import vertex_and_tile_shader

    return AlphaBlendTiledRender, RenderGrid, vertex_and_tile_shader


def _scene():
    mesh, view = scenes.workload_gradient_check()
    _, RenderGrid, _ = _dropin()
    grid = RenderGrid(view.height, view.width, tile_width=16, tile_height=16)
    return mesh, view, view.tcam(device="cuda"), grid


def _render_ok(mesh, tcam, grid):
    """A clean frame after an error: the status word was cleared."""
    _, _, vts = _dropin()
    sorted_ids, *_ = vts(to_dev(mesh.indices), to_dev(mesh.vertices), tcam, grid)
    return sorted_ids


def test_bad_index_is_reported_and_culled(cuda):
    mesh, view, tcam, grid = _scene()
    _, _, vts = _dropin()
    V = len(mesh.vertices)
    bad = mesh.indices.copy()
    bad[5, 2] = V + 10
    bad[17, 0] = -3
    bad[(len(bad) - 1), 3] = 2 ** 31 - 1
    with pytest.raises(C.DeviceStatusError) as ei:
        vts(to_dev(bad), to_dev(mesh.vertices), tcam, grid)
    assert ei.value.bits == C.RM_STATUS_BAD_INDEX and ei.value.code == C.RM_EINVAL
    # the stage itself: the bad tets are culled (zero rows), the others are unchanged
    cam = tcam_to_struct(tcam)
    i_bad, v = to_dev(bad), to_dev(mesh.vertices)
    tiles, rect, vs, cc = R.project_fwd(i_bad, v, cam)
    tiles0, rect0, vs0, cc0 = R.project_fwd(to_dev(mesh.indices), v, cam)
    status = R.frame_status(len(bad), v.device)
    torch.cuda.synchronize()
    assert int(status.item()) == C.RM_STATUS_BAD_INDEX
    status.zero_()
    rows = [5, 17, len(bad) - 1]
    keep = np.setdiff1d(np.arange(len(bad)), rows)
    assert (tiles[rows] == 0).all() and (rect[rows] == 0).all() and (cc[rows] == 0).all()
    assert torch.equal(tiles[keep], tiles0[keep]) and torch.equal(vs[keep], vs0[keep])
    # the next good frame goes through
    _render_ok(mesh, tcam, grid)


@pytest.mark.parametrize("value", [float("nan"), float("inf")])
def test_nonfinite_vertex_is_reported(cuda, value):
    mesh, view, tcam, grid = _scene()
    _, _, vts = _dropin()
    verts = mesh.vertices.copy()
    verts[mesh.indices[3, 1], 2] = value
    with pytest.raises(C.DeviceStatusError) as ei:
        vts(to_dev(mesh.indices), to_dev(verts), tcam, grid)
    assert ei.value.bits == C.RM_STATUS_NONFINITE
    _render_ok(mesh, tcam, grid)


def test_pack_and_features_skip_bad_indices(cuda):
    """Records of tets with a bad index are all zero (never hit) and their
    features zero; no vertex is read for them."""
    mesh, view, tcam, grid = _scene()
    T, V = len(mesh.indices), len(mesh.vertices)
    bad = mesh.indices.copy()
    bad[2, 1] = V
    i, v, cv = to_dev(bad), to_dev(mesh.vertices), to_dev(mesh.cell_values)
    L = C.lib()
    recs = torch.full((T * 32,), 7.0, device="cuda")
    C.check(L.rm_blend_pack_records(C.ptr(i), C.ptr(v), C.ptr(cv), T, V, None, C.ptr(recs), C.stream_handle()))
    torch.cuda.synchronize()
    r = recs.view(T, 32)
    assert (r[2] == 0).all() and (r[3] != 7.0).any()
    from radiance_meshes_b200 import features as F

    g = torch.Generator(device="cuda").manual_seed(0)
    feats = F.activate_output(torch.zeros(3), torch.rand((T, 1), device="cuda", generator=g),
                              torch.rand((T, 3), device="cuda", generator=g),
                              torch.rand((T, 3), device="cuda", generator=g), None, i,
                              torch.rand((T, 3), device="cuda", generator=g), v, 0, 0)
    torch.cuda.synchronize()
    assert (feats[2] == 0).all() and torch.isfinite(feats).all()


def _scan(tiles, ws=None):
    L = C.lib()
    T = tiles.numel()
    off = torch.empty_like(tiles)
    tot = torch.zeros(1, dtype=torch.int64, device=tiles.device)
    ws_n = L.rm_scan_workspace_size(T)
    if ws is None:
        ws = torch.zeros(ws_n, dtype=torch.uint8, device=tiles.device)
    C.check(L.rm_scan_tiles(C.ptr(tiles), T, C.ptr(off), C.ptr(tot), C.ptr(ws), ws_n, C.stream_handle()), "scan")
    st = ctypes.c_uint32(0)
    C.check(L.rm_read_status(C.ptr(ws), ctypes.byref(st), C.stream_handle()))
    return off, tot, st.value


def test_scan_overflow_is_reported(cuda):
    """A pair total above INT32_MAX cannot be held by the int32 offsets (the
    reference's cumsum is int32 too): the scan says so."""
    tiles = torch.full((600_000,), 4096, dtype=torch.int32, device="cuda")  # 2.46e9 pairs
    _, _, st = _scan(tiles)
    assert st & C.RM_STATUS_OVERFLOW
    ok = torch.full((600_000,), 3000, dtype=torch.int32, device="cuda")  # 1.8e9 pairs: fits
    off, tot, st = _scan(ok)
    assert st == 0 and int(tot.item()) == 600_000 * 3000 and int(off[-1].item()) == 600_000 * 3000


def _until(fn, tries=5):
    for _ in range(tries):
        if fn():
            return True
    return False


def test_scan_and_sort_waits_give_up(cuda):
    """With a wait limit of one poll, look-backs whose predecessor has not
    published yet give up: the timeout bit is set and the call returns."""
    L = C.lib()
    rng = np.random.default_rng(3)
    tiles = torch.from_numpy(rng.integers(0, 9, size=4_000_000).astype(np.int32)).cuda()
    n = 4_000_000
    keys = torch.from_numpy(rng.integers(0, 2 ** 45, size=n).astype(np.int64)).cuda()
    vals = torch.arange(n, dtype=torch.int32, device="cuda")

    def sort_times_out():
        ko, vo = torch.empty_like(keys), torch.empty_like(vals)
        ws_n = L.rm_sort_workspace_size(n)
        ws = torch.zeros(ws_n, dtype=torch.uint8, device="cuda")
        status = torch.zeros(1, dtype=torch.int32, device="cuda")
        C.check(L.rm_sort_pairs(C.ptr(keys), C.ptr(vals), n, None, 45, C.ptr(ko), C.ptr(vo), C.ptr(ws), ws_n,
                                C.ptr(status), C.stream_handle()), "sort")
        torch.cuda.synchronize()
        return int(status.item()) & C.RM_STATUS_SORT_TIMEOUT

    try:
        C.set_wait_limit(1)
        assert _until(lambda: _scan(tiles)[2] & C.RM_STATUS_SCAN_TIMEOUT)
        assert _until(sort_times_out)
    finally:
        C.set_wait_limit(0)
    off, tot, st = _scan(tiles)  # the default limit: exact again
    assert st == 0 and int(tot.item()) == int(tiles.sum().item())
    assert not sort_times_out()


def test_dropin_raises_on_timeout(cuda):
    """The drop-in reads the frame's status word with the pair count and
    raises with the timeout code; the next frame at the default limit is
    clean."""
    mesh, view = scenes.workload_training_step(n_points=60_000, seed=2, tile_size=16, height=420, width=648)
    _, RenderGrid, vts = _dropin()
    grid = RenderGrid(view.height, view.width, tile_width=16, tile_height=16)
    tcam = view.tcam(device="cuda")
    i, v = to_dev(mesh.indices), to_dev(mesh.vertices)

    def raises_timeout():
        try:
            vts(i, v, tcam, grid)
        except C.DeviceStatusError as e:
            assert e.code == C.RM_ETIMEOUT
            return True
        return False

    try:
        C.set_wait_limit(1)
        assert _until(raises_timeout)
    finally:
        C.set_wait_limit(0)
    vts(i, v, tcam, grid)
    R.check_status(len(mesh.indices), v.device)


def test_blend_without_frame_state_is_identical(cuda):
    """A copy of the sorted ids carries no projection state: the blend then
    packs every tet and walks the caller's lists, with the same image and
    gradients."""
    AlphaBlendTiledRender, _, vts = _dropin()
    mesh, view, tcam, grid = _scene()
    idx = to_dev(mesh.indices)
    jitter = torch.full((view.height, view.width, 2), 0.5, device="cuda")
    outs = []
    for copy in (False, True):
        verts = to_dev(mesh.vertices).requires_grad_(True)
        cv = to_dev(mesh.cell_values).requires_grad_(True)
        sorted_ids, ranges, *_ = vts(idx, verts, tcam, grid)
        if copy:
            sorted_ids = sorted_ids.clone()
            assert R.frame_of(sorted_ids) is None
        img, dist, _ = AlphaBlendTiledRender.apply(sorted_ids, ranges, idx, verts, cv, grid, tcam, jitter)
        (img[..., :3].sum() + dist.sum() * 1e-3).backward()
        outs.append((img.detach(), verts.grad, cv.grad))
    (a, ga, ca), (b, gb, cb) = outs
    assert (a[..., 3] == b[..., 3]).all()  # log T: bit for bit over 8x8 or caller's lists
    assert (a - b).abs().max() <= 1e-6
    # gradients are sums of float atomics in another order: relative L2 error
    for x, y in ((ga, gb), (ca, cb)):
        assert float((x - y).norm() / y.norm()) <= 1e-5


@pytest.mark.parametrize("bad_id", [-7, 10 ** 6])
def test_blend_skips_list_ids_outside_the_tets(cuda, bad_id):
    """A list id that names no tet (only lists left invalid by a wait that
    gave up, or a caller's corrupt lists, hold one) is never used as an
    address: the blend stages a zero record for it, which no ray hits, and
    sets RM_STATUS_BAD_INDEX.  Forward and backward then equal the passes
    over the intact lists with that tet's density set to zero."""
    mesh, view, tcam, grid = _scene()
    cam = tcam_to_struct(view.tcam())
    i, v = to_dev(mesh.indices), to_dev(mesh.vertices)
    cv = to_dev(mesh.cell_values)
    tiles, rect, vs, _ = R.project_fwd(i, v, cam)
    L = R.build_tile_lists(tiles, rect, vs, cam)
    ids = L.sorted_ids
    g = int(ids[ids.shape[0] // 2])
    bad = ids.clone()
    bad[ids == g] = bad_id
    cv0 = cv.clone()
    cv0[g, 0] = 0.0
    jitter = torch.rand((view.height, view.width, 2), generator=torch.Generator().manual_seed(5)).cuda()
    status = torch.zeros(1, dtype=torch.int32, device="cuda")
    img_b, dist_b, nc_b, ws_b = R.blend_fwd(bad, L.ranges, i, v, cv, jitter, cam, status=status)
    img_r, dist_r, nc_r, ws_r = R.blend_fwd(ids, L.ranges, i, v, cv0, jitter, cam)
    torch.cuda.synchronize()
    assert int(status.item()) & C.RM_STATUS_BAD_INDEX
    assert torch.equal(img_b, img_r) and torch.equal(dist_b, dist_r) and torch.equal(nc_b, nc_r)
    gimg = torch.randn(img_b.shape, generator=torch.Generator().manual_seed(6)).cuda()
    status.zero_()
    gv_b, gc_b = R.blend_bwd(bad, L.ranges, i, v, cv, jitter, cam, img_b, dist_b, nc_b, gimg, None, ws_b,
                             status=status)
    gv_r, gc_r = R.blend_bwd(ids, L.ranges, i, v, cv0, jitter, cam, img_r, dist_r, nc_r, gimg, None, ws_r)
    torch.cuda.synchronize()
    assert int(status.item()) & C.RM_STATUS_BAD_INDEX
    assert float(gc_b[g].abs().max()) == 0.0
    keep = torch.ones(gc_b.shape[0], dtype=torch.bool, device="cuda")
    keep[g] = False
    for x, y in ((gv_b, gv_r), (gc_b[keep], gc_r[keep])):  # float atomics in another order
        assert float((x - y).norm() / y.norm()) <= 1e-6
