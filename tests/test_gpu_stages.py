"""Stages (a)-(c) on the GPU against the oracle: bit-exact integer outputs.

Covers the reference's scenario families (camera inside a tet, on a face,
outside, inside a point cloud, empty lists) from the golden fixtures and the
plain-forward workload (4,096 points, 256x256) computed by the oracle on the fly.
"""
import numpy as np
import pytest
import torch

import golden_util as G
from gpu_util import bits, run_gpu_forward

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name", G.names())
def test_integer_stages_match_golden(cuda, name):
    z, tcam = G.load(name)
    r = run_gpu_forward(z["vertices"], z["indices"], z["cell_values"], tcam, z["jitter"])
    L = r["lists"]
    assert np.array_equal(r["tiles"].cpu().numpy(), z["tiles_touched"])
    assert np.array_equal(r["rect"].cpu().numpy(), z["rect"])
    assert np.array_equal(bits(r["vs"].cpu().numpy()), bits(z["vs"]))
    assert np.array_equal(bits(r["cc"].cpu().numpy()), bits(z["circumcenter"]))
    assert L.n_pairs == len(z["sorted_ids"])
    assert np.array_equal(L.offsets.cpu().numpy(), z["offsets"])
    assert np.array_equal(L.keys.cpu().numpy(), z["keys"])
    assert np.array_equal(L.values.cpu().numpy(), z["values"])
    assert np.array_equal(L.sorted_keys.cpu().numpy(), z["sorted_keys"])
    assert np.array_equal(L.sorted_ids.cpu().numpy(), z["sorted_ids"])
    assert np.array_equal(L.ranges.cpu().numpy(), z["ranges"])


@pytest.mark.parametrize("tile", [4, 8, 16, 32])
def test_integer_stages_plain_forward_workload(cuda, plain_forward_oracle, tile):
    mesh, view, lists, _ = plain_forward_oracle(tile)
    tcam = view.tcam(tile_size=tile)
    jitter = np.full((view.height, view.width, 2), 0.5, np.float32)
    r = run_gpu_forward(mesh.vertices, mesh.indices, mesh.cell_values, tcam, jitter)
    L = r["lists"]
    assert np.array_equal(r["tiles"].cpu().numpy(), lists["tiles_touched"])
    assert np.array_equal(r["rect"].cpu().numpy(), lists["rect"])
    assert np.array_equal(bits(r["vs"].cpu().numpy()), bits(lists["vs"]))
    assert np.array_equal(L.sorted_ids.cpu().numpy(), lists["sorted_ids"])
    assert np.array_equal(L.ranges.cpu().numpy(), lists["ranges"])


def _fine_bits(fp, jb, ox, oy, tw, th, f):
    """Bit q of entry i: the tet with footprint fp[i] can reach fine tile q of
    the coarse tile with pixel origin (ox[i], oy[i]) under the jitter bounds
    jb -- the test of rm_fine_lists (box grown by 1/64 pixel, then the edges of
    the projected vertices' hull with 1/16 pixel), restated in float32 with
    the kernel's operation order."""
    f32 = np.float32
    m, hm = f32(1.0 / 64.0), f32(1.0 / 16.0)
    fp = fp.astype(np.float32)
    jb = jb.astype(np.float32)
    box = fp[:, 0:4]
    oxf, oyf = ox.astype(np.float32), oy.astype(np.float32)
    px = np.stack([fp[:, 4], fp[:, 6], fp[:, 8], fp[:, 10]], 1) - oxf[:, None]
    py = np.stack([fp[:, 5], fp[:, 7], fp[:, 9], fp[:, 11]], 1) - oyf[:, None]
    valid = ~np.isnan(fp[:, 4])
    edges = []
    z = f32(0)
    with np.errstate(invalid="ignore", over="ignore"):
        for a, b, o1, o2 in ((0, 1, 2, 3), (0, 2, 1, 3), (0, 3, 1, 2), (1, 2, 0, 3), (1, 3, 0, 2), (2, 3, 0, 1)):
            nx = py[:, b] - py[:, a]
            ny = px[:, a] - px[:, b]
            ca = nx * px[:, a] + ny * py[:, a]
            s1 = nx * px[:, o1] + ny * py[:, o1] - ca
            s2 = nx * px[:, o2] + ny * py[:, o2] - ca
            pos = (s1 <= 0) & (s2 <= 0)
            neg = ~pos & (s1 >= 0) & (s2 >= 0)
            sg = np.where(pos, f32(1), np.where(neg, f32(-1), f32(0))).astype(np.float32)
            edges.append((np.where(valid, sg * nx, z), np.where(valid, sg * ny, z), np.where(valid, sg * ca, z)))
        w, h = tw // f, th // f
        bits = np.zeros(len(fp), np.int64)
        for q in range(f * f):
            dx, dy = q % f * w, q // f * h
            x0, y0 = ox + dx, oy + dy
            ok = (box[:, 0] - m <= (x0 + w - 1).astype(np.float32) + jb[2]) & \
                 (box[:, 2] + m >= x0.astype(np.float32) + jb[0])
            ok &= (box[:, 1] - m <= (y0 + h - 1).astype(np.float32) + jb[3]) & \
                  (box[:, 3] + m >= y0.astype(np.float32) + jb[1])
            xlo, xhi = f32(dx) + jb[0], f32(dx + w - 1) + jb[2]
            ylo, yhi = f32(dy) + jb[1], f32(dy + h - 1) + jb[3]
            sep = np.zeros(len(fp), bool)
            for nx, ny, c in edges:
                d = (nx * np.where(nx > 0, xlo, xhi).astype(np.float32)
                     + ny * np.where(ny > 0, ylo, yhi).astype(np.float32)) - c
                sep |= d > hm * (np.abs(nx) + np.abs(ny))
            bits |= (ok & ~sep).astype(np.int64) << q
    return bits


def _parallax_px(cam):
    """The library's parallax allowance of a camera (2 x focal x offset of
    cam_pos from the world_view centre / min_t), restated in float64."""
    M = [float(x) for x in cam.world_view]
    R = [[M[4 * i + j] for j in range(3)] for i in range(3)]
    t = [M[4 * i + 3] for i in range(3)]
    off2 = 0.0
    for j in range(3):
        center = -(R[0][j] * t[0] + R[1][j] * t[1] + R[2][j] * t[2])
        d = float(cam.cam_pos[j]) - center
        off2 += d * d
    if off2 == 0.0:
        return np.float32(0.0)
    f = max(abs(float(cam.K[0])), abs(float(cam.K[4])))
    return np.float32(2.0 * f * np.sqrt(off2) / float(np.float32(cam.min_t)))


@pytest.mark.parametrize("tile,jit", [(16, "unit"), (32, "unit"), (16, "half"), (16, "wide")])
def test_fine_lists_split_matches_restatement(cuda, tile, jit):
    """Splitting the sorted coarse lists (rm_fine_lists) keeps, for every fine
    tile, exactly the coarse entries that reach it (float32 restatement of the
    footprint test), in the coarse order, with the fine ranges of that
    order; the projection with footprints equals the plain projection."""
    import torch

    from radiance_meshes_b200 import rasterizer as R
    from radiance_meshes_b200 import scenes
    from radiance_meshes_b200.camera import tcam_to_struct

    mesh, view = scenes.workload_training_step(n_points=20000, seed=2, tile_size=tile, height=420, width=649)
    cam = tcam_to_struct(view.tcam())
    fs = R.fine_shift_for(cam)
    assert fs == (1 if tile == 16 else 2)
    f = 1 << fs
    i = torch.from_numpy(mesh.indices).cuda()
    v = torch.from_numpy(mesh.vertices).cuda()
    tiles, rect, vs, cc, fp = R.project_fwd_fine(i, v, cam)
    t0, r0, vs0, cc0 = R.project_fwd(i, v, cam)
    assert torch.equal(tiles, t0) and torch.equal(rect, r0) and torch.equal(vs, vs0) and torch.equal(cc, cc0)
    fpn = fp.cpu().numpy()
    vis = tiles.cpu().numpy() > 0
    assert (~np.isnan(fpn[vis, 4])).mean() > 0.9  # most visible tets carry their projected vertices
    rng = np.random.default_rng(7)
    shape = (view.height, view.width, 2)
    j = {"unit": rng.uniform(0, 1, shape), "half": np.full(shape, 0.5), "wide": rng.uniform(-1.5, 2.5, shape)}[jit]
    jitter = torch.from_numpy(j.astype(np.float32)).cuda()
    jb = R.jitter_bounds(jitter)
    jj = j.astype(np.float32).reshape(-1, 2)
    assert np.array_equal(jb.cpu().numpy(), np.array([jj[:, 0].min(), jj[:, 1].min(), jj[:, 0].max(),
                                                      jj[:, 1].max()], np.float32))
    coarse = R.build_tile_lists(tiles, rect, vs, cam)
    fine = R.split_fine_lists(coarse.sorted_ids, coarse.ranges, cam, fs, fp, jb, coarse.sorted_keys)
    # restatement: entry e of coarse tile t goes to fine tile q when bit q is set
    ids = coarse.sorted_ids.cpu().numpy()
    rg = coarse.ranges.cpu().numpy()
    G = cam.grid_width * cam.grid_height
    t_of = np.repeat(np.arange(G), rg[:, 1] - rg[:, 0])
    assert len(t_of) == len(ids)
    tx, ty = t_of % cam.grid_width, t_of // cam.grid_width
    # the kernels widen the jitter range by the camera's parallax allowance
    a = _parallax_px(cam)
    jbn = jb.cpu().numpy()
    jbn = np.array([jbn[0] - a, jbn[1] - a, jbn[2] + a, jbn[3] + a], np.float32)
    bits = _fine_bits(fpn[ids], jbn, tx * tile, ty * tile, tile, tile, f)
    fgw = cam.grid_width * f
    e_all, q_all = np.nonzero((bits[:, None] >> np.arange(f * f)[None, :]) & 1)
    fid = (ty[e_all] * f + q_all // f) * fgw + tx[e_all] * f + q_all % f
    order = np.argsort(fid, kind="stable")
    ref_ids = ids[e_all[order]]
    ref_len = np.bincount(fid, minlength=G * f * f)
    n = fine.n_pairs
    assert n == len(ref_ids)
    assert np.array_equal(fine.sorted_ids[:n].cpu().numpy(), ref_ids)
    fr = fine.ranges.cpu().numpy()
    assert np.array_equal(fr[:, 1] - fr[:, 0], ref_len)
    start = np.concatenate([[0], np.cumsum(ref_len)[:-1]])
    ne = ref_len > 0
    assert np.array_equal(fr[ne, 0], start[ne])
    # the hull edges remove entries that the box alone keeps
    fp_box = fpn[ids].copy()
    fp_box[:, 4:] = np.nan
    box_bits = _fine_bits(fp_box, jbn, tx * tile, ty * tile, tile, tile, f)
    assert not np.any(bits & ~box_bits)
    n_box = int(((box_bits[:, None] >> np.arange(f * f)[None, :]) & 1).sum())
    assert n < 0.9 * n_box


@pytest.mark.parametrize("depth_first", [False, True])
def test_pair_buffers_sized_from_the_previous_frame(cuda, depth_first):
    """build_tile_lists sizes the pair buffers from the previous frame's count
    and queues emission, sort and ranges before reading P; a frame with many
    more pairs than the last is rebuilt at its exact size.  The lists equal
    those built with exactly sized buffers, whichever path a frame takes, in
    the reference's order of work and depth first, and the capacity bit of an
    outgrown frame is not left for the next readback."""
    from radiance_meshes_b200 import rasterizer as R
    from radiance_meshes_b200 import scenes
    from radiance_meshes_b200.camera import tcam_to_struct

    small_mesh, small_view = scenes.workload_plain_forward()
    big_mesh, big_view = scenes.workload_training_step(n_points=20000, seed=2, height=420, width=649)

    def lists(mesh, view):
        cam = tcam_to_struct(view.tcam())
        i = torch.from_numpy(mesh.indices).cuda()
        v = torch.from_numpy(mesh.vertices).cuda()
        tiles, rect, vs, cc = R.project_fwd(i, v, cam)
        L = R.build_tile_lists(tiles, rect, vs, cam, keep_debug=not depth_first)
        return L.sorted_ids.clone(), L.ranges.clone(), L.sorted_keys.clone()

    def exact(mesh, view):
        R._PAIR_GUESS.clear()  # no previous frame: buffers of exactly P
        return lists(mesh, view)

    ref_small, ref_big = exact(small_mesh, small_view), exact(big_mesh, big_view)
    for mesh, view, ref in ((small_mesh, small_view, ref_small), (big_mesh, big_view, ref_big),
                            (big_mesh, big_view, ref_big), (small_mesh, small_view, ref_small)):
        got = lists(mesh, view)  # big after small outgrows the small frame's buffers; the others fit
        for a, b in zip(got, ref):
            assert torch.equal(a, b)
    assert ref_big[0].shape[0] > 2 * ref_small[0].shape[0]
    R.check_status(len(small_mesh.indices), torch.device("cuda"))


@pytest.mark.parametrize("n", [0, 1, 1000, 1_000_003])
def test_count_pairs_sums_positive_counts_and_snapshots_status(cuda, n):
    """rm_count_pairs: out[0] = the sum of the positive tile counts (int64),
    out[1] = the status word as the work queued before it left it."""
    from radiance_meshes_b200 import _capi as C

    rng = np.random.default_rng(n + 7)
    tiles_h = rng.integers(-3, 40, size=n).astype(np.int32)
    tiles = torch.from_numpy(tiles_h).cuda()
    status = torch.tensor([C.RM_STATUS_BAD_INDEX | C.RM_STATUS_NONFINITE], dtype=torch.int32, device="cuda")
    out = torch.full((2,), -5, dtype=torch.int64, device="cuda")
    C.check(C.lib().rm_count_pairs(C.ptr(tiles) if n else None, n, C.ptr(status), C.ptr(out), C.stream_handle()),
            "rm_count_pairs")
    got = out.cpu().numpy()
    assert int(got[0]) == int(np.maximum(tiles_h.astype(np.int64), 0).sum())
    assert int(got[1]) == C.RM_STATUS_BAD_INDEX | C.RM_STATUS_NONFINITE
    C.check(C.lib().rm_count_pairs(C.ptr(tiles) if n else None, n, None, C.ptr(out), C.stream_handle()),
            "rm_count_pairs")
    assert int(out[1].item()) == 0
