"""Parity at full size: the 1.32M-tet training frame (200,000 mixture points,
seed 2, 1297x840, 16x16 tiles) against the oracle, with the constant jitter
of render() (0.5) and with the per-pixel random jitter of training
(train.py:244).

  * integer stages bit-exact: tile counts, rectangles, depth keys (bits),
    offsets, emitted and sorted keys and values, ranges, n_contributors;
  * blend forward: log T and the five distortion moments bit-exact, rgb
    within 1e-4 max-abs of the FP32 restatement; the drop-in's 8x8-pixel
    lists give the same image, log T and distortion bit for bit;
  * blend backward (L1 loss): relative L2 error per group <= 1e-4 against
    the FP32 adjoint of the oracle."""
import numpy as np
import pytest
import torch

from gpu_util import bits, to_dev
from oracle import oracle as O
from radiance_meshes_b200 import rasterizer as R
from radiance_meshes_b200 import scenes
from radiance_meshes_b200.camera import tcam_to_struct
from test_gpu_backward import _compare, _groups

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def frame(cuda):
    mesh, view = scenes.workload_training_step(n_points=200_000, seed=2, tile_size=16, height=840, width=1297)
    tcam = view.tcam()
    L = O.rasterize_lists(mesh.indices, mesh.vertices, tcam)
    cam = tcam_to_struct(tcam)
    i, v = to_dev(mesh.indices), to_dev(mesh.vertices)
    tiles, rect, vs, cc = R.project_fwd(i, v, cam)
    lists = R.build_tile_lists(tiles, rect, vs, cam, keep_debug=True)
    torch.cuda.synchronize()
    return dict(mesh=mesh, view=view, L=L, cam=cam, i=i, v=v, tiles=tiles, rect=rect, vs=vs, cc=cc, lists=lists)


def test_config2_integer_stages_bit_exact(frame):
    L, g = frame["L"], frame
    assert len(frame["mesh"].indices) > 1_300_000
    assert np.array_equal(g["tiles"].cpu().numpy(), L["tiles_touched"])
    assert np.array_equal(g["rect"].cpu().numpy(), L["rect"])
    assert np.array_equal(bits(g["vs"].cpu().numpy()), bits(L["vs"]))
    assert np.array_equal(bits(g["cc"].cpu().numpy()), bits(L["circumcenter"]))
    ls = g["lists"]
    assert ls.n_pairs == len(L["keys"]) > 2_000_000
    assert np.array_equal(ls.offsets.cpu().numpy(), L["offsets"])
    assert np.array_equal(ls.keys.cpu().numpy(), L["keys"]) and np.array_equal(ls.values.cpu().numpy(), L["values"])
    assert np.array_equal(ls.sorted_keys.cpu().numpy(), L["sorted_keys"])
    assert np.array_equal(ls.sorted_ids.cpu().numpy(), L["sorted_ids"])
    assert np.array_equal(ls.ranges.cpu().numpy(), L["ranges"])


def _jitter(kind, H, W):
    if kind == "half":
        return np.full((H, W, 2), 0.5, np.float32)
    return np.random.default_rng(244).uniform(0, 1, (H, W, 2)).astype(np.float32)


@pytest.mark.parametrize("kind", ["half", "rand"])
def test_config2_blend_forward_backward(frame, kind):
    mesh, view, L, cam = frame["mesh"], frame["view"], frame["L"], frame["cam"]
    H, W = view.height, view.width
    jit = _jitter(kind, H, W)
    j = to_dev(jit)
    c = to_dev(mesh.cell_values)
    ls = frame["lists"]
    img, dist, nc, recs = R.blend_fwd(ls.sorted_ids, ls.ranges, frame["i"], frame["v"], c, j, cam,
                                      tiles_touched=frame["tiles"], hit_masks=True)
    img32, dist32, nc32 = O.blend_fwd_f32(L, mesh.indices, mesh.vertices, mesh.cell_values, jit)
    g_img, g_dist, g_nc = img.cpu().numpy(), dist.cpu().numpy(), nc.cpu().numpy()[..., 0]
    assert np.array_equal(g_nc, nc32), "n_contributors differ from the oracle"
    assert np.array_equal(bits(g_img[..., 3]), bits(img32[..., 3])), "log T differs from the oracle"
    assert np.array_equal(bits(g_dist), bits(dist32)), "distortion moments differ from the oracle"
    err = np.abs(g_img[..., :3] - img32[..., :3]).max()
    assert err <= 1e-4, f"rgb differs from the FP32 restatement by {err:.3e}"
    # the drop-in's 8x8-pixel lists cut for this jitter: same image bit for bit
    _, _, _, _, fp = R.project_fwd_fine(frame["i"], frame["v"], cam)
    fine = R.split_fine_lists(ls.sorted_ids, ls.ranges, cam, R.fine_shift_for(cam), fp, R.jitter_bounds(j),
                              ls.sorted_keys)
    img_f, dist_f, _, _ = R.blend_fwd(fine.sorted_ids, fine.ranges, frame["i"], frame["v"], c, j, fine.cam,
                                      tiles_touched=frame["tiles"])
    assert torch.equal(img_f, img) and torch.equal(dist_f, dist)
    # backward of an L1 loss against the FP32 adjoint
    target = np.random.default_rng(7).uniform(size=(H, W, 3)).astype(np.float32)
    gimg = np.zeros((H, W, 4), np.float32)
    gimg[..., :3] = np.sign(g_img[..., :3] - target) / (H * W * 3)
    gv, gc = R.blend_bwd(ls.sorted_ids, ls.ranges, frame["i"], frame["v"], c, j, cam, img, dist, nc, to_dev(gimg),
                         None, recs, reuse_records=True, hit_masks=True)
    torch.cuda.synchronize()
    fgv, fgc = O.blend_bwd(L, mesh.indices, mesh.vertices, mesh.cell_values, jit, img32, dist32, nc32, gimg,
                           None, "f32")
    rel = _compare(_groups(gv.cpu().numpy(), gc.cpu().numpy()), _groups(fgv, fgc), 1e-4, what=f"config 2 ({kind})")
    print("relative L2 errors vs FP32 adjoint", rel)
