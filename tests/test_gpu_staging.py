"""The backward's two ways of staging tet records give the same gradients:
per-thread loads, and bulk copies into shared memory with two batches in
flight (RM_BLEND_STAGE_TMA).  The per-hit arithmetic and the batch grouping
are the same, so only the order of the global float atomics differs
(relative L2 error <= 1e-5); both match the oracle's FP32 adjoint."""
import numpy as np
import pytest
import torch

from gpu_util import run_gpu_forward, to_dev
from oracle import oracle as O
from radiance_meshes_b200 import _capi as C
from radiance_meshes_b200 import rasterizer as R
from radiance_meshes_b200 import scenes

pytestmark = pytest.mark.gpu


def _grads(r, gimg, stage_tma, batch_log2=0):
    L = r["lists"]
    saved = R.blend_tuning()
    R.set_blend_tuning(saved[0], batch_log2 << C.RM_BLEND_BATCH_SHIFT if batch_log2 else saved[1])
    R.use_tma_staging(stage_tma)
    try:
        status = torch.zeros(1, dtype=torch.int32, device="cuda")
        gv, gc = R.blend_bwd(L.sorted_ids, L.ranges, r["i"], r["v"], r["c"], r["j"], r["cam"], r["img"], r["dist"],
                             r["nc"], to_dev(gimg), None, r["records"], reuse_records=True, hit_masks=True,
                             status=status)
        torch.cuda.synchronize()
        assert int(status.item()) == 0
    finally:
        R.use_tma_staging(False)
        R.set_blend_tuning(*saved)
    return gv.cpu().numpy(), gc.cpu().numpy()


@pytest.mark.parametrize("workload,batch_log2", [("gradient_check", 0), ("gradient_check", 4), ("gradient_check", 5),
                                                 ("mixture", 0)])
def test_tma_staging_matches_load_staging(cuda, workload, batch_log2):
    if workload == "gradient_check":
        mesh, view = scenes.workload_gradient_check()
    else:
        mesh, view = scenes.workload_training_step(n_points=60_000, seed=2, tile_size=16, height=420, width=648)
    H, W = view.height, view.width
    jit = np.random.default_rng(5).uniform(0, 1, (H, W, 2)).astype(np.float32)
    r = run_gpu_forward(mesh.vertices, mesh.indices, mesh.cell_values, view.tcam(tile_size=8), jit, hit_masks=True)
    img = r["img"].cpu().numpy()
    target = np.random.default_rng(6).uniform(size=(H, W, 3)).astype(np.float32)
    gimg = np.zeros((H, W, 4), np.float32)
    gimg[..., :3] = np.sign(img[..., :3] - target) / (H * W * 3)
    gv0, gc0 = _grads(r, gimg, False, batch_log2)
    gv1, gc1 = _grads(r, gimg, True, batch_log2)
    for a, b in ((gv1, gv0), (gc1, gc0)):
        assert np.linalg.norm(a - b) <= 1e-5 * np.linalg.norm(b)
    if workload == "gradient_check":
        L = r["lists"]
        lists = dict(cam=r["cam"], sorted_ids=L.sorted_ids.cpu().numpy(), ranges=L.ranges.cpu().numpy())
        nc = r["nc"].cpu().numpy()[..., 0]
        img32, dist32, _ = O.blend_fwd_f32(lists, mesh.indices, mesh.vertices, mesh.cell_values, jit)
        fgv, fgc = O.blend_bwd(lists, mesh.indices, mesh.vertices, mesh.cell_values, jit, img32, dist32, nc, gimg,
                               None, "f32")
        assert np.linalg.norm(gv1 - fgv) <= 1e-4 * np.linalg.norm(fgv)
        assert np.linalg.norm(gc1 - fgc) <= 1e-4 * np.linalg.norm(fgc)
