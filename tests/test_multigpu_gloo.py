"""The N>1 path on CPU: two gloo ranks render disjoint views of one mesh with
the oracle (FP32 restatement of the reference forward and backward) and sum
their gradients with allreduce_grads; the result must equal one process
rendering every view."""
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from radiance_meshes_b200 import multigpu as MG
from radiance_meshes_b200 import scenes

N_VIEWS = 3


def _scene():
    mesh, _ = scenes.workload_gradient_check()
    views = scenes.ring_views(N_VIEWS, [(32, 48), (40, 40), (24, 56)], radius=2.9, height_offset=0.3)
    return mesh, views


def _view_grads(mesh, view, seed):
    from oracle import oracle as O

    tcam = view.tcam()
    L = O.rasterize_lists(mesh.indices, mesh.vertices, tcam)
    jit = np.full((view.height, view.width, 2), 0.5, np.float32)
    img, dist_img, nc = O.blend_fwd_f32(L, mesh.indices, mesh.vertices, mesh.cell_values, jit)
    g = np.random.default_rng(seed).normal(size=(view.height, view.width, 4)).astype(np.float32)
    gv, gc = O.blend_bwd(L, mesh.indices, mesh.vertices, mesh.cell_values, jit, img, dist_img, nc, g, None, "f32")
    return torch.from_numpy(gv), torch.from_numpy(gc)


def _worker(rank, world, port, out):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        mesh, views = _scene()
        gv = torch.zeros(len(mesh.vertices), 3, dtype=torch.float64)
        gc = torch.zeros(len(mesh.indices), 7, dtype=torch.float64)
        for k in MG.views_for_rank(N_VIEWS, rank, world):
            a, b = _view_grads(mesh, views[k], seed=k)
            gv += a
            gc += b
        MG.allreduce_grads([gv, gc])
        torch.save((gv, gc), os.path.join(out, f"rank{rank}.pt"))
    finally:
        dist.destroy_process_group()


def _worker_overlapped(rank, world, port, out):
    """Each view's gradient reduced while the rank's next view renders
    (OverlappedGradSum); ranks with fewer views add zeros so the
    collectives line up."""
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        mesh, views = _scene()
        like = [torch.zeros(len(mesh.vertices), 3, dtype=torch.float64),
                torch.zeros(len(mesh.indices), 7, dtype=torch.float64)]
        ex = MG.OverlappedGradSum(like, in_flight=1)
        mine = MG.views_for_rank(N_VIEWS, rank, world)
        for k in mine:
            ex.add_view(list(_view_grads(mesh, views[k], seed=k)))
        for _ in range(MG.views_per_rank(N_VIEWS, world) - len(mine)):
            ex.add_zero_view()
        gv, gc = ex.result()
        assert ex.views == MG.views_per_rank(N_VIEWS, world)
        torch.save((gv, gc), os.path.join(out, f"rank{rank}.pt"))
    finally:
        dist.destroy_process_group()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_views_for_rank_partition():
    for world in (1, 2, 3, 8):
        got = sorted(v for r in range(world) for v in MG.views_for_rank(16, r, world))
        assert got == list(range(16))
    with pytest.raises(ValueError):
        MG.views_for_rank(4, 2, 2)


@pytest.mark.parametrize("worker", [_worker, _worker_overlapped], ids=["one_bucket", "overlapped_per_view"])
def test_two_rank_gradient_sum_matches_single_process(tmp_path, worker):
    mp.start_processes(worker, args=(2, _free_port(), str(tmp_path)), nprocs=2, join=True, start_method="spawn")
    mesh, views = _scene()
    gv = torch.zeros(len(mesh.vertices), 3, dtype=torch.float64)
    gc = torch.zeros(len(mesh.indices), 7, dtype=torch.float64)
    for k in range(N_VIEWS):
        a, b = _view_grads(mesh, views[k], seed=k)
        gv += a
        gc += b
    assert MG.views_per_rank(N_VIEWS, 2) == 2  # rank 1 adds one zero view
    for r in range(2):
        rv, rc = torch.load(os.path.join(tmp_path, f"rank{r}.pt"))
        assert torch.allclose(rv, gv, rtol=1e-12, atol=1e-12)
        assert torch.allclose(rc, gc, rtol=1e-12, atol=1e-12)
    assert float(gv.abs().sum()) > 0
