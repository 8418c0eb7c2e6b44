"""Serving loop: results are the same alone and in the mix; overflow retry
and HBM-budget admission keep that true."""
import numpy as np
import pytest
import torch

from radiance_meshes_b200 import scenes
from radiance_meshes_b200 import serve as S
from radiance_meshes_b200.camera import tcam_to_struct

pytestmark = pytest.mark.gpu

RES = [(48, 64), (96, 128), (160, 96), (77, 131)]


@pytest.fixture(scope="module")
def meshes(cuda):
    m0, _ = scenes.workload_gradient_check()
    m1, _ = scenes.workload_plain_forward()
    return [S.ResidentMesh("ball", m0.indices, m0.vertices, m0.cell_values),
            S.ResidentMesh("cube", m1.indices, m1.vertices, m1.cell_values)]


def _trace(n, seed=11, radius=2.8):
    tr = scenes.serving_trace(n, 500.0, ["ball", "cube"], seed=seed, resolutions=RES, radius=radius)
    return [S.RenderRequest(k, name, tcam_to_struct(view.tcam()), t) for k, (t, name, view) in enumerate(tr)]


def _same(a, b):
    return (torch.equal(a.img.view(torch.int32), b.img.view(torch.int32)) and
            torch.equal(a.dist.view(torch.int32), b.dist.view(torch.int32)) and torch.equal(a.nc, b.nc))


def _calibrate(server, meshes, tile=None):
    cams = [tcam_to_struct(v.tcam(tile_size=tile)) for v in scenes.ring_views(4, RES, radius=2.8)]
    server.calibrate({m.name: cams for m in meshes})


def _views(n, seed=11, radius=2.8):
    return [v for _, _, v in scenes.serving_trace(n, 500.0, ["ball", "cube"], seed=seed, resolutions=RES,
                                                  radius=radius)]


def test_results_same_alone_and_mixed(meshes):
    reqs = _trace(40)
    mixed = S.Server(meshes, streams=3, max_views=5)
    _calibrate(mixed, meshes)
    res = mixed.run_trace(reqs, realtime=False)
    torch.cuda.synchronize()
    assert len(res) == len(reqs)
    assert max(r.batch_views for r in res) > 1  # requests really were batched
    alone = S.Server(meshes, streams=1, max_views=1)
    _calibrate(alone, meshes)
    by_id = {r.rid: r for r in res}
    for q in _trace(40):
        a = alone.render_alone(q)
        assert a.batch_views == 1
        assert _same(a, by_id[q.rid]), q.rid


def test_fine_split_serving_same_alone_and_mixed(meshes):
    reqs = [S.RenderRequest(q.rid, q.mesh, tcam_to_struct(v.tcam(tile_size=16)), q.arrival)
            for q, v in zip(_trace(24, seed=21), _views(24, seed=21))]
    mixed = S.Server(meshes, streams=3, max_views=4, tile=16, fine_shift=1)
    _calibrate(mixed, meshes, tile=16)
    res = {r.rid: r for r in mixed.run_trace(reqs, realtime=False)}
    alone = S.Server(meshes, streams=1, max_views=1, tile=16, fine_shift=1)
    _calibrate(alone, meshes, tile=16)
    for q in reqs:
        assert _same(alone.render_alone(q), res[q.rid]), q.rid


def test_overflow_is_retried(meshes):
    server = S.Server(meshes, streams=2, max_views=4)
    server.pair_slack = 1
    for m in meshes:
        m.pairs_per_pixel = 0.0  # no room: every batch overflows once
    try:
        res = server.run_trace(_trace(12, seed=12), realtime=False)
    finally:
        for m in meshes:
            m.pairs_per_pixel = None
    assert server.n_retries > 0 and all(r.retried for r in res)
    ref = S.Server(meshes, streams=1, max_views=1)
    _calibrate(ref, meshes)
    by_id = {r.rid: r for r in res}
    for q in _trace(12, seed=12):
        assert _same(ref.render_alone(q), by_id[q.rid])


def test_hbm_budget_limits_inflight_memory(meshes):
    reqs = _trace(16, seed=13)
    probe = S.Server(meshes, streams=4, max_views=1)
    _calibrate(probe, meshes)
    from radiance_meshes_b200 import batch as B

    one = max(S.batch_bytes(probe.meshes[q.mesh].T, B.ViewBatch([q.cam]),
                            probe._capacity(probe.meshes[q.mesh], B.ViewBatch([q.cam]))) for q in reqs)
    server = S.Server(meshes, streams=4, max_views=4, hbm_budget=int(one * 1.5))
    _calibrate(server, meshes)
    res = server.run_trace(reqs, realtime=False)
    assert len(res) == len(reqs)
    assert server.peak_reserved <= int(one * 1.5)
    assert server.reserved == 0 and not server.inflight


def test_realtime_trace_latency_summary(meshes):
    server = S.Server(meshes, streams=3, max_views=4, keep_outputs=False)
    _calibrate(server, meshes)
    res = server.run_trace(_trace(60, seed=14), realtime=True)
    s = S.latency_summary(res)
    assert s["requests"] == 60
    assert 0 < s["p50_ms"] <= s["p99_ms"] < 5000
    assert all(r.latency_ms > 0 for r in res)
