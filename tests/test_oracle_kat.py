"""Known-answer tests of the oracle: analytic single-tet and slab integrals,
convergence to the midpoint quadrature of jaxutil/tetra_quad.py, sort
stability and ranges of empty tiles."""
import math

import numpy as np
import pytest

import scenarios
from oracle import oracle as O
from radiance_meshes_b200.camera import make_tcam
from radiance_meshes_b200.scenes import delaunay


def _axis_cam(pos, H=1, W=1, f=1000.0, tile=4, min_t=0.0):
    M = np.eye(4, dtype=np.float32)
    M[:3, 3] = -np.asarray(pos, np.float32)
    K = np.array([[f, 0, W / 2], [0, f, H / 2], [0, 0, 1]], np.float32)
    return make_tcam(M, K, np.asarray(pos, np.float32), H, W, tile, min_t)


def _render(verts, idx, cv, tcam, prec="f64"):
    H, W = int(tcam["image_height"]), int(tcam["image_width"])
    jit = np.full((H, W, 2), 0.5, np.float32)
    L = O.rasterize_lists(idx, verts, tcam)
    if prec == "f32":
        return O.blend_fwd_f32(L, idx, verts, cv, jit), L
    img, dist, nc, own, inv = O.blend_fwd_f64(L, idx, verts.astype(np.float64), cv.astype(np.float64), jit)
    return (img, dist, nc), L


def test_single_tet_axis_ray_closed_form():
    # unit corner tet; the central ray x = y = 0.25 runs along +z, enters at
    # z = 0 and leaves through x + y + z = 1 at z = 0.5
    verts = np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0], [0, 0, 1]], np.float32)
    idx = np.array([[0, 1, 2, 3]], np.int32)
    sigma, base, g = 3.0, np.array([0.2, 0.4, 0.6]), 0.5
    cv = np.array([[sigma, *base, 0.0, 0.0, g]], np.float32)
    base = cv[0, 1:4].astype(np.float64)  # the float32-rounded inputs
    tcam = _axis_cam((0.25, 0.25, -2.0))
    (img, dist, nc), _ = _render(verts, idx, cv, tcam)
    Lseg = 0.5
    # colour along the ray is base + g*z on z in [0, L]:
    # C = int_0^L sigma (b + g z) e^{-sigma z} dz = b (1 - e^{-sL}) + g ((1 - e^{-sL})/s - L e^{-sL})
    e = math.exp(-sigma * Lseg)
    for k in range(3):
        expect = base[k] * (1 - e) + g * ((1 - e) / sigma - Lseg * e)
        assert abs(img[0, 0, k] - expect) < 1e-9
    assert abs(img[0, 0, 3] + sigma * Lseg) < 1e-12
    assert nc[0, 0] == 1
    # distortion moments of one segment: D2 = sigma, D3 = sigma*(a+b)/2, D4 = sigma^2 (b-a)/3
    a, b = 2.0, 2.0 + Lseg
    assert abs(dist[0, 0, 2] - sigma) < 1e-12
    assert abs(dist[0, 0, 3] - sigma * (a + b) / 2) < 1e-9
    assert abs(dist[0, 0, 4] - sigma * sigma * Lseg / 3) < 1e-12
    assert dist[0, 0, 0] == 0 and dist[0, 0, 1] == 0


def test_homogeneous_slab():
    # a cube split into tets with one density and one colour: C = c (1 - exp(-sigma L))
    rng = np.random.default_rng(4)
    g = np.linspace(-0.5, 0.5, 4)
    pts = np.stack(np.meshgrid(g, g, g, indexing="ij"), -1).reshape(-1, 3)
    pts = pts + rng.uniform(-1e-3, 1e-3, pts.shape) * (np.abs(pts) < 0.49)
    pts = pts.astype(np.float32)
    idx = delaunay(pts)
    sigma, c = 2.0, 0.7
    cv = np.tile(np.array([[sigma, c, c, c, 0, 0, 0]], np.float32), (len(idx), 1))
    tcam = _axis_cam((0.013, -0.021, -3.0), H=8, W=8, f=2000.0, tile=8)
    (img, dist, nc), L = _render(verts=pts, idx=idx, cv=cv, tcam=tcam)
    T = np.exp(img[..., 3])
    assert np.allclose(T, math.exp(-sigma * 1.0), atol=1e-9)
    assert np.allclose(img[..., :3], c * (1 - math.exp(-sigma)), atol=1e-9)
    (img32, _, _), _ = _render(pts, idx, cv, tcam, "f32")
    assert np.abs(img32[..., :3] - img[..., :3]).max() < 1e-5


def test_termination_cut():
    # a very dense slab terminates each pixel after the first few entries
    pts = np.array([[-1, -1, 0], [1, -1, 0], [0, 1, 0], [0, 0, 1], [0, 0, -1]], np.float32)
    idx = delaunay(pts)
    cv = np.tile(np.array([[50.0, 1, 1, 1, 0, 0, 0]], np.float32), (len(idx), 1))
    tcam = _axis_cam((0.05, -0.1, -4.0), H=4, W=4, f=400.0, tile=4)
    (img, dist, nc), L = _render(pts, idx, cv, tcam, "f32")
    assert img[..., 3].max() < -5.5
    assert (nc <= L["ranges"][0, 1] - L["ranges"][0, 0]).all()


@pytest.mark.parametrize("view", ["center", "face", "outside"])
def test_single_tet_matches_quadrature(view):
    verts, idx, cv, tcam = scenarios.single_tet(200 + len(view), view)
    cv = cv.copy()
    cv[:, 0] = 2.0  # keep the pixel above the termination threshold
    H, W = 32, 32
    jit = np.full((H, W, 2), 0.5, np.float32)
    L = O.rasterize_lists(idx, verts, tcam)
    v64, c64 = verts.astype(np.float64), cv.astype(np.float64)
    img, _, _, _, _ = O.blend_fwd_f64(L, idx, v64, c64, jit)
    q = O.quadrature_f64(L, idx, v64, c64, jit, 0.0, 4.0, 40001)
    assert np.abs(img[..., :3] - q[..., :3]).max() < 2e-3
    assert np.abs((1 - np.exp(img[..., 3])) - q[..., 3]).max() < 2e-3


@pytest.mark.parametrize("seed,view", [(3, "outside"), (4, "center")])
def test_multi_tet_matches_quadrature(seed, view):
    verts, idx, cv, tcam = scenarios.multi_tet(seed, 20, 10.0, view, 10.0)
    cv = cv.copy()
    cv[:, 0] = 0.05
    H, W = 16, 16
    jit = np.full((H, W, 2), 0.5, np.float32)
    L = O.rasterize_lists(idx, verts, tcam)
    v64, c64 = verts.astype(np.float64), cv.astype(np.float64)
    img, _, _, _, inv = O.blend_fwd_f64(L, idx, v64, c64, jit)
    assert inv == 0  # power order equals front-to-back order along every ray
    q = O.quadrature_f64(L, idx, v64, c64, jit, 0.0, 60.0, 60001)
    assert np.abs(img[..., :3] - q[..., :3]).max() < 2e-3
    assert np.abs((1 - np.exp(img[..., 3])) - q[..., 3]).max() < 2e-3


def test_sort_is_stable_on_masked_bits():
    rng = np.random.default_rng(0)
    keys = (rng.integers(0, 4, 5000).astype(np.int64) << 40) | rng.integers(0, 8, 5000).astype(np.int64)
    vals = np.arange(5000, dtype=np.int32)
    k, v = O.sort_pairs(keys, vals, 3)
    order = np.argsort(keys & 7, kind="stable")
    assert np.array_equal(v, vals[order]) and np.array_equal(k, keys[order])


def test_ranges_empty_tiles():
    keys = (np.array([1, 1, 3, 3, 3, 6], np.int64) << 32)
    r = O.tile_ranges(keys, 8)
    assert r.tolist() == [[0, 0], [0, 2], [0, 0], [2, 5], [0, 0], [0, 0], [5, 6], [0, 0]]


def test_ssim_map_properties():
    import torch

    from radiance_meshes_b200.ssim import ssim_map

    g = torch.Generator().manual_seed(0)
    a = torch.rand(3, 40, 50, generator=g)
    assert torch.allclose(ssim_map(a, a), torch.ones_like(a), atol=1e-6)
    b = (a + 0.1 * torch.randn(3, 40, 50, generator=g)).clamp(0, 1)
    m = ssim_map(a, b)
    assert m.shape == a.shape and float(m.mean()) < 0.99
    assert torch.allclose(m, ssim_map(b, a), atol=1e-6)  # symmetric
    # a constant image against itself shifted by a constant: mean term only
    c1 = torch.full((1, 30, 30), 0.3)
    c2 = torch.full((1, 30, 30), 0.5)
    inner = ssim_map(c1, c2)[0, 10:20, 10:20]
    expect = (2 * 0.3 * 0.5 + 1e-4) / (0.09 + 0.25 + 1e-4)
    assert torch.allclose(inner, torch.full_like(inner, expect), atol=1e-4)  # float32 variance residue


def test_oracle_calc_tet_err_basic():
    """Hit counts of calc_tet_err equal the hits the FP32 forward walk makes
    with its log T starting at 1 (termination at -5.5): on an optically thin
    scene every processed entry with a > 0 counts."""
    import numpy as np

    from oracle import oracle as O
    from radiance_meshes_b200 import scenes

    mesh, view = scenes.workload_gradient_check()
    cv = mesh.cell_values.copy()
    cv[:, 0] = 1e-3  # thin: no pixel terminates
    L = O.rasterize_lists(mesh.indices, mesh.vertices, view.tcam())
    pe = np.ones((view.height, view.width), np.float32)
    se = np.zeros((view.height, view.width), np.float32)
    err, cnt, tmax = O.calc_tet_err(L, mesh.indices, mesh.vertices, cv, pe, se)
    assert cnt.sum() > 0
    assert np.allclose(err[:, 0], err[:, 12]) and np.allclose(err[:, 0], err[:, 1])  # e = 1
    assert np.all(err[:, 5] == 0) and np.all(err[:, 2] == err[:, 1])
    assert np.all(tmax[cnt == 0] == 0)
