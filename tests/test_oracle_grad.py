"""The oracle's hand-derived adjoint (the reference gets it from Slang autodiff)
against FP64 central finite differences.

Protocol of the gradient-check workload: 2,000 points in the unit ball,
densities log-normal(0, 2), 128x128 camera, L1 loss against a uniform random
target, 256 randomly chosen parameters (vertex coordinates, density, base RGB
and colour gradient), central differences with h = 1e-4 on the FP64 forward
(fixed tile lists and per-pixel list cut, which the adjoint treats as
constants).  The L1 loss is evaluated as the linear functional with weights
sign(image - target) / N, its exact local form.  A parameter whose one-sided
differences disagree is a kink inside +-h (a ray crossing a tet edge or a
near-degenerate tet flipping); it is re-checked with h = 1e-6 and, if still
inconsistent, listed as a kink instead of being scored.
"""
import numpy as np

from oracle import oracle as O
from radiance_meshes_b200 import scenes


def _setup():
    mesh, view = scenes.workload_gradient_check()
    tcam = view.tcam()
    L = O.rasterize_lists(mesh.indices, mesh.vertices, tcam)
    H, W = view.height, view.width
    jitter = np.random.default_rng(1).uniform(0, 1, (H, W, 2)).astype(np.float32)
    img32, _, nc = O.blend_fwd_f32(L, mesh.indices, mesh.vertices, mesh.cell_values, jitter)
    v64, c64 = mesh.vertices.astype(np.float64), mesh.cell_values.astype(np.float64)
    img64, dist64, _, own, _ = O.blend_fwd_f64(L, mesh.indices, v64, c64, jitter, cut=nc)
    target = np.random.default_rng(1).uniform(size=(H, W, 3))
    wimg = np.zeros((H, W, 4))
    wimg[..., :3] = np.sign(img64[..., :3] - target) / (H * W * 3)
    return mesh, L, jitter, nc, v64, c64, img64, dist64, wimg


def _tile_mask(L, tets):
    gw, gh = L["cam"].grid_width, L["cam"].grid_height
    m = np.zeros(gw * gh, np.uint8)
    for g in tets:
        r = L["rect"][g]
        for y in range(r[1], r[3]):
            m[y * gw + r[0]: y * gw + r[2]] = 1
    return m


def test_adjoint_matches_central_differences():
    mesh, L, jitter, nc, v64, c64, img64, dist64, wimg = _setup()
    gv, gc = O.blend_bwd(L, mesh.indices, v64, c64, jitter, img64, dist64, nc, wimg, None, "f64")
    vis = np.nonzero(L["tiles_touched"] > 0)[0]
    v2t = {}
    for g in vis:
        for vi in mesh.indices[g]:
            v2t.setdefault(int(vi), []).append(int(g))
    rng = np.random.default_rng(1)
    verts = rng.choice(sorted(v2t), size=128, replace=False)
    tets = rng.choice(vis, size=128, replace=False)
    params = [("v", int(v), int(rng.integers(0, 3))) for v in verts]
    params += [("c", int(g), int(rng.integers(0, 7))) for g in tets]

    def loss(V, C, mask):
        return O.linear_loss_f64(L, mesh.indices, V, C, jitter, nc, wimg, None, mask)

    rel, kinks = [], []
    for kind, idx, comp in params:
        mask = _tile_mask(L, v2t[idx] if kind == "v" else [idx])
        analytic = gv[idx, comp] if kind == "v" else gc[idx, comp]
        ok = False
        for h in (1e-4, 1e-6):
            V, C = v64, c64
            if kind == "v":
                Vp, Vm = v64.copy(), v64.copy()
                Vp[idx, comp] += h
                Vm[idx, comp] -= h
                lp, l0, lm = loss(Vp, C, mask), loss(V, C, mask), loss(Vm, C, mask)
            else:
                Cp, Cm = c64.copy(), c64.copy()
                Cp[idx, comp] += h
                Cm[idx, comp] -= h
                lp, l0, lm = loss(V, Cp, mask), loss(V, C, mask), loss(V, Cm, mask)
            fwd, bwd = (lp - l0) / h, (l0 - lm) / h
            if abs(fwd - bwd) <= 1e-2 * max(abs(fwd), abs(bwd)) + 1e-9:
                fd = (lp - lm) / (2 * h)
                rel.append(abs(fd - analytic) / max(abs(fd), abs(analytic), 1e-9))
                ok = True
                break
        if not ok:
            kinks.append((kind, idx, comp))
    rel = np.array(rel)
    print(f"scored {len(rel)} of {len(params)}; kinks {len(kinks)}; median rel {np.median(rel):.2e}; "
          f"p95 {np.quantile(rel, 0.95):.2e}; max {rel.max():.2e}")
    assert len(kinks) <= 0.05 * len(params)
    assert np.median(rel) < 1e-5
    assert np.quantile(rel, 0.95) < 1e-3


def test_projection_adjoint_matches_central_differences():
    mesh, view = scenes.workload_gradient_check()
    cs = O.camstruct(view.tcam())
    tiles, _, _, _ = O.project(mesh.indices, mesh.vertices, cs)
    vis = np.nonzero(tiles > 0)[0][:400]
    idx = mesh.indices[vis]
    rng = np.random.default_rng(2)
    gvs = np.zeros((len(mesh.indices), 3), np.float32)
    gcc = np.zeros((len(mesh.indices), 3), np.float32)
    gvs[vis, 2] = rng.normal(size=len(vis))
    gcc[vis] = rng.normal(size=(len(vis), 3))
    gv = O.project_bwd(mesh.indices, mesh.vertices, cs, tiles, gvs, gcc)
    v64 = mesh.vertices.astype(np.float64)
    P = np.array(cs.cam_pos[:], np.float64)

    def L(V):
        p, c = O.power_f64(idx, V, P)
        return float((p * gvs[vis, 2]).sum() + (c * gcc[vis]).sum())

    used = np.unique(idx)
    errs = []
    for vi in rng.choice(used, size=40, replace=False):
        for comp in range(3):
            h = 1e-6 * max(1.0, abs(v64[vi, comp]))
            Vp, Vm = v64.copy(), v64.copy()
            Vp[vi, comp] += h
            Vm[vi, comp] -= h
            fd = (L(Vp) - L(Vm)) / (2 * h)
            errs.append(abs(fd - gv[vi, comp]) / max(abs(fd), abs(gv[vi, comp]), 1e-6))
    assert np.median(errs) < 1e-6
    assert np.quantile(errs, 0.95) < 1e-4
