"""The Delaunay update's GPU steps (rm_tets_orient, rm_tets_cull) against the
reference's own formulas, restated in torch on the same device: the
orientation flip of update_triangulation (models/ingp_color.py:538-542, with
topo_utils.tet_volumes = det(v1 - v0, v2 - v0, v3 - v0) / 6) and the
density / alpha culling (:548-554, calc_tet_alpha(mode="min"),
models/base_model.py:82-105), on scipy tetrahedralisations of the
plain-forward (4,096 uniform points, seed 0) and gradient-check (2,000 points
in a ball, seed 1) point sets.  Rows naming a vertex outside the mesh (gDel3D's
point at infinity) are dropped, the rest keep their order."""
import numpy as np
import pytest
import torch

from radiance_meshes_b200 import _capi as C
from radiance_meshes_b200 import delaunay as D
from radiance_meshes_b200 import scenes

pytestmark = pytest.mark.gpu


def _points(name):
    if name == "plain_forward":
        return np.random.default_rng(0).uniform(-1, 1, (4096, 3)).astype(np.float32)
    mesh, _ = scenes.workload_gradient_check()
    return mesh.vertices


def _reference_orient(indices, verts):
    """update_triangulation's flip, as the reference writes it."""
    keep = (indices < verts.shape[0]).all(dim=1)
    indices = indices[keep].clone()
    tets = verts[indices.long()]
    a, b, c = tets[:, 1] - tets[:, 0], tets[:, 2] - tets[:, 0], tets[:, 3] - tets[:, 0]
    vols = torch.det(torch.stack((a, b, c), dim=1)) / 6.0
    rev = vols < 0
    indices[rev] = indices[rev][:, [1, 0, 2, 3]]
    return indices, vols


@pytest.mark.parametrize("name", ["plain_forward", "gradient_check"])
def test_orient_matches_reference_flip(cuda, name):
    pts = torch.from_numpy(_points(name)).cuda()
    raw = D.tetrahedralize(pts).cuda()
    # rows naming the point at infinity (index V), as gDel3D returns them, interleaved
    V = pts.shape[0]
    bad = raw[:7].clone()
    bad[:, 2] = V
    mixed = torch.cat([raw[:100], bad, raw[100:]])
    ours = D.orient_tets(mixed, pts)
    ref, vols = _reference_orient(mixed, pts)
    assert ours.shape == ref.shape == raw.shape
    differ = (ours != ref).any(dim=1)
    # a different sign can only come from a volume at float32 rounding level
    if differ.any():
        scale = (pts.max() - pts.min()).item() ** 3
        assert (vols[differ].abs() < 1e-6 * scale).all()
    assert int(differ.sum()) <= 2
    # every kept tet now has a non-negative volume in double precision
    t = pts.double()[ours.long()]
    vol = torch.det(torch.stack((t[:, 1] - t[:, 0], t[:, 2] - t[:, 0], t[:, 3] - t[:, 0]), dim=1))
    assert (vol >= 0).all()


@pytest.mark.parametrize("name", ["plain_forward", "gradient_check"])
def test_cull_matches_reference_mask(cuda, name):
    pts = torch.from_numpy(_points(name)).cuda()
    indices = D.orient_tets(D.tetrahedralize(pts).cuda(), pts)
    T = indices.shape[0]
    g = torch.Generator(device="cuda").manual_seed(3)
    density = torch.exp(torch.randn(T, device="cuda", generator=g) * 2.0 - 1.0)
    for d_thr, a_thr in ((0.5, 0.0), (0.0, 0.05), (2.0, 0.1)):
        kept, empty = D.cull_tets(indices, pts, density, d_thr, a_thr)
        v = pts[indices.long()]
        el = torch.stack([torch.norm(v[:, i] - v[:, j], dim=1)
                          for i, j in ((0, 1), (0, 2), (0, 3), (1, 2), (1, 3), (2, 3))], dim=0).min(dim=0)[0]
        alpha = 1 - torch.exp(-density * el)
        mask = (density > d_thr) | (alpha > a_thr)
        assert torch.equal(kept, indices[mask]) and torch.equal(empty, indices[~mask])


def test_cull_reports_bad_index(cuda):
    pts = torch.from_numpy(_points("gradient_check")).cuda()
    indices = D.orient_tets(D.tetrahedralize(pts).cuda(), pts)
    bad = indices.clone()
    bad[3, 1] = pts.shape[0] + 5
    with pytest.raises(C.DeviceStatusError) as ei:
        D.cull_tets(bad, pts, torch.ones(bad.shape[0], device="cuda"), 0.5, 0.0)
    assert ei.value.bits == C.RM_STATUS_BAD_INDEX


def test_update_triangulation_end_to_end(cuda):
    pts = torch.from_numpy(_points("gradient_check")).cuda()
    indices, empty = D.update_triangulation(pts)
    assert empty.shape == (0, 4) and indices.dtype == torch.int32
    ref, _ = _reference_orient(D.tetrahedralize(pts).cuda(), pts)
    assert torch.equal(indices, ref)
    dens = lambda idx: torch.full((idx.shape[0],), 0.3, device="cuda")
    kept, empty = D.update_triangulation(pts, density_fn=dens, density_threshold=0.5)
    assert kept.shape[0] + empty.shape[0] == indices.shape[0]
