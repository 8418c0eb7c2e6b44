"""The Delaunay update of the mesh: the reference's update_triangulation
(models/ingp_color.py:523-558).

``update_triangulation(vertices, high_precision=True, density_fn=None,
density_threshold=0.0, alpha_threshold=0.0)`` tetrahedralises the vertices
with scipy's Delaunay (the reference's high-precision mode, :526-527; its
default mode calls gDel3D, a GPU Delaunay library that the reference does not
vendor), then on the GPU drops rows naming a vertex outside the mesh, flips
negatively oriented tets (``rm_tets_orient``) and, given a per-tet density,
splits off the empty tets (``rm_tets_cull``).  Returns ``(indices,
empty_indices)`` as int32 CUDA tensors, like the model's ``indices`` and
``empty_indices``.
"""
from __future__ import annotations

import torch

from . import _capi as C
from . import rasterizer as R

__all__ = ["tetrahedralize", "orient_tets", "cull_tets", "update_triangulation"]


def tetrahedralize(vertices: torch.Tensor):
    """scipy's Delaunay of the vertices (host), as int32 simplices."""
    import numpy as np
    from scipy.spatial import Delaunay

    pts = vertices.detach().to("cpu", torch.float64).numpy()
    return torch.from_numpy(Delaunay(pts).simplices.astype(np.int32))


def _status(dev):
    return torch.zeros(1, dtype=torch.int32, device=dev)


def _raise(status, where):
    bits = int(status.item()) & 0xffffffff
    if bits:
        raise C.DeviceStatusError(bits, where)


def orient_tets(indices: torch.Tensor, vertices: torch.Tensor) -> torch.Tensor:
    """Rows with every index in [0, V), positively oriented (vertices 0 and 1
    swapped where det(v1 - v0, v2 - v0, v3 - v0) < 0), in input order."""
    R._require_cuda(indices=indices, vertices=vertices)
    idx = R._i32(indices)
    v = R._f32(vertices)
    T, dev = idx.shape[0], v.device
    L = C.lib()
    out = torch.empty((T, 4), dtype=torch.int32, device=dev)
    n = torch.zeros(1, dtype=torch.int64, device=dev)
    ws_n = L.rm_tets_workspace_size(T)
    ws = torch.empty(max(ws_n, 256), dtype=torch.uint8, device=dev)
    st = _status(dev)
    R._call("rm_tets_orient", lambda: L.rm_tets_orient(C.ptr(idx), T, C.ptr(v), v.shape[0], C.ptr(out), C.ptr(n),
                                                       C.ptr(ws), ws.numel(), C.ptr(st), R._stream()))
    _raise(st, "orient_tets")
    return out[:int(n.item())]


def cull_tets(indices: torch.Tensor, vertices: torch.Tensor, density: torch.Tensor, density_threshold: float,
              alpha_threshold: float):
    """(kept, empty): tets with density > density_threshold or
    1 - exp(-density * shortest edge) > alpha_threshold, and the rest, each in
    input order."""
    R._require_cuda(indices=indices, vertices=vertices, density=density)
    idx = R._i32(indices)
    v = R._f32(vertices)
    d = R._f32(density.reshape(-1))
    T, dev = idx.shape[0], v.device
    if d.shape[0] != T:
        raise ValueError("one density per tet")
    L = C.lib()
    kept = torch.empty((T, 4), dtype=torch.int32, device=dev)
    empty = torch.empty((T, 4), dtype=torch.int32, device=dev)
    n = torch.zeros(1, dtype=torch.int64, device=dev)
    ws_n = L.rm_tets_workspace_size(T)
    ws = torch.empty(max(ws_n, 256), dtype=torch.uint8, device=dev)
    st = _status(dev)
    R._call("rm_tets_cull", lambda: L.rm_tets_cull(C.ptr(idx), T, C.ptr(v), v.shape[0], C.ptr(d),
                                                   float(density_threshold), float(alpha_threshold), C.ptr(kept),
                                                   C.ptr(empty), C.ptr(n), C.ptr(ws), ws.numel(), C.ptr(st),
                                                   R._stream()))
    _raise(st, "cull_tets")
    k = int(n.item())
    return kept[:k], empty[:T - k]


def update_triangulation(vertices: torch.Tensor, density_fn=None, density_threshold: float = 0.0,
                         alpha_threshold: float = 0.0):
    """(indices, empty_indices) of a new tetrahedralisation of ``vertices``
    (update_triangulation, models/ingp_color.py:523-558, high-precision
    mode).  density_fn(indices) -> per-tet density is called, as the
    reference calls calc_tet_density, only when a threshold is positive."""
    raw = tetrahedralize(vertices).to(vertices.device)
    indices = orient_tets(raw, vertices)
    if density_threshold > 0 or alpha_threshold > 0:
        if density_fn is None:
            raise ValueError("culling needs density_fn")
        return cull_tets(indices, vertices, density_fn(indices), density_threshold, alpha_threshold)
    return indices, torch.empty((0, 4), dtype=indices.dtype, device=indices.device)
