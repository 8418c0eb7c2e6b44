"""Host orchestration of the rasterizer stages over the C ABI.

Each function launches the sm_100a kernels of ``librm_b200.so`` on the current
torch CUDA stream.  Tensors must live on a CUDA device; there is no CPU path.

Stage map (reference file:line in delaunay_rasterization/internal/):
  project_fwd / project_bwd   vertex_shader / vertex_shader.bwd (tile_shader_slang.py:75-150)
  build_tile_lists            cumsum + generate_keys + sort_by_keys + compute_tile_ranges
                              (tile_shader_slang.py:24-72)
  blend_fwd / blend_bwd       splat_tiled / splat_tiled.bwd (alphablend_tiled_slang_interp.py:9-112)
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass

import torch

from . import _capi as C
from .camera import RMCamera, tcam_to_struct

__all__ = [
    "ScratchPool",
    "TileLists",
    "project_fwd",
    "project_bwd",
    "build_tile_lists",
    "blend_fwd",
    "blend_bwd",
    "end_bit_for",
    "read_status",
]


def _require_cuda(**tensors):
    for name, t in tensors.items():
        if t is not None and not t.is_cuda:
            raise RuntimeError(f"{name} must be a CUDA tensor (the rasterizer has no CPU path)")


def _i32(t):
    return t if (t.dtype == torch.int32 and t.is_contiguous()) else t.to(torch.int32).contiguous()


def _f32(t):
    return t if (t.dtype == torch.float32 and t.is_contiguous()) else t.to(torch.float32).contiguous()


class ScratchPool:
    """Grow-only device scratch buffers, one set per (device, name).

    Callers allocate scratch ("workspace") for the C ABI; the pool keeps it
    between calls so steady-state rendering allocates nothing new.
    """

    def __init__(self):
        self._bufs = {}

    def get(self, name: str, nbytes: int, device) -> torch.Tensor:
        key = (str(device), name)
        buf = self._bufs.get(key)
        if buf is None or buf.numel() < nbytes:
            buf = torch.empty(max(int(nbytes), 256), dtype=torch.uint8, device=device)
            self._bufs[key] = buf
        return buf

    def clear(self):
        self._bufs.clear()


_POOL = ScratchPool()


def default_pool() -> ScratchPool:
    return _POOL


def end_bit_for(grid_w: int, grid_h: int) -> int:
    """32 + bit_length(grid_w * grid_h), as in tile_shader_slang.py:57-59."""
    return 32 + int(grid_w * grid_h).bit_length()


@dataclass
class TileLists:
    sorted_ids: torch.Tensor  # [P] int32
    ranges: torch.Tensor  # [G, 2] int32
    n_pairs: int
    offsets: torch.Tensor | None = None  # [T] inclusive scan
    keys: torch.Tensor | None = None  # [P] emission order
    values: torch.Tensor | None = None
    sorted_keys: torch.Tensor | None = None


def _stream():
    return C.stream_handle()


class StageTimer:
    """Records a CUDA event pair around every C-ABI call on the launching
    (current) stream while active; ``totals()`` returns milliseconds per stage."""

    def __init__(self):
        self.events = []

    def __enter__(self):
        global _TIMER
        _TIMER = self
        return self

    def __exit__(self, *exc):
        global _TIMER
        _TIMER = None

    def record(self, name, fn):
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record()
        rc = fn()
        b.record()
        self.events.append((name, a, b))
        return rc

    def totals(self):
        torch.cuda.synchronize()
        out = {}
        for name, a, b in self.events:
            out.setdefault(name, [0.0, 0])
            out[name][0] += a.elapsed_time(b)
            out[name][1] += 1
        return out


_TIMER: StageTimer | None = None


def _call(name, fn):
    if _TIMER is None:
        rc = fn()
    else:
        rc = _TIMER.record(name, fn)
    C.check(rc, name)


def project_fwd(indices: torch.Tensor, vertices: torch.Tensor, cam: RMCamera):
    _require_cuda(indices=indices, vertices=vertices)
    indices = _i32(indices)
    vertices = _f32(vertices)
    T = indices.shape[0]
    dev = vertices.device
    tiles = torch.empty(T, dtype=torch.int32, device=dev)
    rect = torch.empty((T, 4), dtype=torch.int32, device=dev)
    vs = torch.empty((T, 3), dtype=torch.float32, device=dev)
    cc = torch.empty((T, 3), dtype=torch.float32, device=dev)
    _call("rm_project_fwd", lambda: C.lib().rm_project_fwd(C.ptr(indices), C.ptr(vertices), T, vertices.shape[0], ctypes.byref(cam),
                                   C.ptr(tiles), C.ptr(rect), C.ptr(vs), C.ptr(cc), _stream()))
    return tiles, rect, vs, cc


def project_bwd(indices, vertices, cam: RMCamera, tiles, grad_vs, grad_cc, grad_vertices=None):
    indices = _i32(indices)
    vertices = _f32(vertices)
    if grad_vertices is None:
        grad_vertices = torch.zeros_like(vertices)
    gvs = None if grad_vs is None else _f32(grad_vs)
    gcc = None if grad_cc is None else _f32(grad_cc)
    _call("rm_project_bwd", lambda: C.lib().rm_project_bwd(C.ptr(indices), C.ptr(vertices), indices.shape[0], vertices.shape[0],
                                   ctypes.byref(cam), C.ptr(tiles), C.ptr(gvs), C.ptr(gcc), C.ptr(grad_vertices),
                                   _stream()))
    return grad_vertices


def build_tile_lists(tiles: torch.Tensor, rect: torch.Tensor, vs: torch.Tensor, cam: RMCamera,
                     pool: ScratchPool | None = None, keep_debug: bool = False) -> TileLists:
    """Scan, emit, sort and range the tile/tet pairs.

    The pair count P is read back to the host once (the reference reads it
    three times: tile_shader_slang.py:38-44,68)."""
    pool = pool or _POOL
    dev = tiles.device
    T = tiles.shape[0]
    G = cam.grid_width * cam.grid_height
    L = C.lib()
    s = _stream()
    offsets = torch.empty(T, dtype=torch.int32, device=dev)
    total = torch.zeros(1, dtype=torch.int64, device=dev)
    ws_n = L.rm_scan_workspace_size(T)
    ws = pool.get("scan", ws_n, dev)
    _call("rm_scan_tiles", lambda: L.rm_scan_tiles(C.ptr(tiles), T, C.ptr(offsets), C.ptr(total), C.ptr(ws), ws_n, s))
    P = int(total.item())
    keys = torch.empty(P, dtype=torch.int64, device=dev)
    vals = torch.empty(P, dtype=torch.int32, device=dev)
    _call("rm_emit_pairs", lambda: L.rm_emit_pairs(C.ptr(vs), C.ptr(rect), C.ptr(offsets), T, cam.grid_width, P, None, C.ptr(keys),
                            C.ptr(vals), None, s))
    sk = torch.empty(P, dtype=torch.int64, device=dev)
    sv = torch.empty(P, dtype=torch.int32, device=dev)
    if P > 0:
        ws_n = L.rm_sort_workspace_size(P)
        ws = pool.get("sort", ws_n, dev)
        _call("rm_sort_pairs", lambda: L.rm_sort_pairs(C.ptr(keys), C.ptr(vals), P, None, end_bit_for(cam.grid_width, cam.grid_height),
                                C.ptr(sk), C.ptr(sv), C.ptr(ws), ws_n, s))
    ranges = torch.empty((G, 2), dtype=torch.int32, device=dev)
    _call("rm_tile_ranges", lambda: L.rm_tile_ranges(C.ptr(sk), P, None, C.ptr(ranges), G, s))
    if keep_debug:
        return TileLists(sv, ranges, P, offsets, keys, vals, sk)
    return TileLists(sv, ranges, P)


_BLEND_FLAGS = {"fwd": 0, "bwd": 0}


def set_blend_tuning(fwd_flags: int = 0, bwd_flags: int = 0) -> None:
    """Launch tunables (RM_BLEND_STRIP / HEAVY / PAIR_CTAS bits of the flags
    word) used by blend_fwd / blend_bwd; 0 selects the built-in defaults."""
    _BLEND_FLAGS["fwd"] = int(fwd_flags)
    _BLEND_FLAGS["bwd"] = int(bwd_flags)


def blend_tuning() -> tuple[int, int]:
    return _BLEND_FLAGS["fwd"], _BLEND_FLAGS["bwd"]


def blend_fwd(sorted_ids, ranges, indices, vertices, cell_values, ray_jitter, cam: RMCamera,
              tiles_touched=None, records: torch.Tensor | None = None, reuse_records: bool = False):
    _require_cuda(sorted_ids=sorted_ids, ranges=ranges, indices=indices, vertices=vertices,
                  cell_values=cell_values, ray_jitter=ray_jitter)
    indices = _i32(indices)
    vertices = _f32(vertices)
    cell_values = _f32(cell_values)
    ray_jitter = _f32(ray_jitter)
    H, W = cam.image_height, cam.image_width
    dev = vertices.device
    T = indices.shape[0]
    L = C.lib()
    ws_n = L.rm_blend_workspace_size(T, cam.grid_width * cam.grid_height)
    if records is None:
        records = torch.empty(ws_n, dtype=torch.uint8, device=dev)
    img = torch.empty((H, W, 4), dtype=torch.float32, device=dev)
    dist = torch.empty((H, W, 5), dtype=torch.float32, device=dev)
    nc = torch.empty((H, W, 1), dtype=torch.int32, device=dev)
    flags = (C.RM_BLEND_REUSE_RECORDS if reuse_records else 0) | _BLEND_FLAGS["fwd"]
    _call("rm_blend_fwd", lambda: L.rm_blend_fwd(C.ptr(sorted_ids), C.ptr(ranges), C.ptr(indices), C.ptr(vertices), C.ptr(cell_values),
                           T, vertices.shape[0], C.ptr(tiles_touched), C.ptr(ray_jitter), ctypes.byref(cam),
                           C.ptr(img), C.ptr(dist), C.ptr(nc), C.ptr(records), records.numel(), flags, _stream()))
    return img, dist, nc, records


def blend_bwd(sorted_ids, ranges, indices, vertices, cell_values, ray_jitter, cam: RMCamera, img, dist, nc,
              grad_img, grad_dist, records, tiles_touched=None, reuse_records=True,
              grad_vertices=None, grad_cell_values=None):
    indices = _i32(indices)
    vertices = _f32(vertices)
    cell_values = _f32(cell_values)
    ray_jitter = _f32(ray_jitter)
    if grad_img is None:
        grad_img = torch.zeros_like(img)
    grad_img = _f32(grad_img)
    gd = None if grad_dist is None else _f32(grad_dist)
    if grad_vertices is None:
        grad_vertices = torch.zeros_like(vertices)
    if grad_cell_values is None:
        grad_cell_values = torch.zeros_like(cell_values)
    T = indices.shape[0]
    flags = (C.RM_BLEND_REUSE_RECORDS if reuse_records else 0) | _BLEND_FLAGS["bwd"]
    _call("rm_blend_bwd", lambda: C.lib().rm_blend_bwd(C.ptr(sorted_ids), C.ptr(ranges), C.ptr(indices), C.ptr(vertices),
                                 C.ptr(cell_values), T, vertices.shape[0], C.ptr(tiles_touched), C.ptr(ray_jitter),
                                 ctypes.byref(cam), C.ptr(img), C.ptr(dist), C.ptr(nc), C.ptr(grad_img), C.ptr(gd),
                                 C.ptr(grad_vertices), C.ptr(grad_cell_values), C.ptr(records), records.numel(),
                                 flags, _stream()))
    return grad_vertices, grad_cell_values


def read_status(workspace: torch.Tensor) -> int:
    """Read and clear the device status word at the start of a scan/sort workspace."""
    out = ctypes.c_uint32(0)
    C.check(C.lib().rm_read_status(C.ptr(workspace), ctypes.byref(out), _stream()), "rm_read_status")
    return int(out.value)


def camera(tcam: dict) -> RMCamera:
    return tcam_to_struct(tcam)
