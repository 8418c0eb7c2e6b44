"""Batched multi-view rendering: many cameras of one mesh, one launch per stage.

The reference renders one camera per call (``utils/train_util.py:15-77``);
a multi-view step there is N independent passes of
``vertex_and_tile_shader`` + ``AlphaBlendTiledRender``, each with its own
host synchronisations.  Here a batch of up to ``RM_MAX_VIEWS`` cameras runs as:

  rm_project_fwd_multi   every tet projected into every view (vertices read once)
  rm_scan_tiles          one scan over the stacked [n_views * T] tile counts
  rm_emit_pairs_multi    pairs keyed by a global, view-major tile id
  rm_sort_pairs          one radix sort over all views' pairs
  rm_tile_ranges         ranges over the global tiles
  rm_blend_fwd_multi     one persistent launch over all views' tiles
  rm_blend_bwd_multi     its adjoint, gradients summed over the views

Pair buffers have a fixed capacity, and the sort and ranges read the true
pair count from the device, so a frame needs no host synchronisation and the
whole sequence can be captured once in a CUDA graph and replayed.  A frame
whose pairs exceed the capacity sets ``RM_STATUS_CAPACITY``; ``check()``
reads that flag and ``ensure_capacity()`` grows the buffers.

Per view, the results equal the single-camera path's bit for bit (the image,
log T, distortion moments and n_contributors); gradients are the sum of the
per-view gradients up to floating-point summation order.
"""
from __future__ import annotations

from typing import Sequence

import torch

from . import _capi as C
from . import rasterizer as R
from .camera import RMCamera

__all__ = ["ViewBatch", "BatchedRasterizer", "MAX_VIEWS"]

MAX_VIEWS = 32


class ViewBatch:
    """Cameras of one batch (same tile size) and the derived offsets."""

    def __init__(self, cams: Sequence[RMCamera]):
        cams = list(cams)
        if not 1 <= len(cams) <= MAX_VIEWS:
            raise ValueError(f"a batch holds 1..{MAX_VIEWS} views, got {len(cams)}")
        t0 = (cams[0].tile_height, cams[0].tile_width)
        for c in cams:
            if (c.tile_height, c.tile_width) != t0:
                raise ValueError("all views of a batch must share one tile size")
        self.cams = cams
        self.n = len(cams)
        self.array = (RMCamera * self.n)(*cams)
        self.hw = [(c.image_height, c.image_width) for c in cams]
        self.grid = [(c.grid_height, c.grid_width) for c in cams]
        self.tile_base = [0]
        self.pixel_base = [0]
        for (gh, gw), (h, w) in zip(self.grid, self.hw):
            self.tile_base.append(self.tile_base[-1] + gh * gw)
            self.pixel_base.append(self.pixel_base[-1] + h * w)
        self.n_tiles = self.tile_base[-1]
        self.n_pixels = self.pixel_base[-1]
        self.end_bit = 32 + int(self.n_tiles).bit_length()

    def split(self, flat: torch.Tensor) -> list[torch.Tensor]:
        """Per-view [H, W, ...] views of a concatenated [n_pixels, ...] buffer."""
        out = []
        for v, (h, w) in enumerate(self.hw):
            a, b = self.pixel_base[v], self.pixel_base[v + 1]
            out.append(flat[a:b].view(h, w, *flat.shape[1:]))
        return out


class BatchedRasterizer:
    """Renders a ViewBatch of one mesh; forward, backward and a capturable
    fwd+bwd step.

    ``indices`` [T,4] int32, ``vertices`` [V,3] and ``cell_values`` [T,7]
    float32 stay owned by the caller and are read in place on every frame
    (update them with ``copy_`` to render new parameters).  ``jitter`` is the
    concatenated per-pixel ray jitter [n_pixels, 2] (default 0.5).
    """

    def __init__(self, indices: torch.Tensor, vertices: torch.Tensor, cell_values: torch.Tensor,
                 views: ViewBatch, jitter: torch.Tensor | None = None, capacity: int | None = None,
                 fwd_flags: int = 0, bwd_flags: int = 0, records: torch.Tensor | None = None,
                 hit_masks: bool = True, fine_shift: int = 0):
        for name, t in (("indices", indices), ("vertices", vertices), ("cell_values", cell_values)):
            if not t.is_cuda:
                raise RuntimeError(f"{name} must be a CUDA tensor (the rasterizer has no CPU path)")
        if indices.dtype != torch.int32 or not indices.is_contiguous():
            raise ValueError("indices must be contiguous int32")
        if vertices.dtype != torch.float32 or cell_values.dtype != torch.float32:
            raise ValueError("vertices and cell_values must be float32")
        self.indices, self.vertices, self.cell_values = indices, vertices, cell_values
        self.views = views
        # fine_shift > 0: lists are sorted on the cameras' tiles, then split in
        # order into the lists of tiles 2^fine_shift times smaller, which the
        # blend walks (same images; cheaper than sorting at the small tiles)
        self.fine_shift = int(fine_shift)
        self.blend_views = ViewBatch([R.fine_camera(c, self.fine_shift) for c in views.cams]) \
            if self.fine_shift else views
        self.fwd_flags, self.bwd_flags = int(fwd_flags), int(bwd_flags)
        # hit masks (RM_BLEND_HIT_MASKS): the forward records its hits so the
        # backward skips the misses; forward-only users turn them off
        self.hit_masks = bool(hit_masks)
        dev = vertices.device
        self.device = dev
        T, n = indices.shape[0], views.n
        self.T, self.V = T, vertices.shape[0]
        L = C.lib()
        self.tiles = torch.empty(n * T, dtype=torch.int32, device=dev)
        self.rect = torch.empty((n * T, 4), dtype=torch.int32, device=dev)
        self.depth = torch.empty(n * T, dtype=torch.float32, device=dev)
        self.tiles_any = torch.empty(T, dtype=torch.int32, device=dev)
        self.offsets = torch.empty(n * T, dtype=torch.int32, device=dev)
        self.total = torch.zeros(1, dtype=torch.int64, device=dev)
        self.status = torch.zeros(1, dtype=torch.int32, device=dev)
        # zeroed: its first word is the scan's status word, which the scan keeps
        self.scan_ws = torch.zeros(L.rm_scan_workspace_size(n * T), dtype=torch.uint8, device=dev)
        self.ranges = torch.empty((views.n_tiles, 2), dtype=torch.int32, device=dev)
        # records: per-tet blend records packed once per mesh (rm_blend_pack_records), shared by
        # every batch on it; without them each forward packs its own into the workspace
        self.records = records
        ws_tets = 0 if records is not None else T
        bv = self.blend_views
        self._ws_base = int(L.rm_blend_workspace_size(ws_tets, bv.n_tiles))
        if self.fine_shift:
            self.footprint = torch.empty((n * T, 12), dtype=torch.float32, device=dev)
            self.jitter_bounds = torch.empty(4, dtype=torch.float32, device=dev)
            self.jitter_ws = torch.empty(L.rm_jitter_bounds_workspace_size(), dtype=torch.uint8, device=dev)
            self.fine_ranges = torch.empty((bv.n_tiles, 2), dtype=torch.int32, device=dev)
            self.fine_total = torch.zeros(1, dtype=torch.int64, device=dev)
        self.blend_ws = None  # sized with the pair capacity (hit masks) in _alloc_pairs
        Npx = views.n_pixels
        self.jitter = jitter if jitter is not None else torch.full((Npx, 2), 0.5, device=dev)
        self.img = torch.empty((Npx, 4), dtype=torch.float32, device=dev)
        self.dist = torch.empty((Npx, 5), dtype=torch.float32, device=dev)
        self.nc = torch.empty(Npx, dtype=torch.int32, device=dev)
        self._grads = None  # (grad_img, grad_vertices, grad_cell_values), allocated on first use
        self.grad_dist = None
        self.capacity = 0
        self.graph = None
        if capacity is None:
            capacity = self.measure_pairs()
            capacity = int(capacity * 1.05) + 4096
        self._alloc_pairs(capacity)

    # ------------------------------------------------------------ buffers --
    def _grad_bufs(self):
        if self._grads is None:
            self._grads = (torch.zeros((self.views.n_pixels, 4), dtype=torch.float32, device=self.device),
                           torch.zeros_like(self.vertices), torch.zeros_like(self.cell_values))
        return self._grads

    @property
    def grad_img(self):
        return self._grad_bufs()[0]

    @property
    def grad_vertices(self):
        return self._grad_bufs()[1]

    @property
    def grad_cell_values(self):
        return self._grad_bufs()[2]

    def _alloc_pairs(self, capacity: int):
        capacity = max(int(capacity), 1)
        dev = self.device
        self.capacity = capacity
        self.keys = torch.empty(capacity, dtype=torch.int64, device=dev)
        self.vals = torch.empty(capacity, dtype=torch.int32, device=dev)
        self.sorted_keys = torch.empty(capacity, dtype=torch.int64, device=dev)
        self.sorted_ids = torch.empty(capacity, dtype=torch.int32, device=dev)
        self.sort_ws = torch.empty(C.lib().rm_sort_workspace_size(capacity), dtype=torch.uint8, device=dev)
        blend_pairs = capacity
        if self.fine_shift:
            blend_pairs = capacity << (2 * self.fine_shift)  # a coarse entry splits into at most 4^s
            self.fine_ids = torch.empty(blend_pairs, dtype=torch.int32, device=dev)
            fws = C.lib().rm_fine_lists_workspace_size(self.blend_views.n_tiles, capacity, self.fine_shift)
            self.fine_ws = torch.empty(fws, dtype=torch.uint8, device=dev)
        ws = self._ws_base
        if self.hit_masks:
            bv = self.blend_views
            c0 = bv.cams[0]
            ws += int(C.lib().rm_blend_hit_mask_bytes(blend_pairs, bv.n_tiles, c0.tile_width * c0.tile_height))
        self.blend_ws = torch.empty(ws, dtype=torch.uint8, device=dev)
        self.graph = None

    def measure_pairs(self) -> int:
        """Project and scan once, synchronously, and return the pair count."""
        self._project_scan()
        return int(self.total.item())

    def ensure_capacity(self, headroom: float = 1.05) -> bool:
        """Grow the pair buffers if the last frame overflowed them (reads the
        pair count of the last frame); returns True if they were grown."""
        P = int(self.total.item())
        if P <= self.capacity:
            return False
        self._alloc_pairs(int(P * headroom) + 4096)
        return True

    # ------------------------------------------------------------- stages --
    def _project_scan(self):
        L, s, v = C.lib(), C.stream_handle(), self.views
        nT = v.n * self.T
        fp = self.footprint if self.fine_shift else None
        R._call("rm_project_fwd_multi", lambda: L.rm_project_fwd_multi(
            C.ptr(self.indices), C.ptr(self.vertices), self.T, self.V, v.array, v.n, C.ptr(self.tiles),
            C.ptr(self.rect), C.ptr(self.depth), C.ptr(self.tiles_any), None, C.ptr(fp), C.ptr(self.status), s))
        R._call("rm_scan_tiles", lambda: L.rm_scan_tiles(C.ptr(self.tiles), nT, C.ptr(self.offsets), C.ptr(self.total),
                                C.ptr(self.scan_ws), self.scan_ws.numel(), s))
        # the scan's timeout / overflow bits (its workspace's status word) join the batch's status word
        self.status.bitwise_or_(self.scan_ws[:4].view(torch.int32))

    def _lists(self):
        L, s, v = C.lib(), C.stream_handle(), self.views
        # fine_shift 1: the 2x2 coverage bits ride in the sorted values, so the
        # split reads no rectangles
        packed = self.fine_shift == 1 and self.T < (1 << 28)
        if self.fine_shift:
            # the lists of the smaller tiles depend on the ray jitter's range
            R._call("rm_jitter_bounds", lambda: L.rm_jitter_bounds(
                C.ptr(self.jitter), self.jitter.numel() // 2, C.ptr(self.jitter_bounds), C.ptr(self.jitter_ws),
                self.jitter_ws.numel(), s))
        fp = self.footprint if packed else None
        jb = self.jitter_bounds if packed else None
        R._call("rm_emit_pairs_multi", lambda: L.rm_emit_pairs_multi(
            C.ptr(self.depth), C.ptr(self.rect), C.ptr(self.offsets), self.T, v.array, v.n, self.capacity,
            C.ptr(self.total), C.ptr(self.keys), C.ptr(self.vals), C.ptr(self.status), C.ptr(fp), C.ptr(jb), s))
        R._call("rm_sort_pairs", lambda: L.rm_sort_pairs(C.ptr(self.keys), C.ptr(self.vals), self.capacity, C.ptr(self.total), v.end_bit,
                                C.ptr(self.sorted_keys), C.ptr(self.sorted_ids), C.ptr(self.sort_ws),
                                self.sort_ws.numel(), C.ptr(self.status), s))
        R._call("rm_tile_ranges", lambda: L.rm_tile_ranges(C.ptr(self.sorted_keys), self.capacity, C.ptr(self.total), C.ptr(self.ranges),
                                 v.n_tiles, s))
        if self.fine_shift:
            R._call("rm_fine_lists", lambda: L.rm_fine_lists_multi(
                C.ptr(self.sorted_keys), C.ptr(self.sorted_ids), self.capacity, C.ptr(self.total),
                C.ptr(self.ranges), None if packed else C.ptr(self.footprint),
                None if packed else C.ptr(self.jitter_bounds), self.T, v.array, v.n,
                self.fine_shift, self.fine_ids.shape[0], C.ptr(self.fine_ids), C.ptr(self.fine_ranges),
                C.ptr(self.fine_total), C.ptr(self.fine_ws), self.fine_ws.numel(), C.ptr(self.status), s))

    def _blend_lists(self):
        """(sorted ids, ranges, views) that the blend walks."""
        if self.fine_shift:
            return self.fine_ids, self.fine_ranges, self.blend_views
        return self.sorted_ids, self.ranges, self.views

    def _blend_fwd(self):
        L, s = C.lib(), C.stream_handle()
        ids, rg, v = self._blend_lists()
        R._call("rm_blend_fwd_multi", lambda: L.rm_blend_fwd_multi(C.ptr(ids), C.ptr(rg), C.ptr(self.indices),
                                     C.ptr(self.vertices), C.ptr(self.cell_values), self.T, self.V,
                                     C.ptr(self.tiles_any), C.ptr(self.jitter), v.array, v.n, C.ptr(self.img),
                                     C.ptr(self.dist), C.ptr(self.nc), C.ptr(self.records), C.ptr(self.blend_ws), self.blend_ws.numel(),
                                     self.fwd_flags | (C.RM_BLEND_HIT_MASKS if self.hit_masks else 0),
                                     C.ptr(self.status), s))

    def _blend_bwd(self):
        L, s = C.lib(), C.stream_handle()
        ids, rg, v = self._blend_lists()
        self.grad_vertices.zero_()
        self.grad_cell_values.zero_()
        C.check(L.rm_blend_bwd_multi(C.ptr(ids), C.ptr(rg), C.ptr(self.indices),
                                     C.ptr(self.vertices), C.ptr(self.cell_values), self.T, self.V,
                                     C.ptr(self.tiles_any), C.ptr(self.jitter), v.array, v.n, C.ptr(self.img),
                                     C.ptr(self.dist), C.ptr(self.nc), C.ptr(self.grad_img), C.ptr(self.grad_dist),
                                     C.ptr(self.grad_vertices), C.ptr(self.grad_cell_values), C.ptr(self.records), C.ptr(self.blend_ws),
                                     self.blend_ws.numel(), self.bwd_flags | C.RM_BLEND_REUSE_RECORDS |
                                     (C.RM_BLEND_HIT_MASKS if self.hit_masks else 0), C.ptr(self.status), s),
                "rm_blend_bwd_multi")

    # ---------------------------------------------------------------- API --
    def forward(self):
        """Render every view (asynchronous, no host synchronisation).
        Returns the concatenated (img [Npx,4], distortion [Npx,5], n_contrib [Npx])."""
        self._project_scan()
        self._lists()
        self._blend_fwd()
        return self.img, self.dist, self.nc

    def backward(self, grad_img: torch.Tensor | None = None, grad_dist: torch.Tensor | None = None):
        """Adjoint of the last forward; gradients of all views are summed.
        Returns (grad_vertices, grad_cell_values)."""
        if grad_img is not None:
            self.grad_img.copy_(grad_img)
        self.grad_dist = grad_dist
        self._blend_bwd()
        return self.grad_vertices, self.grad_cell_values

    def check(self) -> None:
        """Synchronise and raise if the last frame overflowed the pair buffers
        or a kernel reported an error in the batch's status word (bad index,
        non-finite vertex, int32 overflow, a wait that gave up: raised as
        ``_capi.DeviceStatusError``).  The status word is cleared."""
        P = int(self.total.item())
        bits = int(self.status.item()) & 0xffffffff
        self.status.zero_()
        self.scan_ws[:4].zero_()
        if bits & ~C.RM_STATUS_CAPACITY:
            raise C.DeviceStatusError(bits & ~C.RM_STATUS_CAPACITY, "BatchedRasterizer")
        if P > self.capacity:
            raise RuntimeError(f"pair capacity {self.capacity} exceeded ({P} pairs): call ensure_capacity()")

    def images(self):
        """Per-view (img [H,W,4], distortion [H,W,5], n_contrib [H,W,1])."""
        v = self.views
        return list(zip(v.split(self.img), v.split(self.dist), [x.unsqueeze(-1) for x in v.split(self.nc)]))


def l1_grad_weights(views: ViewBatch, device) -> torch.Tensor:
    """Per-pixel weight 1 / (3 * H_v * W_v): the gradient scale of a sum over
    views of per-view mean L1 losses on the three colour channels."""
    w = torch.empty(views.n_pixels, 1, device=device)
    for v, (h, wd) in enumerate(views.hw):
        w[views.pixel_base[v]:views.pixel_base[v + 1]] = 1.0 / (3.0 * h * wd)
    return w


class L1Step:
    """One capturable multi-view training step: forward, the L1 loss against
    ``target`` [Npx, 3] (sum over views of per-view means) and backward.
    ``capture()`` records the step as a CUDA graph; ``run()`` replays it (or
    launches eagerly before capture)."""

    def __init__(self, rast: BatchedRasterizer, target: torch.Tensor):
        self.r = rast
        self.target = target
        self.w = l1_grad_weights(rast.views, rast.device)
        self.loss = torch.zeros((), device=rast.device)
        self.graph = None

    def _launch(self):
        r = self.r
        r.forward()
        diff = r.img[:, :3] - self.target
        self.loss.copy_((diff.abs() * self.w).sum())
        r.grad_img[:, :3].copy_(torch.sign(diff) * self.w)
        r.grad_img[:, 3].zero_()
        r.grad_dist = None
        r._blend_bwd()

    def capture(self):
        s = torch.cuda.Stream(device=self.r.device)
        s.wait_stream(torch.cuda.current_stream())
        with torch.cuda.stream(s):
            self._launch()  # warm-up outside capture (lazy init, attributes)
        torch.cuda.current_stream().wait_stream(s)
        torch.cuda.synchronize()
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g):
            self._launch()
        self.graph = g
        return g

    def run(self):
        if self.graph is not None:
            self.graph.replay()
        else:
            self._launch()
        return self.loss
