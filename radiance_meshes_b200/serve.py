"""Render serving: resident meshes, HBM-budget admission, continuous batching.

Meshes (indices, vertices, cell values and their packed per-tet blend
records) stay resident in HBM.  Requests (mesh, camera, arrival time) are
queued per mesh; whenever one of the server's streams is free, the scheduler
takes the mesh whose oldest pending request waited longest and launches, on
that stream, one batched forward (``batch.BatchedRasterizer``: every stage
one launch over all views of the batch) over as many of that mesh's pending
requests as fit the batch limit and the free HBM budget.  Views of different
resolutions batch together.  Batches on different streams overlap on the
device, and requests that arrive while others are on the GPU join the next
batch as soon as a stream and memory free up (continuous batching, not a
queue in front of one batch at a time).

Pair buffers are sized from a per-mesh bound on pairs per pixel measured at
load time; a batch whose pairs exceed it sets the device overflow flag and is
re-run with the exact size before its results are released.

Latency = device time at which the batch's results are complete (a CUDA
event) minus the request's arrival time, both relative to the server's
epoch.  A request's image, log T, distortion and n_contributors are the same
bit for bit whether it is rendered alone or inside any batch.

The reference has no serving path (its renders are driven by training and
evaluation scripts, ``utils/train_util.py:15-77``); this module serves the
render call of that path.
"""
from __future__ import annotations

import collections
import gc
import math
import time
from dataclasses import dataclass, field
from typing import Sequence

import numpy as np
import torch

from . import _capi as C
from . import batch as B
from .camera import RMCamera

__all__ = ["RenderRequest", "RenderResult", "ResidentMesh", "Server", "batch_bytes"]


@dataclass
class RenderRequest:
    rid: int
    mesh: str
    cam: RMCamera
    arrival: float = 0.0  # seconds since the server epoch


@dataclass
class RenderResult:
    rid: int
    mesh: str
    latency_ms: float
    done_ms: float
    batch_id: int
    batch_views: int
    retried: bool = False
    img: torch.Tensor | None = None  # [H, W, 4] (r, g, b, log T)
    dist: torch.Tensor | None = None  # [H, W, 5]
    nc: torch.Tensor | None = None  # [H, W, 1]


class ResidentMesh:
    """A mesh kept in HBM with its blend records packed once."""

    def __init__(self, name: str, indices, vertices, cell_values, device=None):
        device = torch.device(device or "cuda")
        self.name = name
        self.indices = torch.as_tensor(indices, dtype=torch.int32).to(device).contiguous()
        self.vertices = torch.as_tensor(vertices, dtype=torch.float32).to(device).contiguous()
        self.cell_values = torch.as_tensor(cell_values, dtype=torch.float32).to(device).contiguous()
        self.T = self.indices.shape[0]
        self.V = self.vertices.shape[0]
        L = C.lib()
        self.records = torch.empty(max(int(L.rm_blend_records_size(self.T)), 16), dtype=torch.uint8, device=device)
        C.check(L.rm_blend_pack_records(C.ptr(self.indices), C.ptr(self.vertices), C.ptr(self.cell_values), self.T,
                                        self.V, None, C.ptr(self.records), C.stream_handle()),
                "rm_blend_pack_records")
        self.pairs_per_pixel = None  # upper bound measured by Server.calibrate

    @property
    def nbytes(self) -> int:
        return (self.indices.numel() * 4 + self.vertices.numel() * 4 + self.cell_values.numel() * 4 +
                self.records.numel())


def batch_bytes(n_tets: int, views: B.ViewBatch, capacity: int, fine_shift: int = 0) -> int:
    """Device bytes a forward batch allocates (projection, lists, sort,
    ranges, fine lists, queue and per-pixel buffers)."""
    n = views.n
    L = C.lib()
    proj = n * n_tets * (4 + 16 + 4 + 4) + n_tets * 4 + int(L.rm_scan_workspace_size(n * n_tets))
    pairs = capacity * (8 + 4 + 8 + 4) + int(L.rm_sort_workspace_size(max(capacity, 1)))
    q = 1 << (2 * fine_shift)
    blend_tiles = views.n_tiles * q
    tiles = views.n_tiles * 8 + int(L.rm_blend_workspace_size(0, blend_tiles))  # no hit masks (forward only)
    if fine_shift:
        tiles += (n * n_tets * 48 + capacity * q * 4 + blend_tiles * 8 + int(L.rm_fine_lists_workspace_size(blend_tiles, capacity, fine_shift))
                  + int(L.rm_jitter_bounds_workspace_size()) + 16)
    pixels = views.n_pixels * (8 + 16 + 20 + 4)
    return proj + pairs + tiles + pixels + 4096


@dataclass
class _Batch:
    bid: int
    mesh: ResidentMesh
    reqs: list
    rast: B.BatchedRasterizer
    stream: torch.cuda.Stream
    done: torch.cuda.Event
    total_host: torch.Tensor  # [pair count, status word] of the batch, copied back with the images
    nbytes: int
    retried: bool = False


class Server:
    """Continuous-batching render server on one GPU.

    meshes: ResidentMesh objects; streams: concurrent batches; max_views:
    views per batch (<= batch.MAX_VIEWS).  The defaults (2 concurrent batches
    of at most 4 views) gave the steadiest tail near capacity on the
    three-mesh serving workload: with 4 batches of up to 8 views, a backlog,
    once formed, grew the batches and drained slowly.  hbm_budget: bytes the in-flight
    batches may hold (default: half the free memory at start); tile:
    tile size of every render; fwd_flags: blend launch flags (autotune.flags).
    """

    def __init__(self, meshes: Sequence[ResidentMesh], streams: int = 2, max_views: int = 4,
                 hbm_budget: int | None = None, tile: int = 16, fwd_flags: int = 0, pair_headroom: float = 1.25,
                 keep_outputs: bool = True, device=None, fine_shift: int = 0):
        self.device = torch.device(device or "cuda")
        self.meshes = {m.name: m for m in meshes}
        self.streams = [torch.cuda.Stream(device=self.device) for _ in range(streams)]
        self.free_streams = list(range(streams))
        self.max_views = min(int(max_views), B.MAX_VIEWS)
        if hbm_budget is None:
            free, _ = torch.cuda.mem_get_info(self.device)
            hbm_budget = free // 2
        self.hbm_budget = int(hbm_budget)
        self.reserved = 0
        self.tile = int(tile)
        self.fwd_flags = int(fwd_flags)
        self.fine_shift = int(fine_shift)  # blend on tiles 2^fine_shift times smaller (split lists)
        self.headroom = float(pair_headroom)
        self.pair_slack = 4096  # extra pair slots per batch
        self.keep_outputs = keep_outputs
        self.pending = collections.OrderedDict((name, collections.deque()) for name in self.meshes)
        self.inflight: list[_Batch] = []
        self.results: list[RenderResult] = []
        self.n_batches = 0
        self.n_retries = 0
        torch.cuda.synchronize(self.device)  # mesh records packed on another stream
        self.epoch = torch.cuda.Event(enable_timing=True)
        self.epoch.record(torch.cuda.current_stream(self.device))
        self.epoch.synchronize()
        self.t0 = time.perf_counter()
        self.peak_reserved = 0

    # ------------------------------------------------------------ set-up --
    def calibrate(self, cams_by_mesh: dict):
        """Measure an upper bound of pairs per pixel for each mesh from sample
        cameras (synchronous; run before serving)."""
        for name, cams in cams_by_mesh.items():
            m = self.meshes[name]
            worst = 0.0
            for cam in cams:
                vb = B.ViewBatch([cam])
                r = B.BatchedRasterizer(m.indices, m.vertices, m.cell_values, vb, capacity=1, records=m.records,
                                        hit_masks=False)
                P = r.measure_pairs()
                worst = max(worst, P / vb.n_pixels)
                del r
            m.pairs_per_pixel = worst

    def now(self) -> float:
        return time.perf_counter() - self.t0

    # -------------------------------------------------------- scheduling --
    def submit(self, req: RenderRequest):
        if req.mesh not in self.meshes:
            raise KeyError(f"unknown mesh {req.mesh!r}")
        if (req.cam.tile_height, req.cam.tile_width) != (self.tile, self.tile):
            raise ValueError(f"request {req.rid}: camera tile size must be {self.tile}")
        self.pending[req.mesh].append(req)

    def _capacity(self, mesh: ResidentMesh, vb: B.ViewBatch) -> int:
        ppp = mesh.pairs_per_pixel if mesh.pairs_per_pixel is not None else 4.0
        return int(ppp * self.headroom * vb.n_pixels) + self.pair_slack

    def _pick(self):
        """Mesh whose oldest pending request arrived first."""
        best, t = None, math.inf
        for name, q in self.pending.items():
            if q and q[0].arrival < t:
                best, t = name, q[0].arrival
        return best

    def _dispatch(self) -> int:
        launched = 0
        while self.free_streams:
            name = self._pick()
            if name is None:
                break
            mesh, q = self.meshes[name], self.pending[name]
            reqs = [q[0]]
            vb = B.ViewBatch([q[0].cam])
            need = batch_bytes(mesh.T, vb, self._capacity(mesh, vb), self.fine_shift)
            for r in list(q)[1:self.max_views]:
                vb2 = B.ViewBatch([x.cam for x in reqs] + [r.cam])
                need2 = batch_bytes(mesh.T, vb2, self._capacity(mesh, vb2), self.fine_shift)
                if self.reserved + need2 > self.hbm_budget:
                    break
                reqs.append(r)
                vb, need = vb2, need2
            if self.reserved + need > self.hbm_budget and self.inflight:
                break  # wait for memory to free up
            for _ in reqs:
                q.popleft()
            self._launch(mesh, reqs, vb, need)
            launched += 1
        return launched

    def _launch(self, mesh: ResidentMesh, reqs, vb: B.ViewBatch, need: int, capacity: int | None = None,
                stream_idx: int | None = None):
        si = self.free_streams.pop(0) if stream_idx is None else stream_idx
        stream = self.streams[si]
        cap = capacity if capacity is not None else self._capacity(mesh, vb)
        with torch.cuda.stream(stream):
            rast = B.BatchedRasterizer(mesh.indices, mesh.vertices, mesh.cell_values, vb, capacity=cap,
                                       fwd_flags=self.fwd_flags, records=mesh.records, hit_masks=False,
                                       fine_shift=self.fine_shift)
            rast.forward()
            total_host = torch.empty(2, dtype=torch.int64, pin_memory=True)
            total_host[0:1].copy_(rast.total, non_blocking=True)
            total_host[1:2].copy_(rast.status, non_blocking=True)
            done = torch.cuda.Event(enable_timing=True)
            done.record(stream)
        self.reserved += need
        self.peak_reserved = max(self.peak_reserved, self.reserved)
        b = _Batch(self.n_batches, mesh, reqs, rast, stream, done, total_host, need)
        b.stream_idx = si
        self.n_batches += 1
        self.inflight.append(b)
        return b

    def _retire(self) -> int:
        finished = 0
        still = []
        for b in self.inflight:
            if not b.done.query():
                still.append(b)
                continue
            P = int(b.total_host[0])
            bits = int(b.total_host[1]) & 0xffffffff & ~C.RM_STATUS_CAPACITY
            if bits:  # bad mesh data or a wait that gave up: the batch's images are not valid
                self.reserved -= b.nbytes
                self.free_streams.append(b.stream_idx)
                self.inflight = [x for x in self.inflight if x is not b]
                raise C.DeviceStatusError(bits, f"serving batch {b.bid} on mesh {b.mesh.name}")
            if P > b.rast.capacity:
                # overflow: re-run this batch with the exact pair count on the same stream
                self.n_retries += 1
                self.reserved -= b.nbytes
                need = batch_bytes(b.mesh.T, b.rast.views, P, self.fine_shift)
                nb = self._launch(b.mesh, b.reqs, b.rast.views, need, capacity=P, stream_idx=b.stream_idx)
                nb.retried = True
                self.inflight.remove(nb)
                still.append(nb)
                continue
            done_ms = self.epoch.elapsed_time(b.done)
            outs = b.rast.images() if self.keep_outputs else [(None, None, None)] * len(b.reqs)
            for r, (img, dist, nc) in zip(b.reqs, outs):
                self.results.append(RenderResult(r.rid, r.mesh, done_ms - 1e3 * r.arrival, done_ms, b.bid,
                                                 len(b.reqs), b.retried, img, dist, nc))
            self.reserved -= b.nbytes
            self.free_streams.append(b.stream_idx)
            finished += 1
        self.inflight = still
        return finished

    def idle(self) -> bool:
        return not self.inflight and not any(self.pending.values())

    def poll(self) -> int:
        """One scheduler iteration: retire finished batches, launch new ones."""
        n = self._retire()
        return n + self._dispatch()

    def drain(self):
        while not self.idle():
            if not self.poll():
                time.sleep(50e-6)

    def run_trace(self, requests: Sequence[RenderRequest], realtime: bool = True) -> list[RenderResult]:
        """Serve a request trace.  With realtime, request i is submitted once
        the wall clock passes its arrival time (relative to now); otherwise
        all requests are submitted at once in arrival order."""
        reqs = sorted(requests, key=lambda r: r.arrival)
        # a collector pause in the middle of a trace delays every launch
        # behind it: collect once, then freeze what exists (the meshes, the
        # process's modules), so that collections during the trace only walk
        # the objects the trace itself creates
        gc.collect()
        gc.freeze()
        try:
            return self._run_trace(reqs, realtime)
        finally:
            gc.unfreeze()

    def _run_trace(self, reqs, realtime: bool) -> list[RenderResult]:
        start = self.now()
        for r in reqs:
            r.arrival += start
        first_result = len(self.results)
        i = 0
        while i < len(reqs) or not self.idle():
            now = self.now()
            while i < len(reqs) and (not realtime or reqs[i].arrival <= now):
                self.submit(reqs[i])
                i += 1
            if not self.poll():
                nxt = reqs[i].arrival - self.now() if i < len(reqs) else 0.0
                time.sleep(min(max(nxt, 0.0), 2e-4) if realtime else 20e-6)
        return self.results[first_result:]

    def render_alone(self, req: RenderRequest) -> RenderResult:
        """Render one request by itself (synchronously)."""
        r = RenderRequest(req.rid, req.mesh, req.cam, self.now())
        self.submit(r)
        self.drain()
        return self.results[-1]


def latency_summary(results: Sequence[RenderResult], skip: int = 0) -> dict:
    lat = np.array([r.latency_ms for r in results[skip:]])
    done = np.array([r.done_ms for r in results[skip:]])
    arr = done - lat
    span_s = (done.max() - arr.min()) * 1e-3 if len(lat) else float("nan")
    return {"requests": int(len(lat)), "p50_ms": float(np.percentile(lat, 50)),
            "p90_ms": float(np.percentile(lat, 90)), "p99_ms": float(np.percentile(lat, 99)),
            "mean_ms": float(lat.mean()), "max_ms": float(lat.max()), "frames_per_s": float(len(lat) / span_s)}
