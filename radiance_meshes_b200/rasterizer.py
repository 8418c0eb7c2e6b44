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
import threading
from dataclasses import dataclass

import torch

from . import _capi as C
from .camera import RMCamera, tcam_to_struct

__all__ = [
    "ScratchPool",
    "TileLists",
    "project_fwd",
    "project_fwd_fine",
    "jitter_bounds",
    "split_fine_lists",
    "fine_shift_for",
    "fine_camera",
    "project_bwd",
    "build_tile_lists",
    "blend_fwd",
    "blend_bwd",
    "calc_tet_err",
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

    def get(self, name: str, nbytes: int, device, zero_head: bool = False) -> torch.Tensor:
        """A buffer of at least ``nbytes``; zero_head: a newly allocated
        buffer gets its first 256 bytes zeroed (a status word lives there)."""
        key = (str(device), name)
        buf = self._bufs.get(key)
        if buf is None or buf.numel() < nbytes:
            buf = torch.empty(max(int(nbytes), 256), dtype=torch.uint8, device=device)
            if zero_head:
                buf[:256].zero_()
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


def frame_status(n_tets: int, device, pool: ScratchPool | None = None) -> torch.Tensor:
    """The device status word (int32 [1]) that the kernels of one frame or
    their RM_STATUS_* bits into: the first 4 bytes of the frame's scan
    workspace, whose other bytes every scan resets.  Projection, scan, sort
    and the fine-list split all report there, and build_tile_lists reads it
    together with the pair count (rm_count_pairs takes both right after the
    projection; the later stages' bits surface at the next readback)."""
    pool = pool or _POOL
    ws = pool.get("scan", C.lib().rm_scan_workspace_size(n_tets), device, zero_head=True)
    return ws[:4].view(torch.int32)


_HOST_READ: dict = {}  # (device, thread) -> pinned int32 [4]: pair count (int64) and status word


def _read_frame(total: torch.Tensor, status: torch.Tensor | None):
    """One synchronisation: the pair count and the frame's status word."""
    key = (str(total.device), threading.get_ident())
    hb = _HOST_READ.get(key)
    if hb is None:
        hb = torch.zeros(4, dtype=torch.int32, pin_memory=True)
        _HOST_READ[key] = hb
    hb[0:2].view(torch.int64).copy_(total.reshape(1), non_blocking=True)
    if status is not None:
        hb[2:3].copy_(status, non_blocking=True)
    else:
        hb[2] = 0
    torch.cuda.current_stream().synchronize()
    return int(hb[0:2].view(torch.int64)[0]), int(hb[2]) & 0xffffffff


def raise_status(bits: int, status: torch.Tensor | None, where: str) -> None:
    """Clear the status word and raise if any RM_STATUS_* bit is set."""
    if bits:
        if status is not None:
            status.zero_()
        raise C.DeviceStatusError(bits, where)


def check_status(n_tets: int, device) -> None:
    """Synchronise the current stream and raise ``_capi.DeviceStatusError``
    if a kernel of this device's frames reported an error that no readback
    has seen yet (the fine-list split runs after a frame's readback, so its
    bits otherwise surface at the next frame)."""
    status = frame_status(n_tets, device)
    torch.cuda.current_stream().synchronize()
    raise_status(int(status.item()) & 0xffffffff, status, "rasterizer")


class StageTimer:
    """Records a CUDA event pair around every C-ABI call on the launching
    (current) stream while active (or only around the stages named in
    ``only``); ``totals()`` returns milliseconds per stage."""

    def __init__(self, only=None):
        self.events = []
        self.only = None if only is None else set(only)

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
    if _TIMER is None or (_TIMER.only is not None and name not in _TIMER.only):
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
    status = frame_status(T, dev)
    _call("rm_project_fwd", lambda: C.lib().rm_project_fwd(C.ptr(indices), C.ptr(vertices), T, vertices.shape[0], ctypes.byref(cam),
                                   C.ptr(tiles), C.ptr(rect), C.ptr(vs), C.ptr(cc), C.ptr(status), _stream()))
    return tiles, rect, vs, cc


def fine_shift_for(cam: RMCamera) -> int:
    """log2 of the split factor that brings the camera's tiles to 8x8 pixels
    (0 when the tiles are already 8 pixels wide or smaller, or not square)."""
    if cam.tile_width != cam.tile_height or cam.tile_width < 16 or cam.tile_width & (cam.tile_width - 1):
        return 0
    return int(cam.tile_width // 8).bit_length() - 1


def fine_camera(cam: RMCamera, fine_shift: int) -> RMCamera:
    """The same camera with tiles 2^fine_shift times smaller on a grid
    2^fine_shift times larger (the grid covers the same pixels)."""
    f = 1 << fine_shift
    out = RMCamera()
    ctypes.memmove(ctypes.byref(out), ctypes.byref(cam), ctypes.sizeof(RMCamera))
    out.tile_width, out.tile_height = cam.tile_width // f, cam.tile_height // f
    out.grid_width, out.grid_height = cam.grid_width * f, cam.grid_height * f
    return out


def project_fwd_fine(indices: torch.Tensor, vertices: torch.Tensor, cam: RMCamera):
    """project_fwd plus each tet's image footprint [T,12] (box, then the four
    projected vertices or NaN; rm_project_fwd_fine), from which the lists of
    smaller tiles are cut."""
    _require_cuda(indices=indices, vertices=vertices)
    indices = _i32(indices)
    vertices = _f32(vertices)
    T = indices.shape[0]
    dev = vertices.device
    tiles = torch.empty(T, dtype=torch.int32, device=dev)
    rect = torch.empty((T, 4), dtype=torch.int32, device=dev)
    vs = torch.empty((T, 3), dtype=torch.float32, device=dev)
    cc = torch.empty((T, 3), dtype=torch.float32, device=dev)
    footprint = torch.empty((T, 12), dtype=torch.float32, device=dev)
    status = frame_status(T, dev)
    _call("rm_project_fwd", lambda: C.lib().rm_project_fwd_fine(
        C.ptr(indices), C.ptr(vertices), T, vertices.shape[0], ctypes.byref(cam), C.ptr(tiles), C.ptr(rect),
        C.ptr(vs), C.ptr(cc), C.ptr(footprint), C.ptr(status), _stream()))
    return tiles, rect, vs, cc, footprint


def jitter_bounds(ray_jitter: torch.Tensor, pool: ScratchPool | None = None) -> torch.Tensor:
    """(min jx, min jy, max jx, max jy) of a per-pixel ray jitter [..., 2], as a
    [4] tensor on the device (rm_jitter_bounds; no host synchronisation)."""
    pool = pool or _POOL
    _require_cuda(ray_jitter=ray_jitter)
    ray_jitter = _f32(ray_jitter)
    if ray_jitter.shape[-1] != 2:
        raise ValueError("ray_jitter must have 2 values per pixel")
    out = torch.empty(4, dtype=torch.float32, device=ray_jitter.device)
    L = C.lib()
    ws_n = L.rm_jitter_bounds_workspace_size()
    ws = pool.get("jitter", ws_n, ray_jitter.device)
    _call("rm_jitter_bounds", lambda: L.rm_jitter_bounds(C.ptr(ray_jitter), ray_jitter.numel() // 2, C.ptr(out),
                                                         C.ptr(ws), ws_n, _stream()))
    return out


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


_PAIR_GUESS: dict = {}  # device -> pair count of the last frame built there
_SIDE: dict = {}  # (device, thread) -> (side stream, pinned int64 [2], its numpy view) for the pair-count read


def _count_read_start(count: torch.Tensor):
    """Copy ``count`` (int64 [2] on the device: pair count, status word) to
    pinned host memory on a side stream that waits for the work queued so
    far only, so the frame's stream goes on with what is queued after this
    call while the host waits in _count_read_finish."""
    dev = count.device
    key = (dev, threading.get_ident())  # threads building frames at once each read their own buffer
    st = _SIDE.get(key)
    if st is None:
        hb = torch.zeros(2, dtype=torch.int64, pin_memory=True)
        st = (torch.cuda.Stream(device=dev), hb, hb.numpy())
        _SIDE[key] = st
    side, hb, hn = st
    side.wait_stream(torch.cuda.current_stream(dev))
    count.record_stream(side)
    with torch.cuda.stream(side):
        hb.copy_(count, non_blocking=True)
    done = torch.cuda.Event()
    done.record(side)
    return done, hn


def _count_read_finish(pending) -> tuple[int, int]:
    done, hn = pending
    done.synchronize()
    return int(hn[0]), int(hn[1]) & 0xffffffff


_LISTS = {"depth_first": True}


def use_depth_first_lists(enabled: bool) -> None:
    """Build the tile lists depth first (sort the visible tets by depth once,
    emit in that order, sort the pairs on the tile bits only: 4 + 2 short
    passes instead of 6 over the pairs) or as the reference does (emit in
    tet order, one sort on 32 + msb bits).  The lists are identical."""
    _LISTS["depth_first"] = bool(enabled)


def build_tile_lists(tiles: torch.Tensor, rect: torch.Tensor, vs: torch.Tensor, cam: RMCamera,
                     pool: ScratchPool | None = None, keep_debug: bool = False) -> TileLists:
    """Scan, emit, sort and range the tile/tet pairs.

    The pair count P is read back to the host once (the reference reads it
    three times: tile_shader_slang.py:38-44,68), together with the frame's
    status word (frame_status): a bad index, a non-finite vertex or a pair
    count beyond int32 raises ``_capi.DeviceStatusError`` there, where the
    reference asserts on the host (tile_shader_slang.py:78).

    By default the lists are built depth first (use_depth_first_lists): P is
    counted right after the projection (rm_count_pairs) and copied to the
    host on a side stream.  After the first frame on a device, the pair
    buffers are sized from the previous frame's count (plus a quarter) and
    the whole build is queued before P is read, so the host goes on while
    the GPU builds the lists; a frame with more pairs than that is built
    again at exactly P.  The first frame waits for the count alone (while the
    GPU orders the visible tets by depth) and builds at exactly P.  Bits that
    the kernels after the count set (a look-back that gave up) surface at the
    next readback of the device: the next frame's, or check_status.

    keep_debug builds the lists in the reference's order of work and also
    returns the tet-order offsets and the emitted keys and values; that path
    sizes its buffers from the previous frame's count (plus a quarter),
    queues emission, sort and ranges before P is read, builds the frame again
    at exactly P should P exceed that, and reads the status word after all of
    its kernels."""
    pool = pool or _POOL
    dev = tiles.device
    T = tiles.shape[0]
    G = cam.grid_width * cam.grid_height
    L = C.lib()
    s = _stream()
    end_bit = end_bit_for(cam.grid_width, cam.grid_height)
    total = torch.zeros(1, dtype=torch.int64, device=dev)
    status = frame_status(T, dev, pool)  # the stages or their RM_STATUS_* bits into it
    depth_first = _LISTS["depth_first"] and not keep_debug and T > 0

    if depth_first:
        # the pair count and the status word as the projection left them,
        # copied to the host on a side stream (read once the build is queued)
        count = torch.empty(2, dtype=torch.int64, device=dev)
        _call("rm_count_pairs", lambda: L.rm_count_pairs(C.ptr(tiles), T, C.ptr(status), C.ptr(count), s))
        pending = _count_read_start(count)
        # visible tets by depth, once; the pairs then need the tile bits only
        dkeys = torch.empty(T, dtype=torch.int64, device=dev)
        dvals = torch.empty(T, dtype=torch.int32, device=dev)
        n_vis = torch.zeros(1, dtype=torch.int64, device=dev)
        dws_n = L.rm_depth_order_workspace_size(T)
        dws = pool.get("depth", dws_n, dev)
        _call("rm_depth_order", lambda: L.rm_depth_order(C.ptr(tiles), C.ptr(vs), T, C.ptr(dkeys), C.ptr(dvals),
                                                         C.ptr(n_vis), C.ptr(dws), dws_n, C.ptr(status), s))
        okeys = torch.empty(T, dtype=torch.int64, device=dev)
        order = torch.empty(T, dtype=torch.int32, device=dev)
        sws_n = L.rm_sort_workspace_size(T)
        sws = pool.get("sort", sws_n, dev)
        _call("rm_sort_pairs", lambda: L.rm_sort_pairs_range(C.ptr(dkeys), C.ptr(dvals), T, C.ptr(n_vis), 0, 32,
                                                             C.ptr(okeys), C.ptr(order), C.ptr(sws), sws_n,
                                                             C.ptr(status), s))
        ews_n = L.rm_emit_ordered_workspace_size(T)
        ews = pool.get("emit", ews_n, dev)
        offsets = None
    else:
        offsets = torch.empty(T, dtype=torch.int32, device=dev)
        ws_n = L.rm_scan_workspace_size(T)
        ws = pool.get("scan", ws_n, dev, zero_head=True)
        _call("rm_scan_tiles", lambda: L.rm_scan_tiles(C.ptr(tiles), T, C.ptr(offsets), C.ptr(total), C.ptr(ws),
                                                       ws_n, s))

    def pairs(cap, n_dev):
        keys = torch.empty(cap, dtype=torch.int64, device=dev)
        vals = torch.empty(cap, dtype=torch.int32, device=dev)
        if depth_first:
            _call("rm_emit_pairs", lambda: L.rm_emit_pairs_ordered(
                C.ptr(vs), C.ptr(rect), C.ptr(tiles), C.ptr(order), T, C.ptr(n_vis), cam.grid_width, cap,
                C.ptr(total), C.ptr(keys), C.ptr(vals), C.ptr(ews), ews_n, C.ptr(status), s))
            n_dev = total
        else:
            _call("rm_emit_pairs", lambda: L.rm_emit_pairs(C.ptr(vs), C.ptr(rect), C.ptr(offsets), T,
                                                           cam.grid_width, cap, C.ptr(n_dev), C.ptr(keys),
                                                           C.ptr(vals), None, s))
        sk = torch.empty(cap, dtype=torch.int64, device=dev)
        sv = torch.empty(cap, dtype=torch.int32, device=dev)
        if cap > 0:
            sws_n = L.rm_sort_workspace_size(cap)
            sws = pool.get("sort", sws_n, dev)
            begin = 32 if depth_first else 0
            _call("rm_sort_pairs", lambda: L.rm_sort_pairs_range(C.ptr(keys), C.ptr(vals), cap, C.ptr(n_dev), begin,
                                                                 end_bit, C.ptr(sk), C.ptr(sv), C.ptr(sws), sws_n,
                                                                 C.ptr(status), s))
        ranges = torch.empty((G, 2), dtype=torch.int32, device=dev)
        _call("rm_tile_ranges", lambda: L.rm_tile_ranges(C.ptr(sk), cap, C.ptr(n_dev), C.ptr(ranges), G, s))
        return keys, vals, sk, sv, ranges

    key = str(dev)
    guess = _PAIR_GUESS.get(key)
    if depth_first:
        out = None
        if guess is not None:  # queued before the count is read: the host does not wait for the GPU
            cap = guess + guess // 4 + 4096
            out = pairs(cap, total)
        P, bits = _count_read_finish(pending)
        raise_status(bits, status, "vertex_and_tile_shader")
        if P > 0x7FFFFFFF:  # the offsets are int32, as the reference's cumsum
            raise C.DeviceStatusError(C.RM_STATUS_OVERFLOW, "vertex_and_tile_shader")
        _PAIR_GUESS[key] = P
        if out is not None and P > cap:
            # expected: the emission into the smaller buffers set the capacity
            # bit; it is cleared (other bits stay for the next readback), and
            # the pairs are built again at exactly P
            torch.cuda.current_stream(dev).synchronize()
            status.fill_(int(status.item()) & ~C.RM_STATUS_CAPACITY)
            out = None
        if out is None:
            out = pairs(P, total)
        keys, vals, sk, sv, ranges = out
        return TileLists(sv[:P], ranges, P, sorted_keys=sk[:P])

    out = None
    if guess is not None:
        cap = guess + guess // 4 + 4096
        out = pairs(cap, total)
        P, bits = _read_frame(total, status)
        if P > cap:
            out = None
    else:
        P, bits = _read_frame(total, status)
    if out is None and bits & C.RM_STATUS_CAPACITY:
        # expected: the buffers were sized before P was known; rebuilt at exactly P below
        bits &= ~C.RM_STATUS_CAPACITY
        if not bits:
            status.zero_()
    raise_status(bits, status, "vertex_and_tile_shader")
    if out is None:
        out = pairs(P, None)
        # the exact-size sort reports now, not at the next frame
        _, bits = _read_frame(total, status)
        raise_status(bits, status, "vertex_and_tile_shader")
    _PAIR_GUESS[key] = P
    keys, vals, sk, sv, ranges = out
    if keep_debug:
        return TileLists(sv[:P], ranges, P, offsets, keys[:P], vals[:P], sk[:P])
    return TileLists(sv[:P], ranges, P, sorted_keys=sk[:P])


@dataclass
class FineLists:
    """Tile lists of one frame on the grid of 8x8-pixel tiles, cut from the
    lists of the caller's (larger) tiles for one ray jitter.  Every entry of a
    coarse list that can reach a ray of a fine tile's pixels is in that fine
    tile's list, in the same order (rm_project_fwd_fine, rm_jitter_bounds,
    rm_fine_lists), so blending over the fine lists with that jitter gives the
    coarse blend's image, log T and distortion bit for bit; n_contributors then
    counts fine-list entries, which only the backward pass reads."""
    shift: int
    cam: RMCamera  # the fine camera
    coarse_key: bytes
    sorted_ids: torch.Tensor  # capacity entries; the first n_pairs are used
    ranges: torch.Tensor
    total: torch.Tensor  # [1] int64 on the device

    @property
    def n_pairs(self) -> int:
        return int(self.total.item())


@dataclass
class PendingFineLists:
    """What the projection leaves on the sorted coarse ids: the coarse ranges,
    the tets' image footprints and the split factor.  The split itself needs the
    ray jitter of the blend, so it runs in fine_lists_of (once per jitter)."""
    shift: int
    coarse_cam: RMCamera
    coarse_key: bytes
    ranges: torch.Tensor
    footprint: torch.Tensor
    sorted_keys: torch.Tensor
    status: torch.Tensor | None = None  # the frame's status word (frame_status)
    tiles_touched: torch.Tensor | None = None  # the projection's counts: the blend packs visible tets only
    jitter: torch.Tensor | None = None  # the jitter of `lists` (kept alive so identity stays meaningful)
    jitter_version: int = -1
    lists: FineLists | None = None


_FINE = {"enabled": True}


def use_fine_lists(enabled: bool) -> None:
    """Switch the drop-in's blending over 8x8-pixel lists on or off."""
    _FINE["enabled"] = bool(enabled)


def fine_lists_enabled() -> bool:
    return _FINE["enabled"]


def _cam_key(cam: RMCamera) -> bytes:
    """Every field of the camera record, as its raw bytes."""
    return bytes(cam)


def attach_fine_lists(sorted_ids: torch.Tensor, ranges: torch.Tensor, cam: RMCamera, fine_shift: int,
                      footprint: torch.Tensor, sorted_keys: torch.Tensor, status: torch.Tensor | None = None,
                      tiles_touched: torch.Tensor | None = None) -> PendingFineLists:
    """Record on ``sorted_ids`` (attribute ``rm_fine``) what fine_lists_of needs
    to cut the 2^fine_shift times smaller tiles' lists from these lists."""
    pend = PendingFineLists(fine_shift, cam, _cam_key(cam), ranges, footprint, sorted_keys, status, tiles_touched)
    sorted_ids.rm_fine = pend
    return pend


@dataclass
class FrameState:
    """What the projection of a frame leaves on its sorted ids (attribute
    ``rm_frame``) for the blend of the same frame: the per-tet tile counts
    (the blend packs records of visible tets only) and the status word."""
    tiles_touched: torch.Tensor
    status: torch.Tensor


def attach_frame(sorted_ids: torch.Tensor, tiles_touched: torch.Tensor, status: torch.Tensor) -> None:
    sorted_ids.rm_frame = FrameState(tiles_touched, status)


def frame_of(sorted_ids: torch.Tensor) -> FrameState | None:
    """The FrameState attached by vertex_and_tile_shader, if ``sorted_ids`` is
    the tensor it returned (a copy or slice carries none; the blend then packs
    every tet, with the same results)."""
    return getattr(sorted_ids, "rm_frame", None)


def split_fine_lists(sorted_ids: torch.Tensor, ranges: torch.Tensor, cam: RMCamera, fine_shift: int,
                     footprint: torch.Tensor, bounds: torch.Tensor, sorted_keys: torch.Tensor,
                     pool: ScratchPool | None = None, status: torch.Tensor | None = None) -> FineLists:
    """Split the sorted coarse lists (ids and keys) into the fine lists for
    the jitter bounds ``bounds`` (rm_fine_lists, no host synchronisation)."""
    pool = pool or _POOL
    dev = sorted_ids.device
    camf = fine_camera(cam, fine_shift)
    Gf = camf.grid_width * camf.grid_height
    cap = max(int(sorted_ids.shape[0]) << (2 * fine_shift), 1)
    fine_ids = torch.empty(cap, dtype=torch.int32, device=dev)
    fine_ranges = torch.empty((Gf, 2), dtype=torch.int32, device=dev)
    total = torch.empty(1, dtype=torch.int64, device=dev)
    L = C.lib()
    P = int(sorted_ids.shape[0])
    ws_n = L.rm_fine_lists_workspace_size(Gf, P, fine_shift)
    ws = pool.get("fine", ws_n, dev)
    _call("rm_fine_lists", lambda: L.rm_fine_lists(C.ptr(sorted_keys), C.ptr(sorted_ids), P, None, C.ptr(ranges),
                                                   C.ptr(footprint), C.ptr(bounds), ctypes.byref(cam), fine_shift,
                                                   cap, C.ptr(fine_ids), C.ptr(fine_ranges), C.ptr(total), C.ptr(ws),
                                                   ws_n, C.ptr(status), _stream()))
    return FineLists(fine_shift, camf, _cam_key(cam), fine_ids, fine_ranges, total)


def fine_lists_of(sorted_ids: torch.Tensor, cam: RMCamera, ray_jitter: torch.Tensor) -> FineLists | None:
    """The fine lists of ``sorted_ids`` for this camera and ray jitter, if the
    projection prepared them (cut on the first call for a jitter tensor and
    kept while that tensor is unchanged)."""
    pend = getattr(sorted_ids, "rm_fine", None)
    if pend is None or not _FINE["enabled"] or pend.coarse_key != _cam_key(cam):
        return None
    if pend.lists is not None and pend.jitter is ray_jitter and pend.jitter_version == ray_jitter._version:
        return pend.lists
    bounds = jitter_bounds(ray_jitter)
    pend.lists = split_fine_lists(sorted_ids, pend.ranges, pend.coarse_cam, pend.shift, pend.footprint, bounds,
                                  pend.sorted_keys, status=pend.status)
    pend.jitter, pend.jitter_version = ray_jitter, ray_jitter._version
    return pend.lists


_BLEND_FLAGS = {"fwd": 0, "bwd": 0}
_STAGE = {"tma": False}


def use_tma_staging(enabled: bool) -> None:
    """Stage the backward's records with bulk copies (RM_BLEND_STAGE_TMA)
    instead of per-thread loads.  Single-GPU processes only by policy."""
    _STAGE["tma"] = bool(enabled)


def tma_staging() -> bool:
    return _STAGE["tma"]


def set_blend_tuning(fwd_flags: int = 0, bwd_flags: int = 0) -> None:
    """Launch tunables (RM_BLEND_STRIP / HEAVY / PAIR_CTAS bits of the flags
    word) used by blend_fwd / blend_bwd; 0 selects the built-in defaults."""
    _BLEND_FLAGS["fwd"] = int(fwd_flags)
    _BLEND_FLAGS["bwd"] = int(bwd_flags)


def blend_tuning() -> tuple[int, int]:
    return _BLEND_FLAGS["fwd"], _BLEND_FLAGS["bwd"]


def blend_fwd(sorted_ids, ranges, indices, vertices, cell_values, ray_jitter, cam: RMCamera,
              tiles_touched=None, records: torch.Tensor | None = None, reuse_records: bool = False,
              hit_masks: bool = False, status: torch.Tensor | None = None):
    """Forward blend.  Returns (img, dist, n_contrib, workspace); pass the
    workspace to blend_bwd.  hit_masks: also store which pixels hit each list
    entry (RM_BLEND_HIT_MASKS) so that a blend_bwd with hit_masks=True skips
    the misses.  status: a device status word (frame_status) for the pass's
    RM_STATUS_* bits (None: the workspace's own word)."""
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
    if hit_masks:
        ws_n += L.rm_blend_hit_mask_bytes(sorted_ids.shape[0], cam.grid_width * cam.grid_height,
                                          cam.tile_width * cam.tile_height)
    if records is None:
        records = torch.empty(ws_n, dtype=torch.uint8, device=dev)
    img = torch.empty((H, W, 4), dtype=torch.float32, device=dev)
    dist = torch.empty((H, W, 5), dtype=torch.float32, device=dev)
    nc = torch.empty((H, W, 1), dtype=torch.int32, device=dev)
    flags = ((C.RM_BLEND_REUSE_RECORDS if reuse_records else 0) | (C.RM_BLEND_HIT_MASKS if hit_masks else 0) |
             _BLEND_FLAGS["fwd"])
    _call("rm_blend_fwd", lambda: L.rm_blend_fwd(C.ptr(sorted_ids), C.ptr(ranges), C.ptr(indices), C.ptr(vertices), C.ptr(cell_values),
                           T, vertices.shape[0], C.ptr(tiles_touched), C.ptr(ray_jitter), ctypes.byref(cam),
                           C.ptr(img), C.ptr(dist), C.ptr(nc), C.ptr(records), records.numel(), flags, C.ptr(status),
                           _stream()))
    return img, dist, nc, records


def blend_bwd(sorted_ids, ranges, indices, vertices, cell_values, ray_jitter, cam: RMCamera, img, dist, nc,
              grad_img, grad_dist, records, tiles_touched=None, reuse_records=True,
              grad_vertices=None, grad_cell_values=None, hit_masks: bool = False,
              status: torch.Tensor | None = None):
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
    flags = ((C.RM_BLEND_REUSE_RECORDS if reuse_records else 0) | (C.RM_BLEND_HIT_MASKS if hit_masks else 0) |
             _BLEND_FLAGS["bwd"])
    if hit_masks and _STAGE["tma"]:
        flags |= C.RM_BLEND_STAGE_TMA
    _call("rm_blend_bwd", lambda: C.lib().rm_blend_bwd(C.ptr(sorted_ids), C.ptr(ranges), C.ptr(indices), C.ptr(vertices),
                                 C.ptr(cell_values), T, vertices.shape[0], C.ptr(tiles_touched), C.ptr(ray_jitter),
                                 ctypes.byref(cam), C.ptr(img), C.ptr(dist), C.ptr(nc), C.ptr(grad_img), C.ptr(gd),
                                 C.ptr(grad_vertices), C.ptr(grad_cell_values), C.ptr(records), records.numel(),
                                 flags, C.ptr(status), _stream()))
    return grad_vertices, grad_cell_values


def calc_tet_err(sorted_ids, ranges, indices, vertices, cell_values, cam: RMCamera, pixel_err, ssim_err,
                 tiles_touched=None, tet_err=None, tet_count=None):
    """Per-tet densification statistics of one view (rm_calc_tet_err):
    accumulates into tet_err [T,16] float32 and tet_count [T,2] int32
    (allocated zeroed when not given) and returns them."""
    _require_cuda(sorted_ids=sorted_ids, ranges=ranges, indices=indices, vertices=vertices,
                  cell_values=cell_values, pixel_err=pixel_err, ssim_err=ssim_err)
    indices = _i32(indices)
    vertices = _f32(vertices)
    cell_values = _f32(cell_values)
    pixel_err = _f32(pixel_err)
    ssim_err = _f32(ssim_err)
    T = indices.shape[0]
    dev = vertices.device
    if tet_err is None:
        tet_err = torch.zeros((T, 16), dtype=torch.float32, device=dev)
    if tet_count is None:
        tet_count = torch.zeros((T, 2), dtype=torch.int32, device=dev)
    L = C.lib()
    ws_n = L.rm_blend_workspace_size(T, cam.grid_width * cam.grid_height)
    ws = _POOL.get("err", ws_n, dev)
    _call("rm_calc_tet_err", lambda: L.rm_calc_tet_err(
        C.ptr(sorted_ids), C.ptr(ranges), C.ptr(indices), C.ptr(vertices), C.ptr(cell_values), T, vertices.shape[0],
        C.ptr(tiles_touched), ctypes.byref(cam), C.ptr(pixel_err), C.ptr(ssim_err), C.ptr(tet_err),
        C.ptr(tet_count), C.ptr(ws), ws_n, 0, _stream()))
    return tet_err, tet_count


def read_status(workspace: torch.Tensor) -> int:
    """Read and clear the device status word at the start of a scan/sort workspace."""
    out = ctypes.c_uint32(0)
    C.check(C.lib().rm_read_status(C.ptr(workspace), ctypes.byref(out), _stream()), "rm_read_status")
    return int(out.value)


def camera(tcam: dict) -> RMCamera:
    return tcam_to_struct(tcam)
