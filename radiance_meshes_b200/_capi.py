"""ctypes binding of ``librm_b200.so`` (declared in ``include/rm_capi.h``).

The library is loaded from ``radiance_meshes_b200/lib``.  There is no fallback:
if the library is missing or a call fails, a ``RuntimeError`` carrying the
library's own message is raised.
"""
from __future__ import annotations

import ctypes
import os
import threading

from .camera import RMCamera

RM_OK = 0
RM_EINVAL = 1
RM_ECAPACITY = 2
RM_ECUDA = 3
RM_ETIMEOUT = 4

RM_STATUS_SCAN_TIMEOUT = 0x1
RM_STATUS_SORT_TIMEOUT = 0x2
RM_STATUS_CAPACITY = 0x4
RM_STATUS_QUEUE_TIMEOUT = 0x8
RM_STATUS_BAD_INDEX = 0x10
RM_STATUS_NONFINITE = 0x20
RM_STATUS_OVERFLOW = 0x40

# what each status bit means, for error messages
STATUS_TEXT = {
    RM_STATUS_SCAN_TIMEOUT: "a scan look-back gave up waiting (offsets invalid)",
    RM_STATUS_SORT_TIMEOUT: "a sort look-back gave up waiting (order invalid)",
    RM_STATUS_CAPACITY: "more pairs than the buffers hold",
    RM_STATUS_QUEUE_TIMEOUT: "a work-queue wait gave up",
    RM_STATUS_BAD_INDEX: "a tet index lies outside [0, n_verts)",
    RM_STATUS_NONFINITE: "a tet vertex is NaN or infinite",
    RM_STATUS_OVERFLOW: "the tile/tet pair count exceeds INT32_MAX",
}

RM_BLEND_REUSE_RECORDS = 0x1
RM_BLEND_HIT_MASKS = 0x2
RM_BLEND_STAGE_TMA = 0x4
RM_BLEND_STRIP_SHIFT = 8
RM_BLEND_HEAVY_SHIFT = 16
RM_BLEND_PAIR_CTAS_SHIFT = 20
RM_BLEND_BATCH_SHIFT = 24

RM_MAX_VIEWS = 32

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "lib", "librm_b200.so")

_lock = threading.Lock()
_lib = None

vp = ctypes.c_void_p
i64 = ctypes.c_int64
i32 = ctypes.c_int32
sz = ctypes.c_size_t
camp = ctypes.POINTER(RMCamera)

# name -> (restype, argtypes); mirrors include/rm_capi.h
SIGNATURES = {
    "rm_last_error": (ctypes.c_char_p, []),
    "rm_abi_version": (ctypes.c_int, []),
    "rm_launch_count": (ctypes.c_uint64, []),
    "rm_read_status": (ctypes.c_int, [vp, vp, vp]),
    "rm_set_wait_limit": (None, [ctypes.c_uint32]),
    "rm_wait_limit": (ctypes.c_uint32, []),
    "rm_project_fwd": (ctypes.c_int, [vp, vp, i64, i64, camp, vp, vp, vp, vp, vp, vp]),
    "rm_project_bwd": (ctypes.c_int, [vp, vp, i64, i64, camp, vp, vp, vp, vp, vp]),
    "rm_scan_workspace_size": (sz, [i64]),
    "rm_scan_tiles": (ctypes.c_int, [vp, i64, vp, vp, vp, sz, vp]),
    "rm_scan_tiles_noalloc": (ctypes.c_int, [vp, i64, vp, vp, vp]),
    "rm_scan_noalloc_read_status": (ctypes.c_int, [vp, vp]),
    "rm_emit_pairs": (ctypes.c_int, [vp, vp, vp, i64, i32, i64, vp, vp, vp, vp, vp]),
    "rm_sort_workspace_size": (sz, [i64]),
    "rm_sort_pairs": (ctypes.c_int, [vp, vp, i64, vp, ctypes.c_int, vp, vp, vp, sz, vp, vp]),
    "rm_tile_ranges": (ctypes.c_int, [vp, i64, vp, vp, i64, vp]),
    "rm_sort_pairs_range": (ctypes.c_int, [vp, vp, i64, vp, ctypes.c_int, ctypes.c_int, vp, vp, vp, sz, vp, vp]),
    "rm_depth_order_workspace_size": (sz, [i64]),
    "rm_depth_order": (ctypes.c_int, [vp, vp, i64, vp, vp, vp, vp, sz, vp, vp]),
    "rm_count_pairs": (ctypes.c_int, [vp, i64, vp, vp, vp]),
    "rm_emit_ordered_workspace_size": (sz, [i64]),
    "rm_emit_pairs_ordered": (ctypes.c_int, [vp, vp, vp, vp, i64, vp, i32, i64, vp, vp, vp, vp, sz, vp, vp]),
    "rm_blend_workspace_size": (sz, [i64, i64]),
    "rm_blend_hit_mask_bytes": (sz, [i64, i64, ctypes.c_int]),
    "rm_blend_status_offset": (sz, [i64, i64]),
    "rm_blend_fwd": (ctypes.c_int, [vp, vp, vp, vp, vp, i64, i64, vp, vp, camp, vp, vp, vp, vp, sz,
                                    ctypes.c_int, vp, vp]),
    "rm_blend_bwd": (ctypes.c_int, [vp, vp, vp, vp, vp, i64, i64, vp, vp, camp, vp, vp, vp, vp, vp,
                                    vp, vp, vp, sz, ctypes.c_int, vp, vp]),
    "rm_project_fwd_fine": (ctypes.c_int, [vp, vp, i64, i64, camp, vp, vp, vp, vp, vp, vp, vp]),
    "rm_jitter_bounds_workspace_size": (sz, []),
    "rm_jitter_bounds": (ctypes.c_int, [vp, i64, vp, vp, sz, vp]),
    "rm_fine_lists_workspace_size": (sz, [i64, i64, ctypes.c_int]),
    "rm_fine_lists": (ctypes.c_int, [vp, vp, i64, vp, vp, vp, vp, camp, ctypes.c_int, i64, vp, vp, vp, vp, sz,
                                     vp, vp]),
    "rm_project_fwd_multi": (ctypes.c_int, [vp, vp, i64, i64, camp, ctypes.c_int, vp, vp, vp, vp, vp, vp, vp,
                                            vp]),
    "rm_fine_lists_multi": (ctypes.c_int, [vp, vp, i64, vp, vp, vp, vp, i64, camp, ctypes.c_int, ctypes.c_int, i64,
                                           vp, vp, vp, vp, sz, vp, vp]),
    "rm_emit_pairs_multi": (ctypes.c_int, [vp, vp, vp, i64, camp, ctypes.c_int, i64, vp, vp, vp, vp, vp, vp, vp]),
    "rm_views_tile_count": (i64, [camp, ctypes.c_int]),
    "rm_calc_tet_err": (ctypes.c_int, [vp, vp, vp, vp, vp, i64, i64, vp, camp, vp, vp, vp, vp, vp, sz,
                                       ctypes.c_int, vp]),
    "rm_activate_features": (ctypes.c_int, [vp, vp, i64, vp, vp, vp, vp, vp, ctypes.c_int, ctypes.c_int, vp, i64,
                                            vp, vp]),
    "rm_activate_features_bwd": (ctypes.c_int, [vp, vp, i64, vp, vp, vp, vp, vp, ctypes.c_int, ctypes.c_int, vp,
                                                i64, vp, vp, vp, vp, vp, vp, vp, vp]),
    "rm_tets_workspace_size": (sz, [i64]),
    "rm_tets_orient": (ctypes.c_int, [vp, i64, vp, i64, vp, vp, vp, sz, vp, vp]),
    "rm_tets_cull": (ctypes.c_int, [vp, i64, vp, i64, vp, ctypes.c_float, ctypes.c_float, vp, vp, vp, vp, sz, vp,
                                    vp]),
    "rm_blend_records_size": (sz, [i64]),
    "rm_blend_pack_records": (ctypes.c_int, [vp, vp, vp, i64, i64, vp, vp, vp]),
    "rm_blend_fwd_multi": (ctypes.c_int, [vp, vp, vp, vp, vp, i64, i64, vp, vp, camp, ctypes.c_int, vp, vp, vp,
                                          vp, vp, sz, ctypes.c_int, vp, vp]),
    "rm_blend_bwd_multi": (ctypes.c_int, [vp, vp, vp, vp, vp, i64, i64, vp, vp, camp, ctypes.c_int, vp, vp, vp,
                                          vp, vp, vp, vp, vp, vp, sz, ctypes.c_int, vp, vp]),
}


def lib():
    """Load the library (once) and bind its signatures."""
    global _lib
    if _lib is None:
        with _lock:
            if _lib is None:
                if not os.path.exists(LIB_PATH):
                    raise RuntimeError(
                        f"{LIB_PATH} is missing: build it with `python -m radiance_meshes_b200.build` "
                        "(there is no CPU fallback)")
                L = ctypes.CDLL(LIB_PATH)
                for name, (res, args) in SIGNATURES.items():
                    fn = getattr(L, name)
                    fn.restype = res
                    fn.argtypes = args
                _lib = L
    return _lib


def last_error() -> str:
    return lib().rm_last_error().decode(errors="replace")


def check(rc: int, what: str = "") -> None:
    if rc != RM_OK:
        raise RuntimeError(f"{what or 'radiance_meshes_b200'} failed (status {rc}): {last_error()}")


def ptr(t) -> int | None:
    """Raw device pointer of a tensor (None for None)."""
    if t is None:
        return None
    return t.data_ptr()


def stream_handle(stream=None) -> int:
    import torch

    s = stream if stream is not None else torch.cuda.current_stream()
    return s.cuda_stream


def status_text(bits: int) -> str:
    """The RM_STATUS_* bits of a device status word, in words."""
    parts = [txt for bit, txt in STATUS_TEXT.items() if bits & bit]
    rest = bits & ~sum(STATUS_TEXT)
    if rest:
        parts.append(f"unknown bits 0x{rest:x}")
    return "; ".join(parts) or "none"


def status_code(bits: int) -> int:
    """The C-ABI status code that a device status word maps to."""
    if bits & (RM_STATUS_SCAN_TIMEOUT | RM_STATUS_SORT_TIMEOUT | RM_STATUS_QUEUE_TIMEOUT):
        return RM_ETIMEOUT
    if bits & RM_STATUS_CAPACITY:
        return RM_ECAPACITY
    return RM_EINVAL if bits else RM_OK


class DeviceStatusError(RuntimeError):
    """A kernel reported an error through a device status word."""

    def __init__(self, bits: int, where: str = ""):
        self.bits = int(bits)
        self.code = status_code(self.bits)
        super().__init__(f"{where or 'radiance_meshes_b200'}: device status 0x{self.bits:x} "
                         f"(code {self.code}): {status_text(self.bits)}")


def set_wait_limit(polls: int) -> None:
    """Iteration limit of the bounded device-side waits (0: the default)."""
    lib().rm_set_wait_limit(int(polls))


def wait_limit() -> int:
    return int(lib().rm_wait_limit())


def launch_count() -> int:
    """Kernels launched by librm_b200.so in this process so far."""
    return int(lib().rm_launch_count())
