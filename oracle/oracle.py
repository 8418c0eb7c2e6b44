"""Python bindings of the CPU oracle (test infrastructure only).

Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline
leg import this module, and only as the checker.  It wraps ``liborc.so``
(built from ``rm_oracle.cpp`` by the Makefile beside it), a C++ restatement of
the reference rasterizer (``delaunay_rasterization/internal/slang/*.slang`` and
``sort_by_keys.cu``); see the header of ``rm_oracle.cpp`` for the file:line map.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None

i32p = np.ctypeslib.ndpointer(np.int32, flags="C_CONTIGUOUS")
i64p = np.ctypeslib.ndpointer(np.int64, flags="C_CONTIGUOUS")
f32p = np.ctypeslib.ndpointer(np.float32, flags="C_CONTIGUOUS")
f64p = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")


def build(force: bool = False) -> str:
    path = os.path.join(_HERE, "liborc.so")
    src = os.path.join(_HERE, "rm_oracle.cpp")
    if force or not os.path.exists(path) or os.path.getmtime(path) < os.path.getmtime(src):
        subprocess.run(["make", "-C", _HERE, "-B", "liborc.so"], check=True, capture_output=True)
    return path


def lib():
    global _LIB
    if _LIB is None:
        path = os.path.join(_HERE, "liborc.so")
        if not os.path.exists(path):
            build()
        L = ctypes.CDLL(path)
        cam = ctypes.c_void_p
        L.orc_project.argtypes = [i32p, f32p, ctypes.c_int64, cam, i32p, i32p, f32p, f32p]
        L.orc_scan_emit.restype = ctypes.c_int64
        L.orc_scan_emit.argtypes = [i32p, i32p, f32p, ctypes.c_int64, ctypes.c_int32, i32p,
                                    ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int64]
        L.orc_sort.argtypes = [i64p, i32p, ctypes.c_int64, ctypes.c_int]
        L.orc_ranges.argtypes = [i64p, ctypes.c_int64, i32p, ctypes.c_int64]
        L.orc_blend_fwd_f32.argtypes = [i32p, i32p, i32p, f32p, f32p, ctypes.c_int64, f32p, cam,
                                        f32p, f32p, i32p]
        L.orc_blend_fwd_f64.argtypes = [i32p, i32p, i32p, f64p, f64p, ctypes.c_int64, f32p, cam,
                                        f64p, f64p, i32p, ctypes.c_void_p, ctypes.c_void_p,
                                        ctypes.c_void_p, ctypes.c_void_p]
        L.orc_blend_bwd_f32.argtypes = [i32p, i32p, i32p, f32p, f32p, ctypes.c_int64, f32p, cam,
                                        f32p, f32p, i32p, f32p, ctypes.c_void_p, f64p, f64p]
        L.orc_blend_bwd_f64.argtypes = [i32p, i32p, i32p, f64p, f64p, ctypes.c_int64, f32p, cam,
                                        f64p, f64p, i32p, f64p, ctypes.c_void_p, f64p, f64p]
        L.orc_calc_tet_err.argtypes = [i32p, i32p, i32p, f32p, f32p, ctypes.c_int64, cam, f32p, f32p, f64p,
                                       i64p, i32p]
        L.orc_linear_loss_f64.restype = ctypes.c_double
        L.orc_linear_loss_f64.argtypes = [i32p, i32p, i32p, f64p, f64p, ctypes.c_int64, f32p, cam,
                                          ctypes.c_void_p, f64p, ctypes.c_void_p, ctypes.c_void_p]
        L.orc_project_bwd.argtypes = [i32p, f32p, ctypes.c_int64, cam, i32p, ctypes.c_void_p,
                                      ctypes.c_void_p, f64p]
        L.orc_power_f64.argtypes = [i32p, f64p, ctypes.c_int64, f64p, f64p, f64p]
        L.orc_quadrature_f64.argtypes = [i32p, i32p, i32p, f64p, f64p, ctypes.c_int64, f32p, cam,
                                         ctypes.c_double, ctypes.c_double, ctypes.c_int, f64p]
        L.orc_blend_fwd_f32_masked.argtypes = [i32p, i32p, i32p, f32p, f32p, ctypes.c_int64, f32p, cam,
                                               f32p, f32p, i32p, ctypes.c_void_p]
        L.orc_blend_bwd_f32_masked.argtypes = [i32p, i32p, i32p, f32p, f32p, ctypes.c_int64, f32p, cam,
                                               f32p, f32p, i32p, f32p, ctypes.c_void_p, f64p, f64p,
                                               ctypes.c_void_p]
        L.orc_max_threads.restype = ctypes.c_int
        L.orc_set_threads.argtypes = [ctypes.c_int]
        _LIB = L
    return _LIB


def _ptr(a):
    return None if a is None else a.ctypes.data_as(ctypes.c_void_p)


def _c(a, dt):
    return np.ascontiguousarray(a, dtype=dt)


def camstruct(tcam):
    from radiance_meshes_b200.camera import tcam_to_struct

    return tcam_to_struct(tcam)


def cam_ref(cs):
    return ctypes.cast(ctypes.pointer(cs), ctypes.c_void_p)


def project(indices, vertices, cs):
    T = len(indices)
    tiles = np.zeros(T, np.int32)
    rect = np.zeros((T, 4), np.int32)
    vs = np.zeros((T, 3), np.float32)
    cc = np.zeros((T, 3), np.float32)
    lib().orc_project(_c(indices, np.int32), _c(vertices, np.float32), T, cam_ref(cs), tiles, rect, vs, cc)
    return tiles, rect, vs, cc


def scan_emit(tiles, rect, vs, grid_w):
    T = len(tiles)
    offsets = np.zeros(T, np.int32)
    P = lib().orc_scan_emit(_c(tiles, np.int32), _c(rect, np.int32), _c(vs, np.float32), T, grid_w,
                            offsets, None, None, 0)
    keys = np.zeros(P, np.int64)
    vals = np.zeros(P, np.int32)
    lib().orc_scan_emit(_c(tiles, np.int32), _c(rect, np.int32), _c(vs, np.float32), T, grid_w, offsets,
                        _ptr(keys), _ptr(vals), P)
    return offsets, keys, vals


def sort_pairs(keys, vals, end_bit):
    k = keys.copy()
    v = vals.copy()
    lib().orc_sort(k, v, len(k), end_bit)
    return k, v


def tile_ranges(sorted_keys, n_tiles):
    r = np.zeros((n_tiles, 2), np.int32)
    lib().orc_ranges(_c(sorted_keys, np.int64), len(sorted_keys), r, n_tiles)
    return r


def end_bit_for(grid_w, grid_h):
    return 32 + int(grid_w * grid_h).bit_length()


def rasterize_lists(indices, vertices, tcam):
    """Stages (a)-(c) of the FP32 restatement: the reference's
    vertex_and_tile_shader (tile_shader_slang.py:24-72) on the CPU."""
    cs = camstruct(tcam)
    tiles, rect, vs, cc = project(indices, vertices, cs)
    offsets, keys, vals = scan_emit(tiles, rect, vs, cs.grid_width)
    sk, sv = sort_pairs(keys, vals, end_bit_for(cs.grid_width, cs.grid_height))
    ranges = tile_ranges(sk, cs.grid_width * cs.grid_height)
    return dict(cam=cs, tiles_touched=tiles, rect=rect, vs=vs, circumcenter=cc, offsets=offsets,
                keys=keys, values=vals, sorted_keys=sk, sorted_ids=sv, ranges=ranges)


def calc_tet_err(lists, indices, vertices, cell_values, pixel_err, ssim_err):
    """calc_tet_err (alphablend_shader_interp.slang:433-599) on the CPU:
    returns (tet_err [T,16] float64, count [T] int64, tmax [T] int32)."""
    T = len(indices)
    err = np.zeros((T, 16), np.float64)
    cnt = np.zeros(T, np.int64)
    tmax = np.zeros(T, np.int32)
    lib().orc_calc_tet_err(_c(lists["sorted_ids"], np.int32), _c(lists["ranges"], np.int32), _c(indices, np.int32),
                           _c(vertices, np.float32), _c(cell_values, np.float32), T, cam_ref(lists["cam"]),
                           _c(pixel_err, np.float32), _c(ssim_err, np.float32), err, cnt, tmax)
    return err, cnt, tmax


def blend_fwd_f32(lists, indices, vertices, cell_values, jitter):
    cs = lists["cam"]
    H, W = cs.image_height, cs.image_width
    img = np.zeros((H, W, 4), np.float32)
    dist = np.zeros((H, W, 5), np.float32)
    nc = np.zeros((H, W), np.int32)
    lib().orc_blend_fwd_f32(_c(lists["sorted_ids"], np.int32), _c(lists["ranges"], np.int32),
                            _c(indices, np.int32), _c(vertices, np.float32), _c(cell_values, np.float32),
                            len(indices), _c(jitter, np.float32), cam_ref(cs), img, dist, nc)
    return img, dist, nc


def blend_fwd_f64(lists, indices, vertices, cell_values, jitter, cut=None, tile_mask=None):
    cs = lists["cam"]
    H, W = cs.image_height, cs.image_width
    img = np.zeros((H, W, 4), np.float64)
    dist = np.zeros((H, W, 5), np.float64)
    nc = np.zeros((H, W), np.int32)
    own = np.zeros((H, W), np.int32)
    inv = np.zeros(1, np.int64)
    cut_a = None if cut is None else _c(cut, np.int32)
    mask_a = None if tile_mask is None else _c(tile_mask, np.uint8)
    lib().orc_blend_fwd_f64(_c(lists["sorted_ids"], np.int32), _c(lists["ranges"], np.int32),
                            _c(indices, np.int32), _c(vertices, np.float64), _c(cell_values, np.float64),
                            len(indices), _c(jitter, np.float32), cam_ref(cs), img, dist, nc, _ptr(cut_a),
                            _ptr(own), _ptr(mask_a), _ptr(inv))
    return img, dist, nc, own, int(inv[0])


def blend_bwd(lists, indices, vertices, cell_values, jitter, img, dist, nc, gimg, gdist=None,
              precision="f64"):
    cs = lists["cam"]
    gv = np.zeros((len(vertices), 3), np.float64)
    gc = np.zeros((len(indices), 7), np.float64)
    if precision == "f32":
        gd = None if gdist is None else _c(gdist, np.float32)
        lib().orc_blend_bwd_f32(_c(lists["sorted_ids"], np.int32), _c(lists["ranges"], np.int32),
                                _c(indices, np.int32), _c(vertices, np.float32),
                                _c(cell_values, np.float32), len(indices), _c(jitter, np.float32),
                                cam_ref(cs), _c(img, np.float32), _c(dist, np.float32), _c(nc, np.int32),
                                _c(gimg, np.float32), _ptr(gd), gv, gc)
    else:
        gd = None if gdist is None else _c(gdist, np.float64)
        lib().orc_blend_bwd_f64(_c(lists["sorted_ids"], np.int32), _c(lists["ranges"], np.int32),
                                _c(indices, np.int32), _c(vertices, np.float64),
                                _c(cell_values, np.float64), len(indices), _c(jitter, np.float32),
                                cam_ref(cs), _c(img, np.float64), _c(dist, np.float64), _c(nc, np.int32),
                                _c(gimg, np.float64), _ptr(gd), gv, gc)
    return gv, gc


def linear_loss_f64(lists, indices, vertices, cell_values, jitter, cut, wimg, wdist=None, tile_mask=None):
    cs = lists["cam"]
    wd = None if wdist is None else _c(wdist, np.float64)
    mask_a = None if tile_mask is None else _c(tile_mask, np.uint8)
    return lib().orc_linear_loss_f64(_c(lists["sorted_ids"], np.int32), _c(lists["ranges"], np.int32),
                                     _c(indices, np.int32), _c(vertices, np.float64),
                                     _c(cell_values, np.float64), len(indices), _c(jitter, np.float32),
                                     cam_ref(cs), _ptr(_c(cut, np.int32)), _c(wimg, np.float64), _ptr(wd),
                                     _ptr(mask_a))


def project_bwd(indices, vertices, cs, tiles, gvs=None, gcc=None):
    gv = np.zeros((len(vertices), 3), np.float64)
    gvs_a = None if gvs is None else _c(gvs, np.float32)
    gcc_a = None if gcc is None else _c(gcc, np.float32)
    lib().orc_project_bwd(_c(indices, np.int32), _c(vertices, np.float32), len(indices), cam_ref(cs),
                          _c(tiles, np.int32), _ptr(gvs_a), _ptr(gcc_a), gv)
    return gv


def power_f64(indices, vertices, cam_pos):
    T = len(indices)
    p = np.zeros(T, np.float64)
    c = np.zeros((T, 3), np.float64)
    lib().orc_power_f64(_c(indices, np.int32), _c(vertices, np.float64), T, _c(cam_pos, np.float64), p, c)
    return p, c


def quadrature_f64(lists, indices, vertices, cell_values, jitter, t0, t1, n_samples):
    cs = lists["cam"]
    out = np.zeros((cs.image_height, cs.image_width, 4), np.float64)
    lib().orc_quadrature_f64(_c(lists["sorted_ids"], np.int32), _c(lists["ranges"], np.int32),
                             _c(indices, np.int32), _c(vertices, np.float64), _c(cell_values, np.float64),
                             len(indices), _c(jitter, np.float32), cam_ref(cs), float(t0), float(t1),
                             int(n_samples), out)
    return out


def max_threads():
    return lib().orc_max_threads()


def set_threads(n):
    lib().orc_set_threads(int(n))


def blend_fwd_bwd_f32_sample(lists, indices, vertices, cell_values, jitter, tile_mask, target):
    """FP32 restatement forward + L1-loss backward over the tiles in tile_mask
    (a bounded sample of a large workload).  Returns the number of pixels in
    the sample."""
    cs = lists["cam"]
    H, W = cs.image_height, cs.image_width
    ids = _c(lists["sorted_ids"], np.int32)
    rg = _c(lists["ranges"], np.int32)
    idx = _c(indices, np.int32)
    v = _c(vertices, np.float32)
    c = _c(cell_values, np.float32)
    j = _c(jitter, np.float32)
    m = _c(tile_mask, np.uint8)
    img = np.zeros((H, W, 4), np.float32)
    dist = np.zeros((H, W, 5), np.float32)
    nc = np.zeros((H, W), np.int32)
    lib().orc_blend_fwd_f32_masked(ids, rg, idx, v, c, len(idx), j, cam_ref(cs), img, dist, nc, _ptr(m))
    gimg = np.zeros((H, W, 4), np.float32)
    gimg[..., :3] = np.sign(img[..., :3] - target) / float(H * W * 3)
    gv = np.zeros((len(v), 3), np.float64)
    gc = np.zeros((len(idx), 7), np.float64)
    lib().orc_blend_bwd_f32_masked(ids, rg, idx, v, c, len(idx), j, cam_ref(cs), img, dist, nc, gimg, None, gv, gc,
                                   _ptr(m))
    return img, gv, gc
