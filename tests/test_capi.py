"""The C-ABI library: loads without a GPU, exports every symbol declared in
include/rm_capi.h, answers size queries and rejects bad arguments before any
device work."""
import ctypes

import numpy as np
import os
import re

import pytest

from radiance_meshes_b200 import _capi as C
from radiance_meshes_b200.camera import RMCamera, tcam_to_struct
from radiance_meshes_b200 import scenes

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    src = open(os.path.join(ROOT, "include", "rm_capi.h")).read()
    return sorted(set(re.findall(r"RM_API\s+[\w\s\*]+?\b(rm_\w+)\s*\(", src)))


def test_all_declared_symbols_exported():
    names = declared_symbols()
    assert len(names) >= 14
    L = C.lib()
    for n in names:
        assert hasattr(L, n), n
        assert n in C.SIGNATURES, f"{n} has no ctypes signature"


def test_struct_layout():
    # 33 floats then 8 int32 (include/rm_capi.h)
    assert ctypes.sizeof(RMCamera) == 164
    assert RMCamera.image_height.offset == 136


def test_size_queries():
    L = C.lib()
    assert L.rm_abi_version() == 2
    assert L.rm_blend_workspace_size(1000, 300) >= 1000 * 128 + 300 * 4
    assert L.rm_scan_workspace_size(5000) >= 16 + 8 * 2
    assert L.rm_sort_workspace_size(1_000_000) > 12 * 1_000_000


def test_tets_argument_checks():
    L = C.lib()
    assert L.rm_tets_workspace_size(1000) >= 8 * 1000
    ws = 256
    assert L.rm_tets_orient(None, 10, 16, 10, 16, 16, ws, 1 << 20, None, None) == C.RM_EINVAL
    assert L.rm_tets_orient(16, 10, 16, 10, 24, 16, ws, 1 << 20, None, None) == C.RM_EINVAL  # misaligned output
    assert L.rm_tets_orient(16, 10, 16, 10, 16, 16, ws, 8, None, None) == C.RM_EINVAL  # workspace too small
    assert "workspace" in C.last_error()
    assert L.rm_tets_cull(16, 10, 16, 10, None, 0.5, 0.0, 16, None, 16, ws, 1 << 20, None, None) == C.RM_EINVAL
    assert L.rm_tets_orient(16, -1, 16, 10, 16, 16, ws, 1 << 20, None, None) == C.RM_EINVAL


def test_blend_status_offset_inside_workspace():
    L = C.lib()
    for T, G in ((0, 1), (1000, 300), (1_300_000, 4346)):
        n = L.rm_blend_workspace_size(T, G)
        off = L.rm_blend_status_offset(T, G)
        assert off % 4 == 0 and off + 4 <= n and off >= n - 256


def test_wait_limit_setting():
    """The bounded-wait limit is a process-wide setting; 0 restores the
    default (no device work involved)."""
    default = C.wait_limit()
    assert default == 1 << 22
    try:
        C.set_wait_limit(7)
        assert C.wait_limit() == 7
    finally:
        C.set_wait_limit(0)
    assert C.wait_limit() == default


def test_status_words_in_words():
    assert C.status_code(C.RM_STATUS_SCAN_TIMEOUT | C.RM_STATUS_BAD_INDEX) == C.RM_ETIMEOUT
    assert C.status_code(C.RM_STATUS_CAPACITY) == C.RM_ECAPACITY
    assert C.status_code(C.RM_STATUS_NONFINITE) == C.RM_EINVAL
    assert C.status_code(0) == C.RM_OK
    err = C.DeviceStatusError(C.RM_STATUS_BAD_INDEX | C.RM_STATUS_OVERFLOW, "x")
    assert isinstance(err, RuntimeError) and err.code == C.RM_EINVAL
    assert "outside [0, n_verts)" in str(err) and "INT32_MAX" in str(err)


def test_noalloc_status_rejects_null():
    assert C.lib().rm_scan_noalloc_read_status(None, None) == C.RM_EINVAL


def _cam():
    mesh, view = scenes.workload_gradient_check()
    return tcam_to_struct(view.tcam())


def test_camera_types_and_distortion():
    """Perspective and fisheye cameras with distortion pass the camera check
    (the call then stops at its NULL buffers); other camera types and NaN
    distortion are rejected."""
    L = C.lib()
    for ctype in (0, 1):
        cam = _cam()
        cam.camera_type = ctype
        cam.distortion[0] = 0.1
        rc = L.rm_project_fwd(None, None, 10, 10, ctypes.byref(cam), None, None, None, None, None, None)
        assert rc == C.RM_EINVAL and "NULL" in C.last_error()
    cam = _cam()
    cam.camera_type = 2
    rc = L.rm_project_fwd(None, None, 10, 10, ctypes.byref(cam), None, None, None, None, None, None)
    assert rc == C.RM_EINVAL and "camera_type" in C.last_error()
    cam = _cam()
    cam.distortion[1] = float("nan")
    rc = L.rm_project_fwd(None, None, 10, 10, ctypes.byref(cam), None, None, None, None, None, None)
    assert rc == C.RM_EINVAL and "NaN" in C.last_error()


def test_rejects_null_and_misaligned():
    L = C.lib()
    cam = _cam()
    assert L.rm_project_fwd(None, None, 10, 10, ctypes.byref(cam), None, None, None, None, None, None) == C.RM_EINVAL
    assert "NULL" in C.last_error()
    assert L.rm_sort_pairs(None, None, 10, None, 0, None, None, None, 0, None, None) == C.RM_EINVAL
    assert L.rm_sort_pairs(None, None, 10, None, 65, None, None, None, 0, None, None) == C.RM_EINVAL
    # unsupported tile size
    cam.tile_width = 5
    cam.tile_height = 5
    cam.grid_width = 26
    cam.grid_height = 26
    rc = L.rm_blend_fwd(None, 16, 16, 16, 16, 10, 10, None, 16, ctypes.byref(cam), 16, 16, 16, 256, 1 << 20, 0,
                        None, None)
    assert rc == C.RM_EINVAL and "tile" in C.last_error()


def test_zero_sizes_are_noops():
    L = C.lib()
    cam = _cam()
    assert L.rm_project_fwd(None, None, 0, 0, ctypes.byref(cam), None, None, None, None, None, None) == C.RM_OK
    assert L.rm_sort_pairs(None, None, 0, None, 40, None, None, None, 0, None, None) == C.RM_OK
    assert L.rm_emit_pairs(None, None, None, 0, 1, 0, None, None, None, None, None) == C.RM_OK


def test_python_camera_validation():
    mesh, view = scenes.workload_gradient_check()
    t = view.tcam()
    t["distortion_params"] = [0.1, 0, 0, 0]
    t["camera_type"] = 1
    assert tcam_to_struct(t).camera_type == 1
    t["camera_type"] = 3
    with pytest.raises(ValueError):
        tcam_to_struct(t)
    t = view.tcam()
    t["distortion_params"] = [float("inf"), 0, 0, 0]
    with pytest.raises(ValueError):
        tcam_to_struct(t)
    t = view.tcam()
    t["grid_width"] = 1
    with pytest.raises(ValueError):
        tcam_to_struct(t)


def test_launch_counter_starts_at_zero_without_gpu():
    assert C.launch_count() >= 0


def _ring_cams(res, tile=16):
    views = scenes.ring_views(len(res), res, tile_size=tile)
    return [tcam_to_struct(v.tcam()) for v in views]


def test_view_batch_offsets_and_tile_count():
    from radiance_meshes_b200 import batch as B

    res = [(840, 1297), (1080, 1920), (480, 640)]
    cams = _ring_cams(res)
    vb = B.ViewBatch(cams)
    grids = [((h + 15) // 16, (w + 15) // 16) for h, w in res]
    assert vb.tile_base == [0, grids[0][0] * grids[0][1], grids[0][0] * grids[0][1] + grids[1][0] * grids[1][1],
                            sum(a * b for a, b in grids)]
    assert vb.pixel_base[-1] == sum(h * w for h, w in res)
    assert vb.end_bit == 32 + vb.n_tiles.bit_length()
    L = C.lib()
    assert L.rm_views_tile_count(vb.array, vb.n) == vb.n_tiles
    assert C.RM_MAX_VIEWS == B.MAX_VIEWS


def test_view_batch_rejects_bad_batches():
    from radiance_meshes_b200 import batch as B

    L = C.lib()
    cams = _ring_cams([(64, 64), (64, 64)], tile=16)
    mixed = cams[:1] + _ring_cams([(64, 64)], tile=8)
    with pytest.raises(ValueError):
        B.ViewBatch(mixed)
    arr = (RMCamera * 2)(*mixed)
    assert L.rm_views_tile_count(arr, 2) == -1
    assert "tile size" in C.last_error()
    many = (RMCamera * (C.RM_MAX_VIEWS + 1))(*([cams[0]] * (C.RM_MAX_VIEWS + 1)))
    assert L.rm_views_tile_count(many, C.RM_MAX_VIEWS + 1) == -1
    assert L.rm_views_tile_count(arr, 0) == -1
    rc = L.rm_project_fwd_multi(None, None, 10, 10, arr, 2, None, None, None, None, None, None, None, None)
    assert rc == C.RM_EINVAL
    ok = (RMCamera * 2)(*cams)
    assert L.rm_project_fwd_multi(None, None, 10, 10, ok, 2, None, None, None, None, None, None, None, None) == C.RM_EINVAL
    assert L.rm_project_fwd_multi(None, None, 0, 0, ok, 2, None, None, None, None, None, None, None, None) == C.RM_OK
    assert L.rm_emit_pairs_multi(None, None, None, 0, ok, 2, 0, None, None, None, None, None, None, None) == C.RM_OK


def test_autotune_flag_packing():
    from radiance_meshes_b200 import autotune as AT

    f = AT.flags(strip=16, heavy_shift=3, pair_ctas=2, batch=64)
    assert (f >> C.RM_BLEND_STRIP_SHIFT) & 0xff == 4
    assert (f >> C.RM_BLEND_HEAVY_SHIFT) & 0xf == 3
    assert (f >> C.RM_BLEND_PAIR_CTAS_SHIFT) & 0xf == 2
    assert (f >> C.RM_BLEND_BATCH_SHIFT) & 0xf == 6
    assert AT.flags() == 0
    for tile in (8, 16, 32):
        for cand in AT.candidates_fwd(tile) + AT.candidates_bwd(tile):
            assert tile * tile % cand["strip"] == 0


def test_serving_trace_is_seeded_poisson():
    tr = scenes.serving_trace(4000, 200.0, ["a", "b", "c"], seed=7)
    tr2 = scenes.serving_trace(4000, 200.0, ["a", "b", "c"], seed=7)
    assert [x[0] for x in tr] == [x[0] for x in tr2]
    gaps = np.diff([0.0] + [x[0] for x in tr])
    assert abs(gaps.mean() - 1 / 200.0) < 0.1 / 200.0
    names = [x[1] for x in tr]
    assert all(abs(names.count(n) / len(names) - 1 / 3) < 0.05 for n in "abc")
    res = [(v.height, v.width) for _, _, v in tr]
    assert set(res) == set(scenes.SERVING_RESOLUTIONS)
    for _, _, v in tr[:50]:
        assert abs(np.linalg.norm(v.cam_pos) - 4.0) < 1e-5


def test_tcam_conversion_cache():
    """tcam_to_struct returns the same camera from its cache for the same
    tensors, a fresh one after an in-place change, and independent copies."""
    import torch

    from radiance_meshes_b200.camera import pinhole_tcam, tcam_to_struct

    tcam = pinhole_tcam((0.0, 0.0, -3.0), (0.0, 0.0, 0.0), 64, 96)
    a = tcam_to_struct(tcam)
    b = tcam_to_struct(tcam)
    assert bytes(a) == bytes(b)
    b.min_t = 7.0  # a copy: the cached camera is untouched
    assert tcam_to_struct(tcam).min_t == a.min_t
    with torch.no_grad():
        tcam["cam_pos"][0] += 1.0
    c = tcam_to_struct(tcam)
    assert c.cam_pos[0] == a.cam_pos[0] + 1.0
    tcam2 = dict(tcam, tile_width=8, tile_height=8, grid_width=12, grid_height=8)
    assert tcam_to_struct(tcam2).tile_width == 8


def test_fine_list_entry_points_validate():
    """The footprint, jitter-bounds and split entry points reject missing or
    misaligned buffers and bad split factors before touching the device, and
    size their workspaces from the fine tiles and pairs."""
    L = C.lib()
    cam = _cam()
    cams = (RMCamera * 1)(cam)
    rc = L.rm_project_fwd_fine(None, None, 10, 10, ctypes.byref(cam), None, None, None, None, None, None, None)
    assert rc == C.RM_EINVAL and "NULL" in C.last_error()
    assert L.rm_project_fwd_fine(None, None, 0, 0, ctypes.byref(cam), None, None, None, None, None, None, None) == C.RM_OK
    assert L.rm_jitter_bounds_workspace_size() >= 16
    assert L.rm_jitter_bounds(None, 10, None, None, 0, None) == C.RM_EINVAL
    assert L.rm_jitter_bounds(8, 10, 16, 16, 0, None) == C.RM_EINVAL and "workspace" in C.last_error()
    assert L.rm_jitter_bounds(4, 10, 16, 16, 1 << 20, None) == C.RM_EINVAL and "misaligned" in C.last_error()
    small = L.rm_fine_lists_workspace_size(1000, 10, 1)
    assert L.rm_fine_lists_workspace_size(1000, 1_000_000, 1) >= small + 1_000_000 - 256
    assert L.rm_fine_lists_workspace_size(1000, 1_000_000, 3) >= 8 * 1_000_000
    ws = 1 << 30
    rc = L.rm_fine_lists(16, 16, 10, None, 16, None, 16, ctypes.byref(cam), 1, 10, 16, 16, 16, 256, ws, None, None)
    assert rc == C.RM_EINVAL and "footprint" in C.last_error()
    rc = L.rm_fine_lists(16, 16, 10, None, 16, 16, None, ctypes.byref(cam), 1, 10, 16, 16, 16, 256, ws, None, None)
    assert rc == C.RM_EINVAL and "jitter_bounds" in C.last_error()
    rc = L.rm_fine_lists(16, 16, 10, None, 16, 16, 16, ctypes.byref(cam), 4, 10, 16, 16, 16, 256, ws, None, None)
    assert rc == C.RM_EINVAL and "fine_shift" in C.last_error()
    rc = L.rm_fine_lists(16, 16, 10, None, 16, 24, 16, ctypes.byref(cam), 1, 10, 16, 16, 16, 256, ws, None, None)
    assert rc == C.RM_EINVAL and "misaligned" in C.last_error()
    # packed bits (no footprint) only for a 2x split
    rc = L.rm_fine_lists_multi(16, 16, 10, None, 16, None, None, 10, cams, 1, 2, 10, 16, 16, 16, 256, ws, None, None)
    assert rc == C.RM_EINVAL and "packed" in C.last_error()
