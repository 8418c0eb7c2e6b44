"""Autotuner for the blend launches of a view batch.

Knobs, all measured on the caller's own mesh and cameras:

* tile size of the sorted lists (8, 16 or 32 pixels square) and of the
  blend (the same, or 2^k times smaller, down to 8: the sorted lists are then
  split in order, rm_fine_lists_multi).  Smaller blend tiles waste fewer
  ray/tet tests per pixel; smaller list tiles cost more pairs to sort.
* work split between the two blend kernels, i.e. pixels per thread: the
  one-thread-per-pixel dense kernel versus the pair kernel that spreads a
  strip's (entry, pixel) tests over four threads per pixel (heavy-tile
  threshold; 1 sends every tile to the pair kernel), and the pair kernel's
  resident CTAs per SM.
* pixels per work item (strip of 16 or 64 pixels).
* tets per shared-memory batch (16, 32 or 64).

Each candidate is timed with CUDA events on one eager fwd / bwd pass after a
warm-up pass.  The winner is cached in a JSON file keyed by the GPU, the mesh
size, the views' resolutions and the tile candidates
(``$RM_AUTOTUNE_CACHE``, default ``~/.cache/radiance_meshes_b200/autotune.json``).
"""
from __future__ import annotations

import json
import math
import os
import threading
from typing import Sequence

import torch

from . import _capi as C
from . import batch as B
from .camera import tcam_to_struct

__all__ = ["flags", "tune_batch", "candidates_fwd", "candidates_bwd", "cache_path", "list_configs"]

_lock = threading.Lock()


def flags(strip: int = 0, heavy_shift: int = 0, pair_ctas: int = 0, batch: int = 0) -> int:
    """Pack blend launch tunables into the flags word (0 = library default)."""
    f = 0
    if strip:
        f |= int(math.log2(strip)) << C.RM_BLEND_STRIP_SHIFT
    if heavy_shift:
        f |= int(heavy_shift) << C.RM_BLEND_HEAVY_SHIFT
    if pair_ctas:
        f |= int(pair_ctas) << C.RM_BLEND_PAIR_CTAS_SHIFT
    if batch:
        f |= int(math.log2(batch)) << C.RM_BLEND_BATCH_SHIFT
    return f


def candidates_fwd(tile: int):
    out = []
    for b in (16, 32, 64):
        for ctas in (2, 3, 4):
            out.append(dict(strip=64 if tile >= 8 else 16, heavy_shift=1, pair_ctas=ctas, batch=b))
    out.append(dict(strip=16, heavy_shift=1, pair_ctas=3, batch=32))
    out.append(dict(strip=64 if tile >= 8 else 16, heavy_shift=3, pair_ctas=2, batch=32))
    return out


def candidates_bwd(tile: int):
    out = []
    for strip in ((16, 64) if tile >= 8 else (16,)):
        for b in (16, 32, 64):
            out.append(dict(strip=strip, heavy_shift=15, pair_ctas=1, batch=b))
    out.append(dict(strip=64 if tile >= 8 else 16, heavy_shift=3, pair_ctas=1, batch=32))
    return out


def cache_path() -> str:
    return os.environ.get("RM_AUTOTUNE_CACHE",
                          os.path.join(os.path.expanduser("~"), ".cache", "radiance_meshes_b200", "autotune.json"))


def _load_cache():
    try:
        with open(cache_path()) as f:
            return json.load(f)
    except (OSError, ValueError):
        return {}


def _store_cache(key, value):
    with _lock:
        data = _load_cache()
        data[key] = value
        path = cache_path()
        try:
            os.makedirs(os.path.dirname(path), exist_ok=True)
            tmp = path + ".tmp"
            with open(tmp, "w") as f:
                json.dump(data, f, indent=1, sort_keys=True)
            os.replace(tmp, path)
        except OSError:
            pass


def _key(device, n_tets, views, tiles, backward):
    p = torch.cuda.get_device_properties(device)
    res = ",".join(f"{v.width}x{v.height}" for v in views)
    return (f"{p.name}|sm{p.multi_processor_count}|T{int(round(math.log2(max(n_tets, 1)) * 4))}|{res}|"
            f"tiles{'/'.join(map(str, tiles))}|{'fwdbwd' if backward else 'fwd'}")


def _time(fn, reps=2):
    fn()  # warm-up (also sets kernel attributes)
    torch.cuda.synchronize()
    best = float("inf")
    for _ in range(reps):
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record()
        fn()
        b.record()
        b.synchronize()
        best = min(best, a.elapsed_time(b))
    return best


def list_configs(tiles):
    """(list tile, fine shift) pairs: lists sorted on `tile`-pixel tiles and
    blended on tiles 2^shift times smaller, down to 8 pixels."""
    out = []
    for t in tiles:
        shift = 0
        while (t >> shift) >= 8:
            out.append((t, shift))
            shift += 1
    return out


def tune_batch(indices: torch.Tensor, vertices: torch.Tensor, cell_values: torch.Tensor, views: Sequence,
               device=None, tiles=(8, 16, 32), backward: bool = True, use_cache: bool = True) -> dict:
    """Pick the list tile size, the blend tile size (fine split) and the blend
    flags for rendering ``views`` (objects with ``tcam(tile_size=...)``, e.g.
    ``scenes.View``) of this mesh.

    Returns {"tile", "fine_shift", "fwd_flags", "bwd_flags", "fwd", "bwd",
    "ms"} where "ms" holds the measured times per configuration
    ("<tile>/<blend tile>": lists, blend fwd, blend bwd).
    """
    device = device or vertices.device
    key = _key(device, indices.shape[0], views, tiles, backward)
    if use_cache:
        hit = _load_cache().get(key)
        if hit is not None:
            return dict(hit, cached=True)
    results = {}
    for tile, shift in list_configs(tiles):
        cams = [tcam_to_struct(v.tcam(tile_size=tile)) for v in views]
        vb = B.ViewBatch(cams)
        br = B.BatchedRasterizer(indices, vertices, cell_values, vb, fine_shift=shift)
        btile = tile >> shift
        t_lists = _time(lambda: (br._project_scan(), br._lists()))
        best_f = None
        for cand in candidates_fwd(btile):
            br.fwd_flags = flags(**cand)
            t = _time(br._blend_fwd)
            if best_f is None or t < best_f[0]:
                best_f = (t, cand)
        br.fwd_flags = flags(**best_f[1])
        br._blend_fwd()
        best_b = (0.0, None)
        if backward:
            br.grad_img.normal_()
            best_b = None
            for cand in candidates_bwd(btile):
                br.bwd_flags = flags(**cand)
                t = _time(br._blend_bwd)
                if best_b is None or t < best_b[0]:
                    best_b = (t, cand)
        pairs = int(br.fine_total.item()) if shift else int(br.total.item())
        results[(tile, shift)] = dict(lists=t_lists, fwd=best_f[0], bwd=best_b[0], fwd_cand=best_f[1],
                                      bwd_cand=best_b[1], pairs=pairs)
        del br
        torch.cuda.empty_cache()
    total = lambda t: results[t]["lists"] + results[t]["fwd"] + results[t]["bwd"]
    fastest = min(results, key=total)
    # Within 3% of the fastest (the timing noise of one sample), take the
    # smallest split: a split of more than one level keeps a footprint of
    # 48 bytes per tet and view in HBM and cuts longer lists per frame.
    near = [t for t in results if total(t) <= 1.03 * total(fastest)]
    best = min(near, key=lambda t: (t[1], total(t)))
    r = results[best]
    name = lambda ts: f"{ts[0]}/{ts[0] >> ts[1]}"
    out = {"tile": best[0], "fine_shift": best[1], "fwd_flags": flags(**r["fwd_cand"]),
           "bwd_flags": flags(**r["bwd_cand"]) if r["bwd_cand"] else 0,
           "fwd": r["fwd_cand"], "bwd": r["bwd_cand"],
           "ms": {name(t): {k: round(v, 4) for k, v in results[t].items() if k in ("lists", "fwd", "bwd")}
                  for t in results},
           "pairs": {name(t): results[t]["pairs"] for t in results}}
    if use_cache:
        _store_cache(key, out)
    return dict(out, cached=False)
