"""Benchmark: fwd+bwd Mpix/s of the tetrahedral tile rasterizer (training step).

Workload (default): 200,000 points drawn as a mixture of 64 anisotropic
Gaussians plus 10% uniform background (seed 2), Delaunay-tetrahedralised
(~1.3M tets), fp32 features with 30% of densities at 1e-4, one 1297x840
camera on a radius-4 ring at height 0.5, 16x16 tiles, L1 loss against a
random target.  A step is: projection, scan/emit/sort/ranges, blend forward,
L1 loss, blend backward (the drop-in autograd path), and on N>1 ranks an
NCCL all-reduce of the vertex and cell-value gradients (each rank renders its
own ring view: data-parallel multi-view training, weak scaling).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]

Rank 0 prints one JSON line.  --impl reference times the CPU restatement of
the reference path (the oracle, OpenMP on all host cores) on a bounded tile
sample of the same workload.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

METRIC = "fwd+bwd Mpix/s @1.3M tets"
UNIT = "Mpix/s"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=150)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["b200", "reference"], default="b200")
    ap.add_argument("--points", type=int, default=200_000)
    ap.add_argument("--tile", type=int, default=16)
    ap.add_argument("--height", type=int, default=840)
    ap.add_argument("--width", type=int, default=1297)
    ap.add_argument("--cpu-seconds", type=float, default=15.0, help="budget of the CPU-baseline sample")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-extras", action="store_true",
                    help="single GPU: skip the multi-view and serving results nested in the training line")
    ap.add_argument("--stage", choices=["ldg", "tma"], default="ldg",
                    help="how the backward stages tet records in shared memory: per-thread loads, or bulk copies "
                         "(cp.async.bulk, two batches in flight); bulk copies only in single-GPU runs")
    ap.add_argument("--pair-ctas", type=int, default=0,
                    help="resident CTAs per SM of the forward's pair kernel (0: the library default)")
    ap.add_argument("--bwd-batch", type=int, default=0, choices=[0, 16, 32, 64],
                    help="tets per shared-memory batch of the backward (0: the library default)")
    ap.add_argument("--profile-steps", type=int, default=0, help="(profiling) run N steps after warmup, print nothing")
    ap.add_argument("--workload", choices=["training", "multiview", "serving", "sort"], default="training",
                    help="training: the 1.3M-tet fwd+bwd step (default line); multiview: 16 views of a "
                         "1M-point mesh, batched CUDA-graph step vs 16 plain per-view steps; serving: "
                         "Poisson requests over three resident meshes, p50/p99 latency; sort: the pair "
                         "sort alone on random keys (--sort-pairs, --sort-bits)")
    ap.add_argument("--sort-pairs", type=int, default=24_000_000)
    ap.add_argument("--sort-bits", default="0,47", help="key bits [begin,end) of the sort workload")
    ap.add_argument("--sv-points", default="250000,1000000,3000000")
    ap.add_argument("--sv-rate", type=float, default=200.0)
    ap.add_argument("--sv-requests", type=int, default=2000)
    ap.add_argument("--sv-warmup", type=int, default=200)
    ap.add_argument("--sv-streams", type=int, default=2, help="concurrent batches of the server")
    ap.add_argument("--sv-max-views", type=int, default=4, help="views per batch of the server")
    ap.add_argument("--sv-tile", type=int, default=0, help="tile size (0: autotuned on the middle mesh)")
    ap.add_argument("--sv-low-rate", type=float, default=120.0,
                    help="a second Poisson run at this rate (0: none): latency below saturation")
    ap.add_argument("--mv-points", type=int, default=1_000_000)
    ap.add_argument("--mv-views", type=int, default=16)
    ap.add_argument("--mv-tile", type=int, default=0, help="tile size of the batched step (0: autotuned)")
    return ap.parse_args()


def dist_env():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def workload(args, rank, world):
    from radiance_meshes_b200 import scenes

    mesh, view = scenes.workload_training_step(n_points=args.points, seed=2, tile_size=args.tile,
                                               height=args.height, width=args.width)
    if world > 1 and rank > 0:
        th = 2.0 * math.pi * rank / world
        view = scenes._view((4.0 * math.cos(th), 0.5, 4.0 * math.sin(th)), (0.0, 0.0, 0.0), args.height,
                            args.width, 60.0, args.tile)
    return mesh, view


# ------------------------------------------------------------------ clocks --
class ClockSampler:
    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index, interval_ms=25):
        vis = os.environ.get("CUDA_VISIBLE_DEVICES")
        if vis:
            ids = [x.strip() for x in vis.split(",") if x.strip()]
            index = ids[index] if index < len(ids) else index
        self.index = index
        self.interval_ms = int(interval_ms)
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.QUERY}", "--format=csv,noheader,nounits",
                                          "-i", str(self.index), "-lms", str(self.interval_ms)], stdout=subprocess.PIPE,
                                         stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except (OSError, FileNotFoundError):
            self.proc = None
        # nvidia-smi's start-up (NVML initialisation) stalls CUDA calls of this
        # process for a while: wait for its first sample before the timed region
        t0 = time.time()
        while self.proc is not None and not self.lines and self.proc.poll() is None and time.time() - t0 < 15:
            time.sleep(0.02)
        self.t_start = time.time()  # the timed region runs inside the with block
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append((time.time(), line.strip()))

    def __exit__(self, *exc):
        self.t_end = time.time()
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        t0, t1 = getattr(self, "t_start", 0.0), getattr(self, "t_end", float("inf"))
        inside = [ln for t, ln in self.lines if t0 <= t <= t1]
        for ln in inside:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for k, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(k)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"], "samples": 0}
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm),
                "interval_ms": self.interval_ms}


def issue_roofline(kernel, launch_ms, tests, clocks, **extra):
    """The blend kernels are bound by instruction issue, not HBM: the
    kernel's warp instructions per launch over its measured launch time,
    against the SM's issue peak (148 SMs x 4 schedulers x the sampled SM
    clock).  The instruction count is smsp__inst_executed.sum of one launch
    on this workload (profiles/issue_1.3Mtets.json, an ncu capture of the
    same code; scaled by this pass's ray/tet tests over the capture's), else
    the tests of this pass x the instructions per test of a smaller capture
    (profiles/issue_model.json)."""
    out = {"ray_tet_tests_per_pass": tests, **extra}
    if not launch_ms:
        return out
    import torch

    sms = torch.cuda.get_device_properties(torch.cuda.current_device()).multi_processor_count
    mhz = clocks.get("sm_mhz") or clocks.get("sm_max_mhz") or 1965.0
    warp_inst, src = None, None
    path = os.path.join(ROOT, "profiles", "issue_1.3Mtets.json")
    if os.path.exists(path):
        with open(path) as f:
            cap = json.load(f).get(kernel)
        if cap and cap.get("ray_tet_tests_per_pass"):
            warp_inst = cap["warp_instructions_per_launch"] * tests / cap["ray_tet_tests_per_pass"]
            src = "profiles/issue_1.3Mtets.json (smsp__inst_executed.sum of one launch on this workload)"
    if warp_inst is None:
        path = os.path.join(ROOT, "profiles", "issue_model.json")
        if not os.path.exists(path):
            return out
        with open(path) as f:
            model = json.load(f).get(kernel)
        if not model:
            return out
        warp_inst = tests * model["thread_instructions_per_test"] / model["active_lanes_per_instruction"]
        src = "profiles/issue_model.json (instructions per test of the 50k-point capture)"
    achieved = warp_inst / (launch_ms * 1e-3) / 1e9
    peak = sms * 4 * mhz * 1e6 / 1e9
    out.update({"bound": "issue", "unit": "G warp instructions/s", "achieved": achieved, "peak": peak,
                "frac": achieved / peak, "warp_instructions_per_launch": warp_inst, "instructions_source": src})
    return out


# ------------------------------------------------------------- b200 arm --
# Algorithmic bytes per launch of each stage (every input read once, every
# output written once; FP32 / int32), over T tets, V vertices, P coarse pairs,
# G coarse tiles, Pb / Gb the pairs and tiles of the lists the blend walks,
# Npx pixels.  The same per-unit figures are listed in DESIGN.md.
def stage_bytes(T, V, T_vis, P, G, Pb, Gb, Npx):
    return {
        # indices + vertices in; count, rect, depth, circumcenter out (+ footprint of the visible tets)
        "rm_project_fwd": 12 * V + 16 * T + 36 * T + 48 * T_vis,
        "rm_scan_tiles": 4 * T + 4 * T,
        # rect, depth, offsets in; key + value out
        "rm_emit_pairs": 24 * T + 12 * P,
        # one logical permutation of (key, value)
        "rm_sort_pairs": 12 * P + 12 * P,
        "rm_tile_ranges": 8 * P + 8 * G,
        "rm_jitter_bounds": 8 * Npx,
        # sorted keys, ids, ranges and the footprints of the entries in; fine ids + ranges out
        "rm_fine_lists": 12 * P + 48 * P + 8 * G + 4 * Pb + 8 * Gb,
        # ranges, ids + 92 B tet record per entry, jitter in; image 16 + distortion 20 + n_contrib 4 out,
        # plus the per-frame record packing of the visible tets (92 B in, 128 B out)
        "rm_blend_fwd": 8 * Gb + 96 * Pb + 8 * Npx + 40 * Npx + 220 * T_vis,
        # ranges, ids + record, saved state 40 + grads 36 + jitter 8 per pixel, gradient read-modify-write
        "rm_blend_bwd": 8 * Gb + 96 * Pb + 84 * Npx + 2 * (28 * T + 12 * V),
        # indices, vertices, grads of depth and circumcenter in; vertex gradient read-modify-write
        "rm_project_bwd": 16 * T + 12 * V + 16 * T + 24 * V,
        # indices, vertices, circumcenter, density, rgb, grd in; features out
        "rm_activate_features": 16 * T + 12 * V + 12 * T + 28 * T + 28 * T,
        "rm_activate_features_bwd": 16 * T + 12 * V + 12 * T + 28 * T + 28 * T + 28 * T + 2 * 12 * V,
    }


def run_b200(args, after_gpu_timing=None):
    import torch
    import torch.distributed as dist

    import radiance_meshes_b200 as RMB
    from radiance_meshes_b200 import _capi
    from radiance_meshes_b200 import features as F
    from radiance_meshes_b200 import multigpu as MG
    from radiance_meshes_b200 import rasterizer as R

    world, rank, local = dist_env()
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        import datetime

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300), device_id=dev)
    RMB.install_dropin()
    from delaunay_rasterization.internal.alphablend_tiled_slang_interp import AlphaBlendTiledRender
    from delaunay_rasterization.internal.render_grid import RenderGrid
    from delaunay_rasterization.internal.tile_shader_slang import vertex_and_tile_shader

    mesh, view = workload(args, rank, world)
    H, W = view.height, view.width
    T, V = len(mesh.indices), len(mesh.vertices)
    tcam = view.tcam(device=dev)
    camst = R.camera(tcam)
    grid = RenderGrid(H, W, tile_width=args.tile, tile_height=args.tile)
    R.use_tma_staging(args.stage == "tma" and world == 1)
    if args.pair_ctas:
        R.set_blend_tuning(args.pair_ctas << _capi.RM_BLEND_PAIR_CTAS_SHIFT, R.blend_tuning()[1])
    if args.bwd_batch:
        R.set_blend_tuning(R.blend_tuning()[0], (args.bwd_batch.bit_length() - 1) << _capi.RM_BLEND_BATCH_SHIFT)
    rng = np.random.default_rng(1000 + rank)
    target_h = torch.from_numpy(rng.uniform(size=(H, W, 3)).astype(np.float32)).pin_memory()
    # The model's raw per-tet outputs (density, base colour, colour gradient),
    # turned into the blend's cell values by activate_output
    # (utils/model_util.py:93-105) at SH degree 0 from the circumcenters, as
    # the reference's get_cell_values does (models/ingp_color.py:361-387), so
    # the projection's backward runs in every step.
    raw = mesh.cell_values
    dens_h = torch.from_numpy(np.ascontiguousarray(raw[:, 0:1])).pin_memory()
    rgb_h = torch.from_numpy(np.ascontiguousarray(raw[:, 1:4])).pin_memory()
    grd_h = torch.from_numpy(np.ascontiguousarray(raw[:, 4:7])).pin_memory()
    verts_h = torch.from_numpy(mesh.vertices).pin_memory()
    idx_h = torch.from_numpy(mesh.indices).pin_memory()
    cam_center = torch.tensor(view.cam_pos, dtype=torch.float32)  # host copy: read without a device sync
    verts = verts_h.to(dev).requires_grad_(True)
    dens = dens_h.to(dev).requires_grad_(True)
    rgb = rgb_h.to(dev).requires_grad_(True)
    grd = grd_h.to(dev).requires_grad_(True)
    idx = idx_h.to(dev)
    target = target_h.to(dev)
    gen = torch.Generator(device=dev).manual_seed(5 + rank)
    flush = torch.empty(256 * 1024 * 1024, dtype=torch.uint8, device=dev)  # > 126 MB L2
    stats = {}
    const_jitter = torch.full((H, W, 2), 0.5, device=dev)

    def step(v, d, c, g, i, tgt, jitter_mode="rand", features_ready=None, target_ready=None):
        """One training step of the reference (train.py:243-258, render() of
        utils/train_util.py:15-77): per-pixel jitter drawn on the device,
        projection and tile lists, cell values, blend, L1 loss, backward."""
        for leaf in (v, d, c, g):
            leaf.grad = None
        if jitter_mode == "rand":
            jitter = torch.rand((H, W, 2), device=dev, generator=gen)  # train.py:244
        else:
            jitter = const_jitter  # render()'s default 0.5
        sorted_ids, ranges, vs, cc, mask, rect = vertex_and_tile_shader(i, v, tcam, grid)
        if features_ready is not None:  # raw features still in flight during the tiling
            torch.cuda.current_stream().wait_event(features_ready)
        cell_values = F.activate_output(cam_center, d, c, g, None, i, cc, v, 0, 0)
        img, distimg, _ = AlphaBlendTiledRender.apply(sorted_ids, ranges, i, v, cell_values, grid, tcam, jitter)
        if target_ready is not None:  # the target image arrives during the blend
            torch.cuda.current_stream().wait_event(target_ready)
        loss = (img[..., :3] - tgt).abs().mean()
        loss.backward()
        if world > 1:
            MG.allreduce_grads([v.grad, d.grad, c.grad, g.grad])
        stats["P"] = int(sorted_ids.shape[0])
        stats["fine"] = R.fine_lists_of(sorted_ids, camst, jitter)  # read after the timed steps
        stats["jitter"] = jitter
        return loss, img

    for _ in range(args.warmup):
        step(verts, dens, rgb, grd, idx, target)
    torch.cuda.synchronize()
    if args.profile_steps:
        for _ in range(args.profile_steps):
            step(verts, dens, rgb, grd, idx, target)
        torch.cuda.synchronize()
        if world > 1:
            dist.destroy_process_group()
        return None

    def timed(jitter_mode, timer=None, sampler=None):
        """K steps, per-step events on the launching stream, L2 flushed between steps."""
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()
        ev = []
        for _ in range(args.steps):
            flush.zero_()
            a = torch.cuda.Event(enable_timing=True)
            b = torch.cuda.Event(enable_timing=True)
            a.record()
            step(verts, dens, rgb, grd, idx, target, jitter_mode)
            b.record()
            ev.append((a, b))
        torch.cuda.synchronize()
        if world > 1:
            dist.barrier()
        ms = sum(a.elapsed_time(b) for a, b in ev)
        if world > 1:
            t = torch.tensor([ms], device=dev)
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            ms = float(t.item())
        return ms

    # ---- device-resident timing (headline: random jitter per step, as in training)
    launches0 = _capi.launch_count()
    # inside the timed region only the blend kernels (the roofline's
    # candidates) get event pairs; the per-stage breakdown comes from a
    # separate pass below
    timer = R.StageTimer(only=("rm_blend_fwd", "rm_blend_bwd"))
    with ClockSampler(local) as clocks, timer:
        total_ms = timed("rand")
    launches = _capi.launch_count() - launches0
    stages = timer.totals()
    total_ms_const = timed("const")  # render()'s default jitter 0.5, beside the headline
    # per-stage breakdown: every C-ABI call timed, over a separate untimed pass
    n_break = min(args.steps, 20)
    breakdown = R.StageTimer()
    with breakdown:
        for _ in range(n_break):
            flush.zero_()
            step(verts, dens, rgb, grd, idx, target)
        torch.cuda.synchronize()
    stage_pass = breakdown.totals()
    # Σ n_contrib of the last frame: the number of ray/tet tests per pass
    # (the issue-rate unit), from a separate untimed forward on the same lists
    with torch.no_grad():
        sorted_ids, ranges, vs, cc, mask, rect = vertex_and_tile_shader(idx, verts, tcam, grid)
        jit = stats["jitter"]
        fine = R.fine_lists_of(sorted_ids, camst, jit)
        if fine is not None:  # the lists the timed blend walked
            sorted_ids, ranges, bcam = fine.sorted_ids, fine.ranges, fine.cam
        else:
            bcam = camst
        cvals = F.activate_output(cam_center, dens, rgb, grd, None, idx, cc, verts, 0, 0)
        _, _, ncs, _ = R.blend_fwd(sorted_ids, ranges, idx, verts.detach(), cvals, jit, bcam,
                                   tiles_touched=mask.to(torch.int32))
        tests = int(ncs.sum().item())
        T_vis = int(mask.sum().item())

    # ---- end to end: host buffers in, loss out, copies inside the timed region
    e2e = None
    if not args.no_e2e:
        bufs = [torch.empty_like(x) for x in (verts, dens, rgb, grd)]
        idx_d = torch.empty_like(idx)
        tgt_d = torch.empty_like(target)
        loss_h = torch.empty(1, dtype=torch.float32).pin_memory()
        # Host->device copies on a copy stream, in the order the step needs
        # them: the tiling starts once the vertices and indices are in, the
        # features once the raw per-tet outputs are, the loss once the target
        # image is.
        copy_stream = torch.cuda.Stream(device=dev)
        e2e_times = []
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()
        for _ in range(args.steps):
            flush.zero_()
            a = torch.cuda.Event(enable_timing=True)
            b = torch.cuda.Event(enable_timing=True)
            a.record()
            geometry_ready = torch.cuda.Event()
            features_ready = torch.cuda.Event()
            target_ready = torch.cuda.Event()
            copy_stream.wait_event(a)
            with torch.cuda.stream(copy_stream):
                idx_d.copy_(idx_h, non_blocking=True)
                bufs[0].detach().copy_(verts_h, non_blocking=True)
                geometry_ready.record()
                for buf, host in zip(bufs[1:], (dens_h, rgb_h, grd_h)):
                    buf.detach().copy_(host, non_blocking=True)
                features_ready.record()
                tgt_d.copy_(target_h, non_blocking=True)
                target_ready.record()
            torch.cuda.current_stream().wait_event(geometry_ready)
            leaves = [x.detach().requires_grad_(True) for x in bufs]
            for x in bufs:  # the copy stream wrote them: keep the allocator from reusing them early
                x.record_stream(copy_stream)
            loss, _ = step(*leaves, idx_d, tgt_d, "rand", features_ready, target_ready)
            loss_h.copy_(loss.detach().reshape(1), non_blocking=True)
            b.record()
            b.synchronize()
            e2e_times.append((a, b))
        e2e_ms = sum(a.elapsed_time(b) for a, b in e2e_times)
        if world > 1:
            t = torch.tensor([e2e_ms], device=dev)
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            e2e_ms = float(t.item())
        h2d = sum(x.numel() * 4 for x in (verts_h, dens_h, rgb_h, grd_h, idx_h, target_h))
        e2e = {"value": world * H * W * args.steps / (e2e_ms * 1e-3) / 1e6, "unit": UNIT,
               "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": 4,
               "ms_per_step": e2e_ms / args.steps,
               "path": "vertex_and_tile_shader + activate_output + AlphaBlendTiledRender.apply (reference "
                       "arguments) + L1 + backward, inputs copied from pinned host memory every step"}

    if world > 1:
        dist.destroy_process_group()
    if rank != 0:
        return None

    Npx = H * W
    P = stats["P"]
    G = grid.grid_width * grid.grid_height
    # the blend walks the 8x8-pixel lists when the drop-in built them
    fine = stats["fine"]
    Pb = fine.n_pairs if fine is not None else P
    Gb = fine.cam.grid_width * fine.cam.grid_height if fine is not None else G
    value = world * Npx * args.steps / (total_ms * 1e-3) / 1e6
    value_const = world * Npx * args.steps / (total_ms_const * 1e-3) / 1e6
    peaks = {}
    pk = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(pk):
        with open(pk) as f:
            peaks = json.load(f)
    hbm_peak = float(peaks.get("hbm_gbs", 6650.0))
    peak_src = "measured" if "hbm_gbs" in peaks else "fallback"
    bytes_alg = stage_bytes(T, V, T_vis, P, G, Pb, Gb, Npx)
    per_stage = {}
    for k, v in stage_pass.items():
        ms = v[0] / n_break
        st = {"ms_per_step": ms, "calls": v[1]}
        if k in bytes_alg and ms > 0:
            gbs = bytes_alg[k] / (ms * 1e-3 / max(1, v[1] // n_break)) / 1e9
            st.update({"algorithmic_bytes": int(bytes_alg[k]), "gb_s": gbs, "hbm_frac": gbs / hbm_peak})
        per_stage[k] = st
    dom = max(stages.items(), key=lambda kv: kv[1][0])[0]
    dom_ms = stages[dom][0] / stages[dom][1]
    achieved = bytes_alg.get(dom, 0) / (dom_ms * 1e-3) / 1e9
    traffic = None
    tp = os.path.join(ROOT, "profiles", "traffic.json")
    if os.path.exists(tp):
        with open(tp) as f:
            traffic = json.load(f).get(dom)
    roof = {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": hbm_peak, "unit": "GB/s",
            "frac": achieved / hbm_peak, "peak_source": peak_src, "traffic": traffic,
            "algorithmic_bytes": int(bytes_alg.get(dom, 0)), "avg_launch_ms": dom_ms,
            "issue": issue_roofline(dom, dom_ms, tests, clocks.summary(),
                                    tests_per_s_fwd_plus_bwd=2 * tests / (total_ms * 1e-3 / args.steps))}
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": total_ms / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": f"training step: {args.points} mixture points, {T} tets, {W}x{H}, "
                               f"tile {args.tile}, torch.rand ray jitter per step, activate_output cell values "
                               f"(SH degree 0), L1 loss", "tets": T, "visible_tets": T_vis,
                   "points": args.points, "image": [H, W], "tile": args.tile, "pairs": P,
                   "blend_lists": ("8x8-pixel lists built beside the 16x16 ones, %d pairs" % Pb) if fine is not None
                   else "caller's tiles", "parallelism": f"dp{world} (views)" if world > 1
                   else "single view", "l2": "flushed between steps (256 MiB write)",
                   "seed": 2, "jitter": "torch.rand per step (train.py:244)",
                   "record_staging": "bulk copies (cp.async.bulk)" if R.tma_staging() else "per-thread loads",
                   "pair_ctas_per_sm": args.pair_ctas or "library default",
                   "bwd_batch": args.bwd_batch or "library default"},
        "value_jitter_0_5": {"value": value_const, "ms_per_step": total_ms_const / args.steps,
                             "jitter": "constant 0.5 (render() default)"},
        "e2e": e2e, "roofline": roof, "stages_ms": per_stage, "stages_pass_steps": n_break,
        "gpu_launches": int(launches), "clocks": clocks.summary(),
    }
    if after_gpu_timing is not None:  # every GPU-timed measurement of this line is done
        after_gpu_timing()
    if world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline(mesh, view, args.cpu_seconds)
    return line


# ------------------------------------------------------- CPU (reference) --
def cpu_sample(mesh, view, budget_s, target_frac=None):
    """FP32 restatement of the reference path (oracle) on a bounded sample:
    full projection / scan / sort / ranges, then blend fwd + L1 bwd on an even
    subset of tiles.  Returns (Mpix/s, seconds, sample description, threads)."""
    from oracle import oracle as O

    tcam = view.tcam()
    H, W = view.height, view.width
    t0 = time.perf_counter()
    L = O.rasterize_lists(mesh.indices, mesh.vertices, tcam)
    t_lists = time.perf_counter() - t0
    G = L["cam"].grid_width * L["cam"].grid_height
    jitter = np.full((H, W, 2), 0.5, np.float32)
    target = np.random.default_rng(1000).uniform(size=(H, W, 3)).astype(np.float32)
    frac = target_frac or 1.0 / 64
    while True:
        stride = max(1, int(round(1.0 / frac)))
        mask = np.zeros(G, np.uint8)
        mask[::stride] = 1
        t0 = time.perf_counter()
        O.blend_fwd_bwd_f32_sample(L, mesh.indices, mesh.vertices, mesh.cell_values, jitter, mask, target)
        t_blend = time.perf_counter() - t0
        if target_frac is not None or t_blend > 0.2 * budget_s or stride == 1:
            break
        frac = min(1.0, frac * max(2.0, 0.5 * budget_s / max(t_blend, 1e-3)))
    sample_tiles = int(mask.sum())
    sample_frac = sample_tiles / G
    px = sample_frac * H * W
    t = t_lists * sample_frac + t_blend
    return px / t / 1e6, t, (f"{sample_tiles}/{G} tiles ({px:.0f} px) fwd+bwd + stages a-c scaled by the tile "
                             f"fraction (stages a-c {t_lists:.2f}s on all {len(mesh.indices)} tets)"), \
        O.max_threads(), frac


def cpu_quadrature(mesh, view, budget_s, n_samples=10000):
    """The reference's FP64 quadrature path (jaxutil/tetra_quad.py:58-99,
    143-224, driven as utils/compare_quad.py:134-139 does: n_samples midpoints
    on [min camera-space depth clipped to min_t, 1.2 x max depth]), restated
    in C++ over each ray's exact segments (oracle), forward only, on an even
    sample of tiles sized to the time budget.  Returns Mpix/s and a
    description."""
    from oracle import oracle as O

    tcam = view.tcam()
    H, W = view.height, view.width
    L = O.rasterize_lists(mesh.indices, mesh.vertices, tcam)
    M = np.asarray(view.world_view, np.float64).reshape(4, 4)
    z = (mesh.vertices.astype(np.float64) @ M[2, :3]) + M[2, 3]
    t0 = max(float(z.min()), float(tcam["min_t"]))
    t1 = float(z.max()) * 1.2
    vd = mesh.vertices.astype(np.float64)
    cd = mesh.cell_values.astype(np.float64)
    jitter = np.full((H, W, 2), 0.5, np.float32)
    G = len(L["ranges"])
    frac = 1.0 / 4096
    while True:
        stride = max(1, int(round(1.0 / frac)))
        keep = np.zeros(G, bool)
        keep[::stride] = True
        lists = dict(L)
        rg = L["ranges"].copy()
        rg[~keep] = 0  # tiles outside the sample walk no list
        lists["ranges"] = rg
        t_a = time.perf_counter()
        O.quadrature_f64(lists, mesh.indices, vd, cd, jitter, t0, t1, n_samples)
        t = time.perf_counter() - t_a
        if t > 0.15 * budget_s or stride == 1:
            break
        frac = min(1.0, frac * max(2.0, 0.5 * budget_s / max(t, 1e-3)))
    tiles = int(keep.sum())
    gw = L["cam"].grid_width
    ys, xs = np.divmod(np.flatnonzero(keep), gw)
    tw, th = L["cam"].tile_width, L["cam"].tile_height
    px = int(sum(min(tw, W - x * tw) * min(th, H - y * th) for x, y in zip(xs, ys)))
    return px / t / 1e6, (f"{tiles}/{G} tiles ({px} px), {n_samples} samples per ray on [{t0:.3f}, {t1:.3f}], "
                          f"forward only")


def cpu_baseline(mesh, view, budget_s):
    from oracle import oracle as O

    q_mpix, q_desc = cpu_quadrature(mesh, view, budget_s)
    mpix, t, desc, threads, _ = cpu_sample(mesh, view, budget_s)
    return {"value": q_mpix, "unit": UNIT, "cores": O.max_threads(), "kind": "port", "sample": q_desc,
            "what": "FP64 midpoint quadrature of the reference's oracle (jaxutil/tetra_quad.py), restated in C++ "
                    "over exact ray/tet segments (oracle/), OpenMP on all host cores; forward only",
            "fp32_port_fwd_bwd": {"value": mpix, "unit": UNIT, "cores": threads, "sample": desc,
                                  "what": "FP32 C++ restatement of the reference's rasterizer (oracle/), "
                                          "stages a-c + blend forward + L1 backward, OpenMP"}}


def run_reference(args):
    world, rank, local = dist_env()
    if rank != 0:
        return
    mesh, view = workload(args, 0, 1)
    frac = None
    for _ in range(args.warmup):
        _, _, _, _, frac = cpu_sample(mesh, view, args.cpu_seconds, frac)
    vals, secs = [], []
    desc, threads = "", 0
    for _ in range(args.steps):
        mpix, t, desc, threads, frac = cpu_sample(mesh, view, args.cpu_seconds, frac)
        vals.append(mpix)
        secs.append(t)
    value = float(np.mean(vals))
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * float(np.mean(secs)),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": f"training step: {args.points} mixture points, {len(mesh.indices)} tets, "
                               f"{view.width}x{view.height}, tile {args.tile}, L1 loss", "tets": len(mesh.indices),
                   "image": [view.height, view.width], "tile": args.tile},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "port", "sample": desc},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "note": "the reference's path is Slang compiled by slangtorch, which is not installable offline; this arm "
                "times the C++ restatement of that path (oracle/) on the host cores",
    }
    print(json.dumps(line), flush=True)


# ------------------------------------------------------- multi-view batch --
def run_multiview(args, prebuilt=None):
    """16 ring cameras (8 x 1297x840, 4 x 1920x1080, 4 x 640x480) of a 1M-point
    mixture mesh; fwd + L1 loss + bwd of all views per step.  Batched: one
    launch per stage over all views, replayed as a CUDA graph.  Per view: the
    plain drop-in path (vertex_and_tile_shader + AlphaBlendTiledRender +
    autograd) once per camera.  frames/s = views / step time."""
    import torch

    import radiance_meshes_b200 as RMB
    from radiance_meshes_b200 import _capi
    from radiance_meshes_b200 import batch as B
    from radiance_meshes_b200 import rasterizer as R
    from radiance_meshes_b200 import scenes
    from radiance_meshes_b200.camera import tcam_to_struct

    world, rank, local = dist_env()
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    RMB.install_dropin()
    from delaunay_rasterization.internal.alphablend_tiled_slang_interp import AlphaBlendTiledRender
    from delaunay_rasterization.internal.render_grid import RenderGrid
    from delaunay_rasterization.internal.tile_shader_slang import vertex_and_tile_shader

    t0 = time.perf_counter()
    if prebuilt is not None:
        mesh, views = prebuilt, scenes.multiview_cameras(16)
    else:
        mesh, views = scenes.workload_multiview(n_points=args.mv_points, seed=3, tile_size=16)
    views = views[:args.mv_views]
    gen_s = time.perf_counter() - t0
    T = len(mesh.indices)
    idx = torch.from_numpy(mesh.indices).to(dev)
    verts = torch.from_numpy(mesh.vertices).to(dev)
    cv = torch.from_numpy(mesh.cell_values).to(dev)
    flush = torch.empty(256 * 1024 * 1024, dtype=torch.uint8, device=dev)

    tile = args.mv_tile
    tuned = None
    if tile == 0:
        from radiance_meshes_b200 import autotune

        tuned = autotune.tune_batch(idx, verts, cv, [v for v in views], device=dev)
        tile, fine_shift = tuned["tile"], tuned["fine_shift"]
        fwd_flags, bwd_flags = tuned["fwd_flags"], tuned["bwd_flags"]
    else:
        fwd_flags = bwd_flags = fine_shift = 0
    cams = [tcam_to_struct(v.tcam(tile_size=tile)) for v in views]
    vb = B.ViewBatch(cams)
    gen = torch.Generator(device=dev).manual_seed(7)
    target = torch.rand(vb.n_pixels, 3, device=dev, generator=gen)
    br = B.BatchedRasterizer(idx, verts, cv, vb, fwd_flags=fwd_flags, bwd_flags=bwd_flags, fine_shift=fine_shift)
    step = B.L1Step(br, target)
    step.run()
    br.check()
    P = int(br.total.item())
    # stage times of one eager step
    with R.StageTimer() as timer:
        step.run()
    stages = {k: v[0] for k, v in timer.totals().items()}
    step.capture()
    for _ in range(args.warmup):
        step.run()
    torch.cuda.synchronize()
    launches0 = _capi.launch_count()
    ev = []
    with ClockSampler(local, interval_ms=50) as clocks:
        for _ in range(args.steps):
            flush.zero_()
            a = torch.cuda.Event(enable_timing=True)
            b = torch.cuda.Event(enable_timing=True)
            a.record()
            step.run()
            b.record()
            ev.append((a, b))
        torch.cuda.synchronize()
    br.check()
    batched_ms = sum(a.elapsed_time(b) for a, b in ev) / args.steps
    graph_launches = _capi.launch_count() - launches0  # replays are not counted by the host counter

    # ---- plain per-view steps through the drop-in autograd path: once with
    # the drop-in's 16x16 tiles and default launch flags, once with the
    # batched step's tile size and flags
    vb16 = B.ViewBatch([tcam_to_struct(v.tcam(tile_size=16)) for v in views])
    tgts = [t.contiguous() for t in vb16.split(target)]
    jits = [torch.full((v.height, v.width, 2), 0.5, device=dev) for v in views]
    vv = verts.clone().requires_grad_(True)
    cc = cv.clone().requires_grad_(True)

    def time_per_view(ts, fflags, bflags):
        tcams = [v.tcam(device=dev, tile_size=ts) for v in views]
        grids = [RenderGrid(v.height, v.width, tile_width=ts, tile_height=ts) for v in views]
        saved = R.blend_tuning()
        R.set_blend_tuning(fflags, bflags)

        def per_view_step():
            vv.grad = None
            cc.grad = None
            for k in range(len(views)):
                sorted_ids, ranges, vs, ccen, mask, rect = vertex_and_tile_shader(idx, vv, tcams[k], grids[k])
                img, _, _ = AlphaBlendTiledRender.apply(sorted_ids, ranges, idx, vv, cc, grids[k], tcams[k],
                                                        jits[k])
                loss = (img[..., :3] - tgts[k]).abs().mean()
                loss.backward()

        try:
            for _ in range(args.warmup):
                per_view_step()
            torch.cuda.synchronize()
            ev = []
            for _ in range(args.steps):
                flush.zero_()
                a = torch.cuda.Event(enable_timing=True)
                b = torch.cuda.Event(enable_timing=True)
                a.record()
                per_view_step()
                b.record()
                ev.append((a, b))
            torch.cuda.synchronize()
        finally:
            R.set_blend_tuning(*saved)
        return sum(a.elapsed_time(b) for a, b in ev) / args.steps

    per_view_ms = time_per_view(16, 0, 0)
    per_view_same_ms = time_per_view(tile, fwd_flags, bwd_flags) if tile != 16 or fwd_flags or bwd_flags \
        else per_view_ms
    nv = len(views)
    line = {
        "metric": "batched multi-view fwd+bwd frames/s", "value": nv / (batched_ms * 1e-3), "unit": "frames/s",
        "n_gpus": 1, "steps": args.steps, "warmup": args.warmup, "ms_per_step": batched_ms,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "per_view_fps": nv / (per_view_ms * 1e-3), "per_view_ms_per_step": per_view_ms,
        "batched_over_per_view": per_view_ms / batched_ms,
        "per_view_same_tuning_fps": nv / (per_view_same_ms * 1e-3),
        "batched_over_per_view_same_tuning": per_view_same_ms / batched_ms,
        "config": {"workload": f"multi-view: {args.mv_points} mixture points (seed 3), {T} tets, {nv} ring views "
                               f"{[(v.width, v.height) for v in views]}, fwd + L1 + bwd",
                   "tets": T, "views": nv, "pixels": vb.n_pixels, "pairs": P, "tile": tile,
                   "blend_tile": tile >> fine_shift,
                   "blend_pairs": int(br.fine_total.item()) if fine_shift else P,
                   "autotune": tuned, "l2": "flushed between steps (256 MiB write)",
                   "batched": "one launch per stage over all views, CUDA graph replay",
                   "per_view": "drop-in autograd path per camera, host sync per view: 16x16 tiles with "
                               "default flags (per_view_fps) and the batched step's tile and flags "
                               "(per_view_same_tuning_fps)"},
        "stages_ms_batched_eager": stages, "mesh_generation_s": gen_s,
        "clocks": clocks.summary(),
    }
    return line


# ----------------------------------------------------------------- serving --
def _serving_mesh(job):
    n, seed = job
    from radiance_meshes_b200 import scenes

    m = scenes.mixture_mesh(n, seed)
    return n, m.vertices, m.indices, m.cell_values


def _mesh_worker_init():
    """Mesh builders yield the host cores to the measurement running beside
    them (the e2e step's launches, the CPU baseline's threads)."""
    try:
        os.nice(19)
    except OSError:
        pass


def _mesh_job(job):
    """(points, seed) -> a mixture mesh (runs in a spawned host process)."""
    from radiance_meshes_b200 import scenes

    return scenes.mixture_mesh(*job)


def run_serving(args, prebuilt=None):
    """Three resident meshes (250k / 1M / 3M mixture points, seeds 4-6), a
    Poisson stream of forward render requests (200 req/s, seed 7), each on a
    uniformly chosen mesh with a camera uniform on the radius-4 sphere and a
    resolution uniform over 640x480 / 1280x720 / 1920x1080; continuous
    batching over streams under an HBM budget.  Reports p50/p99 latency
    (result-ready event minus arrival) over the requests after the warm-up."""
    import multiprocessing as mp

    counts = [int(x) for x in args.sv_points.split(",")]
    seeds = [4, 5, 6][:len(counts)]
    t0 = time.perf_counter()
    if prebuilt is not None:
        built = [(n, m.vertices, m.indices, m.cell_values) for n, m in zip(counts, prebuilt)]
    else:
        with mp.get_context("spawn").Pool(len(counts)) as pool:  # before any CUDA call
            built = pool.map(_serving_mesh, list(zip(counts, seeds)))
    gen_s = time.perf_counter() - t0

    import torch

    from radiance_meshes_b200 import _capi
    from radiance_meshes_b200 import scenes
    from radiance_meshes_b200 import serve as S
    from radiance_meshes_b200.camera import tcam_to_struct

    world, rank, local = dist_env()
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    resident = [S.ResidentMesh(f"mixture{n}", idx, pts, cv, device=dev) for n, pts, idx, cv in built]
    tets = {m.name: m.T for m in resident}
    names = [m.name for m in resident]
    tile, flags, tuned, fine_shift = args.sv_tile, 0, None, 0
    rng = np.random.default_rng(77)
    sample_views = [scenes.sphere_view(rng, h, w) for (h, w) in scenes.SERVING_RESOLUTIONS for _ in range(2)]
    if tile == 0:
        from radiance_meshes_b200 import autotune

        mid = resident[len(resident) // 2]
        tuned = autotune.tune_batch(mid.indices, mid.vertices, mid.cell_values, sample_views[::2], device=dev,
                                    tiles=(8, 16, 32), backward=False)
        tile, flags, fine_shift = tuned["tile"], tuned["fwd_flags"], tuned["fine_shift"]
    else:
        fine_shift = 0
    server = S.Server(resident, streams=args.sv_streams, max_views=args.sv_max_views, tile=tile, fwd_flags=flags,
                      fine_shift=fine_shift, keep_outputs=False, device=dev)
    server.calibrate({m.name: [tcam_to_struct(v.tcam(tile_size=tile)) for v in sample_views] for m in resident})
    n_total = args.sv_warmup + args.sv_requests
    trace = scenes.serving_trace(n_total, args.sv_rate, names, seed=7, tile_size=tile)
    reqs = [S.RenderRequest(k, name, tcam_to_struct(v.tcam(tile_size=tile)), t)
            for k, (t, name, v) in enumerate(trace)]
    launches0 = _capi.launch_count()
    with ClockSampler(local, interval_ms=200) as clocks:  # a seconds-long trace: sparse sampling
        results = server.run_trace(reqs, realtime=True)
    launches = _capi.launch_count() - launches0
    low = None
    if args.sv_low_rate > 0:
        n_low = args.sv_warmup + args.sv_requests // 2
        trace_low = scenes.serving_trace(n_low, args.sv_low_rate, names, seed=9, tile_size=tile)
        reqs_low = [S.RenderRequest(10 ** 6 + k, name, tcam_to_struct(v.tcam(tile_size=tile)), t)
                    for k, (t, name, v) in enumerate(trace_low)]
        res_low = sorted(server.run_trace(reqs_low, realtime=True), key=lambda r: r.rid)
        low = dict(S.latency_summary(res_low, skip=args.sv_warmup), rate_req_per_s=args.sv_low_rate)
    # capacity: the same server fed a backlog (all requests at once), frames/s
    backlog = [S.RenderRequest(n_total + k, name, tcam_to_struct(v.tcam(tile_size=tile)), 0.0)
               for k, (t, name, v) in enumerate(scenes.serving_trace(600, args.sv_rate, names, seed=8,
                                                                       tile_size=tile))]
    t_cap = time.perf_counter()
    cap_res = server.run_trace(backlog, realtime=False)
    torch.cuda.synchronize()
    capacity_fps = len(cap_res) / (time.perf_counter() - t_cap)
    results.sort(key=lambda r: r.rid)
    summ = S.latency_summary(results, skip=args.sv_warmup)
    per_mesh = {}
    for name in names:
        sub = [r for r in results[args.sv_warmup:] if r.mesh == name]
        if sub:
            per_mesh[name] = {k: v for k, v in S.latency_summary(sub).items() if k in ("requests", "p50_ms", "p99_ms")}
    views = np.array([r.batch_views for r in results[args.sv_warmup:]])
    line = {
        "metric": "serving p99 latency ms @200 req/s", "value": summ["p99_ms"], "unit": "ms", "n_gpus": 1,
        "steps": args.sv_requests, "warmup": args.sv_warmup, "higher_is_better": False, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "p50_ms": summ["p50_ms"], "p90_ms": summ["p90_ms"], "p99_ms": summ["p99_ms"], "mean_ms": summ["mean_ms"],
        "max_ms": summ["max_ms"], "frames_per_s": summ["frames_per_s"],
        "capacity_frames_per_s": capacity_fps, "at_lower_rate": low,
        "config": {"workload": f"serving: meshes {counts} mixture points (seeds {seeds}), tets {tets}, Poisson "
                               f"{args.sv_rate} req/s (seed 7), sphere poses r=4, resolutions 640x480/1280x720/"
                               f"1920x1080, forward only",
                   "streams": args.sv_streams, "max_views": args.sv_max_views, "tile": tile, "autotune": tuned,
                   "hbm_budget_bytes": server.hbm_budget, "latency": "result-ready CUDA event minus arrival"},
        "per_mesh": per_mesh, "batches": server.n_batches, "mean_views_per_batch": float(views.mean()),
        "retries": server.n_retries, "peak_reserved_bytes": server.peak_reserved,
        "resident_bytes": sum(m.nbytes for m in resident), "gpu_launches": int(launches),
        "mesh_generation_s": gen_s, "clocks": clocks.summary(),
    }
    return line


def run_sort(args):
    """rm_sort_pairs_range alone on --sort-pairs random keys of the key bits
    --sort-bits (seeded), timed with CUDA events per sort (no L2 flush: the
    keys and the ping-pong buffers exceed L2 from about 5M pairs)."""
    import torch

    from radiance_meshes_b200 import _capi as C

    torch.cuda.set_device(0)
    L = C.lib()
    n = args.sort_pairs
    begin, end = (int(x) for x in args.sort_bits.split(","))
    g = torch.Generator(device="cuda").manual_seed(1)
    hi = torch.randint(0, 1 << max(end - 32, 1), (n,), device="cuda", dtype=torch.int64, generator=g)
    lo = torch.randint(0, 1 << 31, (n,), device="cuda", dtype=torch.int64, generator=g)
    keys = ((hi << 32) | lo) & ((1 << end) - 1)
    vals = torch.arange(n, device="cuda", dtype=torch.int32)
    ko, vo = torch.empty_like(keys), torch.empty_like(vals)
    wsn = L.rm_sort_workspace_size(n)
    ws = torch.empty(wsn, dtype=torch.uint8, device="cuda")
    status = torch.zeros(1, dtype=torch.int32, device="cuda")

    def one():
        C.check(L.rm_sort_pairs_range(C.ptr(keys), C.ptr(vals), n, None, begin, end, C.ptr(ko), C.ptr(vo),
                                      C.ptr(ws), wsn, C.ptr(status), C.stream_handle()), "rm_sort_pairs_range")

    for _ in range(args.warmup):
        one()
    torch.cuda.synchronize()
    times = []
    for _ in range(args.steps):
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        one()
        b.record()
        b.synchronize()
        times.append(a.elapsed_time(b))
    if args.profile_steps:
        return None
    passes = (end - begin + 7) // 8
    ms = float(np.median(times))
    if begin == 0:
        assert bool((ko[1:] >= ko[:-1]).all()), "not sorted"
    assert int(status.item()) == 0
    return {"metric": "pairs sorted per second", "value": n / (ms * 1e-3) / 1e9, "unit": "G pairs/s",
            "n_gpus": 1, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "int64 keys, int32 values",
            "data": "synthetic", "config": {"workload": f"rm_sort_pairs_range, {n} random keys, bits [{begin},{end}), "
                                                        f"{passes} passes of 8 bits", "pairs": n},
            "key_value_gb_s": n * 24 * passes / (ms * 1e-3) / 1e9}


def run_default(args):
    """The training line, with the multi-view and serving results nested in
    it (single GPU): their meshes are built in spawned host processes, started
    after the training line's GPU timings, while its CPU baseline runs."""
    import multiprocessing as mp

    world, rank, local = dist_env()
    extras = world == 1 and not args.no_extras and not args.profile_steps
    pool = jobs = None
    spec = None
    if extras:
        counts = [int(x) for x in args.sv_points.split(",")]
        spec = [(args.mv_points, 3)] + list(zip(counts, [4, 5, 6][:len(counts)]))

    def start_builders():
        """Mesh builders for the nested rows, started once the training line's
        GPU timings are taken (they would compete with its host-side launches):
        one thread each (the variables reach the spawned processes before their
        numpy loads), at the lowest priority, beside the CPU baseline."""
        nonlocal pool, jobs
        saved = {k: os.environ.get(k) for k in ("OMP_NUM_THREADS", "OPENBLAS_NUM_THREADS", "MKL_NUM_THREADS")}
        os.environ.update({k: "1" for k in saved})
        try:
            pool = mp.get_context("spawn").Pool(len(spec), initializer=_mesh_worker_init)
        finally:
            for k, v in saved.items():
                if v is None:
                    os.environ.pop(k, None)
                else:
                    os.environ[k] = v
        jobs = pool.map_async(_mesh_job, spec)

    try:
        line = run_b200(args, after_gpu_timing=start_builders if extras else None)
        if line is None or not extras:
            return line
        t0 = time.perf_counter()
        meshes = jobs.get()
        line["extras_mesh_wait_s"] = time.perf_counter() - t0
        for key, fn, arg in (("multiview", run_multiview, meshes[0]), ("serving", run_serving, meshes[1:])):
            try:
                line[key] = fn(args, arg)
            except Exception as e:  # the training line stands on its own
                line[key] = {"error": f"{type(e).__name__}: {e}"}
        return line
    finally:
        if pool is not None:
            pool.terminate()


def main():
    args = parse()
    if args.impl == "b200" and args.workload == "serving":
        line = run_serving(args)
    elif args.impl == "reference":
        return run_reference(args)
    elif args.workload == "multiview":
        line = run_multiview(args)
    elif args.workload == "sort":
        line = run_sort(args)
    else:
        line = run_default(args)
    if line is not None:
        print(json.dumps(line), flush=True)


if __name__ == "__main__":
    main()
