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
    ap.add_argument("--profile-steps", type=int, default=0, help="(profiling) run N steps after warmup, print nothing")
    ap.add_argument("--workload", choices=["training", "multiview", "serving"], default="training",
                    help="training: the 1.3M-tet fwd+bwd step (default line); multiview: 16 views of a "
                         "1M-point mesh, batched CUDA-graph step vs 16 plain per-view steps; serving: "
                         "Poisson requests over three resident meshes, p50/p99 latency")
    ap.add_argument("--sv-points", default="250000,1000000,3000000")
    ap.add_argument("--sv-rate", type=float, default=200.0)
    ap.add_argument("--sv-requests", type=int, default=2000)
    ap.add_argument("--sv-warmup", type=int, default=200)
    ap.add_argument("--sv-streams", type=int, default=4)
    ap.add_argument("--sv-max-views", type=int, default=8)
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

    def __init__(self, index):
        vis = os.environ.get("CUDA_VISIBLE_DEVICES")
        if vis:
            ids = [x.strip() for x in vis.split(",") if x.strip()]
            index = ids[index] if index < len(ids) else index
        self.index = index
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.QUERY}", "--format=csv,noheader,nounits",
                                          "-i", str(self.index), "-lms", "200"], stdout=subprocess.PIPE,
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
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
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
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm)}


def issue_roofline(kernel, launch_ms, tests, clocks, **extra):
    """The blend kernels are bound by instruction issue, not HBM: the
    kernel's warp instructions per launch (ray/tet tests of this pass x the
    instructions per test of the profiled capture, profiles/issue_model.json)
    over its measured launch time, against the SM's issue peak (148 SMs x 4
    schedulers x the sampled SM clock)."""
    out = {"ray_tet_tests_per_pass": tests, **extra}
    path = os.path.join(ROOT, "profiles", "issue_model.json")
    if not os.path.exists(path):
        return out
    with open(path) as f:
        model = json.load(f).get(kernel)
    if not model or not launch_ms:
        return out
    import torch

    sms = torch.cuda.get_device_properties(torch.cuda.current_device()).multi_processor_count
    mhz = clocks.get("sm_mhz") or clocks.get("sm_max_mhz") or 1965.0
    warp_inst = tests * model["thread_instructions_per_test"] / model["active_lanes_per_instruction"]
    achieved = warp_inst / (launch_ms * 1e-3) / 1e9
    peak = sms * 4 * mhz * 1e6 / 1e9
    out.update({"bound": "issue", "unit": "G warp instructions/s", "achieved": achieved, "peak": peak,
                "frac": achieved / peak, "instructions_per_test_source": "profiles/issue_model.json"})
    return out


# ------------------------------------------------------------- b200 arm --
def run_b200(args):
    import torch
    import torch.distributed as dist

    import radiance_meshes_b200 as RMB
    from radiance_meshes_b200 import _capi
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
    rng = np.random.default_rng(1000 + rank)
    target_h = torch.from_numpy(rng.uniform(size=(H, W, 3)).astype(np.float32))
    verts_h = torch.from_numpy(mesh.vertices).pin_memory()
    idx_h = torch.from_numpy(mesh.indices).pin_memory()
    cv_h = torch.from_numpy(mesh.cell_values).pin_memory()
    target_h = target_h.pin_memory()
    verts = verts_h.to(dev).requires_grad_(True)
    cv = cv_h.to(dev).requires_grad_(True)
    idx = idx_h.to(dev)
    target = target_h.to(dev)
    jitter = torch.full((H, W, 2), 0.5, device=dev)
    flush = torch.empty(256 * 1024 * 1024, dtype=torch.uint8, device=dev)  # > 126 MB L2
    stats = {}

    def step(v, c, i, tgt, features_ready=None, target_ready=None):
        v.grad = None
        c.grad = None
        sorted_ids, ranges, vs, cc, mask, rect = vertex_and_tile_shader(i, v, tcam, grid)
        if features_ready is not None:  # cell values still in flight during the tiling
            torch.cuda.current_stream().wait_event(features_ready)
        img, distimg, _ = AlphaBlendTiledRender.apply(sorted_ids, ranges, i, v, c, grid, tcam, jitter, "cuda",
                                                      mask.to(torch.int32))
        if target_ready is not None:  # the target image arrives during the blend
            torch.cuda.current_stream().wait_event(target_ready)
        loss = (img[..., :3] - tgt).abs().mean()
        loss.backward()
        if world > 1:
            MG.allreduce_grads([v.grad, c.grad])
        stats["P"] = int(sorted_ids.shape[0])
        stats["fine"] = R.fine_lists_of(sorted_ids, camst, jitter)  # read after the timed steps
        return loss, img

    for _ in range(args.warmup):
        step(verts, cv, idx, target)
    torch.cuda.synchronize()
    if args.profile_steps:
        for _ in range(args.profile_steps):
            step(verts, cv, idx, target)
        torch.cuda.synchronize()
        if world > 1:
            dist.destroy_process_group()
        return

    # ---- device-resident timing: K steps, per-step events, L2 flushed between steps
    launches0 = _capi.launch_count()
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    times = []
    # inside the timed region only the blend kernels (the roofline's
    # candidates) get event pairs; the per-stage breakdown comes from a
    # separate pass below
    timer = R.StageTimer(only=("rm_blend_fwd", "rm_blend_bwd"))
    with ClockSampler(local) as clocks, timer:
        for _ in range(args.steps):
            flush.zero_()
            a = torch.cuda.Event(enable_timing=True)
            b = torch.cuda.Event(enable_timing=True)
            a.record()
            loss, img = step(verts, cv, idx, target)
            b.record()
            times.append((a, b))
        torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    launches = _capi.launch_count() - launches0
    total_ms = sum(a.elapsed_time(b) for a, b in times)
    stages = timer.totals()
    # per-stage breakdown: every C-ABI call timed, over a separate untimed pass
    n_break = min(args.steps, 20)
    breakdown = R.StageTimer()
    with breakdown:
        for _ in range(n_break):
            flush.zero_()
            step(verts, cv, idx, target)
        torch.cuda.synchronize()
    stage_pass = breakdown.totals()
    # Σ n_contrib of the last frame: the number of ray/tet tests per pass
    # (the issue-rate unit), from a separate untimed forward
    with torch.no_grad():
        sorted_ids, ranges, vs, cc, mask, rect = vertex_and_tile_shader(idx, verts, tcam, grid)
        fine = R.fine_lists_of(sorted_ids, camst, jitter)
        if fine is not None:  # the lists the timed blend walked
            sorted_ids, ranges, bcam = fine.sorted_ids, fine.ranges, fine.cam
        else:
            bcam = camst
        _, _, ncs, _ = R.blend_fwd(sorted_ids, ranges, idx, verts.detach(), cv.detach(), jitter, bcam,
                                   tiles_touched=mask.to(torch.int32))
        tests = int(ncs.sum().item())
    if world > 1:
        t = torch.tensor([total_ms], device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        total_ms = float(t.item())

    # ---- end to end: host buffers in, loss out, copies inside the timed region
    e2e = None
    if not args.no_e2e:
        verts_d = torch.empty_like(verts)
        cv_d = torch.empty_like(cv)
        idx_d = torch.empty_like(idx)
        tgt_d = torch.empty_like(target)
        loss_h = torch.empty(1, dtype=torch.float32).pin_memory()
        # Host->device copies on a copy stream, in the order the step needs
        # them: the tiling starts once the vertices and indices are in, the
        # blend once the cell values are, the loss once the target image is.
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
                verts_d.detach().copy_(verts_h, non_blocking=True)
                geometry_ready.record()
                cv_d.detach().copy_(cv_h, non_blocking=True)
                features_ready.record()
                tgt_d.copy_(target_h, non_blocking=True)
                target_ready.record()
            torch.cuda.current_stream().wait_event(geometry_ready)
            vd = verts_d.detach().requires_grad_(True)
            cd = cv_d.detach().requires_grad_(True)
            loss, _ = step(vd, cd, idx_d, tgt_d, features_ready, target_ready)
            loss_h.copy_(loss.detach().reshape(1), non_blocking=True)
            b.record()
            b.synchronize()
            e2e_times.append((a, b))
        e2e_ms = sum(a.elapsed_time(b) for a, b in e2e_times)
        if world > 1:
            t = torch.tensor([e2e_ms], device=dev)
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            e2e_ms = float(t.item())
        h2d = (verts_h.numel() * 4 + cv_h.numel() * 4 + idx_h.numel() * 4 + target_h.numel() * 4)
        e2e = {"value": world * H * W * args.steps / (e2e_ms * 1e-3) / 1e6, "unit": UNIT,
               "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": 4,
               "ms_per_step": e2e_ms / args.steps}

    if world > 1:
        dist.destroy_process_group()
    if rank != 0:
        return

    Npx = H * W
    P = stats["P"]
    G = grid.grid_width * grid.grid_height
    # the blend walks the 8x8-pixel lists when the drop-in built them
    fine = stats["fine"]
    Pb = fine.n_pairs if fine is not None else P
    Gb = fine.cam.grid_width * fine.cam.grid_height if fine is not None else G
    value = world * Npx * args.steps / (total_ms * 1e-3) / 1e6
    peaks = {}
    pk = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(pk):
        with open(pk) as f:
            peaks = json.load(f)
    hbm_peak = float(peaks.get("hbm_gbs", 6650.0))
    peak_src = "measured" if "hbm_gbs" in peaks else "fallback"
    # algorithmic bytes per launch of the dominant kernel (blend backward):
    # 8G + 96P read (ranges, ids + 92 B tet record), 84 Npx read (saved state
    # 40, grads 36, jitter 8), 2*(28T + 12V) gradient read-modify-write
    per_stage = {k: {"ms_per_step": v[0] / n_break, "calls": v[1]} for k, v in stage_pass.items()}
    dom = max(stages.items(), key=lambda kv: kv[1][0])[0]
    bytes_alg = {
        "rm_blend_bwd": 8 * Gb + 96 * Pb + 84 * Npx + 2 * (28 * T + 12 * V),
        "rm_blend_fwd": 8 * Gb + 96 * Pb + 8 * Npx + 44 * Npx + T * (16 + 48 + 28 + 128),
        "rm_sort_pairs": 24 * P,
        "rm_project_fwd": 12 * V + 16 * T + 36 * T,
    }
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
                               f"tile {args.tile}, L1 loss", "tets": T, "points": args.points,
                   "image": [H, W], "tile": args.tile, "pairs": P,
                   "blend_lists": ("8x8-pixel lists built beside the 16x16 ones, %d pairs" % Pb) if fine is not None
                   else "caller's tiles", "parallelism": f"dp{world} (views)" if world > 1
                   else "single view", "l2": "flushed between steps (256 MiB write)",
                   "seed": 2},
        "e2e": e2e, "roofline": roof, "stages_ms": per_stage, "stages_pass_steps": n_break, "gpu_launches": int(launches),
        "clocks": clocks.summary(),
    }
    if world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline(mesh, view, args.cpu_seconds)
    print(json.dumps(line), flush=True)


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


def cpu_baseline(mesh, view, budget_s):
    mpix, t, desc, threads, _ = cpu_sample(mesh, view, budget_s)
    return {"value": mpix, "unit": UNIT, "cores": threads, "kind": "port", "sample": desc,
            "what": "FP32 C++ restatement of the reference (oracle/), OpenMP"}


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
def run_multiview(args):
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
    with ClockSampler(local) as clocks:
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
                                                        jits[k], "cuda", mask.to(torch.int32))
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
    print(json.dumps(line), flush=True)


# ----------------------------------------------------------------- serving --
def _serving_mesh(job):
    n, seed = job
    from radiance_meshes_b200 import scenes

    pts = scenes.mixture_points(n, seed)
    idx = scenes.delaunay(pts)
    cv = scenes.make_features(len(idx), seed=seed + 1000, low_density_frac=0.3)
    return n, pts, idx, cv


def run_serving(args):
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
    with ClockSampler(local) as clocks:
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
    print(json.dumps(line), flush=True)


def main():
    args = parse()
    if args.impl == "b200" and args.workload == "serving":
        return run_serving(args)
    if args.impl == "reference":
        run_reference(args)
    elif args.workload == "multiview":
        run_multiview(args)
    else:
        run_b200(args)


if __name__ == "__main__":
    main()
