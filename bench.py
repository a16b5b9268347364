#!/usr/bin/env python
"""Throughput benchmark of the B200-native 2D APIC MPM step (particle-steps/s).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Workload (default): the "plain MPM at scale" scene -- 4096x2048 grid, h=1 m,
2000 uniform Voronoi seeds with 70% of the floes kept, 4 points per cell with
+-0.25h jitter, lognormal(0, 0.3) thickness per floe, Rankine-vortex wind
(20 m/s at 800 cells), uniform 0.1 m/s current, dt=1e-4 s (seeded, synthetic).
One "step" is one MPM sub-step (grid update + fused G2P/P2G) of the whole scene.

Our arm: the chosen form (fixed-point P2G, FP32 state) is timed for K steps
with CUDA events on the library's stream (one event pair around every kernel
and one around the whole region), the plain FP32-atomic form beside it, an
end-to-end run through the C ABI with pinned host buffers, and the FP64 CPU
oracle on the host cores.  Under torchrun every rank runs its own scene
(different seed: weak scaling, no collective in the step); rank 0 prints one
JSON line with the whole-job throughput (max time over ranks).

Beside them, on rank 0 at N=1: the reference's own CUDA step
(simulation/kernels.cuh compiled for sm_100a in oracle/_ref, single
partition, FP64, its own launch shapes) on the same scene, timed with CUDA
events around its sub-step loop ("reference_gpu").

--impl reference: the reference's own kernels (simulation/kernels.cuh,
compiled for the host in oracle/_ref) advance the same scene on the host
cores, P2G's blocks in parallel with atomic adds; rank 0 only.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "particle-steps/s on 1 B200, chosen vs plain at ≤1e-4 err vs FP64; % HBM peak"
UNIT = "particle-steps/s"
WORKLOAD = ("floe field: plain MPM at scale, 4096x2048 grid, h=1 m, 2000 Voronoi floes (70% kept), "
            "4 ppc +-0.25h jitter, lognormal(0,0.3) thickness, Rankine wind 20 m/s @ 800 cells, dt=1e-4 s")
FALLBACK_HBM_GBS = 6650.0
# algorithmic bytes per step: 124 per point + 49 per grid node (FP32/u32 words,
# each word the step consumes read once and each word it modifies written once)
B_POINT, B_NODE = 124, 49
# split of the node bytes: the fused G2P+P2G kernel reads 8 B of velocity and
# flushes 12 B of accumulators per node; the grid update moves the other 29 B
B_NODE_FUSED = 20
# DRAM traffic of one fused-kernel launch per point, grid share included:
# dram__bytes_read.sum + dram__bytes_write.sum of an ncu capture of one
# k_g2p_p2g launch on the floe field at 2048x1024 (the summary in
# profiles/k_g2p_p2g_floe_field_2048x1024.md), scaled by point count (the
# node/point ratio is the same at 4096x2048)
TRAFFIC_B_PER_POINT = 79.57
TRAFFIC_CAPTURE = {"capture": "profiles/k_g2p_p2g_floe_field_2048x1024.md", "points": 5884928,
                   "dram_bytes": 468264960, "scaled_by": "points"}
# the ~8.4M-point variant of the scene reported beside the main line
POINTS_8M = 8_400_000


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", choices=["floe_field", "ensemble"], default="floe_field",
                    help="ensemble: 96 independent scenes of 10k-2M points in one batch (one launch per kernel per sub-step)")
    ap.add_argument("--ensemble-scenes", type=int, default=96)
    ap.add_argument("--max-points", type=int, default=None,
                    help="keep whole floes until this many points (the ~8.4M-point variant)")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-plain", action="store_true")
    ap.add_argument("--cpu-steps", type=int, default=4)
    ap.add_argument("--no-ref-gpu", action="store_true")
    ap.add_argument("--no-8m", action="store_true",
                    help="skip the ~8.4M-point variant timed beside the main line (chosen, fp32, reference CUDA step)")
    ap.add_argument("--ref-gpu-steps", type=int, default=50)
    ap.add_argument("--grid", type=int, nargs=2, default=None, metavar=("GX", "GY"),
                    help="same scene rules on a smaller GX x GY grid (seeds scaled by area), "
                         "for profiling captures")
    return ap.parse_args()


def load_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return FALLBACK_HBM_GBS, "fallback"


class ClockSampler:
    """nvidia-smi clock/throttle sampling during the timed region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.rows = []
        self.proc = None

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                                          "-i", str(self.index), "-lms", "100"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
            return
        self.t = threading.Thread(target=self._read, daemon=True)
        self.t.start()

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append((time.time(), [c.strip() for c in line.split(",")]))

    def mark(self):
        return time.time()

    def stop(self):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self, t0, t1):
        rows = [r for t, r in self.rows if t0 - 0.15 <= t <= t1 + 0.15] or [r for _, r in self.rows[-3:]]
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"], "samples": 0}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in rows for k in range(4) if len(r) > 5 + k and r[5 + k] == "Active"})
        pw = [float(r[3]) for r in rows if r[3].replace(".", "").isdigit()]
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows), "power_w_max": max(pw) if pw else None}


def make_scene(seed, max_points=None, grid=None):
    from icempm_2d_sp_b200 import scenes
    if grid is not None:
        gx, gy = grid
        return scenes.floe_field(seed=seed, gx=gx, gy=gy, n_seeds=max(1, round(2000 * gx * gy / (4096 * 2048))))
    return scenes.floe_field(seed=seed, max_points=max_points)


def run_reference(args, rank):
    """The reference's own step on the host cores: simulation/kernels.cuh
    compiled for the host (oracle/_ref), on the same scene as our arm, one
    sub-step of the whole scene per step, P2G's blocks over all host threads
    with atomic adds as on the GPU."""
    if rank != 0:
        return
    sc = make_scene(1235, max_points=args.max_points, grid=args.grid)
    grid = np.zeros((9, sc.grid_nodes))
    grid[5], grid[6] = sc.current[:sc.grid_nodes], sc.current[sc.grid_nodes:]
    sample = f"the benchmark scene itself (N={sc.n} points, {sc.grid_nodes} nodes), one sub-step per step"
    try:
        from oracle.refbuild import build_ref
        L = build_ref.load()
        cores = int(L.ref_num_threads())
        kind = "reference"
        run = lambda k, first: build_ref.run_steps(sc.prms, sc.soa, sc.n, grid, sc.status, k, first,
                                                   parallel_p2g=True)
        note = ("reference simulation/kernels.cuh compiled for the host (oracle/_ref); P2G, grid update and "
                "G2P blocks over OpenMP threads, P2G's atomicAdd as relaxed atomic adds; compat forcing "
                "(the reference has no wind term)")
    except (FileNotFoundError, OSError):
        import oracle
        cores = oracle.num_threads()
        kind = "port"
        run = lambda k, first: oracle.run_steps(sc.prms, sc.soa, sc.n, grid, sc.status, k, first)
        note = "FP64 oracle port (OpenMP); the reference build was not available"
    run(args.warmup, 0)
    t0 = time.perf_counter()
    run(args.steps, args.warmup)
    dt = time.perf_counter() - t0
    v = sc.n * args.steps / dt
    workload = WORKLOAD if args.grid is None else WORKLOAD.replace("4096x2048", "%dx%d" % tuple(args.grid))
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * dt / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded Voronoi floe-field generator)",
            "config": {"workload": workload, "points": int(sc.n), "grid_nodes": sc.grid_nodes, "same_config": True},
            "cpu_baseline": {"value": v, "unit": UNIT, "cores": cores, "kind": kind, "sample": sample, "note": note},
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def reference_gpu_baseline(args, sc):
    """The reference's CUDA step on the benchmark scene: memset of grid rows
    0-2, partition_kernel_p2g, partition_kernel_update_nodes and
    partition_kernel_g2p per sub-step (gpu_partition.cpp:300-365), timed with
    CUDA events around the loop after warm-up.  The reference has no wind
    term: it runs the current-drag forcing of its update kernel."""
    try:
        from oracle.refbuild import build_ref_gpu
        build_ref_gpu.load()
    except (FileNotFoundError, OSError) as e:
        return {"unavailable": "reference GPU library not built: %s" % e}
    G = sc.grid_nodes
    grid = np.zeros((9, G))
    grid[5], grid[6] = sc.current[:G], sc.current[G:2 * G]
    k = max(1, args.ref_gpu_steps)
    with build_ref_gpu.RefGpuScene(sc.prms, sc.status, grid, sc.n) as s:
        s.upload(sc.soa, sc.n)
        s.run(max(3, args.warmup), 0)
        ms = s.run(k, max(3, args.warmup))
        err, _ = s.download(np.zeros((19, sc.n)))
    return {"value": sc.n * k / (ms * 1e-3), "unit": UNIT, "ms_per_step": ms / k, "steps": k, "dtype": "f64",
            "device_errors": err,
            "note": "reference simulation/kernels.cuh built for sm_100a (oracle/_ref/libicempm_ref_gpu.so), "
                    "single partition, tpb P2G/update/G2P = %d/%d/%d, current-drag forcing only"
                    % (sc.prms.tpb_P2G, sc.prms.tpb_Upd, sc.prms.tpb_G2P)}


def run_ensemble(args, rank, world, local, dist):
    """The ensemble workload: independent scenes (point counts log-uniform in
    10k-2M, Voronoi floes, grids 128x128 to 2048x1024, uniform wind 5-25 m/s
    and current 0-0.3 m/s) advanced by one batched launch of each kernel per
    sub-step in CUDA graphs of 50, kernel shape and sort cadence from the
    project autotuner.  Under torchrun the scenes are split across ranks by
    size (no collective in the step); value = all ranks' particle-steps / the
    slowest rank's device time."""
    from icempm_2d_sp_b200 import capi, scenes
    from icempm_2d_sp_b200.params import Options, VARIANT_FIXED
    specs = scenes.ensemble_specs(args.ensemble_scenes)
    mine = scenes.split_by_size([s["target_points"] for s in specs], world)[rank]
    scs = [scenes.ensemble_scene(**specs[i]) for i in mine]
    ctxs = []
    for sc in scs:
        o = Options.default(variant="fixed", forcing=sc.options.forcing, device=local)
        for f in ("wind_kind", "wind_u", "wind_v"):
            setattr(o, f, getattr(sc.options, f))
        c = capi.Context(sc.prms, sc.status, sc.current, capacity=sc.n, options=o)
        c.upload(sc.soa, sc.n)
        ctxs.append(c)
    n = sum(sc.n for sc in scs)
    G = sum(sc.grid_nodes for sc in scs)
    with capi.Batch(ctxs) as b:
        tuning = b.autotune(trial_steps=50, first_step=0)     # also the warm-up
        b.step(max(3, args.warmup), 250)
        if dist:
            dist.barrier()
        l0 = b.launch_count()
        sampler = ClockSampler(local)
        sampler.start()
        time.sleep(0.3)
        t0 = time.time()
        b.step(args.steps, 300)
        t1 = time.time()
        total = b.timings()[0]
        time.sleep(0.2)
        sampler.stop()
        launches = b.launch_count() - l0
        errs = [c.status()[0] for c in ctxs]
    t_ms, n_tot = combine_ranks(dist, total, n)
    value = n_tot * args.steps / (t_ms * 1e-3)
    peak, peak_src = load_peaks()
    step_bytes = B_POINT * n + B_NODE * G
    achieved = step_bytes / (total * 1e-3 / args.steps) / 1e9
    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": t_ms / args.steps, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f32",
                "data": "synthetic (seeded ensemble generator: Voronoi floe fields of 10k-2M points)",
                "config": {"workload": f"ensemble: {args.ensemble_scenes} scenes, 10k-2M points log-uniform, "
                                       "Voronoi floes, grids 128x128..2048x1024, uniform wind 5-25 m/s, "
                                       "current 0-0.3 m/s", "points": int(n), "points_all_ranks": n_tot,
                           "scenes_this_rank": len(scs), "grid_nodes": G,
                           "variant": "fixed: int64 fixed-point P2G, FP32 state",
                           "tuning": tuning.as_dict(), "parallelism": f"scenes split by size over {world} GPU(s)",
                           "l2": "inputs larger than L2", "device_errors": int(max(errs) if errs else 0)},
                "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                             "frac": achieved / peak, "traffic": None, "peak_source": peak_src,
                             "kernel": "whole sub-step (k_grid_update_batch + k_g2p_p2g_batch)",
                             "step_bytes": step_bytes},
                "cpu_baseline": None, "e2e": None, "gpu_launches": launches,
                "clocks": sampler.summary(t0, t1)}
        print(json.dumps(line), flush=True)
    for c in ctxs:
        c.close()


def cpu_baseline(args, sc):
    import oracle
    soa = sc.soa.copy()
    grid = np.zeros((9, sc.grid_nodes))
    grid[5], grid[6] = sc.current[:sc.grid_nodes], sc.current[sc.grid_nodes:]
    k = max(1, args.cpu_steps)
    t0 = time.perf_counter()
    oracle.run_steps(sc.prms, soa, sc.n, grid, sc.status, k, 0, opts=sc.options)
    dt = time.perf_counter() - t0
    return {"value": sc.n * k / dt, "unit": UNIT, "cores": oracle.num_threads(), "kind": "port",
            "sample": f"the full benchmark scene (N={sc.n}) for {k} sub-steps with the FP64 OpenMP oracle"}


def init_ranks(world, local):
    """One process per GPU under torchrun: NCCL where CUDA is present, gloo on
    CPU-only hosts (the host-side reference arm and the tests).  Returns the
    torch.distributed module, or None for a single process."""
    if world <= 1:
        return None
    import torch
    import torch.distributed as dist
    from datetime import timedelta
    if torch.cuda.is_available():
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=timedelta(seconds=600), device_id=torch.device("cuda", local))
    else:
        dist.init_process_group("gloo", timeout=timedelta(seconds=600))
    return dist


def combine_ranks(dist, t_ms, n):
    """Whole-job figures from per-rank ones: the slowest rank's time and the
    points of all ranks (each rank advances its own scene: weak scaling)."""
    if dist is None:
        return t_ms, n
    import torch
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([float(t_ms)], device=dev, dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    c = torch.tensor([float(n)], device=dev, dtype=torch.float64)
    dist.all_reduce(c, op=dist.ReduceOp.SUM)
    return float(t.item()), int(c.item())


def sum_ranks(dist, x):
    """Sum of a per-rank figure over the ranks (x itself for one process)."""
    if dist is None:
        return x
    import torch
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([float(x)], device=dev, dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())


def main():
    args = parse()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    dist = init_ranks(world, local)
    if args.impl == "ours" and args.workload == "ensemble":
        run_ensemble(args, rank, world, local, dist)
        if dist:
            dist.barrier()
            dist.destroy_process_group()
        return
    if args.impl == "reference":
        run_reference(args, rank)
        if dist:
            dist.barrier()
            dist.destroy_process_group()
        return

    import torch
    from icempm_2d_sp_b200 import capi
    from icempm_2d_sp_b200.params import Options, VARIANT_FIXED, VARIANT_FP32, VARIANT_TEXTBOOK

    def sync_all():
        torch.cuda.synchronize()
        if dist:
            dist.barrier()

    sc = make_scene(1235 + rank, max_points=args.max_points, grid=args.grid)
    n, G = sc.n, sc.grid_nodes
    peak, peak_src = load_peaks()

    def timed(variant, sc=sc):
        n = sc.n
        o = Options.default(forcing=sc.options.forcing)
        for f, _ in Options._fields_:
            setattr(o, f, getattr(sc.options, f))
        o.variant, o.device, o.use_graphs = variant, local, 1
        with capi.Context(sc.prms, sc.status, sc.current, capacity=n, options=o) as ctx:
            ctx.upload(sc.soa, n)
            ctx.step(args.warmup, 0)
            sync_all()
            l0 = ctx.launch_count()
            sampler = ClockSampler(local)
            sampler.start()
            time.sleep(0.3)
            t0 = time.time()
            upd, fused = ctx.phase_times(args.steps)
            t1 = time.time()
            total = ctx.timings()[0]
            time.sleep(0.2)
            sampler.stop()
            sync_all()
            launches = ctx.launch_count() - l0
            err, dis = ctx.status()
        return total, upd, fused, launches, sampler.summary(t0, t1), err

    total, upd, fused, launches, clocks, err = timed(VARIANT_FIXED)
    t_ms, n_tot = combine_ranks(dist, total, n)
    value = n_tot * args.steps / (t_ms * 1e-3)

    # the plain from-scratch FP32 step (three unfused kernels, one point per
    # thread, global FP32 atomics) and the fused engine with FP32 atomics
    plain = fp32_atomics = None
    if not args.no_plain:
        ttot, tupd, tpts, _, _, terr = timed(VARIANT_TEXTBOOK)
        plain = {"value": n * args.steps / (ttot * 1e-3), "ms_per_step": ttot / args.steps,
                 "points_kernels_ms": tpts / args.steps, "grid_update_ms": tupd / args.steps, "device_errors": terr,
                 "variant": "textbook: P2G with 27 global FP32 atomics per point, grid update, G2P; "
                            "one point per thread, unfused (ICEMPM_VARIANT_TEXTBOOK)",
                 "chosen_speedup": ttot / total}
        ptot, pupd, pfused, _, _, _ = timed(VARIANT_FP32)
        fp32_atomics = {"value": n * args.steps / (ptot * 1e-3), "ms_per_step": ptot / args.steps,
                        "fused_kernel_ms": pfused / args.steps,
                        "variant": "the fused engine with FP32 atomics instead of fixed point"}

    # roofline of the dominant kernel (fused G2P+P2G), live events of the timed region
    fused_bytes = B_POINT * n + B_NODE_FUSED * G
    fused_launch_s = fused * 1e-3 / args.steps
    achieved = fused_bytes / fused_launch_s / 1e9
    # DRAM bytes of one fused launch from an ncu capture (dram__bytes_read.sum +
    # dram__bytes_write.sum of profiles/k_g2p_p2g_floe_field_2048x1024.md), per
    # point, scaled to this scene's point count (same node/point ratio)
    traffic = TRAFFIC_B_PER_POINT * n
    roofline = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                "traffic": traffic, "peak_source": peak_src,
                "traffic_source": dict(TRAFFIC_CAPTURE, bytes_per_point=TRAFFIC_B_PER_POINT,
                                       note="measured on the capture, scaled to this launch; not measured live"),
                "dram_frac": traffic / fused_launch_s / 1e9 / peak,
                "kernel": "k_g2p_p2g (fused G2P + P2G)", "algorithmic_bytes_per_launch": fused_bytes,
                "avg_launch_ms": fused * 1e-3 / args.steps * 1e3,
                "step_bytes": B_POINT * n + B_NODE * G,
                "step_achieved_gbs": (B_POINT * n + B_NODE * G) / (total * 1e-3 / args.steps) / 1e9,
                "grid_update_avg_ms": upd / args.steps}

    e2e = None
    if not args.no_e2e:
        e2e = end_to_end(args, sc, local, capi, Options, VARIANT_FIXED)
        # whole job: the slowest rank's wall time, all ranks' points and copies
        t_e2e, n_e2e = combine_ranks(dist, e2e.pop("seconds") * 1e3, n)
        e2e["value"] = n_e2e * args.steps / (t_e2e * 1e-3)
        e2e["h2d_bytes_per_step"] = sum_ranks(dist, e2e["h2d_bytes_per_step"])
        e2e["d2h_bytes_per_step"] = sum_ranks(dist, e2e["d2h_bytes_per_step"])

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        cpu = cpu_baseline(args, sc)
    ref_gpu = None
    if rank == 0 and world == 1 and not args.no_ref_gpu:
        ref_gpu = reference_gpu_baseline(args, sc)
    # the ~8.4M-point variant (whole floes of the same scene kept until 8.4M
    # points): chosen form, FP32 atomics and the reference's CUDA step
    scene_8m = None
    if rank == 0 and world == 1 and not args.no_8m and args.grid is None and args.max_points is None:
        s8 = make_scene(1235, max_points=POINTS_8M)
        t8, u8, f8, _, _, e8 = timed(VARIANT_FIXED, s8)
        p8, _, pf8, _, _, _ = timed(VARIANT_FP32, s8)
        b8, _, _, _, _, _ = timed(VARIANT_TEXTBOOK, s8)
        scene_8m = {"points": int(s8.n), "grid_nodes": s8.grid_nodes,
                    "value": s8.n * args.steps / (t8 * 1e-3), "ms_per_step": t8 / args.steps,
                    "fused_kernel_ms": f8 / args.steps, "grid_update_ms": u8 / args.steps, "device_errors": e8,
                    "plain": {"value": s8.n * args.steps / (b8 * 1e-3), "ms_per_step": b8 / args.steps,
                              "variant": "textbook (see plain)", "chosen_speedup": b8 / t8},
                    "fp32_atomics": {"value": s8.n * args.steps / (p8 * 1e-3), "ms_per_step": p8 / args.steps}}
        if not args.no_ref_gpu:
            r8 = reference_gpu_baseline(args, s8)
            scene_8m["reference_gpu"] = r8
            if "ms_per_step" in r8:
                scene_8m["speedup_vs_reference_gpu"] = r8["ms_per_step"] / (t8 / args.steps)

    if rank == 0:
        workload = WORKLOAD if args.grid is None else WORKLOAD.replace("4096x2048", "%dx%d" % tuple(args.grid))
        line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": t_ms / args.steps, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f32",
                "data": "synthetic (seeded Voronoi floe-field generator)",
                "config": {"workload": workload, "points": int(n), "points_all_ranks": n_tot, "grid_nodes": G,
                           "variant": "fixed: int64 fixed-point P2G, FP32 state (chosen form)",
                           "forcing": "extended (Rankine wind, quadratic water drag)",
                           "parallelism": f"{world} independent scene(s), one per GPU",
                           "l2": "inputs larger than L2 (2.0 GB point state, 0.4 GB grid)",
                           "device_errors": err},
                "plain": plain, "fp32_atomics": fp32_atomics, "reference_gpu": ref_gpu, "scene_8m": scene_8m,
                "roofline": roofline,
                "cpu_baseline": cpu, "e2e": e2e,
                "gpu_launches": launches, "clocks": clocks}
        print(json.dumps(line), flush=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()


def end_to_end(args, sc, local, capi, Options, variant):
    """The reference-facing call sequence through the C ABI with host buffers:
    upload the HSSOA from page-locked memory, then frames of UpdateEveryNthStep
    sub-steps, each followed by the download of the HSSOA, the status word and
    the boundary forces (Model::Step, model.cpp:7-78).  The HSSOA download of
    frame k (icempm_download_points_async into one of two page-locked buffers)
    overlaps the sub-steps of frame k+1; the last one is waited for inside the
    timed region."""
    import torch
    n, G = sc.n, sc.grid_nodes
    src = sc.soa
    dst = [np.zeros_like(src), np.zeros_like(src)]
    fbuf = np.zeros(2 * G)
    for b in [src, fbuf] + dst:
        capi.host_register(b)
    o = Options.default()
    for f, _ in Options._fields_:
        setattr(o, f, getattr(sc.options, f))
    o.variant, o.device = variant, local
    frame = sc.prms.UpdateEveryNthStep
    def run(ctx, steps):
        ctx.upload(src, n)
        done, frames = 0, 0
        while done < steps:
            k = min(frame, steps - done)
            ctx.clear_force_accumulator()
            ctx.step(k, done)
            ctx.status()
            ctx.boundary_forces(k, fbuf)     # before the large copy takes the device-to-host engine
            if frames:
                ctx.download_wait()          # frame k-1 is on the host now
            ctx.download_async(dst[frames % 2])
            done += k
            frames += 1
        ctx.download_wait()
        return frames

    try:
        with capi.Context(sc.prms, sc.status, sc.current, capacity=n, options=o) as ctx:
            # untimed warm-up frame: CUDA graph instantiation, the forces buffer
            # and the copy stream are created on first use
            run(ctx, min(frame, args.steps))
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            frames = run(ctx, args.steps)
            t1 = time.perf_counter()
    finally:
        for b in [src, fbuf] + dst:
            capi.host_unregister(b)
    hssoa_bytes = 19 * 8 * n
    return {"value": n * args.steps / (t1 - t0), "unit": UNIT, "seconds": t1 - t0,
            "h2d_bytes_per_step": hssoa_bytes / args.steps,
            "d2h_bytes_per_step": frames * (hssoa_bytes + 16 * G + 8) / args.steps,
            "frames": frames, "frame_steps": frame,
            "note": "after one untimed warm-up frame: upload from page-locked host memory, per frame: step + "
                    "HSSOA download (overlapping the next frame's sub-steps) + status + boundary forces"}


if __name__ == "__main__":
    main()
