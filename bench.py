#!/usr/bin/env python
"""Benchmark: MPS time steps of the 3D dam break (1,595,308 particles, 1,024,000
fluid) on B200, through the C-ABI of voxarmps_b200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

A step is one full MPS time step (neighbour search, PND, prediction, PPE
assembly + CG to the stated relative residual, gradient, integration,
collision, commit).  ``value`` is whole-job particle-steps/s with the state
resident in HBM; ``e2e`` is the same metric through the public API with host
buffers (state uploaded from pinned host memory and downloaded every step,
through ``mps_step_io``).
Under torchrun each rank advances its own copy of the scene (independent
scenes, no collective on the data path: weak scaling), except that the
batched configuration (--config 4) splits its 64 scenes between the ranks
(strong scaling, still no exchange); timings are the max over ranks.  ``--impl reference`` times the reference's own CPU path
(oracle/_ref, OpenMP on all host cores) on a bounded sample of the workload.
"""
from __future__ import annotations

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

PEAKS_FILE = os.path.join(ROOT, "MEASURED_PEAKS.json")
FALLBACK_HBM_GBS = 6650.0
METRIC = "particle-steps/s"
# ncu capture of k_cg_spmv on the 476,608-particle dam (profiles/
# cg_spmv_dam3d_476k.md): dram read+write per launch / algorithmic bytes of
# that launch.  The traffic grows with the non-zeros, so the full launch's
# traffic is this ratio times its algorithmic bytes.
SPMV_TRAFFIC_OVER_ALGORITHMIC = 810.62 / 742.74


def dist_env():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


def max_over_ranks(v: float, ws: int, device: str = "cuda") -> float:
    """Maximum of a per-rank time over all ranks (every rank gets it)."""
    if ws == 1:
        return v
    import torch
    import torch.distributed as dist
    t = torch.tensor([v], device=device, dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def sum_over_ranks(v: float, ws: int, device: str = "cuda") -> float:
    """Sum of a per-rank count over all ranks (every rank gets it)."""
    if ws == 1:
        return v
    import torch
    import torch.distributed as dist
    t = torch.tensor([v], device=device, dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())


def whole_job_rate(units_per_rank: float, ws: int, ms_max: float) -> float:
    """Units all ranks processed per second, timed by the slowest rank."""
    return units_per_rank * ws / (ms_max * 1e-3)


def peaks():
    try:
        with open(PEAKS_FILE) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.idx = gpu_index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.idx), f"--query-gpu={self.Q}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = float(parts[2])
            except ValueError:
                continue
            for nm, val in zip(names, parts[5:9]):
                if val.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm)}


def spmv_algorithmic_bytes(nnz_a: float, rows: float) -> float:
    """Bytes one FP64 CSR SpMV must move: per stored non-zero a column index
    (4 B) and a value (8 B); per unknown row its (offset, length) pair (8),
    diag (8), the row's own p (8) and the written s (8), and bcon (4).
    Gathers of p_j are L2 hits."""
    return nnz_a * 12.0 + rows * 36.0


def spmv32_algorithmic_bytes(nnz_a: float, rows: float) -> float:
    """Inner SpMV of the mixed-precision PPE: one (column, FP32 value) pair
    (8 B) per non-zero; per row (offset, length) (8), diag (8), FP32 p and s
    (4 each), bcon (4)."""
    return nnz_a * 8.0 + rows * 28.0


def refine_algorithmic_bytes(nnz_a: float, rows: float) -> float:
    """Refinement r -= A64 d, x += d: 12 B per non-zero; per row (offset,
    length) (8), diag (8), bcon, FP32 d (4 each), r and x read and written
    (32)."""
    return nnz_a * 12.0 + rows * 56.0


WORKLOADS = {
    0: "2D dam break, 25x50 fluid (1,250) + 678 wall/dummy particles, l0=0.01, "
       "re=2.1/4.0*l0, dt=1e-4, FP64 Jacobi-PCG to 1e-8",
    1: "3D dam break, 80x160x80 fluid (1,024,000) + 571,308 wall/dummy particles, l0=0.005, "
       "re=2.1/4.0*l0, dt=5e-5, FP64 Jacobi-PCG to 1e-8 relative residual",
    2: "3D dam break, 80x160x80 fluid (1,024,000) + 571,308 wall/dummy particles, l0=0.005, "
       "re=2.1/4.0*l0, dt=5e-5, mixed-precision PPE (FP32 inner CG, FP64 dots and "
       "refinement) to 1e-8 relative residual",
    3: "2D two-phase dam, water 600x100 + Bingham block 150x150 (82,500 fluid), l0=0.002, "
       "SPS-LES Cs=0.12, HB second fluid, dt=1e-4, FP64 Jacobi-PCG to 1e-8 from the learned "
       "initial guess (4-layer message-passing net, width 64, BF16)",
    4: "64 batched 2D dam breaks (splitmix64 seed 0, columns U[0.1,0.4]x U[0.2,0.6] m, "
       "l0=0.005), one context, mixed-precision PPE from the learned initial guess, every "
       "scene's PPE to 1e-8",
}


def build_case(scale: int = 0, which: int = 1, precision=None, rank: int = 0, ws: int = 1):
    """(cfg, case, scenes) of the benchmark scene; scale > 0 selects the
    smaller 3D dam used for profiling captures (config.scaled_dam3d).  The
    batched configuration's independent scenes are split over the ws ranks
    (config.partition_scenes); every other configuration is one scene, which
    each rank advances as its own replica."""
    from voxarmps_b200 import config
    scenes = None
    if scale:
        cfg, case = config.scaled_dam3d(scale)
    elif which == 4:
        base, sc = config.baseline(4)
        if ws > 1:
            part = config.partition_scenes([len(s["x"]) for s in sc], ws)[rank]
            sc = [sc[k] for k in part]
        cfg, case, sid, boxes, pmax = config.batched(base, sc)
        scenes = (sid, boxes, pmax)
    else:
        cfg, case = config.baseline(which)
    cfg = config.solver_semantics(cfg)
    cfg["cg_tol"] = 1e-8
    cfg["cg_max"] = 1000
    # configs 2 and 4 name the mixed-precision PPE
    cfg["precision"] = (1 if which in (2, 4) else 0) if precision is None else precision
    return cfg, case, scenes


def cpu_reference_sample(scale: int = 1, radius: float = 4.0):
    """Bounded CPU sample: 3D dam at the benchmark's spacing, a 10s x 20s x 10s
    fluid column (scale 1: 12,608 particles) and one support radius for every
    stage, as the reference has: 4.0*l0 (the Laplacian radius, so the PPE and
    its IC(0) factorisation cost what they cost in the benchmark; the PND-list
    stages then do more work than the GPU's 2.1*l0) or 2.1*l0 (every stage
    cheaper than the GPU's)."""
    from voxarmps_b200 import config
    cfg, case = config.scaled_dam3d(scale)
    cfg = dict(cfg)
    cfg["re_s"] = cfg["re_l"] = radius * cfg["l0"]
    return cfg, case


def physical_cores() -> int:
    try:
        import psutil
        return int(psutil.cpu_count(logical=False) or os.cpu_count() or 1)
    except Exception:
        return os.cpu_count() or 1


def time_reference(steps: int, warmup: int, nthreads: int, scale: int = 1, radius: float = 4.0):
    """The reference's own CPU path on a bounded sample: OpenMP
    (oracle/_ref/libref_omp.so) with nthreads > 1, the sequential build
    (libref.so) with 1; if it was not built, the C restatement (single
    thread) stands in."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import pyoracle
    cfg, case = cpu_reference_sample(scale, radius)
    n = len(case["x"])
    if pyoracle.ref_available(omp=nthreads > 1):
        kind, h = "reference", pyoracle.RefHarness(cfg, case, nthreads=nthreads)
        cores = nthreads
    else:
        pyoracle.build()
        kind, h = "port", pyoracle.Oracle(dict(cfg, solver=0), case)
        cores = 1
    h.init()
    for _ in range(warmup):
        h.step()
    t0 = time.perf_counter()
    for _ in range(steps):
        h.step()
    el = time.perf_counter() - t0
    h.close()
    fl = int((np.asarray(case["ptype"]) > 0).sum())
    col = "x".join(str(10 * scale * k) for k in (1, 2, 1))
    return {"value": n * steps / el, "unit": METRIC, "cores": cores, "kind": kind,
            "sample": f"3D dam, l0=0.005, one radius {radius}*l0 for every stage, {n} particles "
                      f"({col} fluid, {fl}), {steps} steps after {warmup} warm-up, "
                      f"{'OpenMP, ' + str(cores) + ' threads' if cores > 1 else 'sequential'}",
            "ms_per_step": el / steps * 1e3, "particles": n}


def cpu_series(nthreads: int):
    """Around the headline CPU number: the same sample at the small radius,
    a scaled series (scales 1-3 at 2.1*l0, where the reference's per-step
    cost stays bounded) and the sequential build (OMP_NUM_THREADS=1 form)."""
    out = {"physical_cores": physical_cores(), "logical_cpus": os.cpu_count()}
    r = time_reference(3, 1, nthreads, 1, 2.1)
    out["radius_2.1"] = {k: r[k] for k in ("value", "ms_per_step", "particles", "sample")}
    out["scaled_2.1"] = []
    for sc in (1, 2, 3):
        r = time_reference(2 if sc < 3 else 1, 1 if sc < 3 else 0, nthreads, sc, 2.1)
        out["scaled_2.1"].append({k: r[k] for k in ("value", "ms_per_step", "particles")})
    r = time_reference(1, 0, 1, 1, 4.0)
    out["sequential_4.0"] = {k: r[k] for k in ("value", "ms_per_step", "particles", "sample",
                                                 "kind")}
    out["solver_iterations"] = solver_iterations()
    return out


def solver_iterations():
    """Iterations to the 1e-8 relative residual of the reference's ICCG
    (IC(0) preconditioner) against the Jacobi-PCG the GPU runs and plain CG,
    on the same PPE systems (the oracle's, from the previous pressure), for
    the 2D dam break after 20 steps and a 3D dam at the benchmark's spacing
    and radii after 10 steps."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import pyoracle
    from voxarmps_b200 import cases, config
    out = {}
    c3 = cases.dam_break(3, 0.005, (6, 10, 6), (20, 14, 8))
    f3 = config.reference_defaults(0.005, 3)
    f3.update(re_s=2.1 * 0.005, re_l=4.0 * 0.005, dt=5e-5, gy=-9.81)
    for name, (cfg, case), steps in (("dam2d_config0_step20", config.baseline(0), 20),
                                     ("dam3d_6x10x6_step10", (config.with_box(f3, c3), c3), 10)):
        cfg = config.solver_semantics(cfg)
        o = pyoracle.Oracle(cfg, case)
        o.init()
        prev = None
        for _ in range(steps):
            prev = o.get("p")
            o.step()
        off, nbr, bcon, diag, val, b, _p = pyoracle.ppe_system(cfg, o)
        it = pyoracle.solver_iterations(off, nbr, bcon, diag, val, b, prev)
        out[name] = {"unknowns": int((bcon == 0).sum()), "iccg": it["iccg"],
                     "jacobi_pcg": it["jacobi"], "cg": it["plain"], "tol": 1e-8}
        o.close()
    return out


def run_reference_arm(args):
    ws, rank, _ = dist_env()
    if rank != 0:
        return
    nthreads = physical_cores()
    r = time_reference(args.steps, args.warmup, nthreads)
    line = {"impl": "reference", "metric": METRIC, "value": r["value"], "unit": METRIC,
            "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": r["ms_per_step"], "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": "3D dam break, config-1 spacing and radii, bounded CPU "
                                   "sample (the full 1.6M-particle case is infeasible on CPU)",
                       "particles": 12608},
            "cpu_baseline": {"value": r["value"], "unit": METRIC, "cores": r["cores"],
                             "kind": r["kind"], "sample": r["sample"]},
            "e2e": {"value": r["value"], "unit": METRIC, "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def run_ours(args):
    import torch
    import voxarmps_b200 as vm

    ws, rank, local = dist_env()
    dev = local if torch.cuda.device_count() > 1 else 0
    torch.cuda.set_device(dev)
    if ws > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    cfg, case, scenes = build_case(args.scale, args.config, args.precision, rank, ws)
    split = scenes is not None and ws > 1  # the batch's scenes are shared out
    mixed = cfg["precision"] >= 1
    n = len(case["x"])
    fp = int((case["ptype"] > 0).sum())
    guess = args.guess or ("learned" if args.config in (3, 4) and not args.scale else "previous")
    trained = own = None
    if guess == "learned":
        source = args.guess_train or ("configs" if args.config == 3 and not args.scale else "own")
        if source == "configs":
            trained = train_guess_configs(vm, dev)
            # the same network trained on the scene's own snapshots, for comparison
            own = train_guess(vm, cfg, case, scenes, dev, args.gnn_train_steps)
        else:
            trained = train_guess(vm, cfg, case, scenes, dev, args.gnn_train_steps)
    if guess == "zero":
        cfg["warm_start"] = 0
    if guess == "extrapolated":
        cfg["warm_start"] = 2
    s = vm.Solver(cfg, case, device=dev)
    if scenes is not None:
        s.set_scenes(*scenes)
    s.init()
    if trained is not None:
        s.gnn_create(GNN_LAYERS, 0)
        s.gnn_params(set_to=trained["params"])
        s.gnn_use(True)
        # the network was fitted to the flow over the training steps: time it
        # on the states that follow them (untimed advance, graph mode)
        s.set_graph(bool(args.graph))
        for _ in range(args.gnn_train_steps):
            s.step()
    stream = torch.cuda.ExternalStream(s.stream())

    def barrier():
        if ws > 1:
            torch.distributed.barrier()
        torch.cuda.synchronize()

    def rank_max(v: float) -> float:
        return max_over_ranks(v, ws, "cuda")

    if args.advance:  # profiling later flow states: untimed steps first
        s.set_graph(True)
        for _ in range(args.advance):
            s.step()
    tuning = s.autotune(2) if args.autotune else s.get_tuning()
    s.set_profile(False)
    s.set_graph(bool(args.graph))
    for _ in range(args.warmup):
        s.step()
    # ---- device-resident timed region (graph mode: one launch per step) ----
    iters = []
    sampler = ClockSampler(dev)
    barrier()
    sampler.start()
    l0 = s.scalar("launches")
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    status = 0
    for _ in range(args.steps):
        status |= s.step()
        iters.append(s.scalar("cg_iters"))
    e1.record(stream)
    barrier()
    launches = int(s.scalar("launches") - l0)
    clocks = sampler.stop()
    el_ms = rank_max(e0.elapsed_time(e1))
    relres = s.scalar("cg_relres")
    # ---- the same steps again with CUDA events around every stage and
    # every SpMV launch (eager launches; events cannot sit inside the graph's
    # while node): per-kernel durations for the roofline ----
    s.set_profile(True)
    ppe_ms, inner, outer = [], 0, 0
    stage = {k: [] for k in ("ms_neighbors", "ms_explicit", "ms_ppe", "ms_post")}
    barrier()
    p0, p1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    p0.record(stream)
    for _ in range(args.steps):
        status |= s.step()
        ppe_ms.append(s.scalar("ms_ppe"))
        inner += s.scalar("cg_iters")
        outer += s.scalar("cg_outer")
        for k in stage:
            stage[k].append(s.scalar(k))
    p1.record(stream)
    barrier()
    prof_ms = rank_max(p0.elapsed_time(p1))
    spmv_ms = s.scalar("spmv_ms")
    spmv_n = s.scalar("spmv_launches")
    nnz_a = s.scalar("nnz_a")
    rows = float((s.get("bcon") == 0).sum())
    # ---- end-to-end through the API with host buffers ----
    names = ["x", "y", "z", "u", "v", "w", "p"]
    host = {k: torch.from_numpy(s.get(k)).pin_memory() for k in names}
    ptrs = [host[k].data_ptr() for k in names]
    s.set_profile(False)
    barrier()
    t0 = time.perf_counter()
    e2 = torch.cuda.Event(enable_timing=True)
    e3 = torch.cuda.Event(enable_timing=True)
    e2.record(stream)
    for _ in range(args.steps):
        # mps_step_io: mps_set_state + mps_step + mps_get_state in one call,
        # the copy of u, v, w, p overlapped with the neighbour search
        s.step_io(ptrs, ptrs)
    e3.record(stream)
    barrier()
    e2e_ms = rank_max(max(e2.elapsed_time(e3), (time.perf_counter() - t0) * 1e3))
    bytes_state = 8 * n * len(names)
    peak, peak_kind = peaks()
    spmv_avg_ms = spmv_ms / max(spmv_n, 1)
    if mixed:  # launches of k_ir_spmv: inner FP32 SpMVs and FP64 refinements
        algo = (inner * spmv32_algorithmic_bytes(nnz_a, rows) +
                outer * refine_algorithmic_bytes(nnz_a, rows)) / max(inner + outer, 1)
    else:
        algo = spmv_algorithmic_bytes(nnz_a, rows)
    achieved = algo / (spmv_avg_ms * 1e-3) / 1e9 if spmv_n else None
    # DRAM bytes per launch from the ncu capture of the FP64 SpMV (scaled by
    # its traffic/algorithmic ratio); not captured for the mixed kernel
    traffic = None if mixed else SPMV_TRAFFIC_OVER_ALGORITHMIC * algo
    line = None
    # ---- the flow's later state: untimed steps to step `advanced`, then K
    # steps timed as above (the early steps are the easiest window) ----
    adv = None
    if args.advanced and args.config in (1, 2) and not args.scale:
        s.set_graph(bool(args.graph))
        done = int(s.scalar("steps"))
        for _ in range(max(0, args.advanced - done)):
            s.step()
        barrier()
        a0, a1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        ait = []
        a0.record(stream)
        for _ in range(args.steps):
            status |= s.step()
            ait.append(s.scalar("cg_iters"))
        a1.record(stream)
        barrier()
        adv_ms = rank_max(a0.elapsed_time(a1)) / args.steps
        adv = {"after_steps": max(args.advanced, done), "ms_per_step": adv_ms,
               "value": n * 1e3 / adv_ms * (ws if not split else 1),
               "cg_iters_mean": statistics.mean(ait)}
    if rank == 0:
        cpu = None
        if ws == 1 and args.config in (1, 2) and not args.scale:
            nth = physical_cores()
            cpu = time_reference(steps=3, warmup=1, nthreads=nth)
            if args.cpu_series:
                cpu["series"] = cpu_series(nth)
    # units of the whole job: a split batch counts every rank's own particles
    n_job = sum_over_ranks(float(n), ws) if split else float(n) * ws
    fp_job = sum_over_ranks(float(fp), ws) if split else float(fp) * ws
    if rank == 0:
        value = whole_job_rate(n_job * args.steps, 1, el_ms)
        line = {
            "metric": METRIC, "value": value, "unit": METRIC, "n_gpus": ws, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": el_ms / args.steps, "higher_is_better": True,
            "scaling": "strong" if split else "weak", "vs_baseline": None,
            "dtype": "f32+f64" if mixed else "f64",
            "data": "synthetic",
            "config": {"workload": (WORKLOADS[args.config] if not args.scale else
                                    f"3D dam break scaled x{args.scale} (profiling case)"),
                       "particles": int(n_job) if split else n,
                       "fluid_particles": int(fp_job) if split else fp,
                       "parallelism": ((f"{ws} ranks, the batch's scenes split between them "
                                        f"(rank 0: {int(scenes[2].shape[0])} scenes, {n} "
                                        "particles, in one context), no exchange") if split else
                                       (f"{ws} independent replicas" if ws > 1 else "1 GPU") +
                                       (f", {int(scenes[2].shape[0])} scenes in one context"
                                        if scenes is not None else "")),
                       "l2": "working set (lists, matrix) > 126 MB L2; no flush needed"},
            "fluid_particle_steps_per_s": fp_job * args.steps / (el_ms * 1e-3),
            "graph": bool(args.graph), "ms_per_step_profiled_eager": prof_ms / args.steps,
            "tuning": dict(tuning, autotuned=bool(args.autotune)),
            "ppe_ms_per_step": statistics.mean(ppe_ms), "cg_iters_mean": statistics.mean(iters),
            "precision": ({1: "mixed (FP32 inner CG, FP64 dots/refinement; FP32 viscous sums)",
                           2: "mixed (FP32 inner CG, FP64 dots/refinement; FP32 viscous sums, "
                              "PNUMSTAR and pressure gradient)"}.get(cfg["precision"], "fp64")),
            "cg_outer_mean": outer / args.steps,
            "cg_relres_last": relres, "status_bits": status,
            "stage_ms": {k[3:]: statistics.mean(v) for k, v in stage.items()},
            "roofline": {"kernel": ("k_ir_spmv (mixed PPE: FP32 inner SpMV + FP64 refinement, "
                                    "CSR, warp per row)" if mixed else
                                    "k_cg_spmv (PPE SpMV, FP64 CSR, warp per row)"),
                         "bound": "hbm",
                         "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": (achieved / peak) if achieved else None,
                         "traffic": traffic, "peak_source": peak_kind,
                         "algorithmic_bytes_per_launch": algo,
                         "avg_launch_ms": spmv_avg_ms, "launches_timed": int(spmv_n),
                         "duration_source": "CUDA events around every %s launch over the "
                                            "K profiled steps" % ("k_ir_spmv" if mixed else "k_cg_spmv")},
            "e2e": {"value": whole_job_rate(n_job * args.steps, 1, e2e_ms), "unit": METRIC,
                    "h2d_bytes_per_step": bytes_state, "d2h_bytes_per_step": bytes_state},
            "gpu_launches": launches, "clocks": clocks,
            "cpu_baseline": ({k: cpu[k] for k in ("value", "unit", "cores", "kind", "sample",
                                                  "series") if k in cpu}
                             if cpu else None),
        }
        if adv:
            line["advanced"] = adv
    s.close()
    if line is not None and mixed:
        line["error_vs_fp64"] = mixed_vs_fp64(vm, cfg, case, scenes, dev, steps=10)
    if line is not None:
        line["cg_guess"] = guess
        if args.advance:
            line["advanced_steps_before_warmup"] = args.advance
        if trained is not None:
            line["guess_training"] = trained["info"]
            line["advanced_steps_before_warmup"] = args.gnn_train_steps
            if own is not None:
                line["guess_training_own_scene"] = own["info"]
            line["guess_comparison"] = compare_guesses(
                vm, cfg, case, scenes, dev, trained["params"], args,
                own=None if own is None else own["params"])
    if ws > 1:
        torch.distributed.barrier()
        torch.distributed.destroy_process_group()
    if line:
        print(json.dumps(line), flush=True)


GNN_LAYERS = 4


def train_guess(vm, cfg, case, scenes, dev, steps, iters=2, lr=2e-3):
    """Train the learned CG initial guess online on the benchmark scene's own
    PPE snapshots: each of `steps` solver steps (previous-pressure start) is
    followed by `iters` Adam steps on the relative residual the network's
    guess would have left in that step's system.  Not part of any timed
    region; its cost is reported."""
    import time
    s = vm.Solver(cfg, case, device=dev)
    if scenes is not None:
        s.set_scenes(*scenes)
    s.init()
    s.gnn_create(GNN_LAYERS, 1)
    losses = []
    t0 = time.perf_counter()
    for _ in range(steps):
        s.step()
        losses.append(s.gnn_train(iters, lr, objective="residual"))
    sec = time.perf_counter() - t0
    params = s.gnn_params()
    s.close()
    k = max(1, min(10, steps // 4))
    return {"params": params,
            "info": {"snapshots": steps, "adam_steps_per_snapshot": iters, "lr": lr,
                     "objective": "|b - A x0|^2 / |b|^2 of the guess x0",
                     "loss_first": float(sum(losses[:k]) / k),
                     "loss_last": float(sum(losses[-k:]) / k), "seconds": sec,
                     "network": "4 residual message-passing layers, width 64, BF16 weights "
                                "and activations, FP32 sums"}}


def train_guess_configs(vm, dev, rounds=100, per_round=(20, 1, 1), iters=2, lr=2e-3):
    """Train the learned CG initial guess on PPE snapshots of configs 0, 1 and
    2 (the 2D dam, the 1.6 M-particle 3D dam in FP64 and in mixed precision),
    the training set the two-phase configuration names.  One network: its
    training state (weights, Adam moments and step count) passes from
    context to context; each round takes per_round[k] snapshots of config k
    (the defaults: config 0's whole 2000-step run and the first 100 steps of
    configs 1 and 2, 2,200 snapshots).  Each snapshot is one solver step
    (previous-pressure start) followed by `iters` Adam steps on the relative
    residual the network's guess leaves in that step's system.  Not part of
    any timed region; its cost is reported."""
    import time
    ctxs = []
    for k in (0, 1, 2):
        c, case, _ = build_case(0, k)
        s = vm.Solver(c, case, device=dev)
        s.init()
        s.gnn_create(GNN_LAYERS, 1)
        ctxs.append(s)
    state = ctxs[0].gnn_state()
    P = len(ctxs[0].gnn_params())
    losses = ([], [], [])
    t0 = time.perf_counter()
    for _ in range(rounds):
        for k, s in enumerate(ctxs):
            s.gnn_state(set_to=state)
            for _ in range(per_round[k]):
                s.step()
                losses[k].append(s.gnn_train(iters, lr, objective="residual"))
            state = s.gnn_state()
    sec = time.perf_counter() - t0
    for s in ctxs:
        s.close()

    def ends(v):
        k = max(1, min(10, len(v) // 4))
        return float(sum(v[:k]) / k), float(sum(v[-k:]) / k)
    return {"params": state[:P],
            "info": {"source": "PPE snapshots of configs 0, 1 and 2",
                     "snapshots": {f"config{k}": rounds * per_round[k] for k in range(3)},
                     "adam_steps_per_snapshot": iters, "lr": lr,
                     "objective": "|b - A x0|^2 / |b|^2 of the guess x0",
                     "loss_first_last": {f"config{k}": ends(losses[k]) for k in range(3)},
                     "seconds": sec,
                     "network": "4 residual message-passing layers, width 64, BF16 weights "
                                "and activations, FP32 sums"}}


def compare_guesses(vm, cfg, case, scenes, dev, params, args, steps=20, own=None):
    """CG iterations, initial relative residual and step time for the zero,
    previous-pressure and learned starting points, each in a fresh context
    advanced past the training steps, then timed over `steps` steps (graph
    mode, CUDA events)."""
    import torch
    out = {}
    names = ["zero", "previous", "extrapolated", "learned"] + (["learned_own_scene"] if own is not None
                                                               else [])
    for name in names:
        c = dict(cfg)
        c["warm_start"] = {"zero": 0, "extrapolated": 2}.get(name, 1)
        s = vm.Solver(c, case, device=dev)
        if scenes is not None:
            s.set_scenes(*scenes)
        s.init()
        if name.startswith("learned"):
            s.gnn_create(GNN_LAYERS, 0)
            s.gnn_params(set_to=params if name == "learned" else own)
            s.gnn_use(True)
        s.set_graph(bool(args.graph))
        for _ in range(args.gnn_train_steps + max(args.warmup, 3)):
            s.step()
        st = torch.cuda.ExternalStream(s.stream())
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        its, r0 = [], []
        torch.cuda.synchronize()
        e0.record(st)
        for _ in range(steps):
            s.step()
            its.append(s.scalar("cg_iters"))
            r0.append(s.scalar("cg_r0"))
        e1.record(st)
        torch.cuda.synchronize()
        out[name] = {"cg_iters_mean": sum(its) / steps, "r0_rel_mean": sum(r0) / steps,
                     "ms_per_step": e0.elapsed_time(e1) / steps}
        s.close()
    out["steps"] = steps
    return out


def mixed_vs_fp64(vm, cfg, case, scenes, dev, steps):
    """Max relative differences between the mixed-precision run and the FP64
    run of the same case after the same number of steps (not timed)."""
    import numpy as np
    out = {}
    mixed = cfg["precision"]
    for prec in (mixed, 0):
        c = dict(cfg)
        c["precision"] = prec
        s = vm.Solver(c, case, device=dev)
        if scenes is not None:
            s.set_scenes(*scenes)
        s.init()
        p1 = None
        for k in range(steps):
            s.step()
            if k == 0:
                p1 = s.get("p")
        out[prec] = {"p_step1": p1, **{f: s.get(f) for f in ("x", "y", "z", "u", "v", "w", "p")}}
        s.close()

    def rel(a, b):
        return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))
    res = {"steps": steps, "norm": "max|mixed - fp64| / max|fp64|",
           "p_after_1_step": rel(out[mixed]["p_step1"], out[0]["p_step1"])}
    for f in ("p", "x", "y", "z", "u", "v", "w"):
        res[f] = rel(out[mixed][f], out[0][f])
    return res


# the run length each configuration names (configs 3 and 4 name none)
DEFAULT_STEPS = {0: 2000, 1: 500, 2: 500, 3: 100, 4: 100}
REF_MAX_STEPS = 20


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=None,
                    help="timed steps (default: the configuration's run length, "
                         "2000 / 500 / 500 / 100 / 100 for configs 0-4)")
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--graph", type=int, default=1, choices=[0, 1],
                    help="1: each step is one CUDA graph launch (CG loop as a while node)")
    ap.add_argument("--autotune", type=int, default=1, choices=[0, 1],
                    help="1: pick launch shapes by timing candidates on the first steps")
    ap.add_argument("--guess", default=None, choices=["zero", "previous", "extrapolated", "learned"],
                    help="CG starting point (default: learned for configs 3 and 4)")
    ap.add_argument("--guess-train", default=None, choices=["configs", "own"],
                    help="training snapshots of the learned guess: configs 0-2 (the default "
                         "for config 3, which names them) or the benchmark scene's own")
    ap.add_argument("--gnn-train-steps", type=int, default=300,
                    help="solver steps of online training for the learned guess")
    ap.add_argument("--precision", type=int, default=None, choices=[0, 1, 2],
                    help="0 FP64; 1 mixed PPE and FP32 viscous sums (default for configs 2 "
                         "and 4); 2 as 1 with FP32 PNUMSTAR and pressure gradient")
    ap.add_argument("--config", type=int, default=1, choices=[0, 1, 2, 3, 4],
                    help="benchmark configuration (1: the headline 3D dam break)")
    ap.add_argument("--advance", type=int, default=0,
                    help="profiling only: untimed steps before autotuning and warm-up")
    ap.add_argument("--advanced", type=int, default=500,
                    help="configs 1/2: also time K steps after this many steps (0: skip)")
    ap.add_argument("--cpu-series", type=int, default=1, choices=[0, 1],
                    help="configs 1/2: CPU baseline at the small radius, scaled and sequential")
    ap.add_argument("--scale", type=int, default=0,
                    help="profiling only: smaller 3D dam (10s x 20s x 10s fluid)")
    args = ap.parse_args()
    if args.impl == "reference":
        # the reference CPU path takes ~0.75 s per step of its sample: bounded
        args.steps = min(args.steps or 3, REF_MAX_STEPS)
        run_reference_arm(args)
    else:
        if args.steps is None:
            args.steps = DEFAULT_STEPS[args.config] if not args.scale else 20
        run_ours(args)


if __name__ == "__main__":
    main()
