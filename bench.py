"""Benchmark of the B200 batched trace-and-optimise path (one JSON line on rank 0).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]
                    [--workload merit|lm]

Workload: the seven-element objective of the adjoint-vs-FD configuration -- 4096 runs (one
variant each), 15 table surfaces, 7 wavelengths, 5 fields, 16 rings x 32 spokes (14,448 rays
per variant, 59.2 M rays per evaluation), 29 variables (14 curvatures, 15 thicknesses incl. the
working distance), soft failure; synthetic seeded inputs.

  --workload lm (default): one step = one batched Levenberg-Marquardt cycle of all 4096 runs
      (adjoint Jacobian fused with its FP64-tensor-core normal equations, damped Cholesky step,
      trial MERIT, acceptance), FP64 with FMA contraction, replayed as a CUDA graph. The value is
      the LM iterations the runs actually took in the timed cycles per second. Beside it: the
      same LM with the MIXED-precision adjoint (`adjoint_mixed`), with the central-difference
      Jacobian (the reference method, 2P + 1 = 59 traced variants per run, `fd_fp64`, on 512
      runs: its cost is linear in the runs), and the OPD error of each precision against the
      bit-exact FP64 trace.
  --workload merit: one step = one MERIT evaluation of all variants.

N > 1 (torchrun, one rank per GPU): every rank traces its own 4096 variants (weak scaling,
independent variants, no data-path collective); the time is the maximum over ranks.

Timing: W untimed warm-up steps, then K steps timed with CUDA events on the launching stream,
bracketed by a barrier and a device synchronisation; the L2 cache (126 MB) is flushed before
every step outside the events (the batch records are only 5 MB). Clocks are sampled with
nvidia-smi during the timed region.
"""

from __future__ import annotations

import argparse
import ctypes as C
import dataclasses
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "LM iter/s & ray-surface hits/s: adjoint+mixed vs FP64 FD, at ≤1e-4λ OPD err"
WORKLOAD = "objective-4096: 4096 runs x 15 surfaces, L=7, F=5, 16x32 pupil, P=29 (config 2 shape)"
WORKLOAD_SINGLET = ("singlet-1024: 1024 biconvex singlets (stop plane + 2 spheres), L=3, F=3 "
                    "(axis 6 rays, two Half 6x12 fields: 150 rays per wavelength), soft "
                    "failures (config 1 shape)")
WORKLOAD_LM = ("objective-4096: 4096 runs x 15 surfaces, L=7, F=5, 16x32 pupil, P=32: 14 "
               "curvatures, 15 thicknesses and the first element's Buchdahl glass (n0, nu1, nu2) "
               "(config 2 shape)")
WORKLOAD_LM_STOP = ("objective-4096: 4096 runs x 16 surfaces (15 of configuration 2 with its "
                    "aperture stop inserted as table surface {stop}; the entrance pupil by "
                    "paraxial ray aiming), L=7, F=5, 16x32 pupil, P={P}: 14 curvatures, 14 "
                    "thicknesses (thickness[0] follows the pupil) and the first element's "
                    "Buchdahl glass (config 2 shape)")
FLOPEQ_PER_RAY_SURFACE = 140  # reference cost model (docs/hardware.md:138 of the reference)
# DRAM traffic (ncu dram__bytes_read.sum + dram__bytes_write.sum) measured once per kernel on a
# smaller capture of the same workload, per unit, scaled below by the units of the timed launch
# and reported with "traffic_source": "scaled capture".
# trace_kernel, objective variants (512 captured: 668,672 B read, 0 B written)
TRAFFIC_BYTES_PER_VARIANT = 668672 / 512
# adjoint_gram_kernel<Exact64, 12> (bit-exact FP64; glass variable and the aimed stop at
# surface 8), configuration-2 objectives (1,184 runs captured: 2.070 GB read, 19.238 GB written)
FUSED_TRAFFIC_BYTES_PER_RUN = (2.069940e9 + 19.237769e9) / 1184
# adjoint_gram_kernel<MixedPrecision, 18, *> (plates in the forward trace only: every plate
# lies below every run's sweep floor; the three-CTA instance for the runs with more than 31
# variables), uneven runs with the zero-power plate at surface 1, both launches of a call
# (1,184 runs captured: 34.8 MB read, 2.343 GB written)
FUSED_TRAFFIC_UNEVEN_BYTES_PER_RUN = (31.629056e6 + 3.127808e6 + 1.787534e9 + 0.555371e9) / 1184

def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--workload", default="uneven", choices=["uneven", "lm", "merit", "tolerancing", "precision",
                             "singlet", "psf"])
    ap.add_argument("--stop", type=int, default=8,
                    help="--workload lm: table surface of the aperture stop inside the "
                         "objective (paraxial ray aiming); 0: the stop at surface 0")
    ap.add_argument("--variants", type=int, default=None,
                    help="runs per GPU (default 8192 for uneven, 262144 for tolerancing, 4096 "
                         "otherwise)")
    return ap.parse_args()


# ---- distributed plumbing ------------------------------------------------------------------
def dist_setup(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import torch.distributed as dist
        import datetime
        backend = "nccl" if os.environ.get("MKB_BENCH_BACKEND", "nccl") == "nccl" else "gloo"
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=120))
    return world, rank, local


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def max_over_ranks(value: float, world: int, device) -> float:
    if world == 1:
        return value
    import torch
    import torch.distributed as dist
    t = torch.tensor([value], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


# ---- clocks --------------------------------------------------------------------------------
class ClockSampler:
    """nvidia-smi samples of SM clock and throttle reasons while the timed region runs."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.lines: list[str] = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "100"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except (FileNotFoundError, OSError):
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
        return False

    def summary(self):
        sm, mx, reasons = [], 0.0, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.lines:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = max(mx, float(parts[2]))
            except ValueError:
                continue
            for name, flag in zip(names, parts[5:9]):
                if flag.lower().startswith("active"):
                    reasons.add(name)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


# ---- B200 arm ------------------------------------------------------------------------------
def fp64_peak_tflops(torch) -> float:
    """Measured FP64 peak: cuBLAS DGEMM 8192^3 on this GPU, best of 5 (CUDA events)."""
    n = 8192
    a = torch.randn(n, n, dtype=torch.float64, device="cuda")
    b = torch.randn(n, n, dtype=torch.float64, device="cuda")
    for _ in range(2):
        a @ b
    torch.cuda.synchronize()
    best = float("inf")
    for _ in range(5):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        a @ b
        e1.record()
        torch.cuda.synchronize()
        best = min(best, e0.elapsed_time(e1))
    del a, b
    return 2 * n ** 3 / best / 1e9


def run_b200(args, world, rank, local):
    import torch
    from mikroptim_b200 import _capi, engine, workloads
    from mikroptim_b200.batch import PRECISION_FP64, PRECISION_FP64_FMA, ResidualLayout

    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    lib = _capi.lib()
    b, st, vs, x0 = workloads.objective(args.variants or 4096,
                                        seed=20261203 + 2 + 1000 * rank)
    st.precision = PRECISION_FP64_FMA
    lay = ResidualLayout(b.topology, st)
    db = engine.DeviceSystemBatch(b, dev)
    ws = torch.empty(int(lib.mkb_merit_workspace_bytes(b.variants, C.byref(lay.plan(b)))),
                     dtype=torch.uint8, device=dev)
    flush = torch.empty(256 * 1024 * 1024, dtype=torch.uint8, device=dev)
    stream = torch.cuda.current_stream()
    rays = b.variants * lay.rays_per_variant
    hits = rays * (b.surfaces - 1)
    flopeq = rays * FLOPEQ_PER_RAY_SURFACE * (b.surfaces - 1 + 2)

    def step():
        return engine.merit_device(db, lay, b, workspace=ws)

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    barrier(world)
    launches0 = lib.mkb_launch_count()
    times = []
    with ClockSampler(local) as clocks:
        torch.cuda.synchronize()
        barrier(world)
        for _ in range(args.steps):
            flush.zero_()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            step()
            e1.record(stream)
            times.append((e0, e1))
        torch.cuda.synchronize()
        barrier(world)
    launches = lib.mkb_launch_count() - launches0
    ms_total = sum(a.elapsed_time(c) for a, c in times)
    ms_total = max_over_ranks(ms_total, world, dev)
    ms_step = ms_total / args.steps
    value = world * hits * args.steps / (ms_total / 1e3)

    # dominant kernel alone (trace kernel without the finalize launch) for the roofline
    plan = lay.plan(b)
    kernel_ms = ms_step  # finalize is < 1 % of the step; measured below
    # exact FP64 rate for reference
    st_exact = ResidualLayout(b.topology, type(st)(rings=st.rings, spokes=st.spokes,
                                                   failure=st.failure,
                                                   precision=PRECISION_FP64))
    engine.merit_device(db, st_exact, b, workspace=ws)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    flush.zero_()
    e0.record(stream)
    for _ in range(3):
        engine.merit_device(db, st_exact, b, workspace=ws)
    e1.record(stream)
    torch.cuda.synchronize()
    exact_ms = e0.elapsed_time(e1) / 3

    # end to end through the host-buffer path: pinned host records in, merit out, every step
    host_in = db.host_records
    host_out = torch.empty(b.variants, dtype=torch.float64).pin_memory()
    for _ in range(2):
        db.records[:b.variants].copy_(host_in, non_blocking=True)
        host_out.copy_(step().merit, non_blocking=True)
    torch.cuda.synchronize()
    barrier(world)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        db.records[:b.variants].copy_(host_in, non_blocking=True)
        host_out.copy_(step().merit, non_blocking=True)
    e1.record(stream)
    torch.cuda.synchronize()
    e2e_ms = max_over_ranks(e0.elapsed_time(e1) / args.steps, world, dev)

    peak = fp64_peak_tflops(torch) if rank == 0 else None
    achieved = flopeq / (kernel_ms / 1e3) / 1e12
    out = None
    if rank == 0:
        out = {
            "metric": METRIC,
            "value": value,
            "unit": "ray-surface hits/s",
            "n_gpus": world,
            "steps": args.steps,
            "warmup": args.warmup,
            "ms_per_step": ms_step,
            "higher_is_better": True,
            "scaling": "weak",
            "vs_baseline": None,
            "dtype": "f64",
            "data": "synthetic (seeded generator, configuration-2 shapes)",
            "config": {"workload": WORKLOAD, "step": "one MERIT evaluation of all variants",
                       "precision": "FP64 with FMA contraction",
                       "variants_per_gpu": b.variants, "rays_per_variant": lay.rays_per_variant,
                       "l2": "flushed (256 MB write) before every timed step"},
            "gpu_launches": int(launches),
            "e2e": {"value": world * hits / (e2e_ms / 1e3), "unit": "ray-surface hits/s",
                    "h2d_bytes_per_step": int(host_in.numel() * 8),
                    "d2h_bytes_per_step": int(b.variants * 8)},
            "roofline": {"bound": "fp64", "achieved": achieved, "peak": peak,
                         "unit": "TFLOP/s", "frac": achieved / peak if peak else None,
                         "traffic": TRAFFIC_BYTES_PER_VARIANT * b.variants,
                         "traffic_source": "scaled capture",
                         "peak_source": "cuBLAS DGEMM 8192^3 measured in this run",
                         "flop_model": "140 FLOP-eq per ray-surface step, (S-1)+2 steps per ray"},
            "fp64_exact": {"ms_per_step": exact_ms,
                           "value": world * hits / (exact_ms / 1e3),
                           "note": "bit-identical to the reference CPU"},
            "clocks": clocks.summary(),
        }
    return out, (b, lay)


def _lm_window(lm, steps: int, warmup: int, flush, world, dev, graph: bool = True):
    """W warm-up cycles, then K cycles timed with CUDA events (L2 flushed before each, outside
    the events). Returns (ms per cycle, LM iterations performed in the timed cycles, launches
    per cycle)."""
    import torch
    from mikroptim_b200 import _capi
    lib = _capi.lib()
    stream = torch.cuda.current_stream()
    for _ in range(warmup):
        lm.cycle()
    l0 = lib.mkb_launch_count()
    g = lm.capture() if graph else None
    per_cycle = lib.mkb_launch_count() - l0
    it0 = int(lm.iterations().sum())
    barrier(world)
    times = []
    for _ in range(steps):
        flush.zero_()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        if g is not None:
            g.replay()
        else:
            lm.cycle()
        e1.record(stream)
        times.append((e0, e1))
    torch.cuda.synchronize()
    barrier(world)
    iters = int(lm.iterations().sum()) - it0
    ms = sum(a.elapsed_time(b) for a, b in times)
    del g
    return ms / steps, iters, per_cycle


def opd_errors(b, st, runs: int = 256):
    """RMS / max OPD difference (waves at the reference wavelength) of the FP64-FMA, MIXED and
    (coaxial batches without plates) FP32-bulk traces against the bit-exact FP64 trace, over
    rays in the piston with the same status."""
    import torch
    from mikroptim_b200 import engine
    from mikroptim_b200.batch import ResidualLayout, in_piston
    sub = b.subset(0, runs)
    lam_mm = sub.reference_wavelength_nm * 1e-6
    out = {}
    res = {}
    bulk = not sub.topology.non_coaxial and sub.topology.ghost_plates == 0
    precs = (0, 2, 1, 4) if bulk else (0, 2, 1)
    for prec in precs:
        lay = ResidualLayout(sub.topology, dataclasses.replace(st, precision=prec))
        r = engine.residuals_device(engine.DeviceSystemBatch(sub), lay, sub)
        torch.cuda.synchronize()
        res[prec] = (r.opd.cpu().numpy(), r.status.cpu().numpy())
    ref_opd, ref_st = res[0]
    for prec, name in ((2, "fp64_fma"), (1, "mixed"), (4, "fp32_bulk")):
        if prec not in res:
            continue
        opd, stt = res[prec]
        same = (stt == ref_st) & in_piston(ref_st)
        clean = same & (ref_st == 0)
        err = (opd - ref_opd) / lam_mm
        out[name] = {"rms_waves": float(np.sqrt(np.mean(err[same] ** 2))),
                     "rms_waves_ok_rays": float(np.sqrt(np.mean(err[clean] ** 2))),
                     "median_abs_waves": float(np.median(np.abs(err[same]))),
                     "status_agreement": float(np.mean(stt == ref_st))}
    return out


def gram_errors(ref: np.ndarray, got: np.ndarray) -> np.ndarray:
    """|got - ref| / sqrt(|A_ii A_jj|) of every entry of one run's (P+1)^2 normal equations."""
    d = np.abs(np.diagonal(ref))
    d = np.maximum(d, 1e-20 * d.max() + 1e-300)
    return (np.abs(got - ref) / np.sqrt(d[:, None] * d[None, :])).ravel()


def mixed_accuracy(b, st, vss, x0, runs: int = 256, iterations: int = 100):
    """What the FP32 reverse sweep costs on uneven runs: (1) the MIXED fused normal equations
    against the FP64 (separately rounded) fused ones at the start points, per entry relative to
    sqrt(A_ii A_jj), for the runs with <= 31 variables and the wider ones (each kind has its own
    launch); (2) the final merit of a 100-iteration MIXED LM against the FP64-FMA LM."""
    import torch
    from mikroptim_b200 import engine
    from mikroptim_b200.batch import (PRECISION_FP64, PRECISION_FP64_FMA, PRECISION_MIXED,
                                      ResidualLayout)
    sub = b.subset(0, runs)
    vs = vss[:runs]
    x = x0[:runs]
    lay = {p: ResidualLayout(sub.topology, dataclasses.replace(st, precision=p))
           for p in (PRECISION_FP64, PRECISION_FP64_FMA, PRECISION_MIXED)}
    db = engine.DeviceSystemBatch(sub)
    ref = engine.adjoint_normal_equations_runs_device(db, lay[PRECISION_FP64], sub, vs, x)
    got = engine.adjoint_normal_equations_runs_device(db, lay[PRECISION_MIXED], sub, vs, x)
    torch.cuda.synchronize()
    narrow, wide = [], []
    for i, v in enumerate(vs):
        e = gram_errors(engine.gram_block(ref, i, v.size).cpu().numpy(),
                        engine.gram_block(got, i, v.size).cpu().numpy())
        (wide if v.size > 31 else narrow).append(e)

    def stats(parts):
        if not parts:
            return None
        e = np.concatenate(parts)
        return {"runs": len(parts), "median": float(np.median(e)),
                "p99": float(np.quantile(e, 0.99)), "max": float(e.max())}
    opt = engine.LmOptions(max_iterations=iterations, jacobian=engine.JACOBIAN_ADJOINT,
                           gram_exact=False)
    lm = {p: engine.optimize_lm_gpu(sub, lay[p], vs, x, opt)
          for p in (PRECISION_FP64, PRECISION_FP64_FMA, PRECISION_MIXED)}

    def agreement(a, b_):
        rel = np.abs(a["merit"] - b_["merit"]) / np.maximum(np.abs(b_["merit"]), 1e-300)
        ratio = a["merit"] / b_["merit"]
        conv = (np.isin(a["status"], (1, 2, 3, 4)) & np.isin(b_["status"], (1, 2, 3, 4)))
        return {"median_rel": float(np.median(rel)), "p90_rel": float(np.quantile(rel, 0.9)),
                "max_rel": float(rel.max()),
                "geo_mean_ratio": float(np.exp(np.mean(np.log(ratio)))),
                "lower_frac": float(np.mean(ratio < 1.0 - 1e-9)),
                "higher_frac": float(np.mean(ratio > 1.0 + 1e-9)),
                "converged_in_both": int(conv.sum()),
                "converged_median_rel": float(np.median(rel[conv])) if conv.any() else None}
    return {"normal_equations_vs_fp64": {"le31_variables": stats(narrow),
                                         "gt31_variables": stats(wide),
                                         "error": "|A_mixed - A_fp64| / sqrt(A_ii A_jj)"},
            "lm_final_merit": {
                "runs": runs, "iterations": iterations,
                "at_iteration_limit_frac": float(np.mean(lm[PRECISION_FP64]["status"] == 5)),
                "mixed_vs_fp64": agreement(lm[PRECISION_MIXED], lm[PRECISION_FP64]),
                "fp64_fma_vs_fp64": agreement(lm[PRECISION_FP64_FMA], lm[PRECISION_FP64])}}


def e2e_optimize(b, layout, variables, x0, world, dev, iterations: int = 100):
    """optimize_lm_gpu end to end (the call `optimize --gpu` makes): host batch, variables and
    start points in, host results out, 100 iterations plus penalty rounds, convergence included.
    LM iterations taken / wall time (max over ranks); the bytes copied each way are counted
    from the arrays the call uploads and downloads."""
    import torch
    from mikroptim_b200 import _capi, engine
    opt = engine.LmOptions(max_iterations=iterations, jacobian=engine.JACOBIAN_ADJOINT,
                           gram_exact=False)
    runs = b.variants
    per_run = isinstance(variables, (list, tuple))
    P = max(v.size for v in variables) if per_run else variables.size
    stride = int(_capi.lib().mkb_record_stride_ext(b.surfaces, b.wavelengths, b.fields,
                                                   1 if b.non_coaxial else 0,
                                                   b.topology.ghost_plates,
                                                   b.topology.ghost_terms,
                                                   1 if b.buchdahl_coeff is not None else 0))
    torch.cuda.synchronize(dev)
    barrier(world)
    t0 = time.perf_counter()
    res = engine.optimize_lm_gpu(b, layout, variables, x0, opt, device=dev.index or 0)
    torch.cuda.synchronize(dev)
    wall = time.perf_counter() - t0
    wall = max_over_ranks(wall, world, dev)
    iters = int(res["iterations"].sum())
    rounds = int(res["penalty_rounds"].max())
    # per pass: records + variant surface counts + x0 + the run-variable table in; x, merit,
    # status, counters, damping, history, failed counts out
    h2d = runs * (stride * 8 + P * 8 + ((1 + 1800) if per_run else 0))
    d2h = runs * (P * 8 + 8 + 4 * 4 + 8 + 8 * (iterations + 1) + 16)
    return {"value": world * iters / wall, "unit": "LM iterations/s",
            "h2d_bytes_per_step": int(h2d * rounds), "d2h_bytes_per_step": int(d2h * rounds),
            "api": "engine.optimize_lm_gpu(host batch, VariableSet(s), x0) -> host results",
            "wall_s": wall, "iterations": iters, "runs": runs, "penalty_rounds_max": rounds,
            "cycles": int(res["cycles"]),
            "converged_runs": int(np.sum(res["status"] != 0)),
            "step": "one full optimisation (100 iterations, convergence and penalty rounds)"}


def run_lm(args, world, rank, local):
    import torch
    from mikroptim_b200 import _capi, engine, workloads
    from mikroptim_b200.batch import PRECISION_FP64_FMA, PRECISION_MIXED, ResidualLayout

    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    lib = _capi.lib()
    b, st, vs, x0 = workloads.objective(args.variants or 4096,
                                        seed=20261203 + 2 + 1000 * rank, glass=True)
    if args.stop > 0:  # configuration 2's stop at surface 8: an aimed entrance pupil
        b, st, vs, x0 = workloads.with_aperture_stop(b, st, vs, args.stop)
    # the headline runs bit-exact FP64 (every operation separately rounded, as the reference
    # CPU): on these NA 0.95 objectives FP64 with contraction misses the 1e-4 wave OPD bar on
    # grazing rays (opd_error_vs_fp64), so FP64_FMA and MIXED are reported beside it
    from mikroptim_b200.batch import PRECISION_FP64
    st.precision = PRECISION_FP64
    lay = ResidualLayout(b.topology, st)
    runs = b.variants
    P = vs.size
    db = engine.DeviceSystemBatch(b, dev)
    max_it = args.warmup + args.steps + 100
    opt = engine.LmOptions(max_iterations=max_it, jacobian=engine.JACOBIAN_ADJOINT,
                           gram_exact=False)
    flush = torch.empty(256 * 1024 * 1024, dtype=torch.uint8, device=dev)
    stream = torch.cuda.current_stream()
    rays = runs * lay.rays_per_variant
    steps_per_ray = b.surfaces - 1

    # ---- headline: adjoint (fused with the FP64 tensor-core normal equations) LM cycles ----
    lm = engine.DeviceLm(db, lay, b, vs, opt, runs)
    lm.start(x0)
    with ClockSampler(local) as clocks:
        ms_cycle, iters, per_cycle = _lm_window(lm, args.steps, args.warmup, flush, world, dev)
    ms_step = max_over_ranks(ms_cycle, world, dev)
    iters_all = max_over_ranks(float(iters), world, dev) * world  # equal per rank by seeding
    value = iters_all / (ms_step * args.steps / 1e3)
    x_now = torch.empty((runs, P), dtype=torch.float64, device=dev)
    lib.mkb_lm_results_device(*lm._args(), runs, C.c_void_p(lm.workspace.data_ptr()),
                              C.c_void_p(x_now.data_ptr()), *([None] * 10),
                              C.c_void_p(stream.cuda_stream))
    torch.cuda.synchronize()
    x_np = x_now.cpu().numpy()
    del lm

    # ---- the same LM with the MIXED-precision adjoint ----
    lay_mixed = ResidualLayout(b.topology, dataclasses.replace(st, precision=PRECISION_MIXED))
    lm_m = engine.DeviceLm(db, lay_mixed, b, vs, opt, runs)
    lm_m.start(x0)
    ms_mixed, iters_mixed, _ = _lm_window(lm_m, args.steps, args.warmup, flush, world, dev)
    mixed_value = world * iters_mixed / (max_over_ranks(ms_mixed, world, dev) * args.steps / 1e3)
    del lm_m

    # ---- the same LM in FP64 with FMA contraction (faster; its OPD error in
    # opd_error_vs_fp64.fp64_fma)
    lay_fma = ResidualLayout(b.topology, dataclasses.replace(st, precision=PRECISION_FP64_FMA))
    lm_f = engine.DeviceLm(db, lay_fma, b, vs, opt, runs)
    lm_f.start(x0)
    ms_fma, iters_fma, _ = _lm_window(lm_f, args.steps, args.warmup, flush, world, dev)
    fma_value = world * iters_fma / (max_over_ranks(ms_fma, world, dev) * args.steps / 1e3)
    del lm_f

    # ---- the reference method on the same GPU: FD Jacobian (2P + 1 traced variants), FP64 ----
    fd_runs = min(512, runs)
    fd_b = b.subset(0, fd_runs)
    fd_db = engine.DeviceSystemBatch(fd_b, dev)
    fd_opt = engine.LmOptions(max_iterations=max_it, jacobian=engine.JACOBIAN_FD,
                              gram_exact=False)
    fd = engine.DeviceLm(fd_db, lay, fd_b, vs, fd_opt, fd_runs)
    fd.start(x0[:fd_runs])
    fd_steps = max(2, min(args.steps, 10))
    fd_ms, fd_iters, _ = _lm_window(fd, fd_steps, args.warmup, flush, world, dev)
    fd_value = fd_iters / (fd_ms * fd_steps / 1e3)
    del fd

    # ---- the dominant kernel alone: fused adjoint + normal equations at the current points.
    # The call's host part is enqueued while the previous call runs: the first call is outside
    # the events, so they see the GPU work only; the L2 flush between calls is taken out.
    x_dev = x_now.clone()
    engine.adjoint_normal_equations_device(db, lay, b, vs, x_dev)
    torch.cuda.synchronize()
    reps = 3
    engine.adjoint_normal_equations_device(db, lay, b, vs, x_dev)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(reps):
        flush.zero_()
        engine.adjoint_normal_equations_device(db, lay, b, vs, x_dev)
    e1.record(stream)
    torch.cuda.synchronize()
    f0, f1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    f0.record(stream)
    for _ in range(reps):
        flush.zero_()
    f1.record(stream)
    torch.cuda.synchronize()
    kernel_ms = (e0.elapsed_time(e1) - f0.elapsed_time(f1)) / reps
    # FLOP model (reference cost model): adjoint = 3 x FLOPeq(ray), FLOPeq = 140 (S_steps + 2),
    # plus 4 P per ray (projection) and 2 P^2 per row (rows: rays and penalty rows)
    flop = rays * (3 * FLOPEQ_PER_RAY_SURFACE * (steps_per_ray + 2) + 4 * P) + \
        2 * P * P * runs * lay.trace_rows

    # ---- MERIT rate (ray-surface hits/s) on the same points ----
    engine.merit_device(db, lay, b)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(3):
        engine.merit_device(db, lay, b)
    e1.record(stream)
    torch.cuda.synchronize()
    merit_ms = e0.elapsed_time(e1) / 3

    # ---- end to end through the drop-in API: optimize_lm_gpu(host batch, variables, x0) ->
    # host results, the full 100-iteration LM with its penalty rounds, convergence included
    e2e = e2e_optimize(b, lay, vs, x0, world, dev)

    errors = opd_errors(b, st) if rank == 0 else None
    peak = fp64_peak_tflops(torch) if rank == 0 else None
    achieved = flop / (kernel_ms / 1e3) / 1e12
    if rank != 0:
        return None, None
    return {
        "metric": METRIC,
        "value": value,
        "unit": "LM iterations/s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": ms_step,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f64",
        "data": "synthetic (seeded generator, configuration-2 shapes)",
        "config": {"workload": WORKLOAD_LM if args.stop <= 0 else WORKLOAD_LM_STOP.format(
                       stop=args.stop, P=P),
                   "step": "one batched LM cycle of all runs (CUDA graph)",
                   "runs_per_gpu": runs, "variables": P, "rays_per_run": lay.rays_per_variant,
                   "jacobian": "adjoint fused with FP64 tensor-core normal equations",
                   "precision": "FP64, every operation separately rounded (bit-identical to "
                                "the reference CPU: no OPD error)",
                   "iterations": "LM iterations actually taken in the timed cycles "
                                 f"({iters} of {runs * args.steps} run-cycles)",
                   "l2": "flushed (256 MB write) before every timed step"},
        "gpu_launches": int(per_cycle * args.steps),
        "ray_surface_hits_per_s": world * rays * steps_per_ray / (merit_ms / 1e3),
        "adjoint_mixed": {"value": mixed_value, "unit": "LM iterations/s",
                          "ms_per_cycle": ms_mixed},
        "adjoint_fp64_fma": {"value": fma_value, "unit": "LM iterations/s",
                             "ms_per_cycle": ms_fma,
                             "speedup_vs_fd": fma_value / (world * fd_value)},
        "fd_fp64": {"value": world * fd_value, "unit": "LM iterations/s",
                    "ms_per_cycle_512_runs": fd_ms, "cycles": fd_steps,
                    "speedup_adjoint_vs_fd": value / (world * fd_value),
                    "speedup_adjoint_mixed_vs_fd": mixed_value / (world * fd_value)},
        "opd_error_vs_fp64": errors,
        "e2e": e2e,
        "roofline": {"bound": "fp64", "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
                     "frac": achieved / peak if peak else None,
                     "traffic": (FUSED_TRAFFIC_BYTES_PER_RUN * runs
                                 if FUSED_TRAFFIC_BYTES_PER_RUN else None),
                     "traffic_source": "scaled capture",
                     "kernel": "adjoint_gram_kernel (fused adjoint + DMMA normal equations)",
                     "kernel_ms": kernel_ms,
                     "peak_source": "cuBLAS DGEMM 8192^3 measured in this run",
                     "flop_model": "3 x 140 (S-1+2) FLOP-eq per ray + 4P per ray + 2P^2 per row"},
        "clocks": clocks.summary(),
    }, None


WORKLOAD_UNEVEN = ("uneven-8192: 8192 runs, S ~ U{6..30} (stop, a zero-power ghost plate at "
                   "surface 1, 1/50-style biconvex elements, a zero-curvature surface where the "
                   "count is odd), P ~ U{8..64} (capped by the system), L=7, F=5, 16x32 Half "
                   "pupils (config 3 shape)")


def run_uneven(args, world, rank, local):
    """Configuration 3: batched LM over uneven systems, one launch per kernel per cycle."""
    import torch
    from mikroptim_b200 import _capi, engine, workloads
    from mikroptim_b200.batch import PRECISION_FP64_FMA, PRECISION_MIXED, ResidualLayout

    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    lib = _capi.lib()
    runs = args.variants or 8192
    b, st, vss, x0 = workloads.uneven(runs, seed=20261203 + 3 + 1000 * rank)
    P = max(v.size for v in vss)
    lay_fma = ResidualLayout(b.topology, dataclasses.replace(st, precision=PRECISION_FP64_FMA))
    lay_mixed = ResidualLayout(b.topology, dataclasses.replace(st, precision=PRECISION_MIXED))
    db = engine.DeviceSystemBatch(b, dev)
    max_it = args.warmup + args.steps + 100
    opt = engine.LmOptions(max_iterations=max_it, jacobian=engine.JACOBIAN_ADJOINT,
                           gram_exact=False)
    flush = torch.empty(256 * 1024 * 1024, dtype=torch.uint8, device=dev)
    stream = torch.cuda.current_stream()
    rays = lay_fma.rays_per_variant
    sv = b.variant_surfaces.astype(np.int64)
    hits = int(rays * (sv - 1).sum())

    # ---- headline: adjoint (FP64 trace, FP32 reverse sweep) fused with the normal equations
    lm = engine.DeviceLm(db, lay_mixed, b, vss, opt, runs)
    lm.start(x0)
    with ClockSampler(local) as clocks:
        ms_cycle, iters, per_cycle = _lm_window(lm, args.steps, args.warmup, flush, world, dev)
    ms_step = max_over_ranks(ms_cycle, world, dev)
    value = world * iters / (ms_step * args.steps / 1e3)
    x_now = np.zeros((runs, P))
    res = lm.results()
    x_now = res["x"]
    del lm

    # ---- the same with the FP64-FMA adjoint
    lm_f = engine.DeviceLm(db, lay_fma, b, vss, opt, runs)
    lm_f.start(x0)
    ms_fma, iters_fma, _ = _lm_window(lm_f, args.steps, args.warmup, flush, world, dev)
    fma_value = world * iters_fma / (max_over_ranks(ms_fma, world, dev) * args.steps / 1e3)
    del lm_f

    # ---- the same with the FP32-bulk forward (directions and refraction in FP32; positions,
    # intersection and optical path in FP64) and the FP32 reverse sweep
    # (built for batches without ghost plates: measured then, else reported as not run)
    from mikroptim_b200.batch import PRECISION_FP32_BULK
    bulk_value = ms_bulk = None
    if b.topology.ghost_plates == 0:
        lay_bulk = ResidualLayout(b.topology,
                                  dataclasses.replace(st, precision=PRECISION_FP32_BULK))
        lm_b = engine.DeviceLm(db, lay_bulk, b, vss, opt, runs)
        lm_b.start(x0)
        ms_bulk, iters_bulk, _ = _lm_window(lm_b, args.steps, args.warmup, flush, world, dev)
        bulk_value = world * iters_bulk / (max_over_ranks(ms_bulk, world, dev) * args.steps / 1e3)
        del lm_b

    # ---- the same LM with paraxial constraints on the device (image at the paraxial focus,
    # working distance >= 1 mm, |Petzval curvature| <= 0.02 / mm; analytic adjoint rows): the
    # constrained cycle stays one graph-captured launch sequence
    cons = engine.ParaxialConstraints.of([(3, 0, 1.0, 0.0), (2, 1, 1.0, 1.0), (4, 2, 100.0, 0.02)],
                                         derivative="adjoint")
    opt_c = dataclasses.replace(opt, paraxial=cons)
    lm_c = engine.DeviceLm(db, lay_mixed, b, vss, opt_c, runs)
    lm_c.start(x0)
    ms_con, iters_con, per_cycle_con = _lm_window(lm_c, args.steps, args.warmup, flush, world,
                                                  dev)
    con_value = world * iters_con / (max_over_ranks(ms_con, world, dev) * args.steps / 1e3)
    del lm_c

    # ---- the reference method on the same GPU: FD Jacobian (2P + 1 traced variants), FP64
    fd_runs = min(1024, runs)
    fd_b = b.subset(0, fd_runs)
    fd_db = engine.DeviceSystemBatch(fd_b, dev)
    fd_opt = engine.LmOptions(max_iterations=max_it, jacobian=engine.JACOBIAN_FD,
                              gram_exact=False)
    fd = engine.DeviceLm(fd_db, lay_fma, fd_b, vss[:fd_runs], fd_opt, fd_runs)
    fd.start(x0[:fd_runs])
    fd_steps = max(2, min(args.steps, 10))
    fd_ms, fd_iters, _ = _lm_window(fd, fd_steps, args.warmup, flush, world, dev)
    fd_value = fd_iters / (fd_ms * fd_steps / 1e3)
    del fd

    # ---- the dominant kernel alone: fused adjoint + normal equations of every run
    # FLOP model per run (reference cost model): 3 x 140 (S_v - 1 + 2) per ray + 4 P per ray +
    # 2 P^2 per row (rays and penalty rows)
    pv = np.array([v.size for v in vss], dtype=np.float64)
    flop = float(np.sum(rays * (3 * FLOPEQ_PER_RAY_SURFACE * (sv - 1 + 2) + 4 * pv) +
                        2 * pv * pv * lay_mixed.trace_rows))
    # the call's host part (variable table, run order) is enqueued while the previous call
    # runs: the first call is outside the events, so the events see the GPU work only
    rvars = engine.RunVariables(vss)
    x_dev = torch.from_numpy(np.ascontiguousarray(x_now)).to(dev)
    ws_k = None
    gram_k = engine.adjoint_normal_equations_runs_device(db, lay_mixed, b, rvars, x_dev)
    torch.cuda.synchronize()
    reps = 3
    engine.adjoint_normal_equations_runs_device(db, lay_mixed, b, rvars, x_dev)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(reps):
        flush.zero_()  # L2 flushed between the timed calls; its own time is taken out below
        engine.adjoint_normal_equations_runs_device(db, lay_mixed, b, rvars, x_dev)
    e1.record(stream)
    torch.cuda.synchronize()
    f0, f1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    f0.record(stream)
    for _ in range(reps):
        flush.zero_()
    f1.record(stream)
    torch.cuda.synchronize()
    kernel_ms = (e0.elapsed_time(e1) - f0.elapsed_time(f1)) / reps
    del gram_k, ws_k

    # ---- MERIT rate (ray-surface hits/s) on the uneven batch
    engine.merit_device(db, lay_fma, b)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(3):
        engine.merit_device(db, lay_fma, b)
    e1.record(stream)
    torch.cuda.synchronize()
    merit_ms = e0.elapsed_time(e1) / 3

    # ---- end to end through the drop-in API: optimize_lm_gpu(host batch, variables, x0) ->
    # host results, the full 100-iteration LM with its penalty rounds, convergence included
    e2e = e2e_optimize(b, lay_mixed, vss, x0, world, dev)

    errors = opd_errors(b, st, runs=256) if rank == 0 else None
    accuracy = mixed_accuracy(b, st, vss, x0, runs=256) if rank == 0 else None
    peak = fp64_peak_tflops(torch) if rank == 0 else None
    achieved = flop / (kernel_ms / 1e3) / 1e12
    if rank != 0:
        return None, None
    return {
        "metric": METRIC,
        "value": value,
        "unit": "LM iterations/s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": ms_step,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f64+f32-adjoint",
        "data": "synthetic (seeded generator, configuration-3 shapes)",
        "config": {"workload": WORKLOAD_UNEVEN,
                   "step": "one batched LM cycle of all runs in one launch per kernel "
                           "(CUDA graph), runs ordered by surface count",
                   "runs_per_gpu": runs, "variables_max": P, "rays_per_run": rays,
                   "jacobian": "adjoint fused with FP64 tensor-core normal equations",
                   "precision": "MIXED: FP64 trace and OPD, FP32 adjoint reverse sweep",
                   "iterations": "LM iterations actually taken in the timed cycles "
                                 f"({iters} of {runs * args.steps} run-cycles)",
                   "l2": "flushed (256 MB write) before every timed step"},
        "gpu_launches": int(per_cycle * args.steps),
        "ray_surface_hits_per_s": world * hits / (merit_ms / 1e3),
        "adjoint_fp64_fma": {"value": fma_value, "unit": "LM iterations/s",
                             "ms_per_cycle": ms_fma},
        "adjoint_fp32_bulk": {"value": bulk_value, "unit": "LM iterations/s",
                              "ms_per_cycle": ms_bulk,
                              "precision": "FP32_BULK: forward with FP32 directions and "
                                           "refraction (FP64 positions, intersection, optical "
                                           "path), FP32 reverse sweep; its OPD error in "
                                           "opd_error_vs_fp64.fp32_bulk; not run (null) on "
                                           "batches with ghost plates, which it does not trace"},
        "adjoint_mixed_paraxial_constraints": {
            "value": con_value, "unit": "LM iterations/s", "ms_per_cycle": ms_con,
            "launches_per_cycle": int(per_cycle_con),
            "constraints": "paraxial focus (equal), working distance >= 1 mm, |Petzval| <= "
                           "0.02/mm; rows and analytic adjoint Jacobian on the device, "
                           "graph-captured cycle"},
        "fd_fp64": {"value": world * fd_value, "unit": "LM iterations/s",
                    "ms_per_cycle_1024_runs": fd_ms, "cycles": fd_steps,
                    "speedup_adjoint_mixed_vs_fd": value / (world * fd_value),
                    "speedup_adjoint_fma_vs_fd": fma_value / (world * fd_value)},
        "opd_error_vs_fp64": errors,
        "e2e": e2e,
        "mixed_accuracy": accuracy,
        "roofline": {"bound": "fp64", "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
                     "frac": achieved / peak if peak else None,
                     "traffic": FUSED_TRAFFIC_UNEVEN_BYTES_PER_RUN * runs,
                     "traffic_source": "scaled capture",
                     "kernel": "adjoint_gram_kernel<MixedPrecision> (fused adjoint + DMMA "
                               "normal equations, every run, with its apply kernel)",
                     "kernel_ms": kernel_ms,
                     "peak_source": "cuBLAS DGEMM 8192^3 measured in this run",
                     "flop_model": "3 x 140 (S_v-1+2) FLOP-eq per ray + 4P per ray + 2P^2 "
                                   "per row, summed over the runs"},
        "clocks": clocks.summary(),
    }, None


def run_singlet(args, world, rank, local):
    """Configuration 1: FP64 RESIDUALS + MERIT of 1,024 singlets. One evaluation is ~0.3
    GFLOP-eq (microseconds of GPU work), so a step is one CUDA-graph replay of many
    back-to-back evaluations (each: RESIDUALS with OPD and status, then MERIT), with the L2
    flushed between steps; beside it the same rate over a sweep of batch sizes."""
    import torch
    from mikroptim_b200 import _capi, engine, workloads
    from mikroptim_b200.batch import PRECISION_FP64, PRECISION_FP64_FMA, ResidualLayout

    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    lib = _capi.lib()
    flush = torch.empty(256 * 1024 * 1024, dtype=torch.uint8, device=dev)
    stream = torch.cuda.current_stream()

    def graph_of(V, precision, evals, seed, tplans=None):
        """A CUDA graph of `evals` evaluations of V singlets (outputs preallocated), RESIDUALS
        and MERIT launched with the trace plans `tplans` = (residuals plan, merit plan), each
        (pack_rays, variants_per_cta); None: the defaults."""
        b, st, vs, x0 = workloads.singlet(V, seed=seed)
        st.precision = precision
        lay = ResidualLayout(b.topology, st)
        db = engine.DeviceSystemBatch(b, dev)
        rows, rays = lay.trace_rows, lay.rays_per_variant
        res = torch.empty((V, rows), dtype=torch.float64, device=dev)
        opd = torch.empty((V, rays), dtype=torch.float64, device=dev)
        stat = torch.empty((V, rays), dtype=torch.uint8, device=dev)
        merit = torch.empty(V, dtype=torch.float64, device=dev)
        failed = torch.empty(V, dtype=torch.int64, device=dev)
        hard = torch.empty(V, dtype=torch.int64, device=dev)
        plan = lay.plan(b)
        ws = torch.empty(int(lib.mkb_merit_workspace_bytes(V, C.byref(plan))), dtype=torch.uint8,
                         device=dev)
        bst = db.c_struct()
        opts_r, opts_m = [engine._trace_options(0) if tplans is None else engine._trace_options(
            tp.pack_rays, variants_per_cta=tp.variants_per_cta) for tp in (tplans or (0, 0))]

        def one():
            h = C.c_void_p(torch.cuda.current_stream().cuda_stream)
            _capi.check(lib.mkb_residuals_ex_device(
                C.byref(bst), C.byref(plan), C.byref(opts_r), C.c_void_p(res.data_ptr()), rows,
                C.c_void_p(opd.data_ptr()), C.c_void_p(stat.data_ptr()), h), "residuals")
            _capi.check(lib.mkb_merit_ex_device(
                C.byref(bst), C.byref(plan), C.byref(opts_m), C.c_void_p(merit.data_ptr()),
                C.c_void_p(failed.data_ptr()), C.c_void_p(hard.data_ptr()),
                C.c_void_p(ws.data_ptr()), ws.numel(), h), "merit")

        for _ in range(2):
            one()
        torch.cuda.synchronize()
        g = torch.cuda.CUDAGraph()
        l0 = lib.mkb_launch_count()
        with torch.cuda.graph(g):
            for _ in range(evals):
                one()
        per_graph = lib.mkb_launch_count() - l0
        torch.cuda.synchronize()
        keep = (b, lay, db, res, opd, stat, merit, failed, hard, ws, plan, bst, opts_r, opts_m)
        hits = 2 * V * rays * (b.surfaces - 1) * evals  # RESIDUALS and MERIT trace each ray
        flopeq = 2 * V * rays * FLOPEQ_PER_RAY_SURFACE * (b.surfaces - 1 + 2) * evals
        return g, per_graph, hits, flopeq, keep

    def time_graph(g, steps, warmup):
        for _ in range(warmup):
            g.replay()
        torch.cuda.synchronize()
        times = []
        for _ in range(steps):
            flush.zero_()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            g.replay()
            e1.record(stream)
            times.append((e0, e1))
        torch.cuda.synchronize()
        return sum(a.elapsed_time(c) for a, c in times) / steps

    V = args.variants or 1024
    evals = max(1, 102400 // V)
    seed = 20261203 + 1 + 1000 * rank
    # the autotuner picks the launch shape of each trace (rays per CTA pack and variants per
    # CTA) for this batch shape, outside the timed region; every plan gives the same bits
    from mikroptim_b200 import autotune
    tuner = autotune.TraceAutotuner(launches=20)
    b0, st0, _, _ = workloads.singlet(V, seed=seed)
    st0.precision = PRECISION_FP64
    lay0 = ResidualLayout(b0.topology, st0)
    tuned = {m: tuner.tune(b0, lay0, m) for m in ("residuals", "merit")}
    plan_r = autotune.TracePlan(tuned["residuals"]["pack_rays"],
                                tuned["residuals"]["variants_per_cta"])
    plan_m = autotune.TracePlan(tuned["merit"]["pack_rays"], tuned["merit"]["variants_per_cta"])
    g, per_graph, hits, flopeq, keep = graph_of(V, PRECISION_FP64, evals, seed,
                                                (plan_r, plan_m))
    barrier(world)
    with ClockSampler(local) as clocks:
        ms_step = time_graph(g, args.steps, args.warmup)
    ms_step = max_over_ranks(ms_step, world, dev)
    value = world * hits / (ms_step / 1e3)
    b = keep[0]
    lay = keep[1]
    del g, keep

    # FP64 with contraction on the same batches, and the size sweep (both precisions)
    sweep = []
    fma_value = None
    for n in (1024, 8192, 65536, 262144):
        ev = max(1, 102400 // n)
        row = {"variants": n, "evaluations_per_replay": ev}
        for name, prec in (("fp64", PRECISION_FP64), ("fp64_fma", PRECISION_FP64_FMA)):
            bn, stn, _, _ = workloads.singlet(n, seed=seed)
            stn.precision = prec
            layn = ResidualLayout(bn.topology, stn)
            sweep_tuner = autotune.TraceAutotuner(launches=max(2, 20480 // n))
            tp = [sweep_tuner.tune(bn, layn, m) for m in ("residuals", "merit")]
            tps = tuple(autotune.TracePlan(t["pack_rays"], t["variants_per_cta"]) for t in tp)
            row[name] = {}
            for label, plans in (("default", None), ("tuned", tps)):
                gg, _, hh, ff, kk = graph_of(n, prec, ev, seed, plans)
                ms = time_graph(gg, 3, 2)
                row[name][label] = {"ray_surface_hits_per_s": hh / (ms / 1e3),
                                    "tflopeq_per_s": ff / (ms / 1e3) / 1e12,
                                    "ms_per_replay": ms}
                if n == V and prec == PRECISION_FP64_FMA and label == "tuned":
                    fma_value = world * hh / (ms / 1e3)
                del gg, kk
                torch.cuda.empty_cache()
            row[name]["plans"] = {"residuals": [tps[0].pack_rays, tps[0].variants_per_cta],
                                  "merit": [tps[1].pack_rays, tps[1].variants_per_cta]}
        sweep.append(row)

    # end to end through the public API: host batch in, host residuals / OPD / status and merit
    # out, tranche planning included (TraceEngine.run RESIDUALS then MERIT)
    eng = engine.TraceEngine(local)
    ts = engine.TraceSettings(lay.settings, opd=True)
    out_r, out_m = engine.TraceOutput(), engine.TraceOutput()  # reused, as a caller's loop does
    for _ in range(2):
        eng.run(b, engine.TraceMode.RESIDUALS, ts, out_r)
        eng.run(b, engine.TraceMode.MERIT, ts, out_m)
    torch.cuda.synchronize()
    barrier(world)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        eng.run(b, engine.TraceMode.RESIDUALS, ts, out_r)
        eng.run(b, engine.TraceMode.MERIT, ts, out_m)
    e1.record(stream)
    torch.cuda.synchronize()
    e2e_ms = max_over_ranks(e0.elapsed_time(e1) / args.steps, world, dev)
    rays = lay.rays_per_variant
    stride = int(lib.mkb_record_stride(3, 3, 3))

    peak = fp64_peak_tflops(torch) if rank == 0 else None
    achieved = flopeq / (ms_step / 1e3) / 1e12
    if rank != 0:
        return None, None
    return {
        "metric": METRIC,
        "value": value,
        "unit": "ray-surface hits/s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": ms_step,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f64",
        "data": "synthetic (seeded generator, configuration-1 shapes)",
        "config": {"workload": WORKLOAD_SINGLET,
                   "step": f"one CUDA-graph replay of {evals} back-to-back evaluations, each "
                           "RESIDUALS (with OPD and status) then MERIT of every variant",
                   "precision": "FP64, every operation separately rounded (bit-identical to "
                                "the reference CPU)",
                   "variants_per_gpu": V, "rays_per_variant": rays,
                   "l2": "flushed (256 MB write) before every timed step"},
        "gpu_launches": int(per_graph * args.steps),
        "fp64_fma": {"value": fma_value, "unit": "ray-surface hits/s"},
        "autotuned": {m: {"pack_rays": tuned[m]["pack_rays"],
                          "variants_per_cta": tuned[m]["variants_per_cta"],
                          "ms_per_launch": tuned[m]["ms"],
                          "default_ms_per_launch": next(t[2] for t in tuned[m]["timings"]
                                                        if t[0] == 512 and t[1] == 1)}
                      for m in tuned},
        "size_sweep": sweep,
        "e2e": {"value": world * (hits / evals) / (e2e_ms / 1e3), "unit": "ray-surface hits/s",
                "h2d_bytes_per_step": int(2 * V * stride * 8),
                "d2h_bytes_per_step": int(V * (lay.trace_rows * 8 + rays * 9) + V * 24),
                "path": "TraceEngine.run(RESIDUALS, opd=True) + TraceEngine.run(MERIT) from a "
                        "host SystemBatchHost, one evaluation per step"},
        "roofline": {"bound": "fp64", "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
                     "frac": achieved / peak if peak else None, "traffic": None,
                     "kernel": "trace_kernel<1, 0, 0> + trace_kernel<0, 0, 0> + "
                               "merit_finalize_kernel (graph replay)",
                     "peak_source": "cuBLAS DGEMM 8192^3 measured in this run",
                     "flop_model": "2 traces x 140 (S-1+2) FLOP-eq per ray"},
        "clocks": clocks.summary(),
    }, None


def cpu_baseline_singlet(variants: int = 1024, seed: int = 20261203 + 1, window: float = 2.0):
    """The reference's own residuals_cpu + merit_cpu (oracle/_ref, or the C restatement when
    the reference build is missing) over all host threads, repeated for about `window` s."""
    import oracle.pyoracle as po
    from mikroptim_b200 import workloads
    from mikroptim_b200.batch import ResidualLayout
    b, st, vs, x0 = workloads.singlet(variants, seed=seed)
    lay = ResidualLayout(b.topology, st)
    kind = reference_kind()
    impl = po.reference() if kind == "reference" else po.port()
    threads = os.cpu_count() or 1
    impl.residuals(b, lay, threads=threads)
    impl.merit(b, lay, threads=threads)
    reps, t0 = 0, time.perf_counter()
    while time.perf_counter() - t0 < window:
        impl.residuals(b, lay, threads=threads)
        impl.merit(b, lay, threads=threads)
        reps += 1
    dt = time.perf_counter() - t0
    hits = 2 * b.variants * lay.rays_per_variant * (b.surfaces - 1) * reps
    return {"value": hits / dt, "unit": "ray-surface hits/s", "cores": threads, "kind": kind,
            "sample": f"residuals_cpu + merit_cpu of the {variants} singlets, {reps} times, "
                      f"{dt:.2f} s"}


# ---- CPU baselines (oracle) ----------------------------------------------------------------
def cpu_baseline(kind: str, sample_variants: int = 16, seed: int = 20261203 + 2):
    """The reference's own CPU merit (oracle/_ref) or the C restatement, on all host threads,
    on the first `sample_variants` variants of the same workload."""
    import oracle.pyoracle as po
    from mikroptim_b200 import workloads
    from mikroptim_b200.batch import ResidualLayout
    b, st, vs, x0 = workloads.objective(4096, seed=seed)
    b = b.subset(0, sample_variants)
    lay = ResidualLayout(b.topology, st)
    impl = po.reference() if kind == "reference" else po.port()
    threads = os.cpu_count() or 1
    impl.merit(b, lay, threads=threads)
    t0 = time.perf_counter()
    impl.merit(b, lay, threads=threads)
    dt = time.perf_counter() - t0
    hits = b.variants * lay.rays_per_variant * (b.surfaces - 1)
    return {"value": hits / dt, "unit": "ray-surface hits/s", "cores": threads, "kind": kind,
            "sample": f"MERIT of {sample_variants} of the 4096 variants, {dt:.2f} s"}


def cpu_baseline_lm(kind: str, runs: int = 256, seed: int = 20261203 + 2):
    """LM cycles (adjoint Jacobian, normal equations, step, trial merit) of `runs` runs of the
    same workload on all host threads: the reference's own optimize_lm_cpu (oracle/_ref).
    Three cycles minus one cycle, halved, isolates the cost of a cycle from the start-up."""
    import oracle.pyoracle as po
    from mikroptim_b200 import workloads
    from mikroptim_b200.batch import ResidualLayout
    b, st, vs, x0 = workloads.objective(4096, seed=seed, glass=True)
    b = b.subset(0, runs)
    lay = ResidualLayout(b.topology, st)
    threads = os.cpu_count() or 1
    ref = po.reference()
    t0 = time.perf_counter()
    ref.optimize_lm(b, lay, vs, x0[:runs], max_iterations=1, method="adjoint", threads=threads)
    t1 = time.perf_counter()
    ref.optimize_lm(b, lay, vs, x0[:runs], max_iterations=3, method="adjoint", threads=threads)
    t2 = time.perf_counter()
    per_cycle = max(((t2 - t1) - (t1 - t0)) / 2, 1e-9)
    return {"value": runs / per_cycle, "unit": "LM run-iterations/s", "cores": threads,
            "kind": kind, "sample": f"optimize_lm_cpu (adjoint) of {runs} of the 4096 runs, "
                                     f"1 and 3 cycles, {t2 - t0:.1f} s"}


def uneven_reference_sampler(runs: int = 96, seed: int = 20261203 + 3):
    """The reference's optimize_lm_cpu on a sample of the uneven runs: the reference needs one
    topology and one variable set per call, so every run is its own call (its baseline loops
    over topology groups), the calls spread over all host threads. Returns (sample, threads):
    sample() times one step -- 1 then 3 cycles of every run; three cycles minus one, halved,
    isolates the cost of a cycle from the start-up -- and returns (LM iterations/s, seconds)."""
    import concurrent.futures as cf
    import oracle.pyoracle as po
    from mikroptim_b200 import workloads
    from mikroptim_b200.batch import ResidualLayout
    b, st, vss, x0 = workloads.uneven(runs, seed=seed)
    ref = po.reference()
    threads = os.cpu_count() or 1
    jobs = []
    for v in range(runs):
        one = workloads.unpad(b, v)
        lone = ResidualLayout(one.topology, st)
        vs = type(vss[v])(one.topology, [
            type(var)(2 if (var.type == 1 and var.surface == one.surfaces - 1) else var.type,
                      var.surface, var.lower, var.upper, var.typical)
            for var in vss[v].variables])
        jobs.append((one, lone, vs, x0[v][None, :]))

    def run_all(max_it):
        with cf.ThreadPoolExecutor(max_workers=threads) as ex:
            list(ex.map(lambda j: ref.optimize_lm(*j, max_iterations=max_it, method="adjoint",
                                                  threads=1), jobs))

    def sample():
        t0 = time.perf_counter()
        run_all(1)
        t1 = time.perf_counter()
        run_all(3)
        t2 = time.perf_counter()
        per_cycle = max(((t2 - t1) - (t1 - t0)) / 2, 1e-9)
        return runs / per_cycle, t2 - t0
    return sample, threads


def cpu_baseline_uneven(runs: int = 96, seed: int = 20261203 + 3):
    """One sample of uneven_reference_sampler, as the cpu_baseline of the GPU line."""
    sample, threads = uneven_reference_sampler(runs, seed)
    v, sec = sample()
    return {"value": v, "unit": "LM iterations/s", "cores": threads, "kind": "reference",
            "sample": f"optimize_lm_cpu (adjoint), {runs} of the uneven runs one per call, "
                      f"1 and 3 cycles, {sec:.1f} s"}


def reference_kind() -> str:
    import oracle.pyoracle as po
    return "reference" if os.path.exists(po.REF_LIB) else "port"


def repeated_samples(fn, warmup: int, steps: int):
    """W untimed and K timed calls of a bounded CPU sample fn() -> dict with "value"; returns
    (median of the K values, the last dict)."""
    vals, last = [], None
    for i in range(warmup + steps):
        last = fn()
        if i >= warmup:
            vals.append(last["value"])
    return statistics.median(vals), last


def run_reference(args, world, rank):
    if rank != 0:
        return None
    kind = reference_kind()
    if args.workload == "uneven":
        if kind != "reference":
            return {"impl": "reference", "unavailable": "reference CPU build (oracle/_ref) missing"}
        # W warm-up and K timed steps, each a bounded sample (96 runs; fewer when K + W > 30,
        # so the whole run stays within a few minutes); the value is the median of the K
        n_steps = args.warmup + args.steps
        runs = 96 if n_steps <= 30 else max(24, 96 * 30 // n_steps)
        sample, threads = uneven_reference_sampler(runs)
        rates, total = [], 0.0
        for i in range(n_steps):
            r, sec = sample()
            total += sec
            if i >= args.warmup:
                rates.append(r)
        v = statistics.median(rates)
        return {
            "metric": METRIC, "value": v, "unit": "LM iterations/s", "impl": "reference",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded generator, configuration-3 shapes)",
            "config": {"workload": WORKLOAD_UNEVEN,
                       "step": f"LM cycles of a {runs}-run sample on the host (1 and 3 cycles of "
                               f"every run; the median of the timed steps)"},
            "cpu_baseline": {"value": v, "unit": "LM iterations/s", "cores": threads,
                             "kind": kind,
                             "sample": f"optimize_lm_cpu (adjoint), {runs} of the uneven runs "
                                       f"one per call, {n_steps} steps, {total:.1f} s"},
            "e2e": {"value": v, "unit": "LM iterations/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0},
        }
    if args.workload == "lm":
        if kind != "reference":
            return {"impl": "reference", "unavailable": "reference CPU build (oracle/_ref) missing"}
        n_steps = args.warmup + args.steps  # bounded: fewer runs per step for long runs
        runs = 128 if n_steps <= 30 else max(32, 128 * 30 // n_steps)
        v, base = repeated_samples(lambda: cpu_baseline_lm(kind, runs=runs), args.warmup,
                                   args.steps)
        return {
            "metric": METRIC, "value": v, "unit": "LM run-iterations/s", "impl": "reference",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded generator, configuration-2 shapes)",
            "config": {"workload": WORKLOAD_LM,
                       "step": f"LM cycles of a {runs}-run sample on the host (the median of "
                               f"the timed steps)"},
            "cpu_baseline": {"value": v, "unit": "LM run-iterations/s", "cores": base["cores"],
                             "kind": kind, "sample": base["sample"]},
            "e2e": {"value": v, "unit": "LM run-iterations/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0},
        }
    if args.workload == "singlet":
        n_steps = args.warmup + args.steps
        window = 2.0 if n_steps <= 30 else 2.0 * 30 / n_steps
        v, base = repeated_samples(lambda: cpu_baseline_singlet(window=window), args.warmup,
                                   args.steps)
        return {
            "metric": METRIC, "value": v, "unit": "ray-surface hits/s", "impl": "reference",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded generator, configuration-1 shapes)",
            "config": {"workload": WORKLOAD_SINGLET,
                       "step": "residuals_cpu + merit_cpu of the 1024 singlets on the host"},
            "cpu_baseline": {"value": v, "unit": "ray-surface hits/s", "cores": base["cores"],
                             "kind": base["kind"], "sample": base["sample"]},
            "e2e": {"value": v, "unit": "ray-surface hits/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0},
        }
    samples = []
    for i in range(args.warmup + args.steps):
        r = cpu_baseline(kind, sample_variants=8)
        if i >= args.warmup:
            samples.append(r["value"])
    v = statistics.median(samples)
    base = cpu_baseline(kind, sample_variants=8)
    return {
        "metric": METRIC, "value": v, "unit": "ray-surface hits/s", "impl": "reference",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded generator, configuration-2 shapes)",
        "config": {"workload": WORKLOAD, "step": "MERIT of an 8-variant sample on the host"},
        "cpu_baseline": {"value": v, "unit": "ray-surface hits/s", "cores": base["cores"],
                         "kind": kind, "sample": base["sample"]},
        "e2e": {"value": v, "unit": "ray-surface hits/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }


WORKLOAD_TOL = ("tolerancing-{V}: {V} Monte-Carlo perturbations of one 10-element (20-sphere) "
                "objective, decenter 5 um, tilt 1', dR/R 0.1 %, dt 10 um, dn 2e-4 per glass, "
                "non-coaxial, L=7, F=5, Full 16x32 pupils, P=40 design variables (config 5 shape)")


def run_tolerancing(args, world, rank, local):
    """Configuration 5: per step, the MERIT of every perturbed variant (FP64 with FMA) and its
    gradient with respect to the design variables, 2 J^T r, from the fused adjoint normal
    equations (column P of [J r]^T [J r]; the Gauss-Newton block J^T J comes with it). The
    gradient's reverse sweep runs in MIXED precision (FP64 trace, FP32 sweep); its error
    against the FP64_FMA gradient is reported, and the FP64_FMA gradient is timed beside."""
    import torch
    from mikroptim_b200 import _capi, engine, workloads
    from mikroptim_b200.batch import PRECISION_FP64_FMA, PRECISION_MIXED, ResidualLayout

    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    lib = _capi.lib()
    V = args.variants or 262144
    b, st, vs, x0 = workloads.tolerancing(V, seed=20261203 + 5 + 1000 * rank)
    st.precision = PRECISION_FP64_FMA
    lay = ResidualLayout(b.topology, st)
    lay_mixed = ResidualLayout(b.topology, dataclasses.replace(st, precision=PRECISION_MIXED))
    db = engine.DeviceSystemBatch(b, dev)
    P = vs.size
    cb = db.c_struct()
    plans = {0: lay.plan(b), 1: lay_mixed.plan(b)}
    cvars = vs.c_struct()
    x = torch.from_numpy(np.ascontiguousarray(x0)).to(dev)
    gram = torch.empty((V, P + 1, P + 1), dtype=torch.float64, device=dev)
    ws_g = torch.empty(int(lib.mkb_adjoint_jacobian_workspace_bytes(C.byref(cb), V)),
                       dtype=torch.uint8, device=dev)
    ws_m = torch.empty(int(lib.mkb_merit_workspace_bytes(V, C.byref(plans[0]))),
                       dtype=torch.uint8, device=dev)
    merit = torch.empty(V, dtype=torch.float64, device=dev)
    failed = torch.empty(V, dtype=torch.int64, device=dev)
    hard = torch.empty(V, dtype=torch.int64, device=dev)
    flush = torch.empty(256 * 1024 * 1024, dtype=torch.uint8, device=dev)
    stream = torch.cuda.current_stream()
    sh = C.c_void_p(stream.cuda_stream)

    def merit_call():
        _capi.check(lib.mkb_merit_device(C.byref(cb), C.byref(plans[0]),
                                         C.c_void_p(merit.data_ptr()),
                                         C.c_void_p(failed.data_ptr()),
                                         C.c_void_p(hard.data_ptr()),
                                         C.c_void_p(ws_m.data_ptr()), ws_m.numel(), sh), "merit")

    def gram_call(which):
        _capi.check(lib.mkb_adjoint_normal_equations_device(
            C.byref(cb), C.byref(plans[which]), C.byref(cvars), C.c_void_p(x.data_ptr()), V,
            C.c_void_p(gram.data_ptr()), C.c_void_p(ws_g.data_ptr()), ws_g.numel(), sh),
            "adjoint normal equations")

    def timed(fn, steps):
        ts = []
        for _ in range(steps):
            flush.zero_()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            fn()
            e1.record(stream)
            ts.append((e0, e1))
        torch.cuda.synchronize()
        return sum(a.elapsed_time(c) for a, c in ts) / steps

    def step():
        merit_call()
        gram_call(1)

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    barrier(world)
    l0 = lib.mkb_launch_count()
    with ClockSampler(local) as clocks:
        ms_step = timed(step, args.steps)
    launches = lib.mkb_launch_count() - l0
    barrier(world)
    ms_step = max_over_ranks(ms_step, world, dev)
    ms_merit = timed(merit_call, 2)
    ms_gram_fma = timed(lambda: gram_call(0), 2)
    g_fma = gram[:, :P, P].clone()
    ms_gram = timed(lambda: gram_call(1), 2)
    torch.cuda.synchronize()
    g_mixed = gram[:, :P, P]
    # MIXED gradient error against the FMA one (relative to |g| per sample)
    rel = (torch.linalg.vector_norm(g_mixed - g_fma, dim=1) /
           torch.clamp(torch.linalg.vector_norm(g_fma, dim=1), min=1e-300)).cpu().numpy()

    # end to end: host x in (pinned), merit and gradient out, every step
    x_host = torch.from_numpy(np.ascontiguousarray(x0)).pin_memory()
    out_merit = torch.empty(V, dtype=torch.float64).pin_memory()
    out_grad = torch.empty((V, P), dtype=torch.float64).pin_memory()

    def e2e_step():
        x.copy_(x_host, non_blocking=True)
        step()
        out_merit.copy_(merit, non_blocking=True)
        out_grad.copy_(gram[:, :P, P], non_blocking=True)

    e2e_step()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        e2e_step()
    e1.record(stream)
    torch.cuda.synchronize()
    e2e_ms = max_over_ranks(e0.elapsed_time(e1) / args.steps, world, dev)

    rays = V * lay.rays_per_variant
    S = b.surfaces
    flop = rays * (3 * FLOPEQ_PER_RAY_SURFACE * (S - 1 + 2) + 4 * P) + 2.0 * (P + 1) ** 2 * \
        V * lay.trace_rows
    peak = fp64_peak_tflops(torch) if rank == 0 else None
    achieved = flop / (ms_gram / 1e3) / 1e12
    if rank != 0:
        return None, None
    return {
        "metric": "MC tolerancing samples/s (MERIT + design-variable gradient)",
        "value": world * V / (ms_step / 1e3),
        "unit": "samples/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_step,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64+f32-adjoint",
        "data": "synthetic (seeded generator, configuration-5 shapes)",
        "config": {"workload": WORKLOAD_TOL.format(V=V),
                   "step": "MERIT (FP64, FMA) + fused adjoint normal equations (MIXED: FP64 "
                           "trace, FP32 reverse sweep) of every sample; the gradient is 2 x "
                           "column P",
                   "samples_per_gpu": V, "rays_per_sample": lay.rays_per_variant,
                   "l2": "flushed (256 MB write) before every timed step"},
        "gpu_launches": int(launches),
        "ray_surface_hits_per_s": world * rays * (S - 1) / (ms_merit / 1e3),
        "ms_merit": ms_merit, "ms_gradient_mixed": ms_gram, "ms_gradient_fp64_fma": ms_gram_fma,
        "fp64_fma_gradient": {"value": world * V / ((ms_merit + ms_gram_fma) / 1e3),
                              "unit": "samples/s"},
        "mixed_gradient_rel_error_vs_fp64_fma": {"median": float(np.median(rel)),
                                                 "p99": float(np.percentile(rel, 99))},
        "e2e": {"value": world * V / (e2e_ms / 1e3), "unit": "samples/s",
                "h2d_bytes_per_step": int(V * P * 8),
                "d2h_bytes_per_step": int(V * (P + 1) * 8)},
        "roofline": {"bound": "fp64", "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
                     "frac": achieved / peak if peak else None, "traffic": None,
                     "kernel": "adjoint_gram_kernel<MixedPrecision> (fused adjoint + DMMA "
                               "normal equations) with its apply kernel",
                     "kernel_ms": ms_gram,
                     "peak_source": "cuBLAS DGEMM 8192^3 measured in this run"},
        "clocks": clocks.summary(),
    }, (b, lay)


WORKLOAD_PREC = ("precision-{V}: {V} systems x 20 surfaces (9 configuration-1 style elements + "
                 "a zero-power plate), L=9 (405..700 nm), F=5, Half 32x32 pupils (1,024 rays per "
                 "field and wavelength; config 4 shape)")


def run_precision(args, world, rank, local):
    """Configuration 4: MERIT of every system in FP64 (bit-identical to the reference CPU),
    FP64_FMA and MIXED, timed; OPD of every ray in all three, in tranches, and the FMA / MIXED
    OPD error against the FP64 trace (waves at the reference wavelength, over rays whose status
    agrees and lies in the piston); the normal-equation error of the fused MIXED and FMA
    adjoint against the exact materialised one on a sample."""
    import torch
    from mikroptim_b200 import _capi, engine, workloads
    from mikroptim_b200.batch import (PRECISION_FP64, PRECISION_FP64_FMA, PRECISION_MIXED,
                                      ResidualLayout, in_piston)

    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    lib = _capi.lib()
    V = args.variants or 65536
    b, st, vs, x0 = workloads.sweep(V, seed=20261203 + 4 + 1000 * rank)
    lays = {p: ResidualLayout(b.topology, dataclasses.replace(st, precision=p))
            for p in (PRECISION_FP64, PRECISION_FP64_FMA, PRECISION_MIXED)}
    db = engine.DeviceSystemBatch(b, dev)
    lay0 = lays[PRECISION_FP64]
    ws = torch.empty(int(lib.mkb_merit_workspace_bytes(V, C.byref(lay0.plan(b)))),
                     dtype=torch.uint8, device=dev)
    flush = torch.empty(256 * 1024 * 1024, dtype=torch.uint8, device=dev)
    stream = torch.cuda.current_stream()
    rays = V * lay0.rays_per_variant
    hits = rays * (b.surfaces - 1)

    def merit_ms(p, steps):
        for _ in range(args.warmup):
            engine.merit_device(db, lays[p], b, workspace=ws)
        torch.cuda.synchronize()
        ts = []
        for _ in range(steps):
            flush.zero_()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            engine.merit_device(db, lays[p], b, workspace=ws)
            e1.record(stream)
            ts.append((e0, e1))
        torch.cuda.synchronize()
        return sum(a.elapsed_time(c) for a, c in ts) / steps

    from mikroptim_b200.batch import PRECISION_DF64, PRECISION_FP32_BULK
    for extra in (PRECISION_DF64, PRECISION_FP32_BULK):
        lays[extra] = ResidualLayout(b.topology, dataclasses.replace(st, precision=extra))
    l0 = lib.mkb_launch_count()
    with ClockSampler(local) as clocks:
        ms = {p: merit_ms(p, args.steps) for p in (PRECISION_FP64_FMA, PRECISION_FP64,
                                                   PRECISION_MIXED, PRECISION_DF64,
                                                   PRECISION_FP32_BULK)}
    launches = lib.mkb_launch_count() - l0
    ms = {p: max_over_ranks(v, world, dev) for p, v in ms.items()}

    # OPD errors over every ray, in tranches of variants
    lam_mm = b.reference_wavelength_nm * 1e-6
    acc = {PRECISION_FP64_FMA: [0.0, 0, 0.0, 0, 0], PRECISION_MIXED: [0.0, 0, 0.0, 0, 0],
           PRECISION_DF64: [0.0, 0, 0.0, 0, 0], PRECISION_FP32_BULK: [0.0, 0, 0.0, 0, 0]}
    chunk = 2048
    for first in range(0, V, chunk):
        n = min(chunk, V - first)
        sub = b.subset(first, n)
        dsub = engine.DeviceSystemBatch(sub, dev)
        ref = engine.residuals_device(dsub, lay0, sub)
        ok_ref = ((ref.status == 0) | (ref.status == 5) | (ref.status == 6))
        for p in (PRECISION_FP64_FMA, PRECISION_MIXED, PRECISION_DF64, PRECISION_FP32_BULK):
            r = engine.residuals_device(dsub, lays[p], sub)
            same = (r.status == ref.status) & ok_ref
            err = ((r.opd - ref.opd) / lam_mm)[same]
            a = acc[p]
            a[0] += float((err * err).sum())
            a[1] += int(err.numel())
            a[2] = max(a[2], float(err.abs().max()) if err.numel() else 0.0)
            a[3] += int((r.status == ref.status).sum())
            a[4] += int(r.status.numel())
        del dsub, ref
    errors = {name: {"rms_waves": math.sqrt(acc[p][0] / max(acc[p][1], 1)),
                     "max_waves": acc[p][2],
                     "status_agreement": acc[p][3] / max(acc[p][4], 1),
                     "rays_compared": acc[p][1]}
              for p, name in ((PRECISION_FP64_FMA, "fp64_fma"), (PRECISION_MIXED, "mixed"),
                              (PRECISION_DF64, "df64"), (PRECISION_FP32_BULK, "fp32_bulk"))}

    # normal equations: fused (FMA, MIXED) against the exact materialised J^T J on a sample
    sample = b.subset(0, 64)
    ds = engine.DeviceSystemBatch(sample, dev)
    J, r0, _ = engine.adjoint_jacobian_device(ds, lay0, sample, vs, x0[:64])
    exact = engine.normal_equations_device(J, r0, True)
    # Jacobian entries: the contracted adjoint J against the bit-exact one, each entry relative
    # to its column's largest entry (the precisions whose J is materialised)
    Jf, _, _ = engine.adjoint_jacobian_device(ds, lays[PRECISION_FP64_FMA], sample, vs, x0[:64])
    colmax = J.abs().amax(dim=2, keepdim=True).clamp_min(1e-300)
    jrel = ((Jf - J).abs() / colmax)
    jac_entries = {"fp64_fma": {"median": float(jrel.median()), "max": float(jrel.max()),
                                "entries": int(jrel.numel()),
                                "relative_to": "the largest entry of the column"}}
    del J, Jf, jrel
    jerr = {}
    for p, name in ((PRECISION_FP64_FMA, "fp64_fma"), (PRECISION_MIXED, "mixed")):
        g = engine.adjoint_normal_equations_device(ds, lays[p], sample, vs, x0[:64])
        d = torch.diagonal(exact, dim1=1, dim2=2).abs()
        d = torch.maximum(d, 1e-20 * d.max(dim=1, keepdim=True).values + 1e-300)
        rel = (g - exact).abs() / torch.sqrt(d[:, :, None] * d[:, None, :])
        jerr[name] = {"median": float(rel.median()), "max": float(rel.max())}
    # intercept errors: EVAL (image-plane intercepts on a 32 x 32 grid, vertex reference
    # sphere) in FP64 with contraction (the forward of MIXED) against the bit-exact FP64, on a
    # sample of the systems
    ev = b.subset(0, 512)
    dev_ev = engine.DeviceSystemBatch(ev, dev)
    es = {p: engine.evaluate_device(dev_ev, ev, engine.EvalSettings(
        grid=32, reference=engine.EVAL_VERTEX, precision=p)) for p in (PRECISION_FP64,
                                                                       PRECISION_FP64_FMA)}
    e0_, e1_ = es[PRECISION_FP64], es[PRECISION_FP64_FMA]
    okm = (e0_.status == 0) & (e1_.status == 0)
    dxy = np.hypot(e1_.spot_x[okm] - e0_.spot_x[okm], e1_.spot_y[okm] - e0_.spot_y[okm]) * 1e6
    intercepts = {"fp64_fma_and_mixed": {
        "rms_nm": float(np.sqrt(np.mean(dxy ** 2))) if dxy.size else None,
        "max_nm": float(dxy.max()) if dxy.size else None, "rays_compared": int(dxy.size),
        "status_agreement": float(np.mean(e0_.status == e1_.status)),
        "sample": "512 systems, 9 wavelengths, 5 fields, 32 x 32 grid (EVAL, vertex sphere)"}}
    if rank != 0:
        return None, None
    return {
        "metric": "ray-surface hits/s (MERIT, FP64_FMA) with the OPD error of FP64_FMA and "
                  "MIXED against bit-exact FP64",
        "value": world * hits / (ms[PRECISION_FP64_FMA] / 1e3),
        "unit": "ray-surface hits/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": ms[PRECISION_FP64_FMA],
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded generator, configuration-4 shapes)",
        "config": {"workload": WORKLOAD_PREC.format(V=V),
                   "step": "one MERIT evaluation of every system",
                   "rays_per_evaluation": rays,
                   "l2": "flushed (256 MB write) before every timed step"},
        "gpu_launches": int(launches),
        "merit_ms": {"fp64_fma": ms[PRECISION_FP64_FMA], "fp64_exact": ms[PRECISION_FP64],
                     "mixed": ms[PRECISION_MIXED], "df64": ms[PRECISION_DF64],
                     "fp32_bulk": ms[PRECISION_FP32_BULK]},
        "df64_vs_fp64_fma_time": ms[PRECISION_DF64] / ms[PRECISION_FP64_FMA],
        "opd_error_vs_fp64": errors,
        "normal_equations_rel_error_vs_exact": jerr,
        "jacobian_entry_rel_error_vs_exact": jac_entries,
        "intercept_error_vs_fp64": intercepts,
        "e2e": None,
        "clocks": clocks.summary(),
    }, (b, lay0)


WORKLOAD_PSF = ("psf-{V}: EVAL of {V} objectives (config-2 shape: 15 surfaces, L=7, F=5) on a "
                "{N} x {N} pupil grid, then the scalar PSF and MTF of every (variant, field, "
                "wavelength) tuple with FFT size {M} (zero padding 4), NA {NA} given")


def hbm_peak_gbs() -> tuple[float, str]:
    """The measured copy bandwidth of this pool's B200s (MEASURED_PEAKS.json beside this
    file), else the earlier measurement."""
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "MEASURED_PEAKS.json")
    try:
        with open(path) as fh:
            return float(json.load(fh)["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback"


def run_psf(args, world, rank, local):
    """Scalar PSF and MTF (PsfEngine): one step = the device chain for every tuple -- OPD maps
    from EVAL's device outputs (mkb_psf_maps_device), then mkb_psf_device (row FFTs, column
    FFTs with the intensity, the centred PSF and the projections, MTF cuts); EVAL itself runs
    once before the timed steps. e2e: PsfEngine.compute on host pupils (maps up, PSF and MTF
    down, finish_psf on the host) for a sample of the tuples."""
    import torch
    from mikroptim_b200 import _capi, engine, psf, workloads

    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    lib = _capi.lib()
    V = args.variants or 512
    N, NA = 64, 0.25
    M = psf.psf_fft_size(N, 4.0)
    b, st, _, _ = workloads.objective(V, seed=20261203 + 6 + 1000 * rank)
    db = engine.DeviceSystemBatch(b, dev)
    settings = engine.EvalSettings(grid=N)
    pts, _, _, out = engine.evaluate_device_tensors(db, b, settings)
    res = engine.evaluate_device(db, b, settings)
    col, row, full, half = psf.grid_cells(res)
    T = V * b.fields * b.wavelengths
    n = pts.shape[0]
    params = []
    for v in range(V):
        for f in range(b.fields):
            for l in range(b.wavelengths):
                params.append(_capi.PsfPupilParams(b.wavelength_nm[l] * 1e-6,
                                                   1.0 / (float(full) * full), 1, 1))
    pa = (_capi.PsfPupilParams * T)(*params)
    pd = torch.frombuffer(bytearray(pa), dtype=torch.uint8).to(dev)
    cold = torch.from_numpy(col).to(dev)
    rowd = torch.from_numpy(row).to(dev)
    maps = torch.empty((T, N, N), dtype=torch.float64, device=dev)
    P = torch.empty((T, M, M), dtype=torch.float64, device=dev)
    mtf = torch.empty((T, 2, N + 1), dtype=torch.float64, device=dev)
    nbytes = int(lib.mkb_psf_workspace_bytes(T, N, M))
    ws = torch.empty(nbytes, dtype=torch.uint8, device=dev)
    flush = torch.empty(256 * 1024 * 1024, dtype=torch.uint8, device=dev)
    stream = torch.cuda.current_stream()

    def step():
        _capi.check(lib.mkb_psf_maps_device(T, N, n, int(half), C.c_void_p(out["opd"].data_ptr()),
                                            C.c_void_p(out["st"].data_ptr()),
                                            C.c_void_p(cold.data_ptr()),
                                            C.c_void_p(rowd.data_ptr()),
                                            C.c_void_p(maps.data_ptr()), None), "psf maps")
        _capi.check(lib.mkb_psf_device(T, N, M, C.c_void_p(maps.data_ptr()),
                                       C.c_void_p(pd.data_ptr()), C.c_void_p(P.data_ptr()),
                                       C.c_void_p(mtf.data_ptr()), C.c_void_p(ws.data_ptr()),
                                       nbytes, None), "psf")

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    l0 = lib.mkb_launch_count()
    ts = []
    with ClockSampler(local) as clocks:
        for _ in range(args.steps):
            flush.zero_()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            step()
            e1.record(stream)
            ts.append((e0, e1))
        torch.cuda.synchronize()
    launches = lib.mkb_launch_count() - l0
    ms = max_over_ranks(sum(a.elapsed_time(c) for a, c in ts) / args.steps, world, dev)
    # bytes one step must move: the maps in (EVAL's OPD and status read, maps written and
    # read), the N x M complex row spectra out and back in (the field does not fit on chip),
    # the PSF and MTF out
    per_tuple = (n * 9 + 2 * N * N * 8 + 2 * N * M * 16 + M * M * 8 + 2 * (N + 1) * 8)
    peak, peak_src = hbm_peak_gbs()
    achieved = T * per_tuple / (ms / 1e3) / 1e9
    # e2e through PsfEngine.compute (host pupils in, host results out with finish_psf)
    sample = min(T, 1024)
    pupils = []
    for t in range(sample):
        v, rem = divmod(t, b.fields * b.wavelengths)
        f, l = divmod(rem, b.wavelengths)
        p = psf.make_psf_pupil(b, res, v, f, l, psf.PsfSettings(numerical_aperture=NA))
        pupils.append(p)
    eng = psf.PsfEngine(local)
    eng.compute(pupils[:8], M)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    eng.compute(pupils, M)
    torch.cuda.synchronize()
    e2e_s = time.perf_counter() - t0
    if rank != 0:
        return None, None
    cpu = None
    try:
        cpu = cpu_baseline_psf(pupils[:16], M)
    except Exception as e:  # the baseline is reported, not required
        cpu = {"value": None, "error": str(e)}
    return {
        "metric": "PSF tuples/s (scalar PSF + MTF cuts from EVAL OPD maps)",
        "value": world * T / (ms / 1e3),
        "unit": "PSF tuples/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded generator, configuration-2 shapes)",
        "config": {"workload": WORKLOAD_PSF.format(V=V, N=N, M=M, NA=NA), "tuples": T,
                   "step": "maps from the device EVAL output + mkb_psf_device for every tuple",
                   "l2": "flushed (256 MB write) before every timed step; a step writes about "
                         "10 GB (inputs larger than L2)"},
        "gpu_launches": int(launches),
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "traffic": None, "peak_source": peak_src,
                     "bytes_model": "per tuple: EVAL OPD + status read (9 B/point), map write "
                                    "+ read (2 N^2 x 8), row spectra write + read "
                                    "(2 N M x 16), PSF write (M^2 x 8), MTF"},
        "e2e": {"value": sample / e2e_s, "unit": "PSF tuples/s",
                "h2d_bytes_per_step": sample * (N * N * 8 + 24),
                "d2h_bytes_per_step": sample * (M * M * 8 + 2 * (N + 1) * 8),
                "api": "psf.PsfEngine.compute(host pupils, M) -> PSF, MTF and figures",
                "tuples": sample},
        "clocks": clocks.summary(),
        "cpu_baseline": cpu,
    }, None


def cpu_baseline_psf(pupils, M: int):
    """The reference's psf_cpu (own radix-2 FFT, one thread) on a sample of the tuples."""
    import oracle.pyoracle as po
    ref = po.reference()
    t0 = time.perf_counter()
    for p in pupils:
        ref.psf_pupil(p.grid, M, p.opd, p.full_count, p.wavelength_nm, p.na_x, p.na_y,
                      p.flip_x, p.flip_y)
    dt = time.perf_counter() - t0
    return {"value": len(pupils) / dt, "unit": "PSF tuples/s", "cores": 1,
            "kind": "reference",
            "sample": f"psf_cpu of {len(pupils)} tuples (FFT {M}), {dt:.1f} s"}


def cpu_baseline_tolerancing(samples: int = 8):
    """The reference's CPU MERIT plus adjoint Jacobian (gradient 2 J^T r) of `samples` samples,
    all host threads (oracle/_ref)."""
    import oracle.pyoracle as po
    from mikroptim_b200 import workloads
    from mikroptim_b200.batch import ResidualLayout
    b, st, vs, x0 = workloads.tolerancing(samples)
    lay = ResidualLayout(b.topology, st)
    ref = po.reference()
    threads = os.cpu_count() or 1
    t0 = time.perf_counter()
    ref.merit(b, lay, threads=threads)
    J, r0, _ = ref.adjoint_jacobian(b, lay, vs, x0, threads=threads)
    np.einsum("ipr,ir->ip", J, r0)
    dt = time.perf_counter() - t0
    return {"value": samples / dt, "unit": "samples/s", "cores": threads, "kind": "reference",
            "sample": f"merit_cpu + adjoint_jacobian_cpu of {samples} samples, {dt:.1f} s"}


def main():
    args = parse()
    world, rank, local = dist_setup(args)
    if args.impl == "reference":
        out = run_reference(args, world, rank)
    elif args.workload == "uneven":
        out, _ = run_uneven(args, world, rank, local)
        if rank == 0 and world == 1:
            try:
                out["cpu_baseline"] = cpu_baseline_uneven()
            except Exception as e:  # the baseline is reported, not required
                out["cpu_baseline"] = {"value": None, "error": str(e)}
    elif args.workload == "precision":
        out, _ = run_precision(args, world, rank, local)
    elif args.workload == "psf":
        out, _ = run_psf(args, world, rank, local)
    elif args.workload == "tolerancing":
        out, _ = run_tolerancing(args, world, rank, local)
        if rank == 0 and world == 1:
            try:
                out["cpu_baseline"] = cpu_baseline_tolerancing()
            except Exception as e:  # the baseline is reported, not required
                out["cpu_baseline"] = {"value": None, "error": str(e)}
    elif args.workload == "singlet":
        out, _ = run_singlet(args, world, rank, local)
        if rank == 0 and world == 1:
            try:
                out["cpu_baseline"] = cpu_baseline_singlet()
            except Exception as e:  # the baseline is reported, not required
                out["cpu_baseline"] = {"value": None, "error": str(e)}
    elif args.workload == "lm":
        out, _ = run_lm(args, world, rank, local)
        if rank == 0 and world == 1:
            try:
                out["cpu_baseline"] = cpu_baseline_lm(reference_kind())
            except Exception as e:  # the baseline is reported, not required
                out["cpu_baseline"] = {"value": None, "error": str(e)}
    else:
        out, _ = run_b200(args, world, rank, local)
        if rank == 0 and world == 1:
            try:
                out["cpu_baseline"] = cpu_baseline(reference_kind())
            except Exception as e:  # the baseline is reported, not required
                out["cpu_baseline"] = {"value": None, "error": str(e)}
    if rank == 0:
        print(json.dumps(out))
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
