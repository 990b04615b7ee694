"""Benchmark: laminarSMOKE reaction step (chemistry cells*steps/s) on B200.

Workload (one "step" = one reaction step of every cell of the batch, dt = 1e-5 s):
  POLIMI_H2CO_1412 (14 species, 33 reactions), 1,048,576 cells with uneven
  stiffness: 30 % cold frozen mixing states, 20 % near-ignition states, 50 % hot
  near-equilibrium states (samples, with <= 1e-3 relative perturbation, of a
  pool of 4,096 hot mixtures integrated for 10 ms by the CPU oracle once and
  stored in tests/golden/h2co_hot_pool.npz, so both arms integrate identical
  cells).  Seeded synthetic inputs; no dataset is involved.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

The headline is the mixed-precision batched form (autotuned).  The same run
times the plain FP64 form (warp per cell, the reference's operation order) on
the same cells and reports the ratio, and checks both forms against the CPU
oracle on the cells of the CPU-baseline sample.

Under torchrun (N > 1) every rank integrates its own 1,048,576-cell batch (cells
are independent, no collective on the data path): weak scaling, value = all
cells*steps of all ranks / max-over-ranks time.  --impl reference times the
CPU restatement of the reference step (oracle/) on the host cores instead.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

NCELLS = 1 << 20
DT = 1.0e-5
POOL = os.path.join(ROOT, "tests", "golden", "h2co_hot_pool.npz")   # oracle-integrated hot pool
P_ATM = 101325.0
METRIC = "chemistry cells·steps/s: mixed-prec batched vs plain FP64 on 1 B200 at ≤1e-6 rel T err"
UNIT = "cells*steps/s"
TRANSCENDENTAL_FLOPS = 20.0   # FP64-instruction equivalent charged per exp/log/pow in the work model


# Work model of the reference algorithm (FP64 operations; transcendentals charged
# TRANSCENDENTAL_FLOPS each), split by the kernel that does the work:
#   rhs      F_rhs per RHS call, and per Jacobian (n - 1) F_rhs,T-cached + F_rhs
#            (KernelDense.hpp:111-193: only the T column recomputes k(T));
#   advance  per factorisation 2/3 n^3 + n^2 (G = I - h r0 J and its LU,
#            KernelDense.hpp:195-222), per solve 2 n^2 (:224-245), per Jacobian
#            n^2 (the difference quotients), per BDF step VEC_FLOPS_PER_N n
#            (predictor, corrector updates, error norms, Nordsieck rescale);
#   plain    all of it (one launch integrates every cell).
VEC_FLOPS_PER_N = 30.0


def rhs_flops(arrays):
    nc = int(arrays["dims"][0]); nr = int(arrays["dims"][1])
    nnz = len(arrays["reac_species"]) + len(arrays["prod_species"])
    n_exp = nr + len(arrays["rev_thermo"]) + 3 * len(arrays["fo_rxn"]) + 2
    f_rhs = 40 * nc + 12 * nr + 4 * nnz + TRANSCENDENTAL_FLOPS * (n_exp + 2 * len(arrays["fo_rxn"]))
    f_cached = 15 * nc + 4 * nr + 4 * nnz + TRANSCENDENTAL_FLOPS * 2 * len(arrays["fo_rxn"])
    return f_rhs, f_cached


def work_by_kernel(arrays, counters: np.ndarray):
    """FLOPs of the reference algorithm per kernel kind, summed over the cells' counters."""
    n = int(arrays["dims"][0]) + 1
    f_rhs, f_cached = rhs_flops(arrays)
    c = counters.astype(np.float64).sum(axis=0)
    steps, rhs, jac, fact, solve = c[0], c[1], c[2], c[3], c[4]
    w_rhs = rhs * f_rhs + jac * ((n - 1) * f_cached + f_rhs)
    w_adv = fact * (2.0 / 3.0 * n ** 3 + n * n) + solve * 2.0 * n * n + jac * n * n + steps * VEC_FLOPS_PER_N * n
    return {"rhs": w_rhs, "advance": w_adv, "plain": w_rhs + w_adv, "persistent": w_rhs + w_adv}


def fp64_peak_tflops(device) -> float:
    """Measured FP64 rate of this GPU: a cuBLAS DGEMM (8192^3) timed with CUDA events."""
    import torch
    a = torch.randn(8192, 8192, dtype=torch.float64, device=device)
    b = torch.randn(8192, 8192, dtype=torch.float64, device=device)
    for _ in range(2):
        torch.matmul(a, b)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(5):
        torch.matmul(a, b)
    e1.record()
    torch.cuda.synchronize()
    s = e0.elapsed_time(e1) / 1e3 / 5
    del a, b
    return 2.0 * 8192 ** 3 / s / 1e12


def kernel_roofline(args, ktimes, counters, arrays, fp64_peak, hbm, hbm_src):
    """Roofline of the dominant kernel (largest live CUDA-event time): the reference algorithm's FP64 work
    it does per launch over its average launch time, against the measured FP64 rate.  The same kernel's
    bytes per launch under the step's algorithmic traffic (2 n 8 + 8 per cell-step: read Y, T, write Y, T)
    and its measured DRAM traffic (ncu, profiles/traffic.json) are reported beside it."""
    n = int(arrays["dims"][0]) + 1
    timed = {k: v for k, v in ktimes.items() if v[1] > 0}
    if not timed:
        return None
    dom = max(timed, key=lambda k: timed[k][0])
    ms, nl = timed[dom]
    per_step = nl / max(args.steps, 1)                  # launches of this kernel per step
    avg_s = ms / nl / 1e3
    flops = work_by_kernel(arrays, counters).get(dom, 0.0) / per_step
    achieved = flops / avg_s / 1e12 if avg_s > 0 else None
    ncells = counters.shape[0]
    traffic = None
    tfile = os.path.join(ROOT, "profiles", "traffic.json")
    if os.path.exists(tfile):
        try:
            with open(tfile) as f:
                tr = json.load(f).get("mixed_fp32", {})
            if tr.get("kernel") == dom and tr.get("bytes_per_unit"):
                visits = float(counters[:, 1].sum() + counters[:, 2].sum())
                traffic = tr["bytes_per_unit"] * visits / per_step
        except (OSError, ValueError):
            traffic = None
    step_bytes = (2 * n * 8 + 8) * ncells / per_step
    return {"bound": "fp64", "achieved": achieved, "peak": fp64_peak, "unit": "TFLOP/s",
            "frac": achieved / fp64_peak if achieved else None, "traffic": traffic,
            "kernel": dom, "launch_ms": avg_s * 1e3, "algorithmic_flops_per_launch": flops,
            "peak_source": "measured live in this run: cuBLAS DGEMM 8192^3, CUDA events",
            "hbm_view": {"algorithmic_bytes_per_launch": step_bytes, "achieved_gbs": step_bytes / avg_s / 1e9,
                         "peak_gbs": hbm, "peak_source": hbm_src},
            "note": "latency-bound BDF solver kernel; traffic is its cell-record round trips"}


def tuning_report(ctx, lsg):
    t = ctx.tuning()
    if t is None:
        return None
    tile, width, rates = t
    names = {lsg.LSG_TILE_LANE: f"round scheme, {width} lanes per cell", lsg.LSG_TILE_WARP: "plain warp kernel",
             lsg.LSG_TILE_PERSISTENT: "persistent lane kernel",
             lsg.LSG_TILE_GROUP: f"fused lane-group kernel, {width} blocks per SM",
             lsg.LSG_TILE_BLOCK: "block per cell, " + ("tensor-core inverse" if width else "FP64 LU factors")}
    return {"chosen": names.get(tile, str(tile)), "sample_cells_per_s": {k: round(v) for k, v in rates.items() if v}}


def max_over_ranks(x: float, world: int, device) -> float:
    """The slowest rank's time (every rank calls it, same order, every step)."""
    if world <= 1:
        return float(x)
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def whole_job_rate(cells_per_rank: int, steps: int, ms: float, world: int) -> float:
    """cells*steps/s of all ranks together: every rank integrates its own batch
    (replicas, weak scaling) and the job is as fast as its slowest rank."""
    return world * cells_per_rank * steps / (ms / 1e3)


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=("ours", "reference"), default="ours")
    ap.add_argument("--cells", type=int, default=NCELLS)
    ap.add_argument("--cpu-sample", type=int, default=0,
                    help="cells of the CPU baseline sample (0: sized for about 10 s of CPU work)")
    ap.add_argument("--tile", choices=("auto", "lane", "persistent", "group"), default="auto",
                    help="batched form: autotuned (the first warm-up step times the candidate forms), round "
                         "scheme (lane) or persistent lane kernel")
    ap.add_argument("--factors", choices=("fp32", "fp64"), default="fp32",
                    help="batched form: precision of the LU factors")
    ap.add_argument("--plain-steps", type=int, default=3,
                    help="timed steps of the plain FP64 form (it is ~6x slower; 0 skips it)")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--plain-cells", type=int, default=0,
                    help="large-mechanism workloads: the FP64 arm runs on an evenly strided sample of this many "
                         "of the cells (0: all)")
    ap.add_argument("--workload", choices=("h2co_uneven", "syn120", "syn500", "coflow"), default="h2co_uneven",
                    help="h2co_uneven: the headline (1,048,576 cells); syn120 / syn500: the 120- and 500-species "
                         "synthetic mechanisms (bounded draws); coflow: 50 device-resident steps of the 200 x 400 "
                         "coflow mesh with the 120-species mechanism, replayed from a CUDA graph")
    return ap.parse_args()


# ----------------------------------------------------------------------------
def workload(n: int, seed: int = 2):
    """The uneven-stiffness H2/CO cells; the hot pool is the oracle-integrated one from tests/golden."""
    from laminarsmoke_b200 import cells, mech
    from laminarsmoke_b200.mech import blob
    data, species = mech.load("h2co")
    arrays, _ = blob.unpack(data)
    Y, T = cells.h2co_uneven(species, arrays["mw"], n, cells.pool_from_file(POOL), seed=seed)
    return data, species, arrays, Y, T


def config_dict(ncells: int, world: int) -> dict:
    """The workload's description, identical in both arms (what differs between the arms is in "arm")."""
    return {"workload": "h2co_uneven (30% cold / 20% igniting / 50% near-equilibrium), seed 2",
            "ncells_per_gpu": ncells, "mechanism": "POLIMI_H2CO_1412 (14 species, 33 reactions)",
            "dt": DT, "t0": 0.0, "p": P_ATM, "rtol": 1e-7, "atol": 1e-12,
            "hot_pool": "tests/golden/h2co_hot_pool.npz (4,096 mixtures integrated 10 ms by the oracle)",
            "l2": "GPU arm: flushed (1 GiB write) before every timed step, inputs restored from an HBM copy",
            "parallelism": f"replicas x{world}"}


class ClockSampler:
    """nvidia-smi clocks and throttle reasons during the timed region."""

    def __init__(self, index: int):
        self.index = index
        self.samples = []
        self.proc = None

    def __enter__(self):
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) >= 9:
                self.samples.append(parts)

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"]}
        sm = [float(s[1]) for s in self.samples if s[1].replace(".", "").isdigit()]
        mx = [float(s[2]) for s in self.samples if s[2].replace(".", "").isdigit()]
        reasons = set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for s in self.samples:
            for nm, v in zip(names, s[5:9]):
                if v.strip().lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(self.samples)}


def oracle_sample(data, Y, T, sample: int = 0, seed: int = 7, target_s: float = 10.0):
    """The reference's CPU step (oracle restatement) on the host cores, on a bounded sample of the
    workload's cells.  sample = 0 sizes the sample from a pilot so that it takes about target_s seconds
    (capped at the workload size).  Returns the baseline record, the sampled cell indices and the
    oracle's results for them (Y, T, status, counters)."""
    from oracle.oracle import OracleMechanism
    om = OracleMechanism(data)
    threads = os.cpu_count() or 1
    rng = np.random.default_rng(seed)
    if sample <= 0:
        pilot = rng.choice(Y.shape[0], size=min(256 * threads, Y.shape[0]), replace=False)
        t0 = time.perf_counter()
        om.reaction_step(Y[pilot], T[pilot], DT, nthreads=threads)
        rate = len(pilot) / max(time.perf_counter() - t0, 1e-6)
        sample = int(min(Y.shape[0], max(len(pilot), rate * target_s)))
    pick = np.sort(rng.choice(Y.shape[0], size=min(sample, Y.shape[0]), replace=False))
    t0 = time.perf_counter()
    Yo, To, _, sto, cnto = om.reaction_step(Y[pick], T[pick], DT, nthreads=threads)
    el = time.perf_counter() - t0
    rec = {"value": len(pick) / el, "unit": UNIT, "cores": threads, "kind": "port",
           "sample": f"{len(pick)} cells drawn (seed {seed}) from the {Y.shape[0]}-cell workload, one step, "
                     f"{threads} OpenMP threads, {el:.2f} s"}
    return rec, pick, (Yo, To, sto, cnto), el


def accuracy_vs_oracle(Yg, Tg, stg, cntg, ref) -> dict:
    """A GPU form's results on the sampled cells against the oracle's: the metric's bounds (relative T
    1e-6, absolute Y 1e-9) and a per-cell account of the cells beyond 1e-9 -- whether each took the same
    solver path as the oracle (all eight per-cell counters equal: steps, RHS calls, Jacobians,
    factorisations, solves, error-test and convergence failures, Jacobian RHS calls)."""
    Yo, To, sto, cnto = ref
    dT = np.abs(Tg - To) / To
    dY = np.abs(Yg - Yo).max(axis=1)
    same = (cntg == cnto).all(axis=1)
    miss = dY > 1e-9
    return {"against": "CPU oracle (FP64 restatement of the reference step), same cells",
            "cells": int(len(To)), "statuses_equal": bool(np.array_equal(stg, sto)),
            "max_rel_T": float(dT.max()), "max_abs_Y": float(dY.max()),
            "cells_within_abs_Y_1e-9": float((~miss).mean()),
            "same_solver_path": float(same.mean()),
            "max_abs_Y_same_path": float(dY[same].max()) if same.any() else None,
            "max_rel_T_same_path": float(dT[same].max()) if same.any() else None,
            "cells_beyond_1e-9": int(miss.sum()),
            "cells_beyond_1e-9_same_path": int((miss & same).sum()),
            "max_abs_Y_other_path": float(dY[~same].max()) if (~same).any() else None}


# ----------------------------------------------------------------------------
def run_reference(args, rank: int, world: int):
    """The reference's CPU step (the oracle port of it) on the host cores.  Each step times one bounded
    sample of the workload (about 10 s of CPU work, a fresh seeded draw each step); ms_per_step is the
    measured wall time of those samples and value = cells / s over the timed steps."""
    if rank != 0:
        return 0
    data, species, arrays, Y, T = workload(args.cells)
    cells_done, secs, samples = 0, 0.0, []
    for k in range(args.warmup + args.steps):
        target = 2.0 if k < args.warmup else 10.0
        r, pick, _, el = oracle_sample(data, Y, T, args.cpu_sample, seed=7 + k, target_s=target)
        if k >= args.warmup:
            cells_done += len(pick)
            secs += el
            samples.append(len(pick))
    v = cells_done / secs
    threads = os.cpu_count() or 1
    out = {"impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": args.gpus,
           "steps": args.steps, "warmup": args.warmup, "ms_per_step": secs / args.steps * 1e3,
           "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
           "data": "synthetic", "config": config_dict(args.cells, world),
           "arm": {"impl": "the oracle's FP64 restatement of the reference CPU step",
                   "threads": f"{threads} OpenMP threads on the host cores, rank 0 only"},
           "cells_per_step": {"min": int(min(samples)), "max": int(max(samples)),
                              "note": "each timed step integrates one seeded sample of the workload's cells"},
           "cpu_baseline": {"value": v, "unit": UNIT, "cores": threads, "kind": "port",
                            "sample": f"{args.steps} timed samples of {min(samples)}-{max(samples)} cells drawn "
                                      f"from the {args.cells}-cell workload (seeds {7 + args.warmup}-"
                                      f"{6 + args.warmup + args.steps}), one step each, {threads} OpenMP "
                                      f"threads, {secs:.1f} s in all"},
           "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(out), flush=True)
    return 0


def timed_steps(ctx, Y0, T0, Yw, Tw, flush, status, steps, warmup, counters, stream):
    """W untimed + K timed device-array steps of `ctx` on a fresh copy of (Y0, T0) each time, L2 flushed
    before each step; returns the per-step CUDA-event times (ms).  The warm-up steps fill `counters`."""
    import torch

    def one(cnt=None):
        Yw.copy_(Y0)
        Tw.copy_(T0)
        flush.fill_(1.0)
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        ctx.step_device(Yw, Tw, DT, status=status, counters=cnt)
        e1.record(stream)
        return e0, e1

    for _ in range(warmup):
        one(counters)
    torch.cuda.synchronize()
    ctx.check()
    evs = [one() for _ in range(steps)]
    torch.cuda.synchronize()
    ctx.check()
    return [a.elapsed_time(b) for a, b in evs]


def run_ours(args, rank: int, world: int, local_rank: int):
    import torch
    import torch.distributed as dist
    from laminarsmoke_b200 import lsg

    dev = torch.device("cuda", local_rank)
    torch.cuda.set_device(dev)
    data, species, arrays, Y, T = workload(args.cells, 2 + 1000 * rank)
    n, nc = Y.shape
    m = lsg.Mechanism(data, device=local_rank)
    tile = {"lane": lsg.LSG_TILE_LANE, "persistent": lsg.LSG_TILE_PERSISTENT, "auto": lsg.LSG_TILE_AUTO,
            "group": lsg.LSG_TILE_GROUP}[args.tile]
    prec = lsg.LSG_PRECISION_MIXED if args.factors == "fp32" else lsg.LSG_PRECISION_FP64
    ctx = lsg.ReactionStep(m, tile=tile, precision=prec, kernel_timing=1, autotune=int(args.tile == "auto"))
    plain = lsg.ReactionStep(m, tile=lsg.LSG_TILE_WARP, precision=lsg.LSG_PRECISION_FP64, kernel_timing=1)
    Y0 = torch.tensor(np.ascontiguousarray(Y.T), device=dev)
    T0 = torch.tensor(T, device=dev)
    Yw = torch.empty_like(Y0)
    Tw = torch.empty_like(T0)
    cnt = torch.zeros((n, lsg.NCOUNTERS), dtype=torch.int64, device=dev)
    status = torch.zeros(n, dtype=torch.int32, device=dev)
    flush = torch.empty(64 << 22, dtype=torch.float32, device=dev)  # 1 GiB > L2
    stream = torch.cuda.current_stream()

    # ---- the headline: the mixed-precision batched form ----
    # warm-up (the autotuner's trial runs in the first step), then the timed steps with the clocks sampled
    timed_steps(ctx, Y0, T0, Yw, Tw, flush, status, 0, args.warmup, cnt, stream)
    ctx.kernel_times(reset=True)
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    l0 = ctx.launches()
    with ClockSampler(local_rank) as clk:
        times = timed_steps(ctx, Y0, T0, Yw, Tw, flush, status, args.steps, 0, None, stream)
    launches = ctx.launches() - l0
    ktimes = ctx.kernel_times(reset=True)
    if world > 1:
        dist.barrier()
    ms = max_over_ranks(float(sum(times)), world, dev)
    ms_per_step = ms / args.steps
    value = whole_job_rate(n, args.steps, ms, world)
    st_m = status.cpu().numpy()
    Ym, Tm = Yw.cpu().numpy().T.copy(), Tw.cpu().numpy().copy()
    cnt_m = cnt.cpu().numpy()

    # ---- the plain FP64 form on the same cells (the metric's denominator) ----
    plain_rec = None
    if args.plain_steps > 0:
        pw = min(args.warmup, 3)
        ptimes = timed_steps(plain, Y0, T0, Yw, Tw, flush, status, args.plain_steps, pw, cnt, stream)
        pms = max_over_ranks(float(sum(ptimes)), world, dev)
        pk = plain.kernel_times(reset=True)
        plain_rec = {"value": whole_job_rate(n, args.plain_steps, pms, world), "unit": UNIT,
                     "ms_per_step": pms / args.plain_steps, "steps": args.plain_steps, "warmup": pw,
                     "form": "plain FP64, one warp per cell, the reference's operation order",
                     "kernel_ms_per_step": {k: round(v[0] / args.plain_steps, 3) for k, v in pk.items() if v[1]}}
        st_p = status.cpu().numpy()
        Yp, Tp = Yw.cpu().numpy().T.copy(), Tw.cpu().numpy().copy()
        cnt_p = cnt.cpu().numpy()

    # ---- end to end through the host-array C ABI call: H2D of the inputs, the step, D2H of the results ----
    e2e = None
    if not args.no_e2e:
        Yh = torch.empty((nc, n), dtype=torch.float64).pin_memory()
        Th = torch.empty(n, dtype=torch.float64).pin_memory()
        Yn = np.ascontiguousarray(Y.T)
        tms = []
        for it in range(1 + args.steps):
            Yh.numpy()[:] = Yn
            Th.numpy()[:] = T
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            ctx.step(Yh.numpy(), Th.numpy(), DT)
            tms.append(time.perf_counter() - t0)
        et = max_over_ranks(float(np.mean(tms[1:])), world, dev)
        e2e = {"value": whole_job_rate(n, 1, et * 1e3, world), "unit": UNIT,
               "h2d_bytes_per_step": int(8 * (nc + 1) * n),
               "d2h_bytes_per_step": int(8 * (nc + 1) * n + 8 * n + 4 * n + 4 * n)}

    out = None
    if rank == 0:
        peaks = {}
        try:
            with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
                peaks = json.load(f)
        except OSError:
            pass
        hbm = peaks.get("hbm_gbs")
        hbm_src = "measured (MEASURED_PEAKS.json)" if hbm else "fallback 6650 GB/s"
        hbm = hbm or 6650.0
        fp64 = fp64_peak_tflops(dev)
        roofline = kernel_roofline(args, ktimes, cnt_m, arrays, fp64, hbm, hbm_src)
        w = work_by_kernel(arrays, cnt_m)
        cpu, pick, ref, _ = oracle_sample(data, Y, T, args.cpu_sample)
        acc = {"mixed": accuracy_vs_oracle(Ym[pick], Tm[pick], st_m[pick], cnt_m[pick], ref)}
        if plain_rec is not None:
            acc["plain"] = accuracy_vs_oracle(Yp[pick], Tp[pick], st_p[pick], cnt_p[pick], ref)
        arm = {"form": "mixed", "tile": "autotuned" if args.tile == "auto" else args.tile,
               "lu": "fp32 factors refined on the fp64 residual" if args.factors == "fp32" else "fp64"}
        out = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64+f32" if args.factors == "fp32" else "f64", "data": "synthetic",
            "config": config_dict(n, world),
            "arm": arm,
            "plain": plain_rec,
            "ratio_vs_plain": value / plain_rec["value"] if plain_rec else None,
            "roofline": roofline,
            "kernel_ms_per_step": {k: round(v[0] / args.steps, 3) for k, v in ktimes.items() if v[1]},
            "autotune": tuning_report(ctx, lsg),
            "fp64_work": {"algorithmic_tflops": w["plain"] / (ms_per_step / 1e3) / 1e12,
                          "peak_tflops": fp64, "frac": w["plain"] / (ms_per_step / 1e3) / 1e12 / fp64,
                          "flops_per_cell_step": w["plain"] / n,
                          "counters_per_cell": dict(zip(("steps", "rhs", "jacobians", "factorisations", "solves",
                                                         "error_fails", "conv_fails", "jacobian_rhs"),
                                                        [round(float(x), 3) for x in cnt_m.mean(axis=0)])),
                          "transcendental_flops_each": TRANSCENDENTAL_FLOPS},
            "statuses": {str(k): int(v) for k, v in zip(*np.unique(st_m, return_counts=True))},
            "accuracy": acc,
            "cpu_baseline": cpu,
            "e2e": e2e,
            "gpu_launches": launches,
            "clocks": clk.summary(),
        }
        print(json.dumps(out), flush=True)
    ctx.close()
    plain.close()
    m.close()
    return 0


# ----------------------------------------------------------------------------
# The large-mechanism workloads (one GPU).  syn120: 120 species / 800 reactions, T ~ U[800, 2400] K,
# dt = 5e-6 s; syn500: 500 species / 3,000 reactions, T ~ U[900, 2200] K, dt = 1e-5 s (the mechanisms are the
# seeded synthetic ones with physically bounded barriers and rate constants, mech.load("syn120p" / "syn500p"));
# coflow: the 200 x 400 Burke-Schumann mesh with the 120-species mechanism, 50 steps of 1e-5 s.  The mixed
# form is the block form with the tensor-core inverse (up to 127 species), the plain form the FP64 block form.
LARGE = {"syn120": ("syn120p", (800.0, 2400.0), 5e-6), "syn500": ("syn500p", (900.0, 2200.0), 1e-5),
         "coflow": ("syn120p", None, 1e-5)}


def run_large(args, rank: int, world: int, local_rank: int):
    import torch
    from laminarsmoke_b200 import cells, lsg, mech
    from laminarsmoke_b200.mech import blob
    dev = torch.device("cuda", local_rank)
    torch.cuda.set_device(dev)
    name, trange, dt = LARGE[args.workload]
    data, species = mech.load(name)
    arrays, _ = blob.unpack(data)
    nsteps = 50 if args.workload == "coflow" else 1
    if args.cells == NCELLS:   # the large mechanisms' default batch: enough cells to fill the GPU many times
        args.cells = {"syn120": 16384, "syn500": 2048}.get(args.workload, args.cells)
    if args.workload == "coflow":
        # the 200 x 400 mesh (80,000 cells); --cells below that takes an evenly strided sample of it
        Y, T = cells.coflow_fields(species, arrays["mw"])
        mesh_cells = T.size
        if args.cells < T.size:
            idx = np.linspace(0, T.size - 1, args.cells).astype(np.int64)
            Y, T = Y[idx], T[idx]
    else:
        mesh_cells = None
        Y, T = cells.synthetic_mixing(species, arrays["mw"], args.cells, seed=11, t_range=trange)
    n, nc = Y.shape
    m = lsg.Mechanism(data, device=local_rank)
    forms = {"mixed": lsg.LSG_PRECISION_MIXED, "plain": lsg.LSG_PRECISION_FP64}
    Y0 = torch.tensor(np.ascontiguousarray(Y.T), device=dev)
    T0 = torch.tensor(T, device=dev)
    Yw, Tw = torch.empty_like(Y0), torch.empty_like(T0)
    status = torch.zeros(n, dtype=torch.int32, device=dev)
    cnt = torch.zeros((n, lsg.NCOUNTERS), dtype=torch.int64, device=dev)
    flush = torch.empty(64 << 22, dtype=torch.float32, device=dev)
    stream = torch.cuda.current_stream()
    # the FP64 arm on all cells, or on an evenly strided sample of them (--plain-cells)
    pn = n if args.plain_cells <= 0 or args.plain_cells >= n else args.plain_cells
    pidx = np.arange(n) if pn == n else np.linspace(0, n - 1, pn).astype(np.int64)
    res = {}
    for form, prec in forms.items():
        # the mixed arm autotuned: its first (warm-up) call times the block form with FP64 LU factors against
        # the block form with the tensor-core inverse and keeps the faster
        ctx = lsg.ReactionStep(m, precision=prec, kernel_timing=0, autotune=int(form == "mixed"))
        idx = np.arange(n) if form == "mixed" else pidx
        nf = len(idx)
        Yf0 = Y0 if nf == n else Y0[:, torch.as_tensor(idx, device=dev)].contiguous()
        Tf0 = T0 if nf == n else T0[torch.as_tensor(idx, device=dev)].contiguous()
        Yf = Yw if nf == n else torch.empty_like(Yf0)
        Tf = Tw if nf == n else torch.empty_like(Tf0)
        # warm-up calls (module load, work space, first launches): the same kernels and options on the
        # first min(nf, 256) cells of the batch for single-step workloads, the full call for the graph
        warm = nf if nsteps > 1 else min(nf, 256)
        ms = []
        for it in range(args.warmup + args.steps):
            k = warm if it < args.warmup else nf
            Yf.copy_(Yf0)
            Tf.copy_(Tf0)
            flush.fill_(1.0)
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            if nsteps > 1:
                used = ctx.step_sequence_graph(Yf, Tf[:k], dt, nsteps, status=status[:k])
            else:
                used = False
                ctx.step_device(Yf, Tf[:k], dt, status=status[:k],
                                counters=cnt[:k] if it == args.warmup else None)
            e1.record(stream)
            torch.cuda.synchronize()
            ctx.check()
            if it >= args.warmup:
                ms.append(e0.elapsed_time(e1))
        t = max_over_ranks(float(sum(ms)), world, dev)
        res[form] = {"value": whole_job_rate(nf, args.steps * nsteps, t, world), "cells": nf,
                     "ms_per_call": t / args.steps, "graph": bool(used),
                     "statuses": {str(k): int(v) for k, v in
                                  zip(*np.unique(status[:nf].cpu().numpy(), return_counts=True))},
                     "Y": Yf.cpu().numpy().T.copy(), "T": Tf.cpu().numpy().copy(), "idx": idx,
                     "counters": cnt[:nf].cpu().numpy().mean(axis=0).tolist() if nsteps == 1 else None,
                     "autotune": tuning_report(ctx, lsg) if form == "mixed" else None}
        ctx.close()
    out = None
    if rank == 0:
        acc = None
        if nsteps == 1:   # the oracle on a bounded sample of the same cells (about 20 s of CPU work)
            from oracle.oracle import OracleMechanism
            om = OracleMechanism(data)
            # cells that both arms integrated (the FP64 arm may run on a strided sample)
            pick = np.sort(np.random.default_rng(3).choice(pidx, min(len(pidx), args.cpu_sample or 64),
                                                           replace=False))
            t0 = time.perf_counter()
            Yo, To, _, sto, _ = om.reaction_step(Y[pick], T[pick], dt, nthreads=os.cpu_count() or 1)
            el = time.perf_counter() - t0
            acc = {}
            for form in forms:
                pos = np.searchsorted(res[form]["idx"], pick)
                dT = np.abs(res[form]["T"][pos] - To) / To
                dY = np.abs(res[form]["Y"][pos] - Yo).max(axis=1)
                acc[form] = {"against": "CPU oracle (FP64 restatement of the reference step), same cells",
                             "cells": int(len(pick)), "max_rel_T": float(dT.max()), "max_abs_Y": float(dY.max()),
                             "cells_within_abs_Y_1e-9": float((dY <= 1e-9).mean())}
            cpu = {"value": len(pick) / el, "unit": UNIT, "cores": os.cpu_count() or 1, "kind": "port",
                   "sample": f"{len(pick)} cells (seed 3) of the workload, one step, {el:.1f} s"}
        else:
            cpu = None
        for form in forms:
            res[form].pop("Y")
            res[form].pop("T")
            res[form].pop("idx")
        out = {"metric": METRIC, "value": res["mixed"]["value"], "unit": UNIT, "n_gpus": world, "steps": args.steps,
               "warmup": args.warmup, "ms_per_step": res["mixed"]["ms_per_call"] / nsteps, "higher_is_better": True,
               "scaling": "weak", "vs_baseline": None, "dtype": "f64+f32", "data": "synthetic",
               "config": {"workload": args.workload, "mechanism": f"{name} ({nc} species, {int(arrays['dims'][1])} "
                                                                 f"reactions)", "ncells_per_gpu": n, "dt": dt,
                          "steps_per_call": nsteps, "rtol": 1e-7, "atol": 1e-12,
                          "l2": "flushed (1 GiB write) before every timed call", "parallelism": f"replicas x{world}",
                          **({"sample": f"evenly strided {n} of the {mesh_cells}-cell mesh"}
                             if mesh_cells and n < mesh_cells else {}),
                          "warmup_calls": "the first min(cells, 256) cells of the batch" if nsteps == 1 else
                                          "the full call"},
               "forms": res, "ratio_vs_plain": res["mixed"]["value"] / res["plain"]["value"],
               "accuracy": acc, "cpu_baseline": cpu}
        print(json.dumps(out), flush=True)
    m.close()
    return 0


def main():
    args = parse()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime
        import torch.distributed as dist
        backend = "gloo" if args.impl == "reference" else "nccl"
        if backend == "nccl":
            import torch
            torch.cuda.set_device(local_rank)
        dist.init_process_group(backend=backend, timeout=datetime.timedelta(seconds=600))
    try:
        if args.impl == "reference":
            rc = run_reference(args, rank, world)
        elif args.workload != "h2co_uneven":
            rc = run_large(args, rank, world, local_rank)
        else:
            rc = run_ours(args, rank, world, local_rank)
    finally:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()
    return rc


if __name__ == "__main__":
    sys.exit(main())
