"""Benchmark: PDHG iterations/s of the projector on the bandwidth-roofline workload.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Workload (the largest single-GPU configuration): a synthetic 1,000,000 x
2,000,000 LP relaxation with 20,000,000 nonzeros, Zipf(1.5) row lengths capped
at 10,000 and rescaled to exactly 20M, U[-1, 1] values, half binary columns;
seeded synthetic data stands in for the MIPLIB instances the reference is
measured on.  One step is one projection to a relative KKT tolerance of 1e-4
(gap and dual residual 1e-4, primal residual 1e-5: the pump at its gap floor),
warm-started from the previous projection with 5% of the integer targets
flipped.  `value` = PDHG iterations of the timed projections / their device
time (CUDA events on the library's stream), mixed precision; the plain FP64
form is measured on the same sequence of targets and reported beside it.
With N > 1 every rank solves its own replica (a single projection does not
shard: each iteration would need an all-gather of x_bar and z) and `value` sums
iterations over ranks / max time.

--impl reference times the reference's own CPU algorithm (the C restatement
under oracle/, every host thread) on a bounded sample of the same workload:
each step projects the next target of the same sequence with the whole
pdfp_solve! loop (steps, evaluation windows, restart tests, PID), cut at
--cpu-iterations iterations (one evaluation window by default).

The default line also carries: the plain FP64 form on the same targets; the
mixed form's error per projection (`parity`); the step kernels' rooflines;
the same generator with a locality band (`zipf_lp_banded`); the batched
uneven projections (`batch_uneven`, config 3) and the markshare-shaped pumps
(`pump_markshare`, config 4); and a single-thread CPU baseline.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "PDHG iters/s and HBM GB/s, FP32+FP64 batched vs plain FP64 at 1e-4 KKT"
WORKLOAD = ("zipf-lp 1,000,000 x 2,000,000, 20,000,000 nnz, Zipf(1.5) rows capped at 10,000, "
            "U[-1,1] values, 50% binary; projections warm-started with 5% of integer targets "
            "flipped; eps_opt 1e-4, eps_feas 1e-5")


def log(*a):
    print(*a, file=sys.stderr, flush=True)


def dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600),
                                device_id=torch.device("cuda", local))
        from pdfp_b200 import gpu
        gpu.set_device(local)  # the library's own runtime selects the rank's GPU too
    return world, rank, local


def barrier(world):
    if world > 1:
        import torch
        import torch.distributed as dist
        torch.cuda.synchronize()
        dist.barrier()
        torch.cuda.synchronize()


def allreduce(world, value, op="max"):
    if world == 1:
        return value
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(value)], dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.MAX if op == "max" else dist.ReduceOp.SUM)
    return float(t.item())


class ClockSampler:
    """nvidia-smi clocks and throttle reasons during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.path = os.path.join(tempfile.gettempdir(), f"pdfp_bench_clocks_{os.getpid()}_{gpu_index}.csv")

    def __enter__(self):
        try:
            os.makedirs(os.path.dirname(self.path), exist_ok=True)
            self.fh = open(self.path, "w")
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-i", str(self.gpu), "-lms", "200"], stdout=self.fh, stderr=subprocess.DEVNULL)
        except (OSError, FileNotFoundError):
            self.proc = None
        return self

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
            self.fh.close()

    def summary(self):
        if self.proc is None or not os.path.exists(self.path):
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax.append(float(parts[2]))
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def bench_lib():
    """libpdfp_bench.so, the benchmark's measurement support (pdfp_measure_gather_rate)."""
    import ctypes as C
    L = C.CDLL(os.path.join(ROOT, "pdfp_b200", "lib", "libpdfp_bench.so"))
    L.pdfp_measure_gather_rate.restype = C.c_int
    L.pdfp_measure_gather_rate.argtypes = [C.c_int64, C.c_int32, C.c_int32, C.POINTER(C.c_double)]
    L.pdfp_bench_last_error.restype = C.c_char_p
    return L


def measured_hbm_peak():
    try:
        d = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
        return float(d["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback"


def build_workload(args, scaler="gpu", band=0):
    """The scaled projection problem (host arrays) and the first target.  `scaler` picks
    scale_problem on the GPU (our arm) or in the CPU oracle (the reference arm); band > 0
    builds the zipf-lp variant with locality (columns within +-band of the diagonal)."""
    from pdfp_b200 import synthetic
    t = time.time()
    if args.workload == "zipf-lp":
        milp, xf = synthetic.zipf_lp(seed=1, m=args.m, n=args.n, nnz=args.nnz, band=band)
    else:
        milp, _, _ = synthetic.general_integer(seed=1)
    log(f"[bench] generated {milp.A.shape} nnz={milp.A.nnz} in {time.time() - t:.1f}s")
    n = len(milp.c)
    con_lb = np.where(milp.is_eq, milp.b, -np.inf)
    t = time.time()
    if scaler == "gpu":
        from pdfp_b200 import gpu
        sc = gpu.scale_problem(milp.A, np.zeros(n), milp.l, milp.u, con_lb, milp.b,
                               bound_objective_rescaling=False)
    else:
        from oracle import oracle as O
        sc = O.scale_problem(milp.A, np.zeros(n), milp.l, milp.u, con_lb, milp.b,
                             bound_objective_rescaling=False)
    log(f"[bench] scaled ({scaler}) in {time.time() - t:.1f}s")
    w = np.ones(n)
    w[milp.int_idx] = sc.D_c[milp.int_idx]
    rng = np.random.Generator(np.random.PCG64(7))
    I = milp.int_idx
    xt0 = np.zeros(n)
    xt0[I] = np.round(np.clip(rng.random(len(I)) * (milp.u[I] - milp.l[I]) + milp.l[I],
                              milp.l[I], milp.u[I]))
    return milp, sc, w, xt0, I


def flip_targets(xt, I, milp, rng, frac=0.05):
    """Flip 5% of the integer targets (binary: 1 - v; general: move by one inside the bounds)."""
    xt = xt.copy()
    k = max(1, int(frac * len(I)))
    idx = I[rng.choice(len(I), size=k, replace=False)]
    up = np.minimum(xt[idx] + 1, milp.u[idx])
    dn = np.maximum(xt[idx] - 1, milp.l[idx])
    xt[idx] = np.where(up != xt[idx], up, dn)
    return xt


def host_kkt(prob, state, xt):
    """compute_residual! (src/pdfp.jl:200-218) re-evaluated in FP64 on the host from the
    solver's pdhg_x, pdhg_y, pdhg_z and dual_slack: (rel_primal, rel_dual, rel_gap)."""
    A, At, b, is_eq, is_int, w, D_c = prob
    xts = xt / D_c
    x, y, z, ds = (state.get(k) for k in ("pdhg_x", "pdhg_y", "pdhg_z", "dual_slack"))
    d = A @ x - b
    viol = np.where(is_eq, np.abs(d), np.maximum(d, 0.0))
    rel_p = np.linalg.norm(viol) / (1.0 + np.linalg.norm(b))
    rel_d = np.linalg.norm(At @ z - y - ds) / (1.0 + np.linalg.norm(np.where(is_int, w, 0.0)))
    l1 = np.sum(np.where(is_int, w * np.abs(x - xts), 0.0))
    yt = np.sum(np.where(is_int, y * (xts - x), 0.0))
    gap = abs(yt + z @ d - l1) / (1.0 + np.sum(np.where(is_int, w * np.abs(xts), 0.0)))
    return float(rel_p), float(rel_d), float(gap)


def run_projections(state, xt_seq, x_out, params, timed, kkt_prob=None):
    """Project each target as the pump does -- set_target(x_tilde ./ D_c) -> solve ->
    D_c .* pdhg_x, the scaling on the device -- and collect per-step figures.  The
    targets and x_out are page-locked host arrays.  With kkt_prob, each projection's
    KKT residuals are re-evaluated in FP64 on the host after its timed interval."""
    out = []
    for xt in xt_seq:
        t0 = time.perf_counter()
        state.set_target_unscaled(xt)
        state.solve(params, 1.0)
        x = state.get_unscaled("pdhg_x", out=x_out)
        t1 = time.perf_counter()
        r = state.last
        out.append({"iters": r["total_count"], "device_ms": r["device_ms"], "wall_s": t1 - t0,
                    "status": r["status"], "polished": r["polished"], "rel_gap": r["rel_gap"],
                    "fp64_iterations": r["fp64_iterations"], "l1": r["objective_value"],
                    "kernel_ms_primal": r["kernel_ms_primal"], "kernel_ms_dual": r["kernel_ms_dual"],
                    "kernel_samples": r["kernel_samples"], "x_sum": float(np.sum(x)),
                    "max_singular_value": r["max_singular_value"]})
        if kkt_prob is not None:
            out[-1]["host_kkt"] = host_kkt(kkt_prob, state, xt)
        if timed:
            log(f"[bench]   {r['status']} iters={r['total_count']} device={r['device_ms']:.1f}ms "
                f"wall={1e3 * (t1 - t0):.1f}ms polished={r['polished']} l1={r['objective_value']:.9g}")
    return out


def time_reference_form(sc, w, xt0, is_eq, is_int, warm=20, timed=200):
    """PDHG steps/s of the reference's own GPU step structure on the same problem:
    cuSPARSE SpMV with A', primal kernel, dual_y kernel, cuSPARSE SpMV with A, dual_z
    kernel, FP64 (src/pdfp_kernels.jl).  Steps only: no evaluation is charged to it."""
    from pdfp_b200 import refform
    r = refform.RefFormState(sc.A, sc.con_ub, is_eq, is_int, sc.var_lb, sc.var_ub, w)
    r.reset(xt0 / sc.D_c, np.zeros(len(xt0)))
    step = 0.998 / np.sqrt(2.0)
    r.steps(step, 1.0, 1, warm)
    ms = r.steps(step, 1.0, 1 + warm, timed)
    r.close()
    return {"value": round(timed / (ms * 1e-3), 1), "unit": "iters/s",
            "ms_per_iter": round(ms / timed, 5), "launches_per_iter": 5,
            "note": "steps only (no evaluation windows), FP64, cuSPARSE SpMV"}


def cpu_baseline(sc, w, xt0, is_eq, is_int, threads, iterations, label, max_sv):
    """The oracle's pdfp_solve! (src/pdfp.jl:252-288: steps, evaluation windows, restart
    tests, PID) on the same scaled problem and first target, cut at `iterations`
    iterations: iterations/s on `threads` host threads.  The ||A||_2 cache is seeded with
    the GPU run's estimate (the same algorithm's value), as a pump run has it after its
    first projection."""
    from oracle import oracle as O
    O.set_threads(threads)
    o = O.OraclePDFP(sc.A, sc.con_ub, is_eq, is_int, sc.var_lb, sc.var_ub, w)
    o.set_max_singular_value(max_sv)
    o.set_target(xt0 / sc.D_c)
    p = O.default_params(eps_optimal_relative=1e-4, eps_feasible_relative=1e-5,
                         iteration_limit=iterations)
    t = time.perf_counter()
    o.solve(p, 1.0)
    dt = time.perf_counter() - t
    return {"value": o.total_count / dt, "unit": "iters/s", "cores": threads, "kind": "port",
            "sample": f"the oracle's pdfp_solve! on the first target, {o.total_count} PDHG "
                      f"iterations with their evaluation and restart tests ({label}), {dt:.1f}s"}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", choices=["zipf-lp", "general-integer", "batch-uneven",
                                           "pump-markshare", "pump-p0201"], default="zipf-lp")
    ap.add_argument("--m", type=int, default=1_000_000)
    ap.add_argument("--n", type=int, default=2_000_000)
    ap.add_argument("--nnz", type=int, default=20_000_000)
    ap.add_argument("--no-fp64", action="store_true", help="skip the plain FP64 comparison")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--cpu-iterations", type=int, default=200,
                    help="PDHG iterations of the CPU baseline's sample (one evaluation window)")
    ap.add_argument("--no-extra", action="store_true",
                    help="skip the batch-uneven and pump-markshare figures of the default line")
    ap.add_argument("--no-refform", action="store_true",
                    help="skip the reference-structured FP64 step (cuSPARSE + 3 kernels)")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)

    world, rank, local = dist_setup()
    if args.impl == "reference":
        return reference_arm(args, world, rank)
    if args.workload == "batch-uneven":
        return batch_uneven(args, world, rank, local)
    if args.workload in PUMP_WORKLOADS:
        return pump_bench(args, world, rank)

    from pdfp_b200 import gpu
    from pdfp_b200.params import SolverParameters
    milp, sc, w, xt0, I = build_workload(args)
    is_eq, is_int = milp.is_eq, milp.is_int
    params = SolverParameters(eps_optimal_relative=1e-4, eps_feasible_relative=1e-5,
                              iteration_limit=2_000_000)
    rng = np.random.Generator(np.random.PCG64(11 + 0 * rank))
    seq = [xt0]
    for _ in range(args.warmup + args.steps - 1):
        seq.append(flip_targets(seq[-1], I, milp, rng))
    pinned = []  # the targets in page-locked host memory, as a caller would stage them
    for xt in seq:
        a = gpu.pinned_zeros(len(xt))
        a[:] = xt
        pinned.append(a)
    x_out = gpu.pinned_zeros(len(xt0))
    warm, timed = pinned[:args.warmup], pinned[args.warmup:]
    # the host FP64 re-evaluation of every timed mixed projection (outside its timed interval)
    kkt_prob = (sc.A, sc.A.T.tocsr(), sc.con_ub, is_eq, is_int, w, sc.D_c)

    results = {}
    for precision in (["mixed"] if args.no_fp64 else ["mixed", "fp64"]):
        t = time.time()
        st = gpu.PDFPState(sc.A, sc.con_ub, is_eq, is_int, sc.var_lb, sc.var_ub, w,
                           precision=precision)
        st.set_col_scale(sc.D_c)
        tun = (gpu.C.c_int32 * 8)()
        gpu.L.check(gpu.L.lib().pdfp_get_tuning(st._h, tun))
        stg = (gpu.C.c_int32 * 2)()
        gpu.L.check(gpu.L.lib().pdfp_get_tuning_stages(st._h, stg))
        tuning = {"a_t_stage_bytes": tun[0], "a_t_threads": tun[1], "a_t_tiles": tun[2],
                  "a_t_stages": stg[0], "a_stage_bytes": tun[3], "a_threads": tun[4],
                  "a_tiles": tun[5], "a_stages": stg[1], "a_t_gather_l2": tun[6],
                  "a_gather_l2": tun[7]}
        blk = (gpu.C.c_int32 * 2)()
        gpu.L.check(gpu.L.lib().pdfp_get_tuning_blocks(st._h, blk))
        tuning["a_t_blocks_per_sm_cap"] = blk[0]
        tuning["a_blocks_per_sm_cap"] = blk[1]
        red = (gpu.C.c_int32 * 2)()
        gpu.L.check(gpu.L.lib().pdfp_get_tuning_reducers(st._h, red))
        tuning["a_t_reducers"] = red[0]
        tuning["a_reducers"] = red[1]
        seg = (gpu.C.c_int32 * 2)()
        gpu.L.check(gpu.L.lib().pdfp_get_tuning_seg(st._h, seg))
        tuning["a_long_row_segments"] = seg[0]
        tuning["a_long_row_threshold"] = seg[1]
        tms = (gpu.C.c_float * 256)()
        tcfg = (gpu.C.c_int32 * (7 * 256))()
        cnt = gpu.C.c_int32()
        gpu.L.check(gpu.L.lib().pdfp_get_tuning_table(st._h, tms, tcfg, 256, gpu.C.byref(cnt)))
        for i in range(min(cnt.value, 256)):
            log(f"[bench]   tune side={['At', 'A', 'A+seg'][tcfg[7*i]]} stage={tcfg[7*i+1]} "
                f"nt={tcfg[7*i+2]} l2={tcfg[7*i+3]} stages={tcfg[7*i+4]} cap={tcfg[7*i+5]} "
                f"red={tcfg[7*i+6]}: {tms[i]*1e3:.1f} us")
        log(f"[bench] {precision} handle built in {time.time() - t:.1f}s, tuning {tuning}")
        run_projections(st, warm, x_out, params, False)
        gpu.L.check(gpu.L.lib().pdfp_set_kernel_timing(st._h, 1))
        barrier(world)
        with ClockSampler(local) as clk:
            steps = run_projections(st, timed, x_out, params, True,
                                    kkt_prob if precision == "mixed" else None)
        barrier(world)
        iters = sum(s["iters"] for s in steps)
        dev_s = sum(s["device_ms"] for s in steps) / 1e3
        wall_s = sum(s["wall_s"] for s in steps)
        max_dev = allreduce(world, dev_s, "max")
        max_wall = allreduce(world, wall_s, "max")
        tot_iters = allreduce(world, iters, "sum")
        kp = [s["kernel_ms_primal"] for s in steps if s["kernel_samples"]]
        kd = [s["kernel_ms_dual"] for s in steps if s["kernel_samples"]]
        results[precision] = {"tuning": tuning, "iters": iters, "tot_iters": tot_iters, "dev_s": max_dev,
                              "wall_s": max_wall, "steps": steps, "clocks": clk.summary(),
                              "kp_ms": float(np.mean(kp)) if kp else None,
                              "kd_ms": float(np.mean(kd)) if kd else None}
        if precision == "mixed":
            # the same sequence with both tolerances at 1e-4 (a secondary figure)
            loose = SolverParameters(eps_optimal_relative=1e-4, eps_feasible_relative=1e-4,
                                     iteration_limit=2_000_000)
            run_projections(st, warm, x_out, loose, False)
            barrier(world)
            ls = run_projections(st, timed, x_out, loose, False)
            barrier(world)
            l_dev = allreduce(world, sum(s["device_ms"] for s in ls) / 1e3, "max")
            l_its = allreduce(world, sum(s["iters"] for s in ls), "sum")
            results["loose"] = {"value": round(l_its / l_dev, 1), "unit": "iters/s",
                                "eps_optimal_relative": 1e-4, "eps_feasible_relative": 1e-4,
                                "iterations_per_step": [s["iters"] for s in ls],
                                "status_per_step": [s["status"] for s in ls]}
        del st

    # configs 3 and 4 of the metric: batched uneven projections and the small pumps
    extras = {}
    if args.workload == "zipf-lp" and not args.no_extra:
        extras["zipf_lp_banded"] = banded_variant(args, world, rank, local)
        sub = argparse.Namespace(**vars(args))
        sub.steps, sub.warmup = min(args.steps, 5), 3
        extras["batch_uneven"] = batch_uneven(sub, world, rank, local, embed=True)
        sub.workload = "pump-markshare"
        extras["pump_markshare"] = pump_bench(sub, world, rank, embed=True)
        if rank == 0:
            extras["p0201_published"] = p0201_published()

    refform_line = None
    if not args.no_refform:
        refform_line = time_reference_form(sc, w, xt0, is_eq, is_int)
        log(f"[bench] reference form (FP64, cuSPARSE + 3 kernels): {refform_line}")
    if rank != 0:
        barrier(world)
        return
    mx = results["mixed"]
    A = sc.A
    nnz, n, m = A.nnz, A.shape[1], A.shape[0]
    # algorithmic bytes per PDHG iteration (FP32): both sides read A once (4 B value + 4 B index),
    # row pointers once, every vector once (n-side 8 reads + 3 writes, m-side 3 + 1), and the
    # two gathered vectors once
    bytes_iter32 = 16.0 * nnz + 4.0 * (n + 1) + 4.0 * (m + 1) + 4.0 * 11 * n + 4.0 * 4 * m + 4.0 * (n + m)
    bytes_primal32 = 8.0 * nnz + 4.0 * (n + 1) + 4.0 * 11 * n + 4.0 * m
    value = mx["tot_iters"] / mx["dev_s"]
    peak, peak_kind = measured_hbm_peak()
    roof = None
    if mx["kp_ms"] and mx["kd_ms"]:
        # one entry per step kernel; `roofline` is the one that takes longer per launch
        bytes_dual32 = 8.0 * nnz + 4.0 * (m + 1) + 4.0 * 4 * m + 4.0 * n
        # DRAM bytes of one launch on the default workload, by engine, from ncu captures
        # (dram__bytes_read.sum + dram__bytes_write.sum)
        default = (args.workload, args.m, args.n, args.nnz) == ("zipf-lp", 1_000_000, 2_000_000,
                                                                20_000_000)
        traffic_ncu = {("PrimalOp", "tile"): 242.8e6, ("DualOp", "tile"): 187.9e6,
                       ("PrimalOp", "vec"): 250.2e6, ("DualOp", "vec"): 189.6e6}
        tun = mx["tuning"]

        seg = tun.get("a_long_row_segments", 0)

        def engine(op, threads):
            if op == "DualOp" and seg:
                return "tile+seg"
            return "flat" if threads == 0 else "vec" if threads == 32 else "tile"

        def kname(op, threads):
            if threads == 0:
                return f"flat_spmv_kernel<{op}<float, false, 256>>"
            if threads == 32:
                return f"vec_spmv_kernel<{op}<float, false, 256>>"
            name = f"tile_spmv_kernel<{op}<float, false, {threads}>>"
            if op == "DualOp" and seg:  # the A side in three launches
                name = (f"seg_partials_kernel<{op}<float, false, 256>> + seg_finish_kernel + "
                        f"{name} [rows of >= {tun['a_long_row_threshold']} nonzeros in "
                        f"{seg} column segments]")
            return name

        entries = []
        for label, op, threads, ms, byts in [
                ("A'z + fused primal/y update", "PrimalOp", tun["a_t_threads"], mx["kp_ms"],
                 bytes_primal32),
                ("A x_bar + fused z update", "DualOp", tun["a_threads"], mx["kd_ms"],
                 bytes_dual32)]:
            achieved = byts / (ms * 1e-3) / 1e9
            traffic = traffic_ncu.get((op, engine(op, threads))) if default else None
            entries.append({"bound": "hbm", "achieved": round(achieved, 1), "peak": peak,
                            "unit": "GB/s", "frac": round(achieved / peak, 4),
                            "traffic": traffic,
                            "kernel": f"{kname(op, threads)} ({label})", "peak_kind": peak_kind,
                            "bytes_per_launch": byts, "mean_launch_ms": round(ms, 5)})
        entries.sort(key=lambda e: -e["mean_launch_ms"])
        roof = dict(entries[0])
        roof["other_kernel"] = entries[1]
        # the sampled minor steps' two kernels against the whole PDHG iteration (every
        # step of every window, evaluation and controller included): at most 1
        ms_iter = 1e3 * mx["dev_s"] / max(mx["tot_iters"] / world, 1)
        roof["kernels_per_iteration_ms"] = round(mx["kp_ms"] + mx["kd_ms"], 5)
        roof["iteration_ms"] = round(ms_iter, 5)
        roof["kernel_share_of_iteration"] = round((mx["kp_ms"] + mx["kd_ms"]) / ms_iter, 4)
        roof["sampling"] = ("per evaluation window of the timed solves: CUDA events around a run "
                            "of its middle-half minor steps (no other event inside) give the mean "
                            "step time, split between the two kernels in the proportion measured "
                            "with events around each kernel of 8 single minor steps outside the run")
    line = {
        "metric": METRIC, "value": round(value, 1), "unit": "iters/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": round(1e3 * mx["dev_s"] / args.steps, 3), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32+f64", "data": "synthetic",
        "config": {"workload": WORKLOAD if args.workload == "zipf-lp" else "general-integer 20k x 50k",
                   "m": m, "n": n, "nnz": nnz, "precision": "mixed (FP32 iterates and SpMV, FP64 "
                   "reductions, restart logic and polish)", "parallelism": f"replicas x{world}",
                   "l2": ("inputs larger than L2 (~450 MB streamed per iteration)"
                          if args.workload == "zipf-lp" else
                          "L2-resident (~11 MB per iteration): no L2 flush between steps, the "
                          "roofline is reported but not a bound here"),
                   "tuning": mx["tuning"]},
        "hbm_gbs": round(bytes_iter32 * value / world / 1e9, 1),
        "iterations_per_step": [s["iters"] for s in mx["steps"]],
        "status_per_step": [s["status"] for s in mx["steps"]],
    }
    if "fp64" in results:
        fp = results["fp64"]
        fv = fp["tot_iters"] / fp["dev_s"]
        line["fp64_plain"] = {"value": round(fv, 1), "unit": "iters/s",
                              "ms_per_step": round(1e3 * fp["dev_s"] / args.steps, 3),
                              "iterations_per_step": [s["iters"] for s in fp["steps"]],
                              "kernel_primal_ms": fp["kp_ms"]}
        line["speedup_vs_fp64_plain"] = round(value / fv, 3)
        line["time_speedup_vs_fp64_plain"] = round(fp["dev_s"] / mx["dev_s"], 3)
    if "loose" in results:
        line["mixed_both_tolerances_1e-4"] = results["loose"]
    # the error of every timed mixed projection: its l1 distance against the plain FP64
    # form's (pinned to the oracle) on the same target, and its KKT residuals
    # re-evaluated in FP64 on the host
    kk = [s["host_kkt"] for s in mx["steps"] if "host_kkt" in s]
    par = {"tolerance": {"eps_optimal_relative": 1e-4, "eps_feasible_relative": 1e-5},
           "max_host_kkt": {"rel_primal": max(k[0] for k in kk), "rel_dual": max(k[1] for k in kk),
                            "rel_gap": max(k[2] for k in kk)} if kk else None,
           "fp64_iterations_in_mixed": sum(s["fp64_iterations"] for s in mx["steps"]),
           "polished_steps": sum(s["polished"] for s in mx["steps"])}
    if "fp64" in results:
        rels = [abs(a["l1"] - b["l1"]) / abs(b["l1"])
                for a, b in zip(mx["steps"], results["fp64"]["steps"])]
        par["max_rel_l1_vs_fp64"] = max(rels)
        par["mean_rel_l1_vs_fp64"] = float(np.mean(rels))
        par["reference"] = ("the plain FP64 form on the same targets and tolerance (it takes the "
                            "oracle's steps: same iteration counts, iterates within 1e-10)")
    line["parity"] = par
    if refform_line is not None:
        line["fp64_reference_form"] = refform_line
        line["speedup_vs_fp64_reference_form"] = round(value / refform_line["value"], 3)
    line["roofline"] = roof
    if mx["kp_ms"] and mx["kd_ms"]:
        # the ceiling that binds a scattered sparsity pattern: random 4-byte gathers, from a
        # vector of the size each kernel gathers from (A'z: z, m entries; A x_bar: x_bar, n)
        blib = bench_lib()

        def gather_peak(entries):
            grate = gpu.C.c_double()
            rc = blib.pdfp_measure_gather_rate((nnz // 4) * 4, entries, 20, gpu.C.byref(grate))
            if rc != 0:
                raise RuntimeError(f"pdfp_measure_gather_rate: {blib.pdfp_bench_last_error()}")
            return grate.value / 1e9

        peaks = {"PrimalOp": gather_peak(m), "DualOp": gather_peak(n)}
        ach = {"PrimalOp": nnz / (mx["kp_ms"] * 1e-3) / 1e9, "DualOp": nnz / (mx["kd_ms"] * 1e-3) / 1e9}
        dom = "PrimalOp" if mx["kp_ms"] >= mx["kd_ms"] else "DualOp"
        line["gather_roofline"] = {
            "bound": "random 4-byte gathers", "unit": "Ggathers/s", "peak": round(peaks[dom], 1),
            "kernel": dom, "achieved": round(ach[dom], 1), "frac": round(ach[dom] / peaks[dom], 4),
            "per_kernel": {k: {"achieved": round(v, 1), "peak": round(peaks[k], 1),
                               "frac": round(v / peaks[k], 4),
                               "vector_entries": m if k == "PrimalOp" else n}
                           for k, v in ach.items()},
            "peak_source": "pdfp_measure_gather_rate on this GPU (streamed indices, "
                           f"{(nnz // 4) * 4} gathers from an FP32 vector of the kernel's "
                           "gathered length)"}
    h2d = 8 * n * args.steps
    line["e2e"] = {"value": round(mx["tot_iters"] / mx["wall_s"], 1), "unit": "iters/s",
                   "h2d_bytes_per_step": 8 * n, "d2h_bytes_per_step": 8 * n,
                   "note": "set_target_unscaled (page-locked host -> device, x_tilde ./ D_c on "
                           "the device) + solve + D_c .* pdhg_x (device -> page-locked host) per "
                           "step, host wall clock"}
    windows = mx["iters"] // 200
    line["gpu_launches"] = int(windows * (2 * 200 + 10) + args.steps * 12)
    line["clocks"] = mx["clocks"]
    line.update(extras)
    if not args.no_cpu_baseline and world == 1:  # the host baseline is measured at N = 1 only
        t = time.time()
        line["cpu_baseline"] = cpu_baseline(sc, w, xt0, is_eq, is_int, 1, args.cpu_iterations,
                                            "single thread", mx["steps"][0]["max_singular_value"])
        log(f"[bench] cpu baseline in {time.time() - t:.1f}s")
    else:
        line["cpu_baseline"] = None
    print(json.dumps(line), flush=True)
    barrier(world)


def banded_variant(args, world, rank, local, band=4096, steps=3):
    """The zipf-lp workload with locality: the same generator with each row's columns
    within +-band of its diagonal position, so that a gather finds its neighbours'
    entries in L1.  Mixed form, a few warm-started projections in timing mode: the
    iteration rate and each step kernel's time and HBM fraction."""
    from pdfp_b200 import gpu
    from pdfp_b200.params import SolverParameters
    milp, sc, w, xt0, I = build_workload(args, band=band)
    params = SolverParameters(eps_optimal_relative=1e-4, eps_feasible_relative=1e-5,
                              iteration_limit=2_000_000)
    rng = np.random.Generator(np.random.PCG64(11))
    seq = [xt0]
    for _ in range(2 + steps - 1):
        seq.append(flip_targets(seq[-1], I, milp, rng))
    x_out = gpu.pinned_zeros(len(xt0))
    st = gpu.PDFPState(sc.A, sc.con_ub, milp.is_eq, milp.is_int, sc.var_lb, sc.var_ub, w,
                       precision="mixed")
    st.set_col_scale(sc.D_c)
    run_projections(st, seq[:2], x_out, params, False)
    gpu.L.check(gpu.L.lib().pdfp_set_kernel_timing(st._h, 1))
    barrier(world)
    out = run_projections(st, seq[2:], x_out, params, False)
    barrier(world)
    tun = st.tuning()
    del st
    nnz, n, m = sc.A.nnz, sc.A.shape[1], sc.A.shape[0]
    dev_s = allreduce(world, sum(s["device_ms"] for s in out) / 1e3, "max")
    its = allreduce(world, sum(s["iters"] for s in out), "sum")
    kp = float(np.mean([s["kernel_ms_primal"] for s in out]))
    kd = float(np.mean([s["kernel_ms_dual"] for s in out]))
    peak, peak_kind = measured_hbm_peak()
    bp = 8.0 * nnz + 4.0 * (n + 1) + 4.0 * 11 * n + 4.0 * m
    bd = 8.0 * nnz + 4.0 * (m + 1) + 4.0 * 4 * m + 4.0 * n
    return {"workload": f"zipf-lp with locality: columns within +-{band} of each row's diagonal "
                        "position, otherwise the headline generator", "precision": "mixed",
            "value": round(its / dev_s, 1), "unit": "iters/s", "steps": steps,
            "iterations_per_step": [s["iters"] for s in out],
            "kernel_ms": {"PrimalOp": round(kp, 5), "DualOp": round(kd, 5)},
            "hbm_frac": {"PrimalOp": round(bp / (kp * 1e-3) / 1e9 / peak, 4),
                         "DualOp": round(bd / (kd * 1e-3) / 1e9 / peak, 4)},
            "peak": peak, "peak_kind": peak_kind, "gather_policy": {"PrimalOp": tun[6], "DualOp": tun[7]}}


def batch_uneven(args, world, rank, local, embed=False):
    """64 uneven binary covering/packing projections packed into one batch handle.

    Instances: n log-uniform in [1000, 200000], m = 0.6 n, 10-40 nonzeros per row
    (seed 1, about 36M nonzeros in all).  One step projects a new target for every
    instance (5% of the previous targets flipped) to eps_opt 1e-4 / eps_feas 1e-5,
    each instance with its own restart and termination state.  value = PDHG
    iterations summed over instances / device time of the batched solves.
    """
    from pdfp_b200 import gpu, synthetic
    from pdfp_b200.params import SolverParameters
    t = time.time()
    models = synthetic.covering_packing_batch(seed=1 + rank)
    log(f"[bench] generated {len(models)} models, nnz={sum(mm.A.nnz for mm in models)} "
        f"in {time.time() - t:.1f}s")
    probs, scs, seqs = [], [], []
    rng = np.random.Generator(np.random.PCG64(13))
    for mm in models:
        n = len(mm.c)
        sc = gpu.scale_problem(mm.A, np.zeros(n), mm.l, mm.u, np.where(mm.is_eq, mm.b, -np.inf),
                               mm.b, bound_objective_rescaling=False)
        w = np.ones(n)
        w[mm.int_idx] = sc.D_c[mm.int_idx]
        probs.append((sc.A, sc.con_ub, mm.is_eq, mm.is_int, sc.var_lb, sc.var_ub, w))
        scs.append(sc)
        seq = [np.round(rng.random(n))]
        for _ in range(args.warmup + args.steps - 1):
            seq.append(flip_targets(seq[-1], mm.int_idx, mm, rng))
        pinned = []  # page-locked copies, as a caller would stage them
        for xt in seq:
            a = gpu.pinned_zeros(n)
            a[:] = xt
            pinned.append(a)
        seqs.append(pinned)
    params = SolverParameters(eps_optimal_relative=1e-4, eps_feasible_relative=1e-5,
                              iteration_limit=2_000_000)
    nnz = [p[0].nnz for p in probs]
    ns = [p[0].shape[1] for p in probs]
    ms = [p[0].shape[0] for p in probs]
    bytes32 = [16.0 * a + 52.0 * b + 24.0 * c for a, b, c in zip(nnz, ns, ms)]
    res = {}
    for precision in (["mixed"] if args.no_fp64 else ["mixed", "fp64"]):
        t = time.time()
        bt = gpu.PDFPBatch(probs, precision=precision)
        for p in range(len(probs)):
            bt.set_col_scale(p, scs[p].D_c)
        tun = (gpu.C.c_int32 * 8)()
        gpu.L.check(gpu.L.lib().pdfp_get_tuning(bt._h, tun))
        engine = {0: "flat", 32: "vec"}
        tuning = {"a_t_engine": engine.get(tun[1], "tile"), "a_t_stage_bytes": tun[0],
                  "a_t_threads": tun[1], "a_engine": engine.get(tun[4], "tile"),
                  "a_stage_bytes": tun[3], "a_threads": tun[4]}
        x_outs = [gpu.pinned_zeros(n) for n in ns]
        log(f"[bench] {precision} batch handle built in {time.time() - t:.1f}s")
        per = []
        for s in range(args.warmup + args.steps):
            if s == args.warmup:
                barrier(world)
                clk = ClockSampler(local).__enter__()
            w0 = time.perf_counter()
            for p in range(len(probs)):
                bt.set_target_unscaled(p, seqs[p][s])
            bt.solve(params, 1.0)
            xs = [bt.get_unscaled(p, "pdhg_x", out=x_outs[p]) for p in range(len(probs))]
            w1 = time.perf_counter()
            its = [r["total_count"] for r in bt.results]
            per.append({"iters": sum(its), "its": its, "device_ms": bt.results[0]["device_ms"],
                        "wall_s": w1 - w0, "bytes": sum(b * i for b, i in zip(bytes32, its)),
                        "status": sorted(set(r["status"] for r in bt.results)),
                        "x_sum": float(sum(np.sum(x) for x in xs))})
            if s >= args.warmup:
                log(f"[bench]   {precision} step iters={sum(its)} max={max(its)} "
                    f"device={per[-1]['device_ms']:.1f}ms status={per[-1]['status']}")
        clk.__exit__(None, None, None)
        barrier(world)
        timed = per[args.warmup:]
        dev_s = allreduce(world, sum(p["device_ms"] for p in timed) / 1e3, "max")
        wall_s = allreduce(world, sum(p["wall_s"] for p in timed), "max")
        iters = allreduce(world, sum(p["iters"] for p in timed), "sum")
        byts = allreduce(world, sum(p["bytes"] for p in timed), "sum")
        res[precision] = {"dev_s": dev_s, "wall_s": wall_s, "iters": iters, "bytes": byts,
                          "clocks": clk.summary(), "steps": timed, "tuning": tuning}
        bt.close()
    if rank != 0:
        return
    mx = res["mixed"]
    value = mx["iters"] / mx["dev_s"]
    peak, peak_kind = measured_hbm_peak()
    line = {"metric": METRIC, "value": round(value, 1), "unit": "iters/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": round(1e3 * mx["dev_s"] / args.steps, 3), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32+f64", "data": "synthetic",
            "config": {"workload": "batch-uneven: 64 binary covering/packing models, n log-uniform "
                       "[1000, 200000], m = 0.6 n, 10-40 nnz/row, one batch handle; eps_opt 1e-4, "
                       "eps_feas 1e-5 per instance", "instances": len(probs), "sum_n": sum(ns),
                       "sum_m": sum(ms), "sum_nnz": sum(nnz), "parallelism": f"replicas x{world}",
                       "l2": "inputs larger than L2", "tuning": mx["tuning"]},
            "hbm_gbs": round(mx["bytes"] / mx["dev_s"] / world / 1e9, 1),
            "hbm_frac": round(mx["bytes"] / mx["dev_s"] / world / 1e9 / peak, 4),
            "peak_kind": peak_kind,
            "iterations_per_step": [s["iters"] for s in mx["steps"]],
            "max_instance_iterations_per_step": [max(s["its"]) for s in mx["steps"]],
            "e2e": {"value": round(mx["iters"] / mx["wall_s"], 1), "unit": "iters/s",
                    "h2d_bytes_per_step": 8 * sum(ns), "d2h_bytes_per_step": 8 * sum(ns)},
            "clocks": mx["clocks"]}
    if "fp64" in res:
        fp = res["fp64"]
        line["fp64_plain"] = {"value": round(fp["iters"] / fp["dev_s"], 1), "unit": "iters/s",
                              "ms_per_step": round(1e3 * fp["dev_s"] / args.steps, 3),
                              "hbm_gbs_fp32_bytes": round(fp["bytes"] / fp["dev_s"] / world / 1e9, 1)}
        line["speedup_vs_fp64_plain"] = round(value / (fp["iters"] / fp["dev_s"]), 3)
        line["time_speedup_vs_fp64_plain"] = round(fp["dev_s"] / mx["dev_s"], 3)
    if embed:
        return line
    print(json.dumps(line), flush=True)


PUMP_WORKLOADS = {
    "pump-markshare": ("markshare_like",
                       "pump-markshare: 6 equality rows x (50 binaries + 6 slacks in [0,1000]), "
                       "U{0..99} coefficients, b = floor(rowsum/2), model seeds 1..32, pump seeds "
                       "101 and 201"),
    "pump-p0201": ("covering_p0201_like",
                   "pump-p0201: p0201-shaped binary covering, 133 x 201, 1923 nonzeros, "
                   "coefficients U{1..5}, b = 1 + floor(0.3 rowsum), c U{1..100}, model seeds "
                   "1..32, pump seeds 101 and 201 (flip_parameter 20, restart_period 100)"),
}


# The one run the reference publishes (README.md:36-48): p0201 on an NVIDIA H100 80GB
# HBM3, root LP "OPTIMAL after 600 iterations, 0.03 s", pump "FEASIBLE after 5
# iterations, 0.12 s", "root LP 0.03 s, projections 0.09 s, rounding 0.00 s".
P0201_PUBLISHED_S = {"total": 0.12, "root_lp": 0.03, "projection": 0.09, "root_lp_iterations": 600,
                     "pump_iterations": 5}


def p0201_published(runs: int = 12, warmup: int = 2):
    """The reference's published example run, on the real p0201 instance (the committed
    fixture tests/golden/p0201.npz, made from the reference's examples/p0201.mps.gz):
    the full pump with the drop-in FP64 solvers and the reference's default parameters,
    `runs` pump seeds after `warmup` untimed runs.  Wall-clock times as the reference's
    log reports them; its later pump iterations follow Julia's MersenneTwister draws,
    which this pump does not reproduce, so the iteration counts differ by seed."""
    import scipy.sparse as sp
    from pdfp_b200.milp import MILP
    from pdfp_b200.pump import feasibility_pump
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "tests", "golden", "p0201.npz")
    d = np.load(path)
    A = sp.csr_matrix((d["data"], d["indices"], d["indptr"]), shape=tuple(d["shape"]))
    milp = MILP(d["c"], float(d["c0"]), A, d["b"], ["eq" if e else "le" for e in d["is_eq"]],
                d["l"], d["u"], d["int_idx"], name=str(d["name"]))
    rows = []
    for seed in range(1, warmup + runs + 1):
        r = feasibility_pump(milp, time_limit=60.0, seed=seed, precision="fp64")
        if seed > warmup:
            rows.append(r)
    med = lambda xs: statistics.median(xs)  # noqa: E731
    ours = {"total_s": round(med([r.time for r in rows]), 5),
            "root_lp_s": round(med([r.root_lp_time for r in rows]), 5),
            "projection_s": round(med([r.projection_time for r in rows]), 5),
            "rounding_s": round(med([r.rounding_time for r in rows]), 5),
            "found": sum(r.found for r in rows), "runs": len(rows),
            "pump_iterations": sorted(r.iterations for r in rows),
            "root_lp_status": sorted(set(r.root_lp_status for r in rows))}
    log(f"[bench] p0201 (published run): {ours}")
    return {"workload": "p0201 (the reference's published example: 133 x 201, 1923 nonzeros), "
                        "full pump, FP64 drop-in form, reference defaults, pump seeds "
                        f"{warmup + 1}..{warmup + runs}",
            "ours_median": ours,
            "published_h100": {"total_s": P0201_PUBLISHED_S["total"],
                               "root_lp_s": P0201_PUBLISHED_S["root_lp"],
                               "projection_s": P0201_PUBLISHED_S["projection"],
                               "root_lp_iterations": P0201_PUBLISHED_S["root_lp_iterations"],
                               "pump_iterations": P0201_PUBLISHED_S["pump_iterations"],
                               "source": "reference README.md:36-48 (NVIDIA H100 80GB HBM3)"},
            "time_ratio_published_over_ours": {
                "total": round(P0201_PUBLISHED_S["total"] / ours["total_s"], 1),
                "root_lp": round(P0201_PUBLISHED_S["root_lp"] / ours["root_lp_s"], 1)}}


def pump_bench(args, world, rank, embed=False):
    """Time to first feasible of the pump on 32 small synthetic models.

    pump-markshare: 6 equality knapsack rows over 50 binaries with U{0..99}
    coefficients plus 6 slacks in [0, 1000].  pump-p0201: binary covering models of
    p0201's shape (133 x 201, 1923 nonzeros).  Model seeds 1..32.  Arms: two
    trajectories (pump seeds 101 and 201) batched in one projector handle in mixed
    precision, in lockstep (every pump iteration waits for both projections); the same
    two in FP64; the mixed pair with each trajectory advancing at its own pace
    (asynchronous); and the plain FP64 single-trajectory pump (seed 101), the drop-in
    form of the reference's GPU run.  Reported: p50/p90 of the wall time to the first feasible
    point, root LP and handle construction included.  Ranks split the model seeds.
    """
    from pdfp_b200 import is_feasible, synthetic
    from pdfp_b200.pump import feasibility_pump, feasibility_pump_batched
    gen_name, config_text = PUMP_WORKLOADS[args.workload]
    gen = getattr(synthetic, gen_name)
    seeds = [s for s in range(1, 33) if (s - 1) % world == rank]
    arms = {"mixed_batched": [], "fp64_batched": [], "mixed_batched_async": [], "fp64_plain": []}
    found = {k: 0 for k in arms}
    split = {k: [] for k in arms}  # (root LP, projections, rounding, pump iterations, PDHG iterations)

    def note(k, r, dt):
        arms[k].append(dt)
        split[k].append((r.root_lp_time, r.projection_time, r.rounding_time, r.iterations,
                         r.pdhg_iterations))
    warm = gen(1000)
    for _ in range(args.warmup):
        feasibility_pump_batched(warm, seeds=(101, 201), precision="mixed", time_limit=60,
                                 asynchronous=True)
        feasibility_pump_batched(warm, seeds=(101, 201), precision="mixed", time_limit=60)
        feasibility_pump(warm, seed=101, precision="fp64", time_limit=60)
    for s in seeds:
        m = gen(s)
        t = time.perf_counter()
        r, _ = feasibility_pump_batched(m, seeds=(101, 201), precision="mixed", time_limit=60)
        note("mixed_batched", r, time.perf_counter() - t)
        found["mixed_batched"] += int(r.found and is_feasible(m, r.x))
        t = time.perf_counter()
        r, _ = feasibility_pump_batched(m, seeds=(101, 201), precision="fp64", time_limit=60)
        note("fp64_batched", r, time.perf_counter() - t)
        found["fp64_batched"] += int(r.found and is_feasible(m, r.x))
        t = time.perf_counter()
        r, _ = feasibility_pump_batched(m, seeds=(101, 201), precision="mixed", time_limit=60,
                                        asynchronous=True)
        note("mixed_batched_async", r, time.perf_counter() - t)
        found["mixed_batched_async"] += int(r.found and is_feasible(m, r.x))
        t = time.perf_counter()
        r = feasibility_pump(m, seed=101, precision="fp64", time_limit=60)
        note("fp64_plain", r, time.perf_counter() - t)
        found["fp64_plain"] += int(r.found and is_feasible(m, r.x))
    if world > 1:
        import torch.distributed as dist
        gathered = [None] * world
        dist.all_gather_object(gathered, (arms, found, split))
        arms = {k: sum((g[0][k] for g in gathered), []) for k in arms}
        found = {k: sum(g[1][k] for g in gathered) for k in found}
        split = {k: sum((g[2][k] for g in gathered), []) for k in split}
    if rank != 0:
        return

    def pct(v, q):
        return round(1e3 * float(np.percentile(v, q)), 2)

    def med_split(rows, total):
        a = np.array(rows, dtype=np.float64)
        root, proj, rnd = (round(1e3 * float(np.median(a[:, i])), 2) for i in range(3))
        return {"root_lp_ms": root, "projection_ms": proj, "rounding_ms": rnd,
                "other_host_ms": round(1e3 * float(np.median(np.asarray(total) - a[:, 0] - a[:, 1]
                                                              - a[:, 2])), 2),
                "pump_iterations": float(np.median(a[:, 3])),
                "pdhg_iterations": float(np.median(a[:, 4]))}

    out = {k: {"p50_ms": pct(v, 50), "p90_ms": pct(v, 90), "found": found[k], "runs": len(v),
               "median_split": med_split(split[k], v)}
           for k, v in arms.items()}
    from oracle import oracle as O
    cpu, cpu_split = [], []
    for s in range(1, 9):
        m = gen(s)
        t = time.perf_counter()
        r, _ = feasibility_pump_batched(m, seeds=(101, 201), solvers=O.OracleSolvers(), time_limit=60)
        cpu.append(time.perf_counter() - t)
        cpu_split.append((r.root_lp_time, r.projection_time, r.rounding_time, r.iterations,
                          r.pdhg_iterations))
    line = {"metric": "time to first feasible, pump with 2 batched trajectories",
            "value": out["mixed_batched"]["p50_ms"], "unit": "ms (p50)", "n_gpus": world,
            "steps": len(arms["mixed_batched"]), "warmup": args.warmup,
            "higher_is_better": False, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32+f64", "data": "synthetic",
            "config": {"workload": config_text},
            "arms": out,
            "p90_speedup_vs_fp64_plain": round(out["fp64_plain"]["p90_ms"]
                                               / max(out["mixed_batched"]["p90_ms"], 1e-9), 3),
            "cpu_baseline": {"value": round(1e3 * float(np.median(cpu)), 2), "unit": "ms (p50)",
                             "cores": 1, "kind": "port",
                             "sample": "the same batched pump on the CPU oracle, model seeds 1..8",
                             "median_split": med_split(cpu_split, cpu)}}
    if embed:
        return line
    print(json.dumps(line), flush=True)


def reference_arm(args, world, rank):
    """The reference's CPU path (the oracle's C restatement of pdfp_solve!, every host
    thread) on the same workload: each step projects the next target of the same
    sequence as our arm (warm-started from the previous one) with the whole solve
    loop -- steps, evaluation windows, restart tests, PID -- cut at --cpu-iterations
    iterations (one evaluation window by default).  The first warm-up step fills the
    per-run ||A||_2 cache with the oracle's own power iteration (untimed)."""
    if rank != 0:
        return
    milp, sc, w, xt0, I = build_workload(args, scaler="oracle")
    threads = os.cpu_count() or 1
    per_step = max(1, args.cpu_iterations)
    from oracle import oracle as O
    O.set_threads(threads)
    rng = np.random.Generator(np.random.PCG64(11))
    seq = [xt0]
    for _ in range(args.warmup + args.steps - 1):
        seq.append(flip_targets(seq[-1], I, milp, rng))
    o = O.OraclePDFP(sc.A, sc.con_ub, milp.is_eq, milp.is_int, sc.var_lb, sc.var_ub, w)
    p = O.default_params(eps_optimal_relative=1e-4, eps_feasible_relative=1e-5,
                         iteration_limit=per_step)
    t = time.time()
    for xt in seq[:args.warmup]:
        o.set_target(xt / sc.D_c)
        o.solve(p, 1.0)
    log(f"[bench] reference warm-up (power iteration included) in {time.time() - t:.1f}s")
    iters = 0
    t = time.perf_counter()
    for xt in seq[args.warmup:]:
        o.set_target(xt / sc.D_c)
        o.solve(p, 1.0)
        iters += o.total_count
    dt = time.perf_counter() - t
    value = iters / dt
    line = {"impl": "reference", "metric": METRIC, "value": round(value, 3), "unit": "iters/s",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": round(1e3 * dt / args.steps, 3), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": WORKLOAD, "precision": "fp64 (the reference's CPU path)"},
            "cpu_baseline": {"value": round(value, 3), "unit": "iters/s", "cores": threads,
                             "kind": "port", "sample": f"per step, pdfp_solve! on the next "
                             f"target cut at {per_step} PDHG iterations (evaluation and restart "
                             "tests included), on the C restatement of the reference's CPU path, "
                             f"{threads} threads"},
            "e2e": {"value": round(value, 3), "unit": "iters/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def shutdown():
    try:
        import torch.distributed as dist
        if dist.is_available() and dist.is_initialized():
            dist.destroy_process_group()
    except Exception:  # noqa: BLE001
        pass


if __name__ == "__main__":
    try:
        main()
    finally:
        shutdown()
