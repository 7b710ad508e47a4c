#!/usr/bin/env python
"""Benchmark of the plain FP64 LU + solve (lu2's lumcolumn) on B200.

Workload (default): one dense FP64 system, N = 65536, block width nb = 256,
recursive panels down to 16 columns, partial pivoting; A and b from lu2's
seeded drand48 stream (randomsetmat, seed 1), generated on the device.  A
step is one factor + solve of that system.  The 34 GB matrix exceeds the
126 MB L2, so no flush is needed between steps.

value  : (2/3 N^3 + 2 N^2) / t, device-resident inputs, CUDA events, max over
         ranks; every step restores A from a pristine device copy (inside the
         timed region) and runs factor + back substitution.
e2e    : the same through the reference-facing C entry point lumcolumn() on
         pinned host buffers: host->device copy of A|b, factor, solve,
         device->host copy of the factors and x, all inside the timed region.
roofline: the trailing-update DGEMM (the dominant kernel), its algorithmic
         FLOPs over its CUDA-event time, against the FP64 DGEMM peak measured
         with cuBLAS (torch.matmul float64, 8192^3) in the same run.
cpu_baseline: the reference compiled from its own sources (oracle/_ref:
         lu2.c/lu2tlib.c/lu2lib.c + OpenBLAS), lumcolumn at N = 8192, all host
         cores.

forms  : BF16-LU + IR and FP8 + GMRES-IR on the diagonally dominant system,
         the batched form (20,000 small systems), and the host-pointer DGEMM
         (mydgemm at lu2's update shape, overlapped vs one pass).

--impl reference times that same reference CPU build on a bounded sample
(N = 8192) of the workload, on rank 0 only.
Multi-GPU (--gpus N under torchrun): the plain, BF16 and FP8 forms run as
independent replicas, one system per GPU (LU has no natural sharding at this
scope), weak scaling; the batched form splits its 20,000 systems over the GPUs
by cost (strong scaling), with no data exchange.
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

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "LU GFLOP/s at N=65536: FP64 vs BF16-LU+IR to FP64 residual; batched solves/s"
UNIT = "GFLOP/s"
REF_SAMPLE_N = 8192


def lu_flops(n: int) -> float:
    """Factor + solve FLOPs as the metric defines them: 2/3 N^3 + 2 N^2."""
    return 2.0 / 3.0 * n**3 + 2.0 * n**2


def trailing_flops(n: int, nb: int, nrhs: int = 1) -> float:
    """Algorithmic FLOPs of the top-level trailing updates C -= L21 U12."""
    f = 0.0
    for i in range(0, n, nb):
        w = min(nb, n - i)
        m_rows = n - i - w
        n_cols = n + nrhs - i - w
        f += 2.0 * m_rows * n_cols * w
    return f


def log(*a):
    print(*a, file=sys.stderr, flush=True)


class Clocks:
    """nvidia-smi sampling during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.path = None

    def start(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), "--query-gpu=" + self.Q,
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        rows = []
        for line in open(self.path):
            p = [s.strip() for s in line.split(",")]
            if len(p) < 9:
                continue
            try:
                rows.append((float(p[1]), float(p[2]), float(p[3]), p[5:9]))
            except ValueError:
                continue
        os.unlink(self.path)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        load = [r for r in rows if r[2] > 250.0] or rows
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in load for i, v in enumerate(r[3]) if v.lower() == "active"})
        return {"sm_mhz": statistics.median(r[0] for r in load), "sm_max_mhz": max(r[1] for r in rows),
                "power_w_median": statistics.median(r[2] for r in load), "samples": len(load),
                "reasons": reasons}


def cpu_model() -> str:
    try:
        for line in open("/proc/cpuinfo"):
            if line.startswith("model name"):
                return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def ref_run(ref, n, nb, seed, runs, orc=None):
    """median GFLOP/s of `runs` timed lumcolumn calls (after one untimed) and
    the HPL scaled residual of the last x"""
    ref.lumcolumn(n, nb, seed)
    ts, x = [], None
    for _ in range(runs):
        x, t = ref.lumcolumn(n, nb, seed)
        ts.append(t)
    out = {"gflops": lu_flops(n) / statistics.median(ts) / 1e9, "seconds_median": statistics.median(ts)}
    if orc is not None:
        out["hpl"] = orc.residual(orc.randomsetmat(n, seed), n, x)["hpl"]
    return out


def c1_baseline(cores: int, runs: int = 5) -> dict:
    """The reference CPU lu2 (nompi) on its own CPU-sized case, N = 2048, nb = 64:
    shipped and pivot-fixed builds, seeds 1 and 12345, OpenBLAS on every core
    with one OpenMP thread (the fastest split), median of `runs`; plus the
    default split (OpenMP and OpenBLAS both on every core), timed once."""
    from oracle.oracle import OracleLib, RefLib

    orc = OracleLib()
    out = {}
    for variant in ("shipped", "fixed"):
        ref = RefLib(variant)
        ref.set_threads(cores, 1)
        for seed in (1, 12345):
            r = ref_run(ref, 2048, 64, seed, runs, orc)
            out["c1_%s_s%d_gflops" % (variant, seed)] = r["gflops"]
            out["c1_%s_s%d_hpl" % (variant, seed)] = r["hpl"]
    ref = RefLib("shipped")
    ref.set_threads(cores, cores)
    _, t = ref.lumcolumn(2048, 64, 1)
    out["c1_shipped_s1_default_split_gflops"] = lu_flops(2048) / t / 1e9
    ref.set_threads(cores, 1)
    return out


def cpu_reference_gflops(n: int, nb: int, runs: int) -> dict:
    """The reference's own lumcolumn on the host cores (oracle/_ref): the
    bounded N = n sample of the workload (shipped build, the baseline of
    record; the pivot-fixed build beside it) and the N = 2048, nb = 64 case (c1_*)."""
    cores = os.cpu_count() or 1
    from oracle.oracle import OracleLib, RefLib

    if RefLib.available("shipped") and RefLib.available("fixed"):
        ref = RefLib("shipped")
        ref.set_threads(cores, 1)
        r = ref_run(ref, n, nb, 1, runs)
        fixed = RefLib("fixed")
        fixed.set_threads(cores, 1)
        rf = ref_run(fixed, n, nb, 1, runs)
        out = {"value": r["gflops"], "unit": UNIT, "cores": cores, "kind": "reference",
               "sample": "lu2 lumcolumn (lu2.c:1122) compiled from the reference sources + OpenBLAS 0.3.15, "
                         "N=%d nb=%d seed 1, OpenBLAS %d threads, 1 OpenMP thread, median of %d after an untimed "
                         "run; c1_*: N=2048 nb=64 median of 5" % (n, nb, cores, runs),
               "cpu": cpu_model(), "fixed_gflops": rf["gflops"]}
        out.update(c1_baseline(cores))
        return out
    orc = OracleLib()
    n2 = 2048
    a = orc.randomsetmat(n2, 1)
    t0 = time.perf_counter()
    orc.lumcolumn(a, n2, 64)
    t = time.perf_counter() - t0
    return {"value": lu_flops(n2) / t / 1e9, "unit": UNIT, "cores": 1, "kind": "port",
            "sample": "oracle restatement N=%d nb=64" % n2, "cpu": cpu_model()}


def fp64_peak(device) -> float:
    """cuBLAS DGEMM 8192^3 (torch.matmul float64), best of 5, TFLOP/s."""
    import torch

    n = 8192
    a = torch.rand((n, n), dtype=torch.float64, device=device)
    b = torch.rand((n, n), dtype=torch.float64, device=device)
    c = a @ b
    best = 1e9
    for _ in range(5):
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        torch.matmul(a, b, out=c)
        e1.record()
        torch.cuda.synchronize()
        best = min(best, e0.elapsed_time(e1) / 1e3)
    del a, b, c
    torch.cuda.empty_cache()
    return 2.0 * n**3 / best / 1e12


def read_profile_traffic():
    """Per-launch DRAM traffic of the trailing-update kernel, from the committed
    ncu summary (scaled to one full-size launch there), or None."""
    p = os.path.join(ROOT, "profiles", "dgemm_update_fp64.md")
    if not os.path.exists(p):
        return None
    for line in open(p):
        if line.startswith("traffic_bytes_per_launch_full_size:"):
            try:
                return float(line.split(":", 1)[1].strip())
            except ValueError:
                return None
    return None


def run_mixed(ctx, n, nb_fp64, ld, buf, dev, stream, args, barrier, max_over_ranks, t_fp64_step, world) -> dict:
    """BF16-LU + FP64 IR (lu2gpu_mixed_solve) on the diagonally dominant system
    of order n (lu2's stream with a_ii = sum_j |a_ij|), timed with CUDA events
    after args.warmup untimed solves; x compared with the plain FP64 GPU LU of
    the same system.  `buf` (n x ld FP64) is overwritten."""
    import numpy as np
    import torch

    import lu2_b200 as L

    nb = args.mixed_nb
    ctx.generate(buf, n, ld, 1, 1, kind=1)
    b = buf[:, n].clone()
    # FP64 reference solution of the same system (untimed)
    A = buf.clone()
    if ctx.lusolve(A, n, ld, nb_fp64, 1, L.PIVOT_PARTIAL) != 0:
        raise RuntimeError("FP64 reference solve hit a zero pivot")
    x64 = A[:, n].clone()
    del A
    torch.cuda.empty_cache()
    x = torch.zeros(n, dtype=torch.float64, device=dev)
    res = None
    for _ in range(args.warmup):
        res = ctx.mixed_solve(buf, n, ld, b, x, nb)
    barrier()
    torch.cuda.synchronize()
    ts, results = [], []
    for _ in range(args.steps):
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        res = ctx.mixed_solve(buf, n, ld, b, x, nb)
        e1.record(stream)
        torch.cuda.synchronize()
        ts.append(e0.elapsed_time(e1) / 1e3)
        results.append(res)
    t = max_over_ranks(sum(ts) / len(ts))
    err = ((x - x64).abs().max() / x64.abs().max()).item()
    # per-phase split of one more (untimed) solve
    ctx.set_timing(True)
    ctx.mixed_solve(buf, n, ld, b, x, nb)
    timers = ctx.timers()
    ctx.set_timing(False)
    upd_ms = timers["DGEMMrest"][0]
    # algorithmic HBM bytes of the BF16 trailing updates: FP32 C read + written
    # (8 B) per element per panel plus the BF16 operands (2 B each per element)
    upd_bytes = 0.0
    for i in range(0, n, nb):
        w = min(nb, n - i)
        m_rows, n_cols = n - i - w, n - i - w
        upd_bytes += 8.0 * m_rows * n_cols + 2.0 * w * (m_rows + n_cols)
    value = world * lu_flops(n) / t / 1e9
    return {"metric": "FP64-equivalent GFLOP/s (2/3 N^3 + 2 N^2)/t", "value": value, "seconds": t,
            "speedup_vs_fp64_plain": t_fp64_step / t, "n": n, "nb": nb,
            "matrix": "lu2 drand48 stream, seed 1, diagonal a_ii = sum_j |a_ij| (diagonally dominant)",
            "iterations": results[-1]["iterations"], "hpl_residual": results[-1]["hpl"],
            "factor_s": results[-1]["factor_s"], "refine_s": results[-1]["refine_s"],
            "x_rel_err_vs_fp64_lu": err, "steps": len(ts), "warmup": args.warmup,
            "bf16_update": {"ms": upd_ms, "launches": timers["DGEMMrest"][1],
                            "hbm_gbs": upd_bytes / (upd_ms / 1e3) / 1e9 if upd_ms > 0 else None,
                            "algorithmic_bytes": upd_bytes},
            "phases_ms": {k: {"ms": v[0], "launches": v[1]} for k, v in timers.items()}}


def run_batched(ctx, dev, stream, args, max_over_ranks, world, rank=0) -> dict:
    """Batching form: 20,000 systems, N log-uniform in [16, 512]
    (seed 1), 10% with 8 right-hand sides, each lu2's stream with seed 1+i; FP64,
    one persistent launch replayed from a CUDA graph, launch shape autotuned.
    Compared with a loop of single plain-method solves (lu2gpu_lusolve, nb=64)
    over a sample of the same systems."""
    import numpy as np
    import torch

    import lu2_b200 as L

    count = args.batch_count
    n_all, r_all = L.batch_sizes(count, 1, 16, 512, 0.1, 8)
    # on N GPUs every rank solves its cost-balanced share of the same systems
    idx = L.batch_shard(n_all, r_all, world, rank) if world > 1 else np.arange(count)
    n, r = n_all[idx], r_all[idx]
    b = L.Batch(ctx, n, r)
    b.generate_seeds(1 + idx)
    b.snapshot()
    flops = float(np.sum(2.0 / 3.0 * n_all.astype(np.float64) ** 3 + 2.0 * n_all.astype(np.float64) ** 2 * r_all))

    def timed():
        """autotune, warm up, time args.steps solves (inputs restored untimed)"""
        cfg = b.autotune()
        for _ in range(args.warmup):
            b.restore()
            b.solve()
        ts = []
        for _ in range(args.steps):
            b.restore()
            torch.cuda.synchronize()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            info = b.solve()
            e1.record(stream)
            torch.cuda.synchronize()
            ts.append(e0.elapsed_time(e1) / 1e3)
        return cfg, max_over_ranks(sum(ts) / len(ts)), info, b.residuals(), len(ts)

    # FP32 factors + FP64 refinement first, then the plain FP64 variant
    b.set_mode(L.BATCH_FP32_IR, 10)
    cfg_ir, t_ir, info_ir, res_ir, _ = timed()
    its = b.iterations()
    hmax_ir = max_over_ranks(float(res_ir.max()))
    fp32_ir = {"value": count / t_ir, "unit": "systems/s", "seconds": t_ir,
               "fp64_equivalent_gflops": flops / t_ir / 1e9, "max_hpl_residual": hmax_ir,
               "all_below_16": hmax_ir < 16, "zero_pivots_max_per_rank": max_over_ranks(float((info_ir != 0).sum())),
               "refinement_iterations": {"mean": float(its.mean()), "max": int(max_over_ranks(float(its.max())))},
               "autotuned": cfg_ir}
    b.set_mode(L.BATCH_FP64)
    cfg, t, info, res, nsteps = timed()
    hmax = max_over_ranks(float(res.max()))
    # the loop of single plain-method launches, on a sample of this rank's systems
    rng = np.random.default_rng(0)
    sample = rng.choice(len(idx), size=min(args.batch_loop_sample, len(idx)), replace=False)
    b.restore()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for i in sample:
        ptr, ld = b.system(int(i))
        ctx.lusolve(ptr, int(n[i]), ld, 64, int(r[i]), L.PIVOT_PARTIAL)
    torch.cuda.synchronize()
    t_loop = max_over_ranks((time.perf_counter() - t0) / len(sample))
    b.close()
    sps = count / t
    return {"metric": "batched solves/s", "value": sps, "unit": "systems/s", "seconds": t, "systems": count,
            "gflops": flops / t / 1e9, "flops": flops,
            "scaling": "strong" if world > 1 else None,
            "sharding": "cost-balanced split of the same %d systems over %d GPUs, no data exchange" % (count, world),
            "sizes": "N log-uniform in [16, 512] (seed 1), 10% with 8 right-hand sides, entries lu2 stream seed 1+i",
            "max_hpl_residual": hmax, "all_below_16": hmax < 16,
            "zero_pivots_max_per_rank": max_over_ranks(float((info != 0).sum())), "autotuned": cfg, "steps": nsteps,
            "warmup": args.warmup,
            "loop_baseline": {"solves_per_s": world / t_loop, "sample_systems_per_rank": int(len(sample)),
                              "api": "lu2gpu_lusolve per system (nb=64), host-timed loop on every GPU"},
            "speedup_vs_loop": sps / (world / t_loop), "fp32_lu_fp64_ir": fp32_ir}


def event_median(fn, stream, reps=5, warm=2) -> float:
    """median CUDA-event seconds of fn() on `stream` after `warm` untimed calls"""
    import torch

    for _ in range(warm):
        fn()
    torch.cuda.synchronize()
    ts = []
    for _ in range(reps):
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        fn()
        e1.record(stream)
        torch.cuda.synchronize()
        ts.append(e0.elapsed_time(e1) / 1e3)
    return statistics.median(ts)


def run_swap_profile(ctx, n, nb, dev, stream, rows=None, reps=5) -> dict:
    """The top-level row exchange of the first panel (lu2.c:541-554): pivots of
    rows 0..nb-1 drawn uniformly from the rows below (as partial pivoting on a
    random matrix picks them) applied to columns nb..n of a matrix of `rows`
    rows (default n) and row stride n+16.  Algorithmic bytes: every row the
    exchanges touch is read once and written once over the width."""
    import numpy as np
    import torch

    rows = rows or n
    ld = n + 16
    a = torch.empty((rows, ld), dtype=torch.float64, device=dev)
    a.uniform_(-0.5, 0.5)
    rng = np.random.default_rng(1)
    piv = np.array([rng.integers(k, rows) for k in range(nb)], dtype=np.int32)
    touched = len(set(range(nb)) | set(int(p) for p in piv))
    dpiv = torch.tensor(piv, device=dev)
    dinv = torch.full((nb,), 1.0, dtype=torch.float64, device=dev)
    width = n + 1 - nb
    t = event_median(lambda: ctx.swaprows(a, rows, ld, 0, nb, dpiv, dinv, nb, n + 1), stream, reps)
    moved = 2.0 * 8 * touched * width
    return {"profile_swap": {"n": n, "rows": rows, "nb": nb, "rows_touched": touched, "width": width, "seconds": t,
                             "algorithmic_bytes": moved, "gbs": moved / t / 1e9}}


def run_trsm_profile(ctx, n, nb, dev, stream, reps=5) -> dict:
    """The top-level block-row solve of the first panel (lu2.c:485-521): L11
    the unit lower triangle of a factored nb x nb panel, X an nb x (n+1-nb)
    block of the matrix (row stride n+16), -X^T written to a separate buffer.
    Algorithmic work: nb^2 (n+1-nb) FLOPs (a triangular solve), bytes: X read
    and written and -X^T written once."""
    import torch

    import numpy as np
    import scipy.linalg as sl

    ld = n + 16
    width = n + 1 - nb
    # L11 of an LU with partial pivoting (|l| <= 1), factored on the host so
    # that the only solve launches are the measured ones
    _, lo, _ = sl.lu(np.random.default_rng(3).uniform(-0.5, 0.5, (nb, nb)))
    t_host = np.zeros((nb, nb + 16))
    t_host[:, :nb] = np.tril(lo, -1)
    t_blk = torch.tensor(t_host, device=dev)
    x = torch.empty((nb, ld), dtype=torch.float64, device=dev)
    x.uniform_(-0.5, 0.5)
    x0 = x.clone()
    bt = torch.empty((width, nb), dtype=torch.float64, device=dev)

    def fn():
        x.copy_(x0)
        ctx.solve_triangle(nb, t_blk, nb + 16, x[:, nb:], ld, width, bt)

    t_copy = event_median(lambda: x.copy_(x0), stream, reps)
    t = event_median(fn, stream, reps) - t_copy
    flops = float(nb) * nb * width
    moved = 3.0 * 8 * nb * width
    return {"profile_trsm": {"n": n, "nb": nb, "width": width, "seconds": t, "flops": flops,
                             "tflops": flops / t / 1e12, "algorithmic_bytes": moved, "gbs": moved / t / 1e9}}


def run_backsolve_profile(ctx, n, nb, dev, stream, reps=5) -> dict:
    """backward_sub (lu2.c:110-116) alone on a factored order-n system: the
    upper triangle (8 n^2 / 2 bytes) read once per solve."""
    import torch

    import lu2_b200 as L

    ld = L.device_ld(n)
    a = torch.empty((n, ld), dtype=torch.float64, device=dev)
    ctx.generate(a, n, ld, 1)
    if ctx.factor(a, n, ld, nb, 1, L.PIVOT_PARTIAL) != 0:
        raise RuntimeError("zero pivot")
    y = a[:, n].clone().reshape(n, 1).contiguous()
    x = y.clone()

    def fn():
        x.copy_(y)
        ctx.backsolve(a, n, ld, x, 1, 1)

    t = event_median(fn, stream, reps) - event_median(lambda: x.copy_(y), stream, reps)
    moved = 8.0 * n * n / 2
    return {"profile_backsolve": {"n": n, "seconds": t, "algorithmic_bytes": moved, "gbs": moved / t / 1e9}}


def headline(value, hplres, e2e, roofline, forms) -> dict:
    """The figures of every form in one short object, printed last on the line."""
    h = {"fp64_gflops": round(value, 1), "fp64_hpl": hplres, "dgemm_frac_of_cublas": round(roofline["frac"], 4)}
    if e2e:
        h["e2e_pinned_gflops"] = round(e2e["value"], 1)
        if "pageable_value" in e2e:
            h["e2e_pageable_gflops"] = round(e2e["pageable_value"], 1)
    m = forms.get("bf16_ir")
    if m:
        h.update({"bf16_ir_gflops": round(m["value"], 1), "bf16_ir_speedup_vs_fp64": round(m["speedup_vs_fp64_plain"], 3),
                  "bf16_ir_iterations": m["iterations"], "bf16_ir_hpl": m["hpl_residual"],
                  "bf16_ir_x_err_vs_fp64": m["x_rel_err_vs_fp64_lu"]})
    f = forms.get("fp8_gmres_ir")
    if f:
        dd = [v for k, v in f.items() if k.startswith("diagonally_dominant_n")]
        gen = [v for k, v in f.items() if k.startswith("general_n")]
        chk = [v for k, v in f.items() if k.startswith("check_n")]
        if dd:
            h.update({"fp8_dd_gflops": round(dd[0]["value"], 1), "fp8_dd_gmres_iters": dd[0]["gmres_iterations"],
                      "fp8_dd_hpl": dd[0]["hpl_residual"]})
        if gen:
            h.update({"fp8_general_converged": gen[0]["converged"], "fp8_general_hpl": gen[0]["hpl_residual"]})
            fac = gen[0].get("factors")
            if fac:
                h["fp8_general_factors_finite"] = fac["factors_finite"]
                h["fp8_general_pivot_max_last_quarter"] = fac["pivot_max_by_quarter"][-1]
        if chk:
            h["fp8_fwd_err_dd"] = chk[0]["diagonally_dominant"]["fwd_err_vs_fp64"]
            h["fp8_fwd_err_general"] = chk[0]["general"]["fwd_err_vs_fp64"]
    b = forms.get("batched_fp64")
    if b:
        h.update({"batched_fp64_systems_s": round(b["value"]), "batched_fp64_max_hpl": b["max_hpl_residual"],
                  "batched_speedup_vs_loop": round(b["speedup_vs_loop"], 1),
                  "batched_fp32ir_systems_s": round(b["fp32_lu_fp64_ir"]["value"]),
                  "batched_fp32ir_max_hpl": b["fp32_lu_fp64_ir"]["max_hpl_residual"]})
    d = forms.get("host_dgemm")
    if d:
        h["host_dgemm_overlap_speedup"] = round(d["speedup"], 3)
    return h


def fp8_update_bytes(n: int, nb: int) -> float:
    """Algorithmic HBM bytes of the FP8 trailing updates of an order-n factorization:
    FP32 C read and written (8 B per element) plus the E4M3 operands (1 B each)."""
    tot = 0.0
    for i in range(0, n, nb):
        w = min(nb, n - i)
        m = n - i - w
        tot += 8.0 * m * m + 1.0 * w * 2 * m
    return tot


def run_host_dgemm(max_over_ranks, barrier) -> dict:
    """The board-replacement DGEMM on host pointers (mydgemm, lu2lib.c:2079;
    gdr_dgemm_ underneath): lu2's trailing-update shape C -= L21 U12 with
    M = N = 16384, K = 256, row-major, every operand in pinned host memory;
    overlapped (C in column blocks through three streams) against one pass
    (LU2GPU_DGEMM_OVERLAP=0: copies in, product, copy out)."""
    import numpy as np
    import torch

    import lu2_b200 as L

    m = n = 16384
    k = 256
    na = nb = nc = n + 16
    a = torch.empty((m, na), dtype=torch.float64, pin_memory=True).numpy()
    b = torch.empty((k, nb), dtype=torch.float64, pin_memory=True).numpy()
    c = torch.empty((m, nc), dtype=torch.float64, pin_memory=True).numpy()
    rng = np.random.default_rng(3)
    a[...] = rng.uniform(-0.5, 0.5, a.shape)
    b[...] = rng.uniform(-0.5, 0.5, b.shape)
    c.fill(0.25)
    flops = 2.0 * m * n * k
    moved = 8.0 * (m * k + k * n + 2 * m * n)
    out = {"shape": "row-major C[16384][16384] -= A[16384][256] B[256][16384], pinned host operands",
           "api": "mydgemm (lu2lib.h) on host pointers"}
    for label, env in (("overlapped", "1"), ("one_pass", "0")):
        os.environ["LU2GPU_DGEMM_OVERLAP"] = env
        ts = []
        for it in range(4):
            barrier()
            t0 = time.perf_counter()
            L.mydgemm(m, n, k, -1.0, a, na, b, nb, 1.0, c, nc)
            ts.append(time.perf_counter() - t0)
        s = max_over_ranks(float(np.median(ts[1:])))
        out[label] = {"seconds": s, "gflops": flops / s / 1e9, "pcie_gbs": moved / s / 1e9}
    os.environ.pop("LU2GPU_DGEMM_OVERLAP", None)
    out["speedup"] = out["one_pass"]["seconds"] / out["overlapped"]["seconds"]
    log("host dgemm: overlapped %.1f ms, one pass %.1f ms" % (1e3 * out["overlapped"]["seconds"],
                                                               1e3 * out["one_pass"]["seconds"]))
    return out


def lowp_diagnostics(ctx, a, n, ld, nb, update, dev) -> dict:
    """The precision form's factors of a (lu2gpu_lowp_factor): whether they are
    finite (the first column holding a non-finite value), and the median and
    largest |pivot| of each quarter of the factorization (E4M3 noise makes the
    pivots grow away from the FP32 factorization's)."""
    import torch

    f = torch.empty((n, n), dtype=torch.float32, device=dev)
    rc = ctx.lowp_factor(a, n, ld, nb, update, f, n)
    first_bad = None
    for c0 in range(0, n, 4096):
        ok = torch.isfinite(f[:, c0:c0 + 4096]).all(dim=0)
        if not bool(ok.all()):
            first_bad = c0 + int((~ok).nonzero()[0])
            break
    piv = f.diagonal().abs().double()
    q = n // 4
    out = {"status": rc, "factors_finite": first_bad is None, "first_nonfinite_column": first_bad,
           "pivot_median_by_quarter": [float(piv[i:i + q].median()) for i in range(0, 4 * q, q)],
           "pivot_max_by_quarter": [float(piv[i:i + q].max()) for i in range(0, 4 * q, q)]}
    del f, piv
    torch.cuda.empty_cache()
    return out


def run_fp8(ctx, dev, stream, args, max_over_ranks, world) -> dict:
    """FP8 form: lu2's factorization of an FP32 copy with E4M3 trailing updates
    (per-128x128-tile power-of-two scales, FP32 accumulation), then GMRES-IR
    (restart 30) in FP64.  Forward error against the plain FP64 GPU solve at
    N = args.fp8_check_n (general and diagonally dominant matrices); timed solve
    of the diagonally dominant matrix at N = args.fp8_n; the general matrix at
    N = args.fp8_n with a bounded GMRES iteration budget."""
    import torch

    import lu2_b200 as L

    out = {"update": "FP8 E4M3 operands, per-128x128-tile power-of-two scales, FP32 accumulation (tcgen05 "
                     "kind::f8f6f4); FP32 panel; GMRES(30)-IR in FP64 preconditioned by the FP32/FP8 factors",
           "nb": args.fp8_nb}
    nb = args.fp8_nb

    def system(n, kind):
        ld = L.device_ld(n)
        a = torch.empty((n, ld), dtype=torch.float64, device=dev)
        ctx.generate(a, n, ld, 1, 1, kind=kind)
        return a, ld, a[:, n].clone()

    # forward error against the plain FP64 solve of the same system
    nc = args.fp8_check_n
    checks = {}
    for kind, name in ((0, "general"), (1, "diagonally_dominant")):
        a, ld, b = system(nc, kind)
        a64 = a.clone()
        if ctx.lusolve(a64, nc, ld, 256, 1, L.PIVOT_PARTIAL) != 0:
            raise RuntimeError("FP64 reference solve hit a zero pivot")
        x64 = a64[:, nc].clone()
        del a64
        x = torch.zeros(nc, dtype=torch.float64, device=dev)
        res = ctx.gmres_solve(a, nc, ld, b, x, nb, update=L.UPDATE_FP8, restart=30,
                              max_iter=args.fp8_general_iters)
        res["fwd_err_vs_fp64"] = ((x - x64).abs().max() / x64.abs().max()).item()
        res["converged"] = res.pop("status") == 0
        res["factors"] = lowp_diagnostics(ctx, a, nc, ld, nb, L.UPDATE_FP8, dev)
        checks[name] = res
        del a, b, x, x64
        torch.cuda.empty_cache()
    out["check_n%d" % nc] = checks

    n = args.fp8_n
    a, ld, b = system(n, 1)
    x = torch.zeros(n, dtype=torch.float64, device=dev)
    for _ in range(args.fp8_warmup):
        ctx.gmres_solve(a, n, ld, b, x, nb, update=L.UPDATE_FP8, restart=30, max_iter=100)
    torch.cuda.synchronize()
    ts, res = [], None
    for _ in range(args.fp8_steps):
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        res = ctx.gmres_solve(a, n, ld, b, x, nb, update=L.UPDATE_FP8, restart=30, max_iter=100)
        e1.record(stream)
        torch.cuda.synchronize()
        ts.append(e0.elapsed_time(e1) / 1e3)
    t = max_over_ranks(sum(ts) / len(ts))
    ctx.set_timing(True)
    ctx.gmres_solve(a, n, ld, b, x, nb, update=L.UPDATE_FP8, restart=30, max_iter=100)
    timers = ctx.timers()
    ctx.set_timing(False)
    upd_ms = timers["DGEMMrest"][0]
    upd_bytes = fp8_update_bytes(n, nb)
    out["diagonally_dominant_n%d" % n] = {
        "metric": "FP64-equivalent GFLOP/s (2/3 N^3 + 2 N^2)/t", "value": world * lu_flops(n) / t / 1e9,
        "seconds": t, "steps": len(ts), "warmup": args.fp8_warmup, "converged": res["status"] == 0,
        "refinements": res["refinements"], "gmres_iterations": res["gmres_iterations"], "hpl_residual": res["hpl"],
        "factor_s": res["factor_s"], "refine_s": res["refine_s"],
        "fp8_update": {"ms": upd_ms, "launches": timers["DGEMMrest"][1], "algorithmic_bytes": upd_bytes,
                       "hbm_gbs": upd_bytes / (upd_ms / 1e3) / 1e9 if upd_ms > 0 else None},
        "phases_ms": {k: {"ms": v[0], "launches": v[1]} for k, v in timers.items()}}
    del a, b, x
    torch.cuda.empty_cache()

    a, ld, b = system(n, 0)
    x = torch.zeros(n, dtype=torch.float64, device=dev)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    res = ctx.gmres_solve(a, n, ld, b, x, nb, update=L.UPDATE_FP8, restart=30, max_iter=args.fp8_general_iters)
    e1.record(stream)
    torch.cuda.synchronize()
    out["general_n%d" % n] = {"converged": res["status"] == 0, "hpl_residual": res["hpl"],
                              "gmres_iterations": res["gmres_iterations"], "iteration_budget": args.fp8_general_iters,
                              "refinements": res["refinements"], "preconditioner_output_finite": res["finite_factors"],
                              "factor_s": res["factor_s"],
                              "refine_s": res["refine_s"], "seconds": e0.elapsed_time(e1) / 1e3}
    del x
    torch.cuda.empty_cache()
    out["general_n%d" % n]["factors"] = lowp_diagnostics(ctx, a, n, ld, nb, L.UPDATE_FP8, dev)
    del a, b
    torch.cuda.empty_cache()
    return out


def run_reference(args, rank: int) -> None:
    if rank != 0:
        return
    from oracle.oracle import RefLib

    cores = os.cpu_count() or 1
    n, nb = REF_SAMPLE_N, args.nb
    if not RefLib.available("shipped"):
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref (the compiled reference) not present"}))
        return
    c1 = c1_baseline(cores)
    ref = RefLib("shipped")
    ref.set_threads(cores, 1)
    for _ in range(args.warmup):
        ref.lumcolumn(n, nb, 1)
    ts = []
    for _ in range(args.steps):
        _, t = ref.lumcolumn(n, nb, 1)
        ts.append(t)
    tot = sum(ts)
    value = args.steps * lu_flops(n) / tot / 1e9
    sample = ("lu2 lumcolumn compiled from the reference sources (lu2.c, lu2tlib.c, lu2lib.c) + OpenBLAS 0.3.15, "
              "N=%d nb=%d seed 1 per step (bounded sample of the N=%d workload), %d threads" % (n, nb, args.n, cores))
    out = {"metric": METRIC, "value": value, "unit": UNIT, "impl": "reference", "n_gpus": args.gpus,
           "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * tot / args.steps,
           "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
           "config": {"workload": "plain FP64 LU+solve (reference CPU lu2), N=%d sample of N=%d, nb=%d" %
                                  (n, args.n, nb), "n": n, "nb": nb, "seed": 1},
           "cpu_baseline": dict({"value": value, "unit": UNIT, "cores": cores, "kind": "reference", "sample": sample,
                                 "cpu": cpu_model()}, **c1),
           "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(out))


def main() -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=2)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--n", type=int, default=65536)
    ap.add_argument("--nb", type=int, default=256)
    ap.add_argument("--e2e-steps", type=int, default=2)
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-e2e-pageable", action="store_true",
                    help="skip lumcolumn on pageable host memory (one untimed + one timed step)")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-mixed", action="store_true", help="skip the BF16-LU + IR measurement")
    ap.add_argument("--mixed-nb", type=int, default=256)
    ap.add_argument("--no-batched", action="store_true", help="skip the batched-systems measurement")
    ap.add_argument("--batch-count", type=int, default=20000)
    ap.add_argument("--batch-loop-sample", type=int, default=400)
    ap.add_argument("--profile", action="store_true",
                    help="profiling run for ncu: generate the matrix and run exactly one factor+solve step")
    ap.add_argument("--profile-mixed", action="store_true",
                    help="profiling run for ncu: one BF16-LU + IR solve of the diagonally dominant system")
    ap.add_argument("--profile-fp8", action="store_true",
                    help="profiling run for ncu: one FP8-LU + GMRES-IR solve of the diagonally dominant system")
    ap.add_argument("--profile-batched", action="store_true",
                    help="profiling run for ncu: one FP64 batched solve of the batch-count systems")
    ap.add_argument("--profile-swap", action="store_true",
                    help="row exchange alone: one panel's pivots (nb random rows below the panel) applied to the "
                         "full width of the order-n matrix through lu2gpu_swaprows_dev, timed with CUDA events")
    ap.add_argument("--swap-rows", type=int, default=0,
                    help="--profile-swap on a matrix of this many rows (pivots drawn below the panel within them; "
                         "0: n rows), so a capture of the full width holds a few GB")
    ap.add_argument("--profile-trsm", action="store_true",
                    help="block-row solve alone: U12 = L11^-1 A12 for an nb x n block (lu2gpu_solve_triangle_dev, "
                         "L11 from a real panel), timed with CUDA events")
    ap.add_argument("--profile-backsolve", action="store_true",
                    help="back substitution alone: factor the order-n system, then time lu2gpu_backsolve")
    ap.add_argument("--batch-ir", action="store_true",
                    help="--profile-batched in the FP32-LU + FP64 IR mode")
    ap.add_argument("--batch-nmin", type=int, default=16, help="--profile-batched: smallest order")
    ap.add_argument("--batch-nmax", type=int, default=512, help="--profile-batched: largest order")
    ap.add_argument("--batch-config", default=None,
                    help="threads,panel_width,ctas_per_sm for --profile-batched (default: autotune)")
    ap.add_argument("--no-fp8", action="store_true", help="skip the FP8 + GMRES-IR measurement")
    ap.add_argument("--no-host-dgemm", action="store_true", help="skip the host-pointer DGEMM measurement")
    ap.add_argument("--fp8-n", type=int, default=98304)
    ap.add_argument("--fp8-nb", type=int, default=256)
    ap.add_argument("--fp8-check-n", type=int, default=32768)
    ap.add_argument("--fp8-warmup", type=int, default=1)
    ap.add_argument("--fp8-steps", type=int, default=1)
    ap.add_argument("--fp8-general-iters", type=int, default=60,
                    help="GMRES iteration budget for the general (not diagonally dominant) matrices")
    args = ap.parse_args()

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        run_reference(args, rank)
        return 0

    import torch
    import torch.distributed as dist

    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        from datetime import timedelta

        dist.init_process_group("nccl", timeout=timedelta(seconds=600), device_id=dev)

    import numpy as np

    import lu2_b200 as L

    def barrier():
        if world > 1:
            dist.barrier()

    def max_over_ranks(v: float) -> float:
        if world == 1:
            return v
        t = torch.tensor([v], dtype=torch.float64, device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    n, nb = args.n, args.nb
    ctx = L.Context(local)
    stream = torch.cuda.current_stream()
    ctx.set_stream(stream.cuda_stream)
    if args.profile_batched:
        n_b, r_b = L.batch_sizes(args.batch_count, 1, args.batch_nmin, args.batch_nmax, 0.1, 8)
        b = L.Batch(ctx, n_b, r_b)
        b.generate_seeds(1 + np.arange(args.batch_count))
        b.snapshot()  # the original systems, for the residuals
        if args.batch_ir:
            b.set_mode(L.BATCH_FP32_IR, 10)
        if args.batch_config:
            t_, pw_, g_ = (int(v) for v in args.batch_config.split(","))
            b.set_config(t_, pw_, g_)
            cfg = {"threads": t_, "pw": pw_, "ctas_per_sm": g_}
        else:
            cfg = b.autotune()
            b.restore()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        info = b.solve()
        torch.cuda.synchronize()
        flops = float(np.sum(2.0 / 3.0 * n_b.astype(np.float64) ** 3 + 2.0 * n_b.astype(np.float64) ** 2 * r_b))
        print(json.dumps({"profile_batched_s": time.perf_counter() - t0, "count": args.batch_count,
                          "orders": [args.batch_nmin, args.batch_nmax], "gflop": flops / 1e9,
                          "config": cfg, "zero_pivots": int((info != 0).sum()),
                          "max_hpl_residual": float(b.residuals().max())}))
        b.close()
        ctx.close()
        return 0
    if args.profile_swap:
        print(json.dumps(run_swap_profile(ctx, n, nb, dev, stream, rows=args.swap_rows or n)))
        ctx.close()
        return 0
    if args.profile_trsm:
        print(json.dumps(run_trsm_profile(ctx, n, nb, dev, stream)))
        ctx.close()
        return 0
    if args.profile_backsolve:
        print(json.dumps(run_backsolve_profile(ctx, n, nb, dev, stream)))
        ctx.close()
        return 0
    ld = L.device_ld(n)
    pristine = torch.empty((n, ld), dtype=torch.float64, device=dev)
    A = torch.empty_like(pristine)
    ctx.generate(pristine, n, ld, 1)
    lib = L.load()
    launches0 = lib.lu2gpu_kernel_launches()

    def step():
        A.copy_(pristine)
        info = ctx.lusolve(A, n, ld, nb, 1, L.PIVOT_PARTIAL)
        if info != 0:
            raise RuntimeError("zero pivot at column %d" % (info - 1))

    if args.profile_mixed or args.profile_fp8:
        ctx.generate(pristine, n, ld, 1, 1, kind=1)
        b = pristine[:, n].clone()
        x = torch.zeros(n, dtype=torch.float64, device=dev)
        if args.profile_fp8:
            res = ctx.gmres_solve(pristine, n, ld, b, x, args.fp8_nb, update=L.UPDATE_FP8, restart=30, max_iter=100)
        else:
            res = ctx.mixed_solve(pristine, n, ld, b, x, args.mixed_nb)
        torch.cuda.synchronize()
        print(json.dumps({"profile_fp8" if args.profile_fp8 else "profile_mixed": res, "n": n}))
        ctx.close()
        return 0
    if args.profile:
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        step()
        torch.cuda.synchronize()
        print(json.dumps({"profile_step_s": time.perf_counter() - t0, "n": n, "nb": nb,
                          "launches": lib.lu2gpu_kernel_launches() - launches0}))
        ctx.close()
        return 0

    log("warmup x%d (n=%d nb=%d)" % (args.warmup, n, nb))
    for _ in range(args.warmup):
        step()
    clocks = Clocks(local)
    barrier()
    torch.cuda.synchronize()
    clocks.start()
    launches0 = lib.lu2gpu_kernel_launches()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        step()
    e1.record(stream)
    torch.cuda.synchronize()
    launches = lib.lu2gpu_kernel_launches() - launches0
    clk = clocks.stop()
    barrier()
    t = max_over_ranks(e0.elapsed_time(e1) / 1e3)
    value = world * args.steps * lu_flops(n) / t / 1e9
    log("timed: %.3f s for %d steps -> %.1f GFLOP/s" % (t, args.steps, value))

    # accuracy of the last step: HPL scaled residual on the device (float64)
    x = A[:, n].clone()
    A0 = pristine[:, :n]
    b0 = pristine[:, n]
    r = (A0 @ x - b0).abs().max().item()
    hplres = r / (2.0**-53 * (A0.abs().sum(1).max().item() * x.abs().max().item() + b0.abs().max().item()) * n)
    del x, A0, b0  # views of pristine: they would keep its 34 GB alive

    # instrumented step: per-phase CUDA-event timers (not part of the timed region)
    ctx.set_timing(True)
    step()
    torch.cuda.synchronize()
    timers = ctx.timers()
    ctx.set_timing(False)
    gemm_ms, gemm_launches = timers["DGEMMrest"]
    gemm_flops = trailing_flops(n, nb)
    achieved = gemm_flops / (gemm_ms / 1e3) / 1e12
    peak = fp64_peak(dev)
    roofline = {"bound": "tensor", "kernel": "dgemm_tn_kernel (trailing update C -= L21 U12)",
                "achieved": achieved, "peak": peak, "unit": "TFLOP/s", "frac": achieved / peak,
                "peak_source": "FP64 DGEMM measured in this run: cuBLAS via torch.matmul float64 8192^3, best of 5",
                "traffic": read_profile_traffic(), "launches_per_step": gemm_launches,
                "avg_launch_ms": gemm_ms / max(gemm_launches, 1),
                "flops_per_step": gemm_flops}
    phases = {k: {"ms": v[0], "launches": v[1]} for k, v in timers.items()}

    # end to end through the reference-facing C entry point on pinned host memory
    e2e = None
    if not args.no_e2e:
        A = None  # the working matrix (34 GB at N = 65536) is not needed any more
        torch.cuda.empty_cache()
        host = torch.empty((n, n + 16), dtype=torch.float64, pin_memory=True)
        bvec = torch.empty(n, dtype=torch.float64, pin_memory=True)
        pv = np.zeros(nb, dtype=np.int32)
        assert ld == n + 16, "device and host row strides differ"
        lib.lu2gpu_set_stream(lib.lu2gpu_default_context(), stream.cuda_stream)
        hn, bn = host.numpy(), bvec.numpy()
        ts = []
        for it in range(1 + args.e2e_steps):
            host.copy_(pristine, non_blocking=False)  # untimed restore of the input
            torch.cuda.synchronize()
            barrier()
            f0 = torch.cuda.Event(enable_timing=True)
            f1 = torch.cuda.Event(enable_timing=True)
            f0.record(stream)
            rc = L.lumcolumn(hn, bn, nb, pv, L.PIVOT_PARTIAL)
            f1.record(stream)
            torch.cuda.synchronize()
            if rc != 0:
                raise RuntimeError("lumcolumn status %d" % rc)
            if it > 0:
                ts.append(f0.elapsed_time(f1) / 1e3)
        te = max_over_ranks(sum(ts))
        e2e = {"value": world * len(ts) * lu_flops(n) / te / 1e9, "unit": UNIT,
               "h2d_bytes_per_step": n * (n + 1) * 8, "d2h_bytes_per_step": n * (n + 1) * 8 + n * 8 + nb * 4,
               "steps": len(ts), "api": "lumcolumn() C entry point, pinned host buffers"}
        del host, bvec
        # the same on pageable host memory, as lu2's main allocates a
        # (malloc, lu2.c:1261-1262): lumcolumn page-locks it for the call
        if not args.no_e2e_pageable:
            hp = np.empty((n, n + 16))
            bp = np.empty(n)
            ts = []
            for it in range(2):
                hp[...] = pristine.cpu().numpy()  # untimed restore of the input
                barrier()
                f0 = torch.cuda.Event(enable_timing=True)
                f1 = torch.cuda.Event(enable_timing=True)
                f0.record(stream)
                rc = L.lumcolumn(hp, bp, nb, pv, L.PIVOT_PARTIAL)
                f1.record(stream)
                torch.cuda.synchronize()
                if rc != 0:
                    raise RuntimeError("lumcolumn status %d" % rc)
                if it > 0:
                    ts.append(f0.elapsed_time(f1) / 1e3)
            tp = max_over_ranks(sum(ts))
            e2e["pageable_value"] = world * len(ts) * lu_flops(n) / tp / 1e9
            e2e["pageable_steps"] = len(ts)
            del hp, bp
        lib.lu2gpu_release()

    # precision form: BF16-LU + FP64 iterative refinement on the
    # diagonally dominant system of the same order, against this run's FP64 LU
    # rebinding, not locals(): a locals() snapshot would keep the 34 GB matrices alive
    A = None
    torch.cuda.empty_cache()
    forms = {}
    if not args.no_mixed:
        torch.cuda.empty_cache()
        forms["bf16_ir"] = run_mixed(ctx, n, nb, ld, pristine, dev, stream, args, barrier, max_over_ranks,
                                     t / args.steps, world)
    pristine = None
    torch.cuda.empty_cache()
    if not args.no_batched:
        forms["batched_fp64"] = run_batched(ctx, dev, stream, args, max_over_ranks, world, rank)
    if not args.no_fp8:
        forms["fp8_gmres_ir"] = run_fp8(ctx, dev, stream, args, max_over_ranks, world)
    if not args.no_host_dgemm:
        forms["host_dgemm"] = run_host_dgemm(max_over_ranks, barrier)

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        cpu = cpu_reference_gflops(REF_SAMPLE_N, nb, 3)

    if rank == 0:
        out = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
               "warmup": args.warmup, "ms_per_step": 1e3 * t / args.steps, "higher_is_better": True,
               "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
               "config": {"workload": "plain FP64 LU+solve (lumcolumn), N=%d, nb=%d, panels split to 16, "
                                      "partial pivoting, drand48 seed 1" % (n, nb),
                          "n": n, "nb": nb, "leaf": 16, "pivoting": "partial", "seed": 1,
                          "parallelism": "replicas" if world > 1 else "single",
                          "l2": "inputs (%.1f GB) larger than L2, no flush" % (n * ld * 8 / 1e9)},
               "gpu_launches": int(launches), "hpl_residual": hplres, "clocks": clk, "roofline": roofline,
               "e2e": e2e, "cpu_baseline": cpu, "phases_ms": phases, "forms": forms,
               "headline": headline(value, hplres, e2e, roofline, forms)}
        print(json.dumps(out))
    ctx.close()
    if world > 1:
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
