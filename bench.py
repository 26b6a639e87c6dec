#!/usr/bin/env python
"""Benchmark of the ADMIXTURE Adam-EM hot path on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--precision f64|f32|bf16|f16] [--config c3|c2|c1|c3s]

Workload (default ``c3``): N=200,000 samples, M=500,000 SNPs, K=10; a seeded synthetic
admixed cohort (Balding-Nichols F=0.02; Q 70% Dirichlet(0.05) / 30% Dirichlet(1); 1%
missing) sampled on the device straight into the 2-bit packed layout (25 GB resident).
A step is one Adam-EM iteration of the reference loop (adamixture/model/em_adam_gpu.py:
330-353): one fused E-step sweep over all genotypes + the EM targets and the Adam move,
with the float64 log-likelihood check every 5th iteration (read back to the host, as the
reference's ``.item()`` does). P/Q start from the reference's random EM initialisation
(adamixture/src/adamixture.py:140-156). Inputs (25 GB) exceed L2 (126 MB), so no flush is
needed between steps.

One JSON line on rank 0. The headline ``value`` (EM iterations/s, device-timed, max over
ranks) is float64 arithmetic throughout, the reference GPU path's own arithmetic
(``--precision`` changes it). ``variants`` repeats the measurement for the float32 sweep
and the two tensor-core sweeps (FP16 / BF16 operands, FP32 accumulation), each with its
own roofline, from the same start. ``time_to_target`` times whole fits from the
reference's default start (randomized SVD + ALS) to the first check within 1e-6 relative
of the plain float32 fit's log-likelihood: float32, FP16, and the learned warm start in
front of FP16. ``e2e`` = the headline iterations through the public Python API starting
from pinned host buffers (packed G, P, Q) and ending with P/Q back on the host;
``roofline`` = the headline's E-step sweep kernel alone: for the float64 sweep, bound by
the float64 tensor-core pipe, its 8 M N K useful flops per launch against a cuBLAS float64
GEMM timed in the same run (the HBM figures, algorithmic bytes ceil(M/4)*N + 4K(3M+2N)
per launch against the measured copy bandwidth, in its ``hbm`` entry); for the other
sweeps those HBM figures;
``cpu_baseline`` = the reference's own CPU Adam-EM step (its Cython kernels compiled from
source into oracle/_ref) with its every-5th log-likelihood check, on a 25,000-row SNP
slice of the same cohort, scaled linearly to the full M.
``--impl reference`` prints the reference arm: that CPU implementation as the headline,
each step on one of two 25,000-row slices (50,000 rows in all).
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "time-to-converged loglik & EM iter/s at N=200k,M=500k,K=10; genotype GB/s vs HBM"
UNIT = "EM iter/s"

CONFIGS = {
    "c3": dict(workload="Adam-EM, N=200000 samples, M=500000 SNPs, K=10, F=0.02, Q 0.7*Dir(0.05)+0.3*Dir(1), 1% missing",
               N=200_000, M=500_000, K=10, F=0.02, alpha=((0.7, 0.05), (0.3, 1.0)), miss=0.01, seed=2000),
    "c2": dict(workload="Adam-EM, N=10000 samples, M=200000 SNPs, K=8, F=0.05, Q Dir(0.3), 0.5% missing",
               N=10_000, M=200_000, K=8, F=0.05, alpha=0.3, miss=0.005, seed=1000),
    "c1": dict(workload="Adam-EM, N=1000 samples, M=10000 SNPs, K=3, F=0.1, Q Dir(0.5), 1% missing",
               N=1_000, M=10_000, K=3, F=0.1, alpha=0.5, miss=0.01, seed=0),
    "c4": dict(workload="K sweep K=2..12 with 5-fold CV (10 % of entries per fold, seeded hash), N=20000 samples, M=100000 SNPs, true K=6, F=0.08, Q Dir(0.5), 1% missing",
               N=20_000, M=100_000, K=6, F=0.08, alpha=0.5, miss=0.01, seed=4000),
    "c5": dict(workload="learned warm start vs the ALS start, held-out cohort N=100000 samples, M=300000 SNPs, K=8, F=0.05, Q Dir(0.5), 1% missing",
               N=100_000, M=300_000, K=8, F=0.05, alpha=0.5, miss=0.01, seed=6000),
    # the c3 cohort's generator at one tenth of its SNPs (2.5 GB packed): the size profiled
    # under ncu, whose full capture saves and restores device memory on every pass
    "c3s": dict(workload="Adam-EM, N=200000 samples, M=50000 SNPs, K=10, F=0.02, Q 0.7*Dir(0.05)+0.3*Dir(1), 1% missing",
                N=200_000, M=50_000, K=10, F=0.02, alpha=((0.7, 0.05), (0.3, 1.0)), miss=0.01, seed=2000),
}
TC_PRECISIONS = ("bf16", "f16")   # the tensor-core sweep
FP64_NOMINAL_TFLOPS = 40.0        # B200 float64 (vector and tensor core), NVIDIA's datasheet
CHECK = 5
HP = dict(lr=0.005, beta1=0.80, beta2=0.88, eps=1e-8)


def peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def peaks_tensor():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        try:
            return float(json.loads(p.read_text())["bf16_tflops"])
        except (ValueError, KeyError):
            pass
    return 1590.0


_FP64_PEAK = {}


def fp64_gemm_peak(dev):
    """Float64 tensor-core peak measured on this GPU in this run: a cuBLAS float64 GEMM of
    8192^3 (2 n^3 flops), best of 5 launches between CUDA events after one warm-up. The
    driver's measured-peaks file has HBM and BF16 figures only, so the float64 sweep's
    denominator is measured here the same way (a library GEMM, burst)."""
    import torch

    if dev in _FP64_PEAK:
        return _FP64_PEAK[dev]
    n = 8192
    a = torch.rand((n, n), dtype=torch.float64, device=dev)
    b = torch.rand((n, n), dtype=torch.float64, device=dev)
    c = torch.matmul(a, b)
    torch.cuda.synchronize(dev)
    best = float("inf")
    for _ in range(5):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        torch.matmul(a, b, out=c)
        e1.record()
        torch.cuda.synchronize(dev)
        best = min(best, e0.elapsed_time(e1))
    del a, b, c
    _FP64_PEAK[dev] = 2.0 * n ** 3 / (best * 1e-3) / 1e12
    return _FP64_PEAK[dev]


def alg_bytes(M, N, K):
    return ((M + 3) // 4) * N + 4 * K * (3 * M + 2 * N)


# ---------------------------------------------------------------- clocks

class Clocks:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, dev_uuid: str | None):
        self.proc = None
        self.uuid = dev_uuid

    def __enter__(self):
        cmd = ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits", "-lms", "200"]
        if self.uuid:
            cmd += ["-i", self.uuid]
        try:
            self.proc = subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except (FileNotFoundError, OSError):
            self.proc = None
        return self

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.out, _ = self.proc.communicate(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
                self.out = ""
        return False

    def summary(self):
        if self.proc is None or not getattr(self, "out", ""):
            return None
        sm, smax, reasons = [], [], set()
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        for line in self.out.strip().splitlines():
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax.append(float(f[2]))
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(smax), "samples": len(sm),
                "reasons": sorted(reasons)}


# ---------------------------------------------------------------- CPU (reference) arm

REF_SLICE_ROWS = 25_000   # SNP rows per timed reference step
REF_SLICES = 2            # the reference arm alternates over this many slices (50,000 rows)


def cpu_reference_sample(cfg, slices, steps, warmup):
    """Time the reference's own Adam-EM CPU iteration on SNP-row slices of the cohort, all
    host cores: ``adamStep`` (em.P_step, em.Q_step, em.adamUpdateP/Q;
    adamixture/model/em_adam.py:12-54) and, every 5th step, its log-likelihood check
    (tools.loglikelihood; em_adam.py:136-160), the same step the GPU arm times. Step s runs
    on ``slices[s % len(slices)]``. A step's full-M time scales the SNP-side work (P_step,
    adamUpdateP, the check) by M / slice rows; the sample-side work (Q_step, adamUpdateQ)
    does not depend on M and is counted once. Returns (seconds per full-M iteration, info)."""
    cores = os.cpu_count() or 1
    os.environ["OMP_NUM_THREADS"] = str(cores)
    from oracle import refmods  # the compiled reference kernels (test/baseline infrastructure)

    kind = "reference" if refmods.available() else "port"
    N, K, M = cfg["N"], cfg["K"], cfg["M"]
    rng = np.random.default_rng(cfg["seed"])
    Q = np.clip(rng.random((N, K)), 1e-5, 1 - 1e-5)
    Q /= Q.sum(1, keepdims=True)
    states = []
    for G_rows in slices:
        Ms = G_rows.shape[0]
        P = np.clip(rng.random((Ms, K)), 1e-5, 1 - 1e-5)
        states.append(dict(G=G_rows, Ms=Ms, P=P, P1=np.zeros_like(P), mP=np.zeros_like(P),
                           vP=np.zeros_like(P)))
    T = np.zeros_like(Q)
    Q1 = np.zeros_like(Q)
    qb = np.zeros(N)
    mQ, vQ = np.zeros_like(Q), np.zeros_like(Q)
    t = [0]
    if kind == "reference":
        em = refmods.load("em")
        tools = refmods.load("tools")

        def step(st, check):
            a = time.perf_counter()
            em.P_step(st["G"], st["P"], st["P1"], Q, T, qb, K, st["Ms"], N)
            b = time.perf_counter()
            em.Q_step(Q, Q1, T, qb, K, N)
            t[0] += 1
            c = time.perf_counter()
            em.adamUpdateP(st["P"], st["P1"], st["mP"], st["vP"], HP["lr"], HP["beta1"], HP["beta2"],
                           HP["eps"], t[0], st["Ms"], K)
            d = time.perf_counter()
            em.adamUpdateQ(Q, Q1, mQ, vQ, HP["lr"], HP["beta1"], HP["beta2"], HP["eps"], t[0], N, K)
            e = time.perf_counter()
            chk = 0.0
            if check:
                f0 = time.perf_counter()
                tools.loglikelihood(st["G"], st["P"], Q)
                chk = time.perf_counter() - f0
            return (b - a) + (d - c), (c - b) + (e - d), chk
        threads = cores
    else:
        from oracle import em_oracle as orc
        ad = orc.Adam(HP["lr"], HP["beta1"], HP["beta2"], HP["eps"]).init(states[0]["P"], Q)

        def step(st, check):
            a = time.perf_counter()
            A, B, Tt, q = orc.em_stats(st["G"], st["P"], Q)
            orc.adam_step(ad, st["P"], Q, *orc.em_final(st["P"], Q, A, B, Tt, q))
            snp = time.perf_counter() - a
            chk = 0.0
            if check:
                f0 = time.perf_counter()
                orc.loglik(st["G"], st["P"], Q)
                chk = time.perf_counter() - f0
            return snp, 0.0, chk
        threads = 1
    for it in range(warmup):
        step(states[it % len(states)], (it + 1) % CHECK == 0)
    full, sl = [], []
    for it in range(steps):
        st = states[it % len(states)]
        snp, smp, chk = step(st, (it + 1) % CHECK == 0)
        full.append((snp + chk) * (M / st["Ms"]) + smp)
        sl.append(snp + smp + chk)
    if steps < CHECK:
        # too few steps for a check among them: one check, timed on its own, counts as
        # 1/CHECK of a check per step
        chk = step(states[0], True)[2]
        full = [f + chk * (M / states[0]["Ms"]) / CHECK for f in full]
        sl = [x + chk / CHECK for x in sl]
    per = float(np.mean(full))
    rows = sum(st["Ms"] for st in states)
    info = {"kind": kind, "cores": threads,
            "sample": f"{len(states)} slice(s) of {states[0]['Ms']} SNP rows ({rows} of {M} rows in all) x all "
                      f"{N} samples, K={K}; step s on slice s mod {len(states)}; mean of {steps} reference "
                      f"Adam-EM steps (adamStep + the log-likelihood check every {CHECK}th step), SNP-side "
                      f"time scaled x{M / states[0]['Ms']:.1f} to the full M (its cost is linear in M)",
            "timed_slice_ms": 1e3 * float(np.mean(sl)), "scale": M / states[0]["Ms"], "sample_rows": rows}
    return per, info


def host_slices(coh, M, n_slices, rows):
    """The cohort's first ``n_slices * rows`` SNP rows, unpacked, sampled on the host."""
    rows = min(rows, max(4, M // n_slices))
    return [coh.genotypes_parallel(s * rows, rows) for s in range(n_slices)]


def run_reference_arm(args, cfg, rank):
    if rank != 0:
        return
    from adamixture_b200.src.simulate import make_cohort

    coh = make_cohort(cfg["N"], cfg["M"], cfg["K"], cfg["F"], cfg["alpha"], cfg["miss"], cfg["seed"])
    slices = host_slices(coh, cfg["M"], REF_SLICES, int(args.cpu_snps))
    full, info = cpu_reference_sample(cfg, slices, args.steps, args.warmup)
    v = 1.0 / full
    line = {
        "impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": full * 1e3,
        "higher_is_better": True, "scaling": "strong", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic", "config": {"workload": cfg["workload"], "sample_rows": info["sample_rows"],
                                        "check_every": CHECK},
        "cpu_baseline": dict(value=v, unit=UNIT, **info),
        "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------- GPU arm

def _sweep_kernel_name(prec, K):
    if prec in TC_PRECISIONS:
        return f"em_sweep_tc_kernel<{prec == 'f16'}>"
    if prec == "f64" and K <= 16:
        return f"em_sweep_dmma_kernel<{(K + 3) // 4}>"
    return f"em_sweep_kernel<{'double' if prec == 'f64' else 'float'},{ops_kmax(K)}>"


def time_steps(prec, G, P0, Q0, M_loc, N, K, dev, steps, warmup, sharded, clocks=None):
    """Adam-EM steps at one E-step arithmetic from (P0, Q0): ``warmup`` untimed steps, then
    ``steps`` steps between CUDA events on the launching stream (barrier + synchronize on
    both sides, max over ranks when sharded). Returns the step time, the kernel launches of
    the timed region and the final P/Q (for the sweep's roofline)."""
    import torch

    from adamixture_b200 import ops
    from adamixture_b200.model.em_adam_dist import CudaBackend, ShardedAdamEM
    from adamixture_b200.model.em_adam_gpu import EMAdamOptimizer

    P = torch.from_numpy(P0).to(dev)
    Q = torch.from_numpy(Q0).to(dev)
    P32, Q32 = P.float(), Q.float()
    ws = ops.Workspace.get(dev, ops.em_workspace_bytes(M_loc, N, K, prec))
    llp = "f64" if prec == "f64" else "f32"
    Pll, Qll = (P, Q) if llp == "f64" else (P32, Q32)
    launches = {"n": 0}
    fold = {"need": True}
    if not sharded:
        opt = EMAdamOptimizer(P.shape, Q.shape, HP["lr"], HP["beta1"], HP["beta2"], HP["eps"], dev, prec)
        per_iter = 3 if prec in TC_PRECISIONS else 2
        if opt.can_fold_check(K):
            # float64: as the optimiser runs it, the check after every 5th iteration is folded
            # into the next iteration's sweep (kernels: the sweep, the partials' sum and the
            # update, read back as the reference's .item()); other iterations are fused

            def one_step(it):
                if fold["need"]:
                    float(opt.sweep_with_loglik(G, P, Q, M_loc, ws).item())
                    opt.apply_update(P, Q, None, None, M_loc, ws)
                    launches["n"] += 3
                    fold["need"] = False
                else:
                    opt.fused_iteration(G, P, Q, P32, Q32, M_loc, ws)
                    launches["n"] += 2
                if (it + 1) % CHECK == 0:
                    fold["need"] = True
        else:
            # kernels per fused iteration: sweep (+ the 16-bit copy of Q for the tensor-core
            # sweep) and the update kernel; per check: the log-likelihood kernel and its final sum

            def one_step(it):
                opt.fused_iteration(G, P, Q, P32, Q32, M_loc, ws)
                launches["n"] += per_iter
                if (it + 1) % CHECK == 0:
                    float(ops.loglik_device(G, Pll, Qll, M_loc, llp).item())
                    launches["n"] += 2
    else:
        # SNP-sharded: local sweep + statistics, all-reduce of T, targets, Adam (Q replicated)
        run = ShardedAdamEM(G, P, Q, M_loc, K, HP["beta1"], HP["beta2"], HP["eps"], HP["lr"],
                            backend=CudaBackend(prec))
        per_iter = (3 if prec in TC_PRECISIONS else 2) + 2

        def one_step(it):
            run.iteration()
            launches["n"] += per_iter
            if (it + 1) % CHECK == 0:
                run.loglik()
                launches["n"] += 2

    torch.cuda.synchronize()
    for it in range(warmup):
        one_step(it)
    torch.cuda.synchronize()
    launches["n"] = 0
    # folded checks: the timed steps hold a check every 5th step, the first at step 0 (the
    # check due after the last warm-up step)
    fold["need"] = True
    if sharded:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    stream = torch.cuda.current_stream(dev)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    import contextlib
    with (clocks if clocks is not None else contextlib.nullcontext()):
        e0.record(stream)
        for it in range(steps):
            one_step(it)
        e1.record(stream)
        torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    if sharded:
        torch.distributed.barrier()
        t = torch.tensor([ms], device=dev)
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        ms = float(t.item())
    if ops.em_status(ws, M_loc, N, K, prec) != 0:
        raise RuntimeError(f"E-step sweep reported a nonzero status ({prec})")
    return {"ms_per_step": ms / steps, "launches": launches["n"], "P": P, "Q": Q}


def sweep_roofline(prec, G, P, Q, M_loc, N, K, dev, reps):
    """The E-step sweep kernel alone (this rank's rows): mean of ``reps`` launches between
    CUDA events on its stream, after one warm-up launch; algorithmic bytes per launch
    ceil(M/4) N + 4K(3M+2N) against the measured HBM copy bandwidth, and for the float64
    sweep (bound by the float64 tensor-core pipe) 8 M N K flops against the float64 GEMM
    peak measured in this run."""
    import torch

    from adamixture_b200 import ops

    Pin, Qin = (P, Q) if prec == "f64" else (P.float(), Q.float())
    ws = ops.Workspace.get(dev, ops.em_workspace_bytes(M_loc, N, K, prec))
    stream = torch.cuda.current_stream(dev)
    ops.em_sweep(G, Pin, Qin, M_loc, prec, ws)
    torch.cuda.synchronize()
    s0, s1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    s0.record(stream)
    for _ in range(reps):
        ops.em_sweep(G, Pin, Qin, M_loc, prec, ws)
    s1.record(stream)
    torch.cuda.synchronize()
    sweep_ms = s0.elapsed_time(s1) / reps
    hbm, peak_kind = peaks()
    ab = alg_bytes(M_loc, N, K)
    achieved = ab / (sweep_ms * 1e-3) / 1e9
    roof = {"bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s",
            "frac": achieved / hbm, "traffic": traffic_per_launch(M_loc, N, K, prec),
            "kernel": _sweep_kernel_name(prec, K), "launch_ms": sweep_ms, "alg_bytes": ab,
            "peak_kind": peak_kind, "entries_per_s": M_loc * N / (sweep_ms * 1e-3),
            "snp_rows_per_rank": M_loc}
    flops = 8.0 * M_loc * N * K
    if prec in TC_PRECISIONS:
        # the contractions (h, 1-h, A, B, T: 8 M N K flops of useful work; K padded to 16 in
        # the MMAs) against the measured dense BF16 peak (FP16's dense rate is the same)
        tf = peaks_tensor()
        roof["tensor"] = {"achieved_tflops": flops / (sweep_ms * 1e-3) / 1e12, "peak_tflops": tf,
                          "frac": flops / (sweep_ms * 1e-3) / 1e12 / tf if tf else None,
                          "flops_per_launch": flops}
    elif prec == "f64":
        # The float64 sweep is bound by the float64 tensor-core pipe, not by HBM (8 M N K
        # flops against 0.25 B per entry): its roofline is the useful contraction flops
        # against the float64 GEMM peak measured in this run; the HBM figures stay beside it.
        # (the peak itself is measured after the other timings: finish_fp64_roofline)
        tflops = flops / (sweep_ms * 1e-3) / 1e12
        hbm_part = {k: roof[k] for k in ("achieved", "peak", "unit", "frac", "peak_kind")}
        roof.update({"bound": "tensor", "achieved": tflops, "peak": None, "unit": "TFLOP/s", "frac": None,
                     "peak_kind": "measured in this run: cuBLAS float64 GEMM 8192^3, best of 5",
                     "flops_per_launch": flops, "hbm": hbm_part,
                     "fp64_nominal": {"peak_tflops": FP64_NOMINAL_TFLOPS,
                                      "frac": tflops / FP64_NOMINAL_TFLOPS}})
    return roof


def finish_fp64_roofline(roof, dev):
    """Fill in the float64 sweep's roofline denominator, timed after every other
    measurement of the run so that its buffers touch none of them."""
    if roof.get("bound") == "tensor" and roof.get("peak") is None:
        pk = fp64_gemm_peak(dev)
        roof["peak"] = pk
        roof["frac"] = roof["achieved"] / pk
    return roof


def run_gpu_arm(args, cfg, rank, world, local_rank):
    import torch

    from adamixture_b200 import ops
    from adamixture_b200.model.em_adam_gpu import resolve_precision
    from adamixture_b200.src.simulate import make_cohort

    dev = torch.device("cuda", local_rank)
    torch.cuda.set_device(dev)
    N, M, K = cfg["N"], cfg["M"], cfg["K"]
    prec = resolve_precision(K, args.precision or "f64")
    sharded = world > 1 or args.shard
    if sharded:
        import datetime

        import torch.distributed as dist
        os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
        os.environ.setdefault("MASTER_PORT", "29531")
        os.environ.setdefault("RANK", str(rank))
        os.environ.setdefault("WORLD_SIZE", str(world))
        dist.init_process_group("nccl", device_id=dev, timeout=datetime.timedelta(minutes=10))

    from adamixture_b200.model.em_adam_dist import shard_rows
    from adamixture_b200.src.simulate import shard_keys

    coh = make_cohort(N, M, K, cfg["F"], cfg["alpha"], cfg["miss"], cfg["seed"])
    # this rank's SNP rows (all of them on one GPU); exactly that slice of the cohort
    j0, j1 = shard_rows(M, world, rank) if world > 1 else (0, M)
    M_loc = j1 - j0
    Pq = torch.from_numpy(coh.Pq[j0:j1].astype(np.int32)).to(dev)
    Qq = torch.from_numpy(coh.Qq.astype(np.int32)).to(dev)
    G = ops.simulate_packed(Pq, Qq, coh.miss_q, shard_keys(coh.keys, j0, N))
    del Pq, Qq
    rng = np.random.default_rng(cfg["seed"])
    P0 = np.clip(rng.random((M, K)), 1e-5, 1 - 1e-5)[j0:j1].copy()
    Q0 = np.clip(rng.random((N, K)), 1e-5, 1 - 1e-5)
    Q0 /= Q0.sum(1, keepdims=True)

    uuid = None
    try:
        uuid = "GPU-" + str(torch.cuda.get_device_properties(dev).uuid)
    except Exception:
        pass
    clk = Clocks(uuid)
    head = time_steps(prec, G, P0, Q0, M_loc, N, K, dev, args.steps, args.warmup, sharded, clocks=clk)
    ms_per_step = head["ms_per_step"]
    reps = max(3, min(10, args.steps))
    roof = sweep_roofline(prec, G, head["P"], head["Q"], M_loc, N, K, dev, reps)
    del head["P"], head["Q"]

    # the other E-step arithmetics from the same start, each with its own sweep roofline
    variants = {}
    if not args.no_variants:
        for vp in ("f32", "f16", "bf16"):
            if vp == prec or (vp in TC_PRECISIONS and K > 16):
                continue
            r = time_steps(vp, G, P0, Q0, M_loc, N, K, dev, args.steps, args.warmup, sharded)
            variants[vp] = {"value": 1000.0 / r["ms_per_step"], "unit": UNIT, "ms_per_step": r["ms_per_step"],
                            "dtype": vp, "gpu_launches": r["launches"],
                            "roofline": sweep_roofline(vp, G, r["P"], r["Q"], M_loc, N, K, dev, reps)}
            del r
        torch.cuda.synchronize()

    # e2e through the public API from pinned host buffers, at the headline arithmetic
    e2e = None
    if not args.no_e2e:
        if not sharded:
            e2e = run_e2e(args, G, P0, Q0, M, N, K, prec, dev)
        else:
            e2e = run_e2e_dist(args, G, P0, Q0, M_loc, N, K, prec, dev, world)

    # whole fits to the converged log-likelihood (one GPU)
    ttt = None
    if not args.no_converge and not sharded:
        ttt = converge_runs(args, cfg, G, dev, ("f32", "f16", "warm_f16"))

    cpu = None
    if not args.no_cpu and rank == 0 and world == 1:
        rows = min(M, int(args.cpu_snps))
        G_rows = ops.unpack_u8(G, 0, rows, M).cpu().numpy()
        full, info = cpu_reference_sample(cfg, [G_rows], 2, 0)
        cpu = dict(value=1.0 / full, unit=UNIT, **info)

    finish_fp64_roofline(roof, dev)
    if rank == 0:
        line = {
            "metric": METRIC, "value": 1000.0 / ms_per_step, "unit": UNIT,
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": ms_per_step, "higher_is_better": True, "scaling": "strong",
            "vs_baseline": None, "dtype": prec, "data": "synthetic",
            "config": {"workload": cfg["workload"], "precision": prec, "check_every": CHECK,
                       "l2": "inputs (packed G) larger than L2; no flush",
                       "genotype_GBps": ((M + 3) // 4) * N / (ms_per_step * 1e-3) / 1e9,
                       "parallelism": "single GPU" if not sharded else
                       f"SNP rows sharded over {world} rank(s) (one all-reduce of T per iteration)"},
            "roofline": roof, "variants": variants, "time_to_target": ttt,
            "cpu_baseline": cpu, "e2e": e2e,
            "gpu_launches": head["launches"], "clocks": clk.summary(),
        }
        print(json.dumps(line), flush=True)
    if sharded:
        torch.distributed.destroy_process_group()


def ops_kmax(K):
    for km in (2, 3, 4, 6, 8, 10, 12, 16, 24, 32, 48, 64):
        if K <= km:
            return km
    return K


def traffic_per_launch(M, N, K, prec):
    """DRAM bytes per sweep launch from the committed ncu capture, scaled by entries."""
    f = ROOT / "profiles" / "traffic.json"
    if not f.exists():
        return None
    try:
        d = json.loads(f.read_text())
        e = d.get(f"em_sweep_{prec}_K{K}")
        if not e:
            return None
        return e["bytes"] * (M * N) / (e["M"] * e["N"])
    except (ValueError, KeyError):
        return None


def run_e2e(args, G_dev, P0, Q0, M, N, K, prec, dev):
    import torch

    from adamixture_b200.model.em_adam_gpu import optimize_parameters_gpu

    try:
        G_host = torch.empty(G_dev.shape, dtype=torch.uint8, pin_memory=True)
        pinned = True
    except RuntimeError:
        G_host = torch.empty(G_dev.shape, dtype=torch.uint8)
        pinned = False
    G_host.copy_(G_dev)
    P_host = torch.from_numpy(P0).pin_memory() if pinned else torch.from_numpy(P0)
    Q_host = torch.from_numpy(Q0).pin_memory() if pinned else torch.from_numpy(Q0)
    iters = args.steps
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    trace = []
    # host tensors in: the packed matrix is uploaded in pieces, each swept by the priming
    # iteration as it lands (float64, K <= 16; other forms upload it first)
    Pb, Qb = optimize_parameters_gpu(G_host, P_host, Q_host, HP["lr"], HP["beta1"], HP["beta2"], HP["eps"],
                                     iters, CHECK, K, M, N, 0.5, 1e-4, 3, 0.1, dev, 8192, 512,
                                     precision=prec, trace=trace)
    Pr, Qr = Pb.cpu(), Qb.cpu()
    el = time.perf_counter() - t0
    del Pb, Qb
    nchecks = len(trace) + 1
    return {"value": iters / el, "unit": UNIT,
            "h2d_bytes_per_step": (G_host.numel() + P0.nbytes + Q0.nbytes) / iters,
            "d2h_bytes_per_step": (Pr.numel() * 8 + Qr.numel() * 8 + 8 * nchecks) / iters,
            "pinned": pinned, "seconds": el,
            "note": "one optimize_parameters_gpu call with max_iter=steps on host tensors: "
                    "H2D of packed G/P/Q (G in pieces overlapping the priming sweep), priming + "
                    "steps iterations, loglik checks read back, best P/Q copied to the host"}


def run_graphs(args):
    """Adam-EM iterations launched one by one (two kernels each, through the Python wrapper)
    against the same iterations replayed from a captured CUDA graph (runs of 4, as between
    the optimiser's checks every 5th iteration, and one run of 20), at the small configs
    where an iteration takes tens of microseconds. CUDA events around 20 iterations after 3
    warm-up ones (the events see the gaps the host leaves between launches)."""
    import torch

    from adamixture_b200 import ops
    from adamixture_b200.model.em_adam_gpu import EMAdamOptimizer
    from adamixture_b200.src.simulate import make_cohort

    dev = torch.device("cuda", 0)
    out = []
    for name in ("c1", "c2"):
        cfg = CONFIGS[name]
        N, M, K = cfg["N"], cfg["M"], cfg["K"]
        coh = make_cohort(N, M, K, cfg["F"], cfg["alpha"], cfg["miss"], cfg["seed"])
        Pq = torch.from_numpy(coh.Pq.astype(np.int32)).to(dev)
        Qq = torch.from_numpy(coh.Qq.astype(np.int32)).to(dev)
        G = ops.simulate_packed(Pq, Qq, coh.miss_q, coh.keys)
        del Pq, Qq
        rng = np.random.default_rng(cfg["seed"])
        P0 = torch.from_numpy(np.clip(rng.random((M, K)), 1e-5, 1 - 1e-5)).to(dev)
        Q0 = np.clip(rng.random((N, K)), 1e-5, 1 - 1e-5)
        Q0 = torch.from_numpy(Q0 / Q0.sum(1, keepdims=True)).to(dev)
        for prec in ("f64", "f32", "f16"):
            P, Q = P0.clone(), Q0.clone()
            P32, Q32 = (P.float(), Q.float()) if prec != "f64" else (None, None)
            opt = EMAdamOptimizer(P.shape, Q.shape, HP["lr"], HP["beta1"], HP["beta2"], HP["eps"], dev, prec)
            ws = ops.em_workspace(M, N, K, prec, dev)
            for _ in range(3):
                opt.fused_iteration(G, P, Q, P32, Q32, M, ws)
            stream = torch.cuda.current_stream(dev)
            row = {"config": name, "N": N, "M": M, "K": K, "precision": prec}
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)

            def timed(fn):
                torch.cuda.synchronize()
                e0.record(stream)
                fn()
                e1.record(stream)
                torch.cuda.synchronize()
                return e0.elapsed_time(e1) / 20 * 1000.0   # us per iteration

            def eager():
                for _ in range(20):
                    opt.fused_iteration(G, P, Q, P32, Q32, M, ws)
            row["eager_us"] = timed(eager)
            for n in (4, 20):
                g = ops.EmGraph(G, P, Q, P32, Q32, opt.m_P, opt.v_P, opt.m_Q, opt.v_Q, opt.q_bat, M, n, opt.lr,
                                opt.beta1, opt.beta2, opt.reg_adam, prec, ws)
                g.launch(opt._t)     # warm-up replay (the first launch uploads the graph)
                opt._t += n

                def replay():
                    for _ in range(20 // n):
                        g.launch(opt._t)
                        opt._t += n
                row[f"graph{n}_us"] = timed(replay)
                g.close()
            out.append(row)
            print(json.dumps(row), flush=True)
    return out


def run_sweep_by_k(args):
    """Sweep time of the float32 SIMT form against the FP16 tensor-core form for K = 2..16
    at two shapes (CUDA events, mean of 10 launches after 3 warm-up launches): the
    measurement behind auto's choice of E-step arithmetic."""
    import torch

    from adamixture_b200 import ops
    from adamixture_b200.src.simulate import make_cohort

    dev = torch.device("cuda", 0)
    out = []
    for N, M in ((10_000, 200_000), (200_000, 50_000)):
        for K in (2, 4, 6, 8, 10, 16):
            coh = make_cohort(N, M, K, 0.05, 0.3, 0.005, 11)
            Pq = torch.from_numpy(coh.Pq.astype(np.int32)).to(dev)
            Qq = torch.from_numpy(coh.Qq.astype(np.int32)).to(dev)
            G = ops.simulate_packed(Pq, Qq, coh.miss_q, coh.keys)
            del Pq, Qq
            P = torch.from_numpy(coh.P).to(dev).float().clamp(1e-5, 1 - 1e-5).contiguous()
            Q = torch.from_numpy(coh.Q).to(dev).float().contiguous()
            row = {"N": N, "M": M, "K": K}
            for prec in ("f32", "f16"):
                ws = torch.zeros(ops.em_workspace_bytes(M, N, K, prec), dtype=torch.uint8, device=dev)
                for _ in range(3):
                    ops.em_sweep(G, P, Q, M, prec, ws)
                s0, s1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                torch.cuda.synchronize()
                s0.record()
                for _ in range(10):
                    ops.em_sweep(G, P, Q, M, prec, ws)
                s1.record()
                torch.cuda.synchronize()
                if ops.em_status(ws, M, N, K, prec) != 0:
                    raise RuntimeError(f"sweep status nonzero at N={N} M={M} K={K} {prec}")
                row[f"{prec}_ms"] = s0.elapsed_time(s1) / 10
                del ws
            out.append(row)
            del G
    print(json.dumps({"metric": "E-step sweep ms by K", "rows": out}), flush=True)


def run_tiles(args):
    """``--tiles``: the float64 sweep under each of its tile layouts for K = 2..12 at the
    config-4 shape (N=20,000 x M=100,000) and at K=3 / 8 / 10 at the c1, c2 and c3 shapes
    (``--config c3s``: K=8 at N=200,000 x M=50,000 only, the profiled case); CUDA events,
    mean of min(5, --steps) launches after one warm-up, with the autotuner's pick for each
    (its own timing, a partial sweep over whole waves). The layouts give bit-identical
    partial sums; the line says so per row."""
    import torch

    from adamixture_b200 import ops, tune
    from adamixture_b200.src.simulate import make_cohort

    dev = torch.device("cuda", 0)
    if args.config == "c3s":
        # the profiled case: the c3 generator at one tenth of its SNPs (2.5 GB packed), K=8
        cases = [(200_000, 50_000, 8)]
    else:
        cases = [(20_000, 100_000, K) for K in range(2, 13)] + [(1_000, 10_000, 3), (10_000, 200_000, 8),
                                                              (200_000, 500_000, 8), (200_000, 500_000, 10)]
    reps = max(1, min(5, args.steps))
    rows, cache = [], {}
    for N, M, K in cases:
        if (N, M) not in cache:
            cache.clear()
            torch.cuda.empty_cache()
            coh = make_cohort(N, M, 6, 0.05, 0.3, 0.01, 21)
            cache[(N, M)] = ops.simulate_packed(torch.from_numpy(coh.Pq.astype(np.int32)).to(dev),
                                                torch.from_numpy(coh.Qq.astype(np.int32)).to(dev),
                                                coh.miss_q, coh.keys)
        G = cache[(N, M)]
        rng = np.random.default_rng(K)
        P = torch.from_numpy(np.clip(rng.random((M, K)), 1e-5, 1 - 1e-5)).to(dev)
        Qn = np.clip(rng.random((N, K)), 1e-5, 1 - 1e-5)
        Q = torch.from_numpy(Qn / Qn.sum(1, keepdims=True)).to(dev)
        ws = ops.em_workspace(M, N, K, "f64", dev)
        row = {"N": N, "M": M, "K": K}
        parts = []
        for tile in range(tune.tiles(K)):
            tune.set_tile(K, tile, 0)
            ops.em_sweep(G, P, Q, M, "f64", ws)
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            for _ in range(reps):
                ops.em_sweep(G, P, Q, M, "f64", ws)
            e1.record()
            torch.cuda.synchronize()
            row[f"layout{tile}_ms"] = e0.elapsed_time(e1) / reps
            parts.append(ws.clone())
        row["bit_identical"] = all(torch.equal(parts[0], x) for x in parts[1:])
        tune.set_tile(K, 0, 0)
        row["tuned"] = tune.tune_dmma(G, P, Q, M, workspace=ws, force=True)
        rows.append(row)
        del ws, parts, P, Q
        torch.cuda.synchronize()
    print(json.dumps({"metric": "float64 E-step sweep ms by tile layout", "rows": rows}), flush=True)


def run_kernels(args, cfg):
    """Per-kernel timings at the config's shape (CUDA events, mean of ``reps`` launches after
    one warm-up): the randomized-SVD products, the log-likelihood, BVLS, the BR-QN
    gradient/Hessian passes and SQP solves, CV masking + deviance, and the warm-start network.
    One JSON line with achieved GB/s (algorithmic bytes) and GFLOP/s per kernel."""
    import torch

    from adamixture_b200 import ops
    from adamixture_b200.model import warm_start as ws
    from adamixture_b200.src.simulate import make_cohort

    dev = torch.device("cuda", 0)
    N, M, K = cfg["N"], cfg["M"], cfg["K"]
    coh = make_cohort(N, M, K, cfg["F"], cfg["alpha"], cfg["miss"], cfg["seed"])
    G = ops.simulate_packed(torch.from_numpy(coh.Pq.astype(np.int32)).to(dev),
                            torch.from_numpy(coh.Qq.astype(np.int32)).to(dev), coh.miss_q, coh.keys)
    rng = np.random.default_rng(1)
    P = torch.from_numpy(np.clip(rng.random((M, K)), 1e-5, 1 - 1e-5)).to(dev)
    Q = torch.from_numpy(rng.dirichlet(np.ones(K), N)).to(dev)
    f = ops.allele_frequency(G, M)
    hbm, _ = peaks()
    gbytes = ((M + 3) // 4) * N
    out = {}

    def timed(name, fn, nbytes=None, flops=None, reps=3):
        fn()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(reps):
            fn()
        e1.record()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / reps
        r = {"ms": ms}
        if nbytes:
            r["GBps"] = nbytes / (ms * 1e-3) / 1e9
            r["hbm_frac"] = r["GBps"] / hbm
        if flops:
            r["GFLOPps"] = flops / (ms * 1e-3) / 1e9
        out[name] = r

    L = 20
    B = torch.randn((N, L), device=dev)
    Y = torch.randn((M, L), device=dev)
    timed("rsvd_rows_L20", lambda: ops.rsvd_rows(G, f, B, M), gbytes + 4 * L * (M + N), 2.0 * M * N * L)
    timed("rsvd_cols_L20", lambda: ops.rsvd_cols(G, f, Y, M), gbytes + 4 * L * (M + N), 2.0 * M * N * L)
    timed("loglik_f64", lambda: ops.loglik_device(G, P, Q, M, "f64"), gbytes + 8 * K * (M + N), 4.0 * M * N * K)
    P32, Q32 = P.float().contiguous(), Q.float().contiguous()
    timed("loglik_f32", lambda: ops.loglik_device(G, P32, Q32, M, "f32"), gbytes + 4 * K * (M + N), 4.0 * M * N * K)
    A = (Q.T @ Q).contiguous()
    Bt = (P @ A).contiguous()
    timed("bvls_M_rows", lambda: ops.bvls(A, Bt, 0.0, 1.0), 16 * M * K)
    v_kk = torch.linalg.svd(torch.ones((1, K), dtype=torch.float64), full_matrices=True)[2].t().contiguous().to(dev)
    if not args.kernels_skip_hessian:
        XtX_q, Xtz_q = ops.grad_hess_q(G, P, Q, M)
        XtX_p, Xtz_p = ops.grad_hess_p(G, P, Q, M)
        timed("grad_hess_q", lambda: ops.grad_hess_q(G, P, Q, M, XtX_q, Xtz_q), gbytes + 8 * N * K * (K + 1),
              2.0 * M * N * K * (K + 1), reps=1)
        timed("grad_hess_p", lambda: ops.grad_hess_p(G, P, Q, M, XtX_p, Xtz_p), gbytes + 8 * M * K * (K + 1),
              1.0 * M * N * K * (K + 1), reps=1)
        Xn = (-Xtz_q).contiguous()
        timed("sqp_q_N_rows", lambda: ops.sqp_solve_q(XtX_q, Xn, Q, v_kk, N, K), 8 * N * K * (K + 2))
        Xp = (-Xtz_p).contiguous()
        timed("sqp_p_M_rows", lambda: ops.sqp_solve_p(XtX_p, Xp, P, M, K), 8 * M * K * (K + 2))
        del XtX_q, XtX_p
    Gm = ops.masked_copy(G)
    timed("cv_mask_hash", lambda: ops.cv_mask_hash(Gm, G, M, 42, 5, 0), 2 * gbytes)
    timed("cv_deviance_hash", lambda: ops.cv_deviance_hash(G, P, Q, M, 42, 5, 0), gbytes + 8 * K * (M + N))
    del Gm
    net = ws.WarmStartMLP(dev)
    X = torch.randn((N, ws.D_IN), device=dev)
    prior = torch.zeros((N, ws.KMAX), device=dev)
    T = torch.full((N, ws.KMAX), 1.0 / ws.KMAX, device=dev)
    fwd_flops = 2.0 * N * (ws.D_IN * ws.H + ws.H * ws.H + ws.H * ws.KMAX)
    timed("mlp_forward", lambda: net.forward(X, prior), None, fwd_flops)
    timed("mlp_forward_backward", lambda: net.gradients(X, prior, T), None, 3 * fwd_flops)
    # host: the .P text writer (all host threads) against np.savetxt, the same bytes
    import tempfile

    from adamixture_b200.src import utils as src_utils

    Ph = np.random.default_rng(0).uniform(1e-5, 1 - 1e-5, (M, K))
    with tempfile.TemporaryDirectory() as d:
        t0 = time.perf_counter()
        src_utils.write_outputs(Ph, "native", K, d)
        t_native = time.perf_counter() - t0
        t0 = time.perf_counter()
        np.savetxt(os.path.join(d, "ref.P"), Ph, delimiter=" ")
        t_np = time.perf_counter() - t0
        same = Path(d, f"native.{K}.Q").read_bytes() == Path(d, "ref.P").read_bytes()
    out["write_P_text_host"] = {"ms": t_native * 1e3, "np_savetxt_ms": t_np * 1e3, "identical": same,
                                "host_threads": os.cpu_count(), "values": M * K}
    line = {"metric": "kernel timings", "config": {"workload": cfg["workload"], "N": N, "M": M, "K": K,
            "note": "CUDA events, mean of 3 launches after one warm-up (Hessian passes: 1); GBps from "
                    "algorithmic bytes, hbm_frac against the measured copy bandwidth"}, "kernels": out}
    print(json.dumps(line), flush=True)


CONVERGE_RUNS = ("f32", "bf16", "f16", "mixed", "warm_f16")


def converge_runs(args, cfg, G, dev, which=CONVERGE_RUNS):
    """Time to the converged log-likelihood on the resident cohort G: from the reference's
    default start (randomized SVD + ALS, seed 42), plain float32 Adam-EM to its stop, then
    the other runs in ``which`` (BF16 / FP16 tensor-core sweeps, mixed: tensor-core then
    float32, warm_f16: the learned warm start in front of the FP16 sweep), each timed to
    the first check within 1e-6 relative of the plain float32 run's best log-likelihood."""
    import torch

    from adamixture_b200.model import warm_start as ws
    from adamixture_b200.model.em_adam_gpu import loglikelihood_gpu, optimize_parameters_gpu

    N, M, K = cfg["N"], cfg["M"], cfg["K"]
    tc = 8 <= K <= 16
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    U, S, V, P0, Q0 = ws.init_als(G, N, M, K, seed=42)
    torch.cuda.synchronize()
    t_init = time.perf_counter() - t0
    runs = {}
    precs = {"f32": "f32", "bf16": "bf16" if tc else "f32", "f16": "f16" if tc else "f32",
             "mixed": "mixed", "warm_f16": "f16" if tc else "f32"}
    # load every kernel instance the fits use before any of them is timed (the first
    # launch of a kernel loads its module)
    for prec in sorted({precs[w] for w in which} | {"f32"}):
        optimize_parameters_gpu(G, P0.clone(), Q0.clone(), HP["lr"], HP["beta1"], HP["beta2"], HP["eps"],
                                CHECK, CHECK, K, M, N, 0.5, 1e-4, 3, 0.1, dev, 8192, 256, precision=prec)
    loglikelihood_gpu(G, P0, Q0, M, N, 8192, dev, 256)
    torch.cuda.synchronize()

    def fit(name, P_start, Q_start, prec, extra_s=0.0):
        tr = []
        torch.cuda.synchronize()
        t = time.perf_counter()
        P, Q = optimize_parameters_gpu(G, P_start.clone(), Q_start.clone(), HP["lr"], HP["beta1"], HP["beta2"],
                                       HP["eps"], args.converge_max_iter, CHECK, K, M, N, 0.5, 1e-4, 3, 0.1, dev,
                                       8192, 256, precision=prec, trace=tr)
        torch.cuda.synchronize()
        el = time.perf_counter() - t
        L = loglikelihood_gpu(G, P, Q, M, N, 8192, dev, 256)
        runs[name] = {"precision": prec, "seconds": el + extra_s, "iterations": tr[-1][0] if tr else 0,
                      "loglik": L, "trace": [(it, Lc, sec + extra_s) for it, Lc, sec in tr],
                      "extra_seconds": extra_s}

    fit("f32", P0, Q0, "f32")
    target = max(e[1] for e in runs["f32"]["trace"])
    for w in which:
        if w in ("f32", "warm_f16"):
            continue
        fit(w, P0, Q0, precs[w])
    if "warm_f16" in which:
        net = ws.WarmStartMLP.load(ws.DEFAULT_WEIGHTS, dev)
        torch.cuda.synchronize()
        t = time.perf_counter()
        Pw, Qw = ws.predict(net, G, M, U, S, V, Q0, P0)
        torch.cuda.synchronize()
        fit("warm_f16", Pw, Qw, precs["warm_f16"], extra_s=time.perf_counter() - t)
    out = {}
    base = runs["f32"]
    base_reach = next(((it, sec) for it, L, sec in base["trace"] if L >= target - 1e-6 * abs(target)), None)
    for name, r in runs.items():
        reach = next(((it, sec) for it, L, sec in r["trace"] if L >= target - 1e-6 * abs(target)), None)
        out[name] = {"precision": r["precision"], "seconds_to_target": reach[1] if reach else None,
                     "iterations_to_target": reach[0] if reach else None,
                     "frac_of_f32_time": (reach[1] / base_reach[1]) if (reach and base_reach) else None,
                     "seconds_to_stop": r["seconds"], "iterations_to_stop": r["iterations"],
                     "loglik": r["loglik"],
                     "rel_gap_to_f32": (base["loglik"] - r["loglik"]) / abs(base["loglik"])}
        if r["extra_seconds"]:
            out[name]["warm_start_seconds"] = r["extra_seconds"]
    return {"target": "first check within 1e-6 relative of the plain float32 run's best (traced) "
                      "log-likelihood; seconds are wall time of optimize_parameters_gpu on the resident "
                      "cohort (warm_f16 includes the network's prediction)",
            "start": "randomized SVD (k=max(K,16), power 5) + ALS, seed 42", "init_seconds": t_init,
            "check_every": CHECK, "max_iter": args.converge_max_iter, "target_loglik": target,
            "runs": out}


def run_converge(args, cfg):
    """``--converge``: the time-to-target runs of every arithmetic as one JSON line."""
    import torch

    from adamixture_b200 import ops
    from adamixture_b200.src.simulate import make_cohort

    dev = torch.device("cuda", 0)
    N, M, K = cfg["N"], cfg["M"], cfg["K"]
    coh = make_cohort(N, M, K, cfg["F"], cfg["alpha"], cfg["miss"], cfg["seed"])
    Pq = torch.from_numpy(coh.Pq.astype(np.int32)).to(dev)
    Qq = torch.from_numpy(coh.Qq.astype(np.int32)).to(dev)
    G = ops.simulate_packed(Pq, Qq, coh.miss_q, coh.keys)
    del Pq, Qq
    res = converge_runs(args, cfg, G, dev)
    print(json.dumps({"metric": "time-to-converged loglik", "config": {"workload": cfg["workload"]}, **res}),
          flush=True)


def run_errors(args, cfg):
    """``--errors``: each E-step arithmetic against the float64 run of the same iterations.
    From the benchmark's start (P0, Q0), the priming step and ``--error-iters`` iterations
    in float64, float32, FP16 and BF16 (tensor-core forms where K <= 16); after each
    iteration, max |P - P_f64|, max |Q - Q_f64| and the float64 log-likelihood's relative
    gap to the float64 run's. One JSON line."""
    import torch

    from adamixture_b200 import ops
    from adamixture_b200.model.em_adam_gpu import EMAdamOptimizer
    from adamixture_b200.src.simulate import make_cohort

    dev = torch.device("cuda", 0)
    N, M, K = cfg["N"], cfg["M"], cfg["K"]
    coh = make_cohort(N, M, K, cfg["F"], cfg["alpha"], cfg["miss"], cfg["seed"])
    G = ops.simulate_packed(torch.from_numpy(coh.Pq.astype(np.int32)).to(dev),
                            torch.from_numpy(coh.Qq.astype(np.int32)).to(dev), coh.miss_q, coh.keys)
    rng = np.random.default_rng(cfg["seed"])
    P0 = np.clip(rng.random((M, K)), 1e-5, 1 - 1e-5)
    Q0 = np.clip(rng.random((N, K)), 1e-5, 1 - 1e-5)
    Q0 /= Q0.sum(1, keepdims=True)
    n = args.error_iters
    ref = []
    out = {}
    for prec in ("f64", "f32", "f16", "bf16"):
        if prec in TC_PRECISIONS and K > 16:
            continue
        P = torch.from_numpy(P0).to(dev)
        Q = torch.from_numpy(Q0).to(dev)
        P32, Q32 = P.float(), Q.float()
        ws = ops.Workspace.get(dev, ops.em_workspace_bytes(M, N, K, prec))
        opt = EMAdamOptimizer(P.shape, Q.shape, HP["lr"], HP["beta1"], HP["beta2"], HP["eps"], dev, prec)
        rows = []
        for it in range(n + 1):
            opt.fused_iteration(G, P, Q, P32, Q32, M, ws)
            L = float(ops.loglik_device(G, P, Q, M, "f64").item())
            if prec == "f64":
                ref.append((P.clone(), Q.clone(), L))
                rows.append({"iteration": it, "loglik": L})
            else:
                Pr, Qr, Lr = ref[it]
                rows.append({"iteration": it, "max_abs_dP": float((P - Pr).abs().max()),
                             "max_abs_dQ": float((Q - Qr).abs().max()),
                             "rel_loglik_gap": (Lr - L) / abs(Lr), "loglik": L})
        if ops.em_status(ws, M, N, K, prec) != 0:
            raise RuntimeError(f"E-step sweep reported a nonzero status ({prec})")
        out[prec] = rows
        del P, Q, P32, Q32, opt
        torch.cuda.synchronize()
    print(json.dumps({"metric": "E-step arithmetic error against float64", "config": {
        "workload": cfg["workload"], "start": "reference random EM start, default_rng(seed)",
        "iterations": "0 = after the priming step; then Adam-EM iterations",
        "loglik": "float64 log-likelihood of each run's own P, Q"}, "runs": out}), flush=True)


def run_batch_sweeps(G, M, N, Ks, starts, dev):
    """``--config c4 --batch-sweeps``: one float64 sweep launch per K alone, the batched
    entry point with that one problem, all K in one batched launch, and all K on fold 0's
    masked copy (CUDA events, mean of 5 launches after one warm-up; 3 for the batches)."""
    import torch

    from adamixture_b200 import ops
    from adamixture_b200.model.em_adam_batch import fold_copy

    def timed(fn, reps=5):
        fn()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(reps):
            fn()
        e1.record()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / reps

    out = {}
    for K in Ks:
        ws = ops.Workspace.get(dev, ops.em_workspace_bytes(M, N, K, "f64"))
        out[f"single_K{K}"] = timed(lambda: ops.em_sweep(G, starts[K][0], starts[K][1], M, "f64", ws))
        b1 = ops.EmBatch(M, N, [K], dev)
        out[f"batch1_K{K}"] = timed(lambda: b1.sweep([G], [starts[K][0]], [starts[K][1]]))
    b = ops.EmBatch(M, N, Ks, dev)
    out["batch_all"] = timed(lambda: b.sweep([G] * len(Ks), [starts[K][0] for K in Ks], [starts[K][1] for K in Ks]), 3)
    out["sum_single"] = sum(out[f"single_K{K}"] for K in Ks)
    Gf = fold_copy(G, M, 42, 10, 0)
    out["batch_fold0_all"] = timed(lambda: b.sweep([Gf] * len(Ks), [starts[K][0] for K in Ks],
                                                   [starts[K][1] for K in Ks]), 3)
    print(json.dumps({"metric": "float64 sweep launch ms, single vs batched", "N": N, "M": M, "ms": out}),
          flush=True)


def run_cv_batch(args, cfg):
    """``--config c4``: the K sweep K=2..12 and 5-fold cross-validation (10 % of the
    entries per fold by the seeded hash rule) as batched problems -- every iteration one
    launch of the batched float64 sweep over all live problems -- against the same problems
    run one at a time through the single-problem path. Reports both wall times, the largest
    difference between their P/Q, and the CV index per K. One JSON line."""
    import torch

    from adamixture_b200 import ops
    from adamixture_b200.model.em_adam_batch import cross_validate
    from adamixture_b200.src.simulate import make_cohort

    dev = torch.device("cuda", 0)
    N, M = cfg["N"], cfg["M"]
    coh = make_cohort(N, M, cfg["K"], cfg["F"], cfg["alpha"], cfg["miss"], cfg["seed"])
    G = ops.simulate_packed(torch.from_numpy(coh.Pq.astype(np.int32)).to(dev),
                            torch.from_numpy(coh.Qq.astype(np.int32)).to(dev), coh.miss_q, coh.keys)
    Ks = list(range(2, 13))
    starts = {}
    for K in Ks:
        rng = np.random.default_rng(cfg["seed"] + K)
        P0 = np.clip(rng.random((M, K)), 1e-5, 1 - 1e-5)
        Q0 = np.clip(rng.random((N, K)), 1e-5, 1 - 1e-5)
        Q0 /= Q0.sum(1, keepdims=True)
        starts[K] = (torch.from_numpy(P0).to(dev), torch.from_numpy(Q0).to(dev))
    if args.batch_sweeps:
        run_batch_sweeps(G, M, N, Ks, starts, dev)
        return
    kw = dict(n_folds=5, n_buckets=10, seed=42, polish_iters=args.cv_polish, max_iter=args.cv_max_iter)
    # load the kernel instances both paths use before timing
    cross_validate(G, M, N, [2, 12], starts, **{**kw, "max_iter": 5, "polish_iters": 1}, batched=True)
    cross_validate(G, M, N, [2, 12], starts, **{**kw, "max_iter": 5, "polish_iters": 1}, batched=False)
    b = cross_validate(G, M, N, Ks, starts, batched=True, **kw)
    s = cross_validate(G, M, N, Ks, starts, batched=False, **kw)
    dmax = 0.0
    for K in Ks:
        for x, y in zip(b["fits"][K], s["fits"][K]):
            dmax = max(dmax, float((x - y).abs().max()))
        for f in range(5):
            for x, y in zip(b["folds"][(K, f)], s["folds"][(K, f)]):
                dmax = max(dmax, float((x - y).abs().max()))
    cv_rel = max(abs(b["cv"][K] - s["cv"][K]) / abs(s["cv"][K]) for K in Ks)
    line = {"metric": "K sweep + cross-validation, batched vs one problem at a time",
            "config": {"workload": cfg["workload"], "Ks": Ks, "folds": 5, "fold_rule": "reference hash, 10 buckets, "
                       "folds 0..4", "polish_iters": args.cv_polish, "max_iter": args.cv_max_iter,
                       "arithmetic": "float64 (tensor-core MMA sweep)"},
            "batched_seconds": b["seconds"], "sequential_seconds": s["seconds"],
            "speedup": (s["seconds"]["fits"] + s["seconds"]["folds"]) / (b["seconds"]["fits"] + b["seconds"]["folds"]),
            "max_abs_diff_PQ": dmax, "max_rel_diff_cv": cv_rel,
            "cv_index": {str(K): b["cv"][K] for K in Ks}, "best_K": min(b["cv"], key=b["cv"].get),
            "held_out_fraction": {str(f): v / (float(ops.sample_counts(G, M).sum().item()) / 2)
                                  for f, v in b["held_out"].items()}}
    print(json.dumps(line), flush=True)


def run_warm_start(args, cfg):
    """``--config c5``: the learned warm start on the held-out cohort. With ``--train``, the
    network is first trained on 50 seeded cohorts (N=20,000, M=50,000, K in 6..10, F in
    0.02..0.15; 5 more choose the epoch) by this library's kernels, targets the converged Q
    of plain EM from the ALS start, and written to ``--weights-out``; otherwise the shipped
    weights are used. Then plain EM from the ALS start and EM from the warm start run on the
    held-out cohort with the default arithmetic: iterations and seconds to the first check
    within 1e-6 relative of the plain run's converged log-likelihood. One JSON line."""
    import torch

    from adamixture_b200.model import warm_start as ws

    dev = torch.device("cuda", 0)
    out = {"metric": "learned warm start vs ALS start", "config": {"workload": cfg["workload"]}}
    if args.train:
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        rep = ws.train_default(dev, out=args.weights_out, n_train=50, n_val=5, size=(20_000, 50_000), epochs=30)
        torch.cuda.synchronize()
        out["training"] = {"seconds": time.perf_counter() - t0, "cohorts": len(rep["cohorts"]),
                           "train_loss": rep["train_loss"], "val_loss": rep["val_loss"],
                           "weights": str(args.weights_out)}
        net = ws.WarmStartMLP.load(args.weights_out, dev)
    else:
        net = ws.WarmStartMLP.load(ws.DEFAULT_WEIGHTS, dev)
    N, M, K = cfg["N"], cfg["M"], cfg["K"]
    G, _ = ws.simulate(N, M, K, cfg["F"], cfg["seed"], dev, alpha=cfg["alpha"], miss=cfg["miss"])
    # load the kernel instances the fits use before timing them
    ws.warm_start_fit(net, G[: (20_000 + 3) // 4], N, 20_000, K, seed=42)
    r = ws.warm_start_fit(net, G, N, M, K, seed=42)
    r.pop("P"), r.pop("Q")
    out["held_out"] = r
    print(json.dumps(out), flush=True)


def run_e2e_dist(args, G_dev, P0, Q0, M_loc, N, K, prec, dev, world):
    """e2e at N GPUs: each rank's packed rows and P rows plus Q from pinned host memory,
    ``optimize_parameters_dist`` for ``steps`` iterations, P rows and Q back to the host;
    max over ranks of the wall time."""
    import torch
    import torch.distributed as dist

    from adamixture_b200.model.em_adam_dist import CudaBackend, optimize_parameters_dist

    G_host = torch.empty(G_dev.shape, dtype=torch.uint8, pin_memory=True)
    G_host.copy_(G_dev)
    P_host = torch.from_numpy(P0).pin_memory()
    Q_host = torch.from_numpy(Q0).pin_memory()
    dist.barrier()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    Gd = G_host.to(dev, non_blocking=True)
    Pd = P_host.to(dev, non_blocking=True)
    Qd = Q_host.to(dev, non_blocking=True)
    Pb, Qb = optimize_parameters_dist(Gd, Pd, Qd, HP["lr"], HP["beta1"], HP["beta2"], HP["eps"], args.steps, CHECK,
                                      K, M_loc, N, 0.5, 1e-4, 3, 0.1, backend=CudaBackend(prec))
    Pr, Qr = Pb.cpu(), Qb.cpu()
    el = torch.tensor([time.perf_counter() - t0], device=dev)
    dist.all_reduce(el, op=dist.ReduceOp.MAX)
    el = float(el.item())
    del Gd
    iters = args.steps
    return {"value": iters / el, "unit": UNIT,
            "h2d_bytes_per_step": (G_host.numel() + P0.nbytes + Q0.nbytes) * world / iters,
            "d2h_bytes_per_step": (Pr.numel() * 8 + Qr.numel() * 8) * world / iters,
            "pinned": True, "seconds": el,
            "note": "optimize_parameters_dist on every rank with max_iter=steps from pinned host shards; "
                    "bytes summed over ranks; max over ranks of the wall time"}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--precision", default=None)
    ap.add_argument("--config", choices=sorted(CONFIGS), default="c3")
    ap.add_argument("--cpu-snps", dest="cpu_snps", type=int, default=REF_SLICE_ROWS,
                    help="SNP rows per timed reference step")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-variants", dest="no_variants", action="store_true",
                    help="skip the float32 / FP16 / BF16 variant measurements")
    ap.add_argument("--no-converge", dest="no_converge", action="store_true",
                    help="skip the time-to-target fits")
    ap.add_argument("--shard", action="store_true",
                    help="use the SNP-sharded path (NCCL all-reduce of T) even on one GPU")
    ap.add_argument("--converge", action="store_true",
                    help="instead of the throughput line, time runs to the converged log-likelihood")
    ap.add_argument("--converge-max-iter", dest="converge_max_iter", type=int, default=300)
    ap.add_argument("--kernels", action="store_true", help="per-kernel timings at the config's shape")
    ap.add_argument("--errors", action="store_true",
                    help="per-iteration error of each E-step arithmetic against the float64 run")
    ap.add_argument("--error-iters", dest="error_iters", type=int, default=20)
    ap.add_argument("--cv-max-iter", dest="cv_max_iter", type=int, default=200,
                    help="c4: iteration cap of the full-data fits")
    ap.add_argument("--cv-polish", dest="cv_polish", type=int, default=10,
                    help="c4: Adam-EM iterations per fold")
    ap.add_argument("--train", action="store_true", help="c5: train the warm-start network first")
    ap.add_argument("--weights-out", dest="weights_out", default="warm_start_weights.npz",
                    help="c5 --train: where the trained weights go")
    ap.add_argument("--batch-sweeps", dest="batch_sweeps", action="store_true",
                    help="c4: time single and batched sweep launches instead of the CV runs")
    ap.add_argument("--kernels-skip-hessian", dest="kernels_skip_hessian", action="store_true")
    ap.add_argument("--tiles", action="store_true",
                    help="float64 sweep time per tile layout and the autotuner's pick, K = 2..12 and c1-c3")
    ap.add_argument("--sweep-by-k", dest="sweep_by_k", action="store_true",
                    help="float32 vs FP16 tensor-core sweep time for K = 2..16")
    ap.add_argument("--graphs", action="store_true",
                    help="eager vs graph-replayed Adam-EM iterations at the small configs")
    args = ap.parse_args()
    if args.warmup < 3:
        print("bench.py: --warmup must be >= 3", file=sys.stderr)
        args.warmup = 3
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    cfg = CONFIGS[args.config]
    if args.impl == "reference":
        run_reference_arm(args, cfg, rank)
        return
    if args.converge:
        if rank == 0:
            run_converge(args, cfg)
        return
    if args.kernels:
        if rank == 0:
            run_kernels(args, cfg)
        return
    if args.errors:
        if rank == 0:
            run_errors(args, cfg)
        return
    if args.config == "c4":
        if rank == 0:
            run_cv_batch(args, cfg)
        return
    if args.config == "c5":
        if rank == 0:
            run_warm_start(args, cfg)
        return
    if args.tiles:
        run_tiles(args)
        return
    if args.sweep_by_k:
        if rank == 0:
            run_sweep_by_k(args)
        return
    if args.graphs:
        if rank == 0:
            run_graphs(args)
        return
    run_gpu_arm(args, cfg, rank, world, local_rank)


if __name__ == "__main__":
    main()
