#!/usr/bin/env python
"""Benchmark of the ADMIXTURE Adam-EM hot path on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--precision auto|f32|f64|bf16|f16] [--config c3|c2|c1]

Workload (default ``c3``): N=200,000 samples, M=500,000 SNPs, K=10; a seeded synthetic
admixed cohort (Balding-Nichols F=0.02; Q 70% Dirichlet(0.05) / 30% Dirichlet(1); 1%
missing) sampled on the device straight into the 2-bit packed layout (25 GB resident).
A step is one Adam-EM iteration of the reference loop (adamixture/model/em_adam_gpu.py:
330-353): one fused E-step sweep over all genotypes + the EM targets and the Adam move,
with the float64 log-likelihood check every 5th iteration (read back to the host, as the
reference's ``.item()`` does). P/Q start from the reference's random EM initialisation
(adamixture/src/adamixture.py:140-156). Inputs (25 GB) exceed L2 (126 MB), so no flush is
needed between steps.

One JSON line on rank 0. ``value`` = EM iterations/s (device-timed, max over ranks);
``e2e`` = the same iterations through the public Python API starting from pinned host
buffers (packed G, P, Q) and ending with P/Q back on the host; ``roofline`` = the E-step
sweep kernel alone (algorithmic bytes: ceil(M/4)*N + 4K(3M+2N) per launch) against the
measured HBM copy bandwidth; ``cpu_baseline`` = the reference's own CPU Adam-EM step
(its Cython kernels compiled from source into oracle/_ref) on a SNP-row slice of the same
cohort, scaled linearly to the full M.
``--impl reference`` prints the reference arm: that CPU implementation as the headline.
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
    # the c3 cohort's generator at one tenth of its SNPs (2.5 GB packed): the size profiled
    # under ncu, whose full capture saves and restores device memory on every pass
    "c3s": dict(workload="Adam-EM, N=200000 samples, M=50000 SNPs, K=10, F=0.02, Q 0.7*Dir(0.05)+0.3*Dir(1), 1% missing",
                N=200_000, M=50_000, K=10, F=0.02, alpha=((0.7, 0.05), (0.3, 1.0)), miss=0.01, seed=2000),
}
TC_PRECISIONS = ("bf16", "f16")   # the tensor-core sweep
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

def cpu_reference_sample(cfg, coh, sample_snps, steps, warmup, G_rows=None):
    """Time the reference's own Adam-EM CPU step (``adamStep``: em.P_step, em.Q_step,
    em.adamUpdateP/Q; adamixture/model/em_adam.py:12-54) on the first ``sample_snps``
    SNP rows of the cohort, all host cores. Returns (seconds per full-M iteration, info)."""
    cores = os.cpu_count() or 1
    os.environ["OMP_NUM_THREADS"] = str(cores)
    from oracle import refmods  # the compiled reference kernels (test/baseline infrastructure)

    kind = "reference" if refmods.available() else "port"
    N, K, M = cfg["N"], cfg["K"], cfg["M"]
    Ms = min(sample_snps, M)
    if G_rows is None:
        G_rows = np.empty((Ms, N), dtype=np.uint8)
        blk = max(4, (1 << 24) // max(N, 1))
        for s in range(0, Ms, blk):
            G_rows[s:s + blk] = coh.genotypes(s, min(blk, Ms - s))
    rng = np.random.default_rng(cfg["seed"])
    P = np.clip(rng.random((Ms, K)), 1e-5, 1 - 1e-5)
    Q = np.clip(rng.random((N, K)), 1e-5, 1 - 1e-5)
    Q /= Q.sum(1, keepdims=True)
    T = np.zeros_like(Q)
    P1 = np.zeros_like(P)
    Q1 = np.zeros_like(Q)
    qb = np.zeros(N)
    mP, vP, mQ, vQ = (np.zeros_like(P), np.zeros_like(P), np.zeros_like(Q), np.zeros_like(Q))
    t = [0]
    if kind == "reference":
        em = refmods.load("em")

        def step():
            em.P_step(G_rows, P, P1, Q, T, qb, K, Ms, N)
            em.Q_step(Q, Q1, T, qb, K, N)
            t[0] += 1
            em.adamUpdateP(P, P1, mP, vP, HP["lr"], HP["beta1"], HP["beta2"], HP["eps"], t[0], Ms, K)
            em.adamUpdateQ(Q, Q1, mQ, vQ, HP["lr"], HP["beta1"], HP["beta2"], HP["eps"], t[0], N, K)
        threads = cores
    else:
        from oracle import em_oracle as orc
        st = orc.Adam(HP["lr"], HP["beta1"], HP["beta2"], HP["eps"]).init(P, Q)

        def step():
            A, B, Tt, q = orc.em_stats(G_rows, P, Q)
            orc.adam_step(st, P, Q, *orc.em_final(P, Q, A, B, Tt, q))
        threads = 1
    for _ in range(warmup):
        step()
    times = []
    for _ in range(steps):
        t0 = time.perf_counter()
        step()
        times.append(time.perf_counter() - t0)
    per = float(np.median(times))
    full = per * (M / Ms)
    info = {"kind": kind, "cores": threads,
            "sample": f"{Ms} of {M} SNP rows x all {N} samples, K={K}; median of {steps} adamStep "
                      f"calls, scaled x{M / Ms:.1f} to the full M (cost is linear in M)"}
    return full, info


def run_reference_arm(args, cfg, rank):
    if rank != 0:
        return
    from adamixture_b200.src.simulate import make_cohort

    coh = make_cohort(cfg["N"], cfg["M"], cfg["K"], cfg["F"], cfg["alpha"], cfg["miss"], cfg["seed"])
    sample = max(64, min(cfg["M"], int(args.cpu_snps)))
    full, info = cpu_reference_sample(cfg, coh, sample, args.steps, args.warmup)
    v = 1.0 / full
    line = {
        "impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": full * 1e3,
        "higher_is_better": True, "scaling": "strong", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic", "config": {"workload": cfg["workload"], "sample_snps": sample},
        "cpu_baseline": dict(value=v, unit=UNIT, **info),
        "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------- GPU arm

def run_gpu_arm(args, cfg, rank, world, local_rank):
    import torch

    from adamixture_b200 import ops
    from adamixture_b200.model.em_adam_gpu import EMAdamOptimizer, optimize_parameters_gpu, resolve_precision
    from adamixture_b200.src.simulate import make_cohort

    dev = torch.device("cuda", local_rank)
    torch.cuda.set_device(dev)
    N, M, K = cfg["N"], cfg["M"], cfg["K"]
    prec = resolve_precision(K, args.precision)
    sharded = world > 1 or args.shard
    if sharded:
        import datetime

        import torch.distributed as dist
        os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
        os.environ.setdefault("MASTER_PORT", "29531")
        os.environ.setdefault("RANK", str(rank))
        os.environ.setdefault("WORLD_SIZE", str(world))
        dist.init_process_group("nccl", device_id=dev, timeout=datetime.timedelta(minutes=10))

    from adamixture_b200.model.em_adam_dist import CudaBackend, ShardedAdamEM, shard_rows
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
    P = torch.from_numpy(P0).to(dev)
    Q = torch.from_numpy(Q0).to(dev)
    P32, Q32 = P.float(), Q.float()
    ws = ops.Workspace.get(dev, ops.em_workspace_bytes(M_loc, N, K, prec))
    llp = "f64" if prec == "f64" else "f32"
    Pll, Qll = (P, Q) if llp == "f64" else (P32, Q32)
    launches = {"n": 0}

    if not sharded:
        # kernels per fused iteration: sweep (+ the BF16 copy of Q for the tensor-core sweep)
        # and the update kernel; per check: the log-likelihood kernel and its final sum
        opt = EMAdamOptimizer(P.shape, Q.shape, HP["lr"], HP["beta1"], HP["beta2"], HP["eps"], dev, prec)
        per_iter = 3 if prec in TC_PRECISIONS else 2

        def one_step(it):
            opt.fused_iteration(G, P, Q, P32, Q32, M, ws)
            launches["n"] += per_iter
            if (it + 1) % CHECK == 0:
                float(ops.loglik_device(G, Pll, Qll, M, llp).item())
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
    for it in range(args.warmup):
        one_step(it)
    torch.cuda.synchronize()
    launches["n"] = 0
    if sharded:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    uuid = None
    try:
        uuid = "GPU-" + str(torch.cuda.get_device_properties(dev).uuid)
    except Exception:
        pass
    stream = torch.cuda.current_stream(dev)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with Clocks(uuid) as clk:
        e0.record(stream)
        for it in range(args.steps):
            one_step(it)
        e1.record(stream)
        torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    if sharded:
        t = torch.tensor([ms], device=dev)
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        ms = float(t.item())
    ms_per_step = ms / args.steps

    # roofline: the sweep kernel alone (this rank's rows), CUDA events on its stream
    Pin, Qin = (P, Q) if prec == "f64" else (P.float(), Q.float())
    reps = max(3, min(10, args.steps))
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
            "kernel": f"em_sweep_tc_kernel<{prec == 'f16'}>" if prec in TC_PRECISIONS else f"em_sweep_kernel<{'double' if prec == 'f64' else 'float'},{ops_kmax(K)}>",
            "launch_ms": sweep_ms, "alg_bytes": ab, "peak_kind": peak_kind,
            "entries_per_s": M_loc * N / (sweep_ms * 1e-3), "snp_rows_per_rank": M_loc}
    if prec in TC_PRECISIONS:
        # the contractions (h, 1-h, A, B, T: 8 M N K flops of useful work; K padded to 16 in
        # the MMAs) against the measured dense BF16 peak (FP16's dense rate is the same), for
        # the tensor-core sweep
        tf = peaks_tensor()
        flops = 8.0 * M_loc * N * K
        roof["tensor"] = {"achieved_tflops": flops / (sweep_ms * 1e-3) / 1e12, "peak_tflops": tf,
                          "frac": flops / (sweep_ms * 1e-3) / 1e12 / tf if tf else None,
                          "flops_per_launch": flops}

    # e2e through the public API from pinned host buffers
    e2e = None
    if not args.no_e2e:
        if not sharded:
            e2e = run_e2e(args, G, P0, Q0, M, N, K, prec, dev)
        else:
            e2e = run_e2e_dist(args, G, P0, Q0, M_loc, N, K, prec, dev, world)

    cpu = None
    if not args.no_cpu and rank == 0 and world == 1:
        G_rows = ops.unpack_u8(G, 0, min(M, args.cpu_snps), M).cpu().numpy()
        full, info = cpu_reference_sample(cfg, coh, min(M, args.cpu_snps), 3, 1, G_rows=G_rows)
        cpu = dict(value=1.0 / full, unit=UNIT, **info)

    if rank == 0:
        line = {
            "metric": METRIC, "value": 1000.0 / ms_per_step, "unit": UNIT,
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": ms_per_step, "higher_is_better": True, "scaling": "strong",
            "vs_baseline": None, "dtype": {"f64": "f64", "f32": "f32", "bf16": "bf16", "f16": "f16"}[prec],
            "data": "synthetic",
            "config": {"workload": cfg["workload"], "precision": prec, "check_every": CHECK,
                       "l2": "inputs (packed G) larger than L2; no flush",
                       "genotype_GBps": ((M + 3) // 4) * N / (ms_per_step * 1e-3) / 1e9,
                       "parallelism": "single GPU" if not sharded else
                       f"SNP rows sharded over {world} rank(s) (one all-reduce of T per iteration)"},
            "roofline": roof, "cpu_baseline": cpu, "e2e": e2e,
            "gpu_launches": launches["n"], "clocks": clk.summary(),
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
    Gd = G_host.to(dev, non_blocking=True)
    Pd = P_host.to(dev, non_blocking=True)
    Qd = Q_host.to(dev, non_blocking=True)
    trace = []
    Pb, Qb = optimize_parameters_gpu(Gd, Pd, Qd, HP["lr"], HP["beta1"], HP["beta2"], HP["eps"],
                                     iters, CHECK, K, M, N, 0.5, 1e-4, 3, 0.1, dev, 8192, 512,
                                     precision=prec, trace=trace)
    Pr, Qr = Pb.cpu(), Qb.cpu()
    el = time.perf_counter() - t0
    del Gd
    nchecks = len(trace) + 1
    return {"value": iters / el, "unit": UNIT,
            "h2d_bytes_per_step": (G_host.numel() + P0.nbytes + Q0.nbytes) / iters,
            "d2h_bytes_per_step": (Pr.numel() * 8 + Qr.numel() * 8 + 8 * nchecks) / iters,
            "pinned": pinned, "seconds": el,
            "note": "one optimize_parameters_gpu call with max_iter=steps from host tensors: "
                    "H2D of packed G/P/Q, priming + steps iterations, loglik checks read back, "
                    "best P/Q copied to the host"}


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


def run_converge(args, cfg):
    """Time to the converged log-likelihood at the config: from the reference's default
    start (randomized SVD + ALS), plain float32 Adam-EM to its stop, then the BF16 and FP16
    tensor-core sweeps, mixed (tensor-core then float32) and the learned warm start with
    the default arithmetic, each timed to the first check within 1e-6 relative of the plain
    float32 run's best log-likelihood. One JSON line."""
    import torch

    from adamixture_b200 import ops
    from adamixture_b200.model import warm_start as ws
    from adamixture_b200.model.em_adam_gpu import loglikelihood_gpu, optimize_parameters_gpu
    from adamixture_b200.src.simulate import make_cohort

    dev = torch.device("cuda", 0)
    N, M, K = cfg["N"], cfg["M"], cfg["K"]
    coh = make_cohort(N, M, K, cfg["F"], cfg["alpha"], cfg["miss"], cfg["seed"])
    Pq = torch.from_numpy(coh.Pq.astype(np.int32)).to(dev)
    Qq = torch.from_numpy(coh.Qq.astype(np.int32)).to(dev)
    G = ops.simulate_packed(Pq, Qq, coh.miss_q, coh.keys)
    del Pq, Qq
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    U, S, V, P0, Q0 = ws.init_als(G, N, M, K, seed=42)
    torch.cuda.synchronize()
    t_init = time.perf_counter() - t0
    runs = {}
    # load every kernel instance the fits use before any of them is timed (the first
    # launch of a kernel loads its module)
    for prec in ("f32", "bf16", "f16"):
        if prec in TC_PRECISIONS and K > 16:
            continue
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
                      "loglik": L, "trace": tr}

    fit("plain_f32", P0, Q0, "f32")
    target = max(e[1] for e in runs["plain_f32"]["trace"])
    fit("bf16", P0, Q0, "bf16" if 8 <= K <= 16 else "f32")
    fit("f16", P0, Q0, "f16" if 8 <= K <= 16 else "f32")
    fit("mixed", P0, Q0, "mixed")
    net = ws.WarmStartMLP.load(ws.DEFAULT_WEIGHTS, dev)
    torch.cuda.synchronize()
    t = time.perf_counter()
    Pw, Qw = ws.predict(net, G, M, U, S, V, Q0, P0)
    torch.cuda.synchronize()
    fit("warm_auto", Pw, Qw, "auto", extra_s=time.perf_counter() - t)
    out = {}
    for name, r in runs.items():
        reach = next(((it, sec) for it, L, sec in r["trace"] if L >= target - 1e-6 * abs(target)), None)
        out[name] = {"precision": r["precision"], "seconds_to_stop": r["seconds"], "iterations_to_stop": r["iterations"],
                     "loglik": r["loglik"], "rel_gap_to_plain_f32": (runs["plain_f32"]["loglik"] - r["loglik"])
                     / abs(runs["plain_f32"]["loglik"]),
                     "iterations_to_target": reach[0] if reach else None,
                     "seconds_to_target": reach[1] if reach else None}
    line = {"metric": "time-to-converged loglik", "config": {"workload": cfg["workload"],
            "start": "randomized SVD (k=max(K,16), power 5) + ALS, seed 42", "check_every": CHECK,
            "max_iter": args.converge_max_iter, "target": "first check within 1e-6 relative of the plain float32 "
            "run's best (traced) log-likelihood"}, "init_seconds": t_init, "runs": out}
    print(json.dumps(line), flush=True)


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
    ap.add_argument("--cpu-snps", dest="cpu_snps", type=int, default=4096)
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--shard", action="store_true",
                    help="use the SNP-sharded path (NCCL all-reduce of T) even on one GPU")
    ap.add_argument("--converge", action="store_true",
                    help="instead of the throughput line, time runs to the converged log-likelihood")
    ap.add_argument("--converge-max-iter", dest="converge_max_iter", type=int, default=300)
    ap.add_argument("--kernels", action="store_true", help="per-kernel timings at the config's shape")
    ap.add_argument("--kernels-skip-hessian", dest="kernels_skip_hessian", action="store_true")
    ap.add_argument("--sweep-by-k", dest="sweep_by_k", action="store_true",
                    help="float32 vs FP16 tensor-core sweep time for K = 2..16")
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
    if args.sweep_by_k:
        if rank == 0:
            run_sweep_by_k(args)
        return
    run_gpu_arm(args, cfg, rank, world, local_rank)


if __name__ == "__main__":
    main()
