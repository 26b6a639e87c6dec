"""Regenerate the golden fixtures in tests/golden/ from the reference implementation.

Run from the repository root, in a tree that has the reference sources and the
compiled reference modules (``make -C oracle``):

    python tests/golden/make_golden.py [edge synth demo demo_gpu solvers cv_proj align supervised]

What it records (all from the reference's own code, imported from its source tree;
its ``torch.compile`` wrappers run eagerly as float64 torch code on the CPU, with the
CUDA unpack op replaced by a bit-shift unpacker of the same packed layout):

* ``demo.npz``: the reference demo cohort (105 samples x 8451 SNPs): raw BED rows,
  the reference reader's packed and unpacked output (checked here against the
  reference's reader fixtures), allele frequencies, the reference's GPU ALS init
  (``demo/outputs/gpu/adamem/demo_run.als.*``), one ``EMAdamOptimizer.run_em_step``
  from that init (A, B, T, q_bat, P_EM, Q_EM), a 20-iteration Adam-EM trace
  (float32 P/Q snapshots after the priming step and after iterations 1, 2, 3, 5, 10,
  15, 20, and every iteration's log-likelihood), and the converged ``optimize_parameters_gpu`` result.
* ``synth.npz``: a seeded synthetic cohort (N=301, M=2003, K=8, 2% missing) with the
  same records (trace of 10 iterations).
* ``edge.npz``: a tiny cohort (N=37, M=29, K=4) with an all-missing sample and an
  all-missing SNP, with one E-step and the log-likelihood.
* ``demo_gpu.npz``: the reference's GPU golden files of the demo run (SVD, ALS, BR-QN and
  Adam-EM results).
* ``solvers.npz``: the reference's CPU BVLS (K = 1..64), gradient/Hessian and SQP
  outputs on seeded problems.
* ``supervised.npz``: the reference's supervised initialisation and its Adam-EM (GPU path,
  run on the CPU) and SQP + ZAL (CPU path) fits on a cohort with 40 % labelled samples.
* ``align.npz``: the reference's cluster alignment across K on seeded Q matrices.
* ``cv_proj.npz``: the reference's cross-validation index (5 folds, seed 42) and fold
  rules, and its Adam-EM and SQP + ZAL projections, on a seeded cohort (N=90, M=700, K=3).
* ``c2_trace.npz`` (only when named: about 20 minutes on 8 cores): the reference's
  Adam-EM iterations on the mid-size benchmark cohort (N=10,000, M=200,000, K=8,
  Balding-Nichols F=0.05, Q Dirichlet(0.3), 0.5 % missing; the seeded sampler of
  adamixture_b200/src/simulate.py, seed 1000) from the reference's random EM start
  drawn with default_rng(1000): the priming step and 20 iterations, each recorded as P on
  1,024 seeded SNP rows and Q on 1,024 seeded samples (float32) plus the column sums of
  the full P and Q (float64), and the log-likelihood after iterations 0, 5, 10, 15, 20.
"""
from __future__ import annotations

import os
import sys
from pathlib import Path

os.environ.setdefault("TORCHDYNAMO_DISABLE", "1")
ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

import numpy as np  # noqa: E402
import torch  # noqa: E402

from oracle import refmods  # noqa: E402

OUT = Path(__file__).resolve().parent
torch.set_num_threads(os.cpu_count() or 1)


def torch_unpacker(G, start, count, M):
    j = torch.arange(start, start + count)
    rows = G[j >> 2].to(torch.int32)
    return ((rows >> ((j & 3) * 2).to(torch.int32)[:, None]) & 3).to(torch.uint8)


def reference():
    refmods.import_reference()
    from adamixture.model import em_adam_gpu
    from adamixture.src import utils

    utils.get_unpacker = lambda device, tpb: torch_unpacker
    em_adam_gpu.utils.get_unpacker = utils.get_unpacker
    return em_adam_gpu, utils


HP = dict(lr=0.005, beta1=0.80, beta2=0.88, reg_adam=1e-8, check=5, lr_decay=0.5,
          min_lr=1e-4, patience=3, tol=0.1)


def run_records(em, utils, Gp, M, N, K, P0, Q0, trace_iters, converge=True):
    """E-step, trace and converged run from (P0, Q0) through the reference code."""
    dev = torch.device("cpu")
    G = torch.from_numpy(Gp)
    P = torch.from_numpy(P0.copy())
    Q = torch.from_numpy(Q0.copy())
    rec = {}
    opt = em.EMAdamOptimizer(P.shape, Q.shape, HP["lr"], HP["beta1"], HP["beta2"], HP["reg_adam"], dev)
    P_EM, Q_EM = opt.run_em_step(G, P, Q, M, 8192, torch_unpacker)
    rec.update(A=opt.A_accum.numpy().copy(), B=opt.B_accum.numpy().copy(),
               T=opt.T_accum.numpy().copy(), q_bat=opt.q_bat.numpy().copy(),
               P_EM=P_EM.numpy().copy(), Q_EM=Q_EM.numpy().copy())
    rec["loglik0"] = np.float64(em.loglikelihood_gpu(G, P, Q, M, N, 8192, dev, 1))
    # The reference loop (em_adam_gpu.py:318-337) step by step, recording snapshots.
    opt = em.EMAdamOptimizer(P.shape, Q.shape, HP["lr"], HP["beta1"], HP["beta2"], HP["reg_adam"], dev)
    opt.run_em_step(G, P, Q, M, 8192, torch_unpacker)
    opt.step(P, Q, opt.P_EM, opt.Q_EM)
    snapsP, snapsQ, lls = [P.numpy().copy()], [Q.numpy().copy()], []
    for it in range(trace_iters):
        opt.run_em_step(G, P, Q, M, 8192, torch_unpacker)
        opt.step(P, Q, opt.P_EM, opt.Q_EM)
        snapsP.append(P.numpy().copy())
        snapsQ.append(Q.numpy().copy())
        lls.append(em.loglikelihood_gpu(G, P, Q, M, N, 8192, dev, 1))
    keep = [t for t in (0, 1, 2, 3, 5, 10, 15, 20) if t <= trace_iters]
    rec["trace_iters"] = np.array(keep)
    # float32 snapshots: the per-iteration parity bar is 1e-5 absolute
    rec["trace_P"] = np.stack([snapsP[t] for t in keep]).astype(np.float32)
    rec["trace_Q"] = np.stack([snapsQ[t] for t in keep]).astype(np.float32)
    rec["trace_loglik"] = np.array(lls)
    if converge:
        Pc, Qc = em.optimize_parameters_gpu(
            G, torch.from_numpy(P0.copy()), torch.from_numpy(Q0.copy()), HP["lr"], HP["beta1"],
            HP["beta2"], HP["reg_adam"], 10000, HP["check"], K, M, N, HP["lr_decay"],
            HP["min_lr"], HP["patience"], HP["tol"], dev, 8192, 1)
        rec["conv_P"] = Pc.numpy().copy()
        rec["conv_Q"] = Qc.numpy().copy()
        rec["conv_loglik"] = np.float64(em.loglikelihood_gpu(G, Pc, Qc, M, N, 8192, dev, 1))
    return rec


def demo(em, utils):
    tree = refmods.REFERENCE_TREE / "adamixture" / "demo"
    bed = tree / "data" / "demo_data.bed"
    Gp_t, N, M = utils.read_data(str(bed), packed=True, chunk_size=8192, verbose=False)
    G_u, N2, M2 = utils.read_data(str(bed), packed=False, chunk_size=8192, verbose=False)
    assert (N, M) == (N2, M2)
    Gp = Gp_t.numpy()
    exp_p = np.loadtxt(tree / "outputs" / "reader" / "demo_data.G.packed.expected").astype(np.uint8)
    exp_u = np.loadtxt(tree / "outputs" / "reader" / "demo_data.G.expected").astype(np.uint8)
    assert np.array_equal(exp_p, Gp), "reference reader disagrees with its packed fixture"
    assert np.array_equal(exp_u, G_u), "reference reader disagrees with its unpacked fixture"
    nb = (N + 3) // 4
    bed_rows = np.fromfile(bed, dtype=np.uint8, offset=3).reshape(-1, nb)
    f = utils.calculate_frequencies_cpu(G_u, M, N, 8192)
    als = tree / "outputs" / "gpu" / "adamem"
    P0 = np.loadtxt(als / "demo_run.als.P.expected")
    Q0 = np.loadtxt(als / "demo_run.als.Q.expected")
    K = P0.shape[1]
    rec = run_records(em, utils, Gp, M, N, K, P0, Q0, trace_iters=20)
    np.savez_compressed(OUT / "demo.npz", N=N, M=M, K=K, bed_rows=bed_rows, packed=Gp,
                        unpacked=G_u, freq=f, P0=P0, Q0=Q0, **rec)
    print("demo.npz", N, M, K, rec["conv_loglik"])


def synth(em, utils):
    from adamixture_b200.src.simulate import make_cohort

    N, M, K = 301, 2003, 8
    coh = make_cohort(N, M, K, F=0.05, alpha=0.3, miss=0.02, seed=7)
    Gp = coh.packed()
    rng = np.random.default_rng(11)
    P0 = np.clip(coh.P + rng.normal(0, 0.05, coh.P.shape), 1e-5, 1 - 1e-5)
    Q0 = np.clip(coh.Q + rng.uniform(0, 0.2, coh.Q.shape), 1e-5, 1 - 1e-5)
    Q0 /= Q0.sum(1, keepdims=True)
    rec = run_records(em, utils, Gp, M, N, K, P0, Q0, trace_iters=10)
    np.savez_compressed(OUT / "synth.npz", N=N, M=M, K=K, packed=Gp, P0=P0, Q0=Q0,
                        Pq=coh.Pq, Qq=coh.Qq, miss_q=coh.miss_q,
                        keys=np.array(coh.keys, dtype=np.uint64), **rec)
    print("synth.npz", rec["conv_loglik"])


def edge(em, utils):
    from adamixture_b200.src.packing import pack

    N, M, K = 37, 29, 4
    rng = np.random.default_rng(3)
    G = rng.integers(0, 3, size=(M, N)).astype(np.uint8)
    G[rng.random((M, N)) < 0.1] = 3
    G[:, 5] = 3      # a sample with no observed SNP
    G[11, :] = 3     # a SNP with no observed sample
    Gp = pack(G)
    P0 = np.clip(rng.random((M, K)), 1e-5, 1 - 1e-5)
    Q0 = rng.random((N, K))
    Q0 /= Q0.sum(1, keepdims=True)
    rec = run_records(em, utils, Gp, M, N, K, P0, Q0, trace_iters=3, converge=False)
    np.savez_compressed(OUT / "edge.npz", N=N, M=M, K=K, packed=Gp, unpacked=G, P0=P0, Q0=Q0, **rec)
    print("edge.npz", rec["loglik0"])


def demo_gpu():
    """The reference's GPU golden files for the demo run (K=7, seed 42, power 5, tol_svd
    0.1): randomized SVD, ALS init (shared by both optimisers), converged BR-QN and
    Adam-EM P/Q (adamixture/demo/outputs/gpu/*, checked by tests/test_cuda.py there)."""
    out = refmods.REFERENCE_TREE / "adamixture" / "demo" / "outputs" / "gpu"
    rec = {}
    for nm in ("svd.U", "svd.S", "svd.V", "als.P", "als.Q"):
        rec[nm.replace(".", "_")] = np.loadtxt(out / "adamem" / f"demo_run.{nm}.expected")
    for alg in ("adamem", "brqn"):
        for nm in ("P", "Q"):
            rec[f"{alg}_{nm}"] = np.loadtxt(out / alg / f"demo_run.{alg}.{nm}.expected")
    np.savez_compressed(OUT / "demo_gpu.npz", **rec)
    print("demo_gpu.npz", {k: v.shape for k, v in rec.items()})


def solvers():
    """Inputs and outputs of the reference's CPU BVLS, gradient/Hessian and SQP kernels
    (the compiled bvls.pyx / sqp.pyx) on seeded problems."""
    from adamixture_b200.src.simulate import make_cohort

    bv = refmods.load("bvls")
    sq = refmods.load("sqp")
    rec = {}
    rng = np.random.default_rng(21)
    for K in (1, 3, 7, 12, 20, 40, 64):
        X = rng.normal(size=(3 * K + 5, K))
        A = X.T @ X + 0.1 * np.eye(K)
        xt = rng.uniform(-0.6, 1.6, size=(96, K))
        B = xt @ A + rng.normal(0, 0.05, size=(96, K))
        out = np.zeros_like(B)
        bv.batch_bvls_bpp(A, np.ascontiguousarray(B), out, 0.0, 1.0)
        rec[f"bvls{K}_A"], rec[f"bvls{K}_B"], rec[f"bvls{K}_X"] = A, B, out
    _, _, vt = torch.linalg.svd(torch.ones((1, 1), dtype=torch.float64), full_matrices=True)
    for tag, (N, M, K, seed) in {"a": (61, 150, 5, 5), "b": (40, 90, 12, 6), "c": (33, 70, 2, 8)}.items():
        coh = make_cohort(N, M, K, F=0.1, alpha=0.5, miss=0.05, seed=seed)
        G = np.ascontiguousarray(coh.genotypes())
        r2 = np.random.default_rng(seed)
        P = np.clip(coh.P + r2.normal(0, 0.1, coh.P.shape), 1e-5, 1 - 1e-5)
        Q = np.clip(coh.Q + r2.uniform(0, 0.3, coh.Q.shape), 1e-5, 1 - 1e-5)
        Q /= Q.sum(1, keepdims=True)
        _, _, vt = torch.linalg.svd(torch.ones((1, K), dtype=torch.float64), full_matrices=True)
        v_kk = np.ascontiguousarray(vt.t().numpy())
        XtX_q = np.zeros((N, K, K)); Xtz_q = np.zeros((N, K))
        XtX_p = np.zeros((M, K, K)); Xtz_p = np.zeros((M, K))
        Q_next = np.zeros((N, K)); P_next = np.zeros((M, K))
        sq.update_q_sqp(G, Q, Q_next, P, XtX_q, Xtz_q, v_kk, M, N, K)
        sq.update_p_sqp(G, Q, P, P_next, XtX_p, Xtz_p, M, N, K)
        rec.update({f"{tag}_packed": coh.packed(), f"{tag}_G": G, f"{tag}_P": P, f"{tag}_Q": Q,
                    f"{tag}_v_kk": v_kk, f"{tag}_XtX_q": XtX_q, f"{tag}_Xtz_q": Xtz_q,
                    f"{tag}_XtX_p": XtX_p, f"{tag}_Xtz_p": Xtz_p, f"{tag}_Q_next": Q_next,
                    f"{tag}_P_next": P_next})
    np.savez_compressed(OUT / "solvers.npz", **rec)
    print("solvers.npz", len(rec))


def cv_proj(em, utils):
    """The reference's CPU cross-validation (cv.py run_cross_validation: shuffled-list folds,
    5 BR-QN polish iterations, deviance score) and its hash fold rule, plus its GPU-path
    Adam-EM projection run on the CPU and its CPU SQP + ZAL projection, on a seeded cohort."""
    from argparse import Namespace

    from adamixture.src import cv, projection
    from adamixture_b200.src.simulate import make_cohort

    projection.utils.get_unpacker = utils.get_unpacker
    N, M, K = 90, 700, 3
    coh = make_cohort(N, M, K, F=0.1, alpha=0.5, miss=0.02, seed=31)
    G = np.ascontiguousarray(coh.genotypes())
    P = np.clip(coh.P, 1e-5, 1 - 1e-5)
    Q = np.clip(coh.Q, 1e-5, 1 - 1e-5)
    Q /= Q.sum(1, keepdims=True)
    rec = dict(packed=coh.packed(), G=G, P=P, Q=Q)
    flat = np.flatnonzero(G != 3).astype(np.int32)
    rec["cv_shuffled"] = cv._shuffle_non_missing(flat, 42)
    rec["cv_index"] = np.float64(cv.run_cross_validation(Namespace(cv=5, seed=42), G.copy(), N, M, K, P, Q))
    probe = (np.arange(20000, dtype=np.int64) * 104729 + 17) % (1 << 40)
    rec["hash_probe"] = probe
    rec["hash_fold"] = np.stack([cv._hash_fold_mask(probe, 42, 5, f) for f in range(5)]).argmax(0).astype(np.uint8)
    rng = np.random.default_rng(42)
    Q0 = rng.random(size=(N, K))
    Q0 /= Q0.sum(1, keepdims=True)
    rec["proj_Q0"] = Q0
    dev = torch.device("cpu")
    Qa = projection.optimize_projection_gpu(
        torch.from_numpy(coh.packed()), torch.from_numpy(P.copy()), torch.from_numpy(Q0.copy()),
        HP["lr"], HP["beta1"], HP["beta2"], HP["reg_adam"], 10000, HP["check"], M, HP["lr_decay"],
        HP["min_lr"], HP["patience"], HP["tol"], dev, 8192, 1)
    rec["proj_adamem_Q"] = Qa.numpy().copy()
    rec["proj_brqn_Q"] = projection.optimize_projection_original(G, P.copy(), Q0.copy(), 10000, K, M, N, 0.1, 3, 3)
    np.savez_compressed(OUT / "cv_proj.npz", **rec)
    print("cv_proj.npz cv_index", rec["cv_index"])


def supervised(em, utils):
    """The reference's supervised mode on a seeded cohort with 40 % of the samples labelled:
    its initialisation (supervised_entry.py:309-315), its GPU-path Adam-EM run on the CPU
    and its CPU SQP + ZAL run."""
    from adamixture.src import supervised as sup
    from adamixture_b200.src.simulate import make_cohort

    sup.utils.get_unpacker = utils.get_unpacker
    N, M, K = 120, 900, 3
    coh = make_cohort(N, M, K, F=0.1, alpha=0.3, miss=0.02, seed=41)
    G = np.ascontiguousarray(coh.genotypes())
    rng_lab = np.random.default_rng(4)
    y = np.where(rng_lab.random(N) < 0.4, np.argmax(coh.Q, 1) + 1, 0).astype(np.int64)
    rng = np.random.default_rng(42)
    P = sup.init_p_supervised(G, y, K, M)
    P_packed = sup.init_p_supervised_packed(torch.from_numpy(coh.packed()), y, K, M)
    Q = rng.random(size=(N, K)).astype(np.float64)
    sup.init_q_supervised(Q, y, K)
    dev = torch.device("cpu")
    Pa, Qa = sup.optimize_supervised_gpu(
        torch.from_numpy(coh.packed()), torch.from_numpy(P.copy()), torch.from_numpy(Q.copy()), y,
        HP["lr"], HP["beta1"], HP["beta2"], HP["reg_adam"], 10000, HP["check"], M, HP["lr_decay"],
        HP["min_lr"], HP["patience"], HP["tol"], dev, 8192, 1)
    # the first 40 iterations with every check an improvement: P_best is the 40th iterate
    P40, Q40 = sup.optimize_supervised_gpu(
        torch.from_numpy(coh.packed()), torch.from_numpy(P.copy()), torch.from_numpy(Q.copy()), y,
        HP["lr"], HP["beta1"], HP["beta2"], HP["reg_adam"], 40, 1, M, HP["lr_decay"],
        HP["min_lr"], HP["patience"], -1e30, dev, 8192, 1)
    Pb, Qb = sup.optimize_supervised_original(G, P.copy(), Q.copy(), y, 10000, K, M, N, 0.1, 3, 3)
    np.savez_compressed(OUT / "supervised.npz", packed=coh.packed(), G=G, y=y, P0=P, P0_packed=P_packed, Q0=Q,
                        adamem_P=Pa.numpy(), adamem_Q=Qa.numpy(), adamem40_P=P40.numpy(), adamem40_Q=Q40.numpy(),
                        brqn_P=Pb, brqn_Q=Qb)
    print("supervised.npz")


def align():
    """The reference's cluster alignment across K (plot.py align_clusters_clumppling) on
    seeded Q matrices of equal, larger and smaller K."""
    refmods.import_reference()
    from adamixture.src.plot import align_clusters_clumppling

    rng = np.random.default_rng(77)
    rec = {}
    for c, (Kr, Kq) in enumerate([(3, 3), (3, 4), (4, 6), (5, 4), (7, 7), (2, 5)]):
        base = rng.dirichlet(np.full(max(Kr, Kq), 0.4), 200)
        ref = base[:, :Kr] / base[:, :Kr].sum(1, keepdims=True)
        perm = rng.permutation(Kq)
        q = np.clip(base[:, :Kq] + rng.normal(0, 0.02, (200, Kq)), 1e-5, None)[:, perm]
        q /= q.sum(1, keepdims=True)
        rec[f"c{c}_ref"], rec[f"c{c}_query"] = ref, q
        rec[f"c{c}_perm"] = np.asarray(align_clusters_clumppling(ref, q))
    np.savez_compressed(OUT / "align.npz", **rec)
    print("align.npz", len(rec))


C2 = dict(N=10_000, M=200_000, K=8, F=0.05, alpha=0.3, miss=0.005, seed=1000)


def c2_cohort():
    """The mid-size benchmark cohort (the same generator, parameters and seed as the
    benchmark's c2 configuration) and its reference random start."""
    from adamixture_b200.src.packing import pack
    from adamixture_b200.src.simulate import make_cohort

    c = C2
    coh = make_cohort(c["N"], c["M"], c["K"], c["F"], c["alpha"], c["miss"], c["seed"])
    rng = np.random.default_rng(c["seed"])
    P0 = np.clip(rng.random((c["M"], c["K"])), 1e-5, 1 - 1e-5)
    Q0 = np.clip(rng.random((c["N"], c["K"])), 1e-5, 1 - 1e-5)
    Q0 /= Q0.sum(1, keepdims=True)
    return coh, P0, Q0, pack


def c2_trace(em, utils):
    coh, P0, Q0, pack = c2_cohort()
    M, N, K = coh.M, coh.N, coh.K
    Gp = np.zeros(((M + 3) // 4, N), dtype=np.uint8)
    blk = 8192
    for s in range(0, M, blk):
        g = coh.genotypes_parallel(s, min(blk, M - s))
        Gp[s // 4: s // 4 + (g.shape[0] + 3) // 4] = pack(g)
    sel = np.random.default_rng(7)
    rows_P = np.sort(sel.choice(M, 1024, replace=False))
    rows_Q = np.sort(sel.choice(N, 1024, replace=False))
    dev = torch.device("cpu")
    G = torch.from_numpy(Gp)
    P = torch.from_numpy(P0.copy())
    Q = torch.from_numpy(Q0.copy())
    opt = em.EMAdamOptimizer(P.shape, Q.shape, HP["lr"], HP["beta1"], HP["beta2"], HP["reg_adam"], dev)
    tP, tQ, sP, sQ, ll = [], [], [], [], {}
    for it in range(21):
        opt.run_em_step(G, P, Q, M, 8192, torch_unpacker)
        opt.step(P, Q, opt.P_EM, opt.Q_EM)
        Pn, Qn = P.numpy(), Q.numpy()
        tP.append(Pn[rows_P].astype(np.float32))
        tQ.append(Qn[rows_Q].astype(np.float32))
        sP.append(Pn.sum(0))
        sQ.append(Qn.sum(0))
        if it % 5 == 0:
            ll[it] = em.loglikelihood_gpu(G, P, Q, M, N, 8192, dev, 1)
        print("c2 iteration", it, flush=True)
    np.savez_compressed(OUT / "c2_trace.npz", N=N, M=M, K=K, seed=C2["seed"], rows_P=rows_P, rows_Q=rows_Q,
                        trace_P=np.stack(tP), trace_Q=np.stack(tQ), colsum_P=np.stack(sP),
                        colsum_Q=np.stack(sQ), loglik_iters=np.array(sorted(ll)),
                        loglik=np.array([ll[k] for k in sorted(ll)]))
    print("c2_trace.npz")


if __name__ == "__main__":
    which = set(sys.argv[1:]) or {"edge", "synth", "demo", "demo_gpu", "solvers", "cv_proj", "align", "supervised"}
    if which & {"edge", "synth", "demo", "cv_proj", "supervised"}:
        em, utils = reference()
        if "edge" in which:
            edge(em, utils)
        if "synth" in which:
            synth(em, utils)
        if "demo" in which:
            demo(em, utils)
        if "cv_proj" in which:
            cv_proj(em, utils)
        if "supervised" in which:
            supervised(em, utils)
    if "c2" in which:
        em, utils = reference()
        c2_trace(em, utils)
    if "demo_gpu" in which:
        demo_gpu()
    if "solvers" in which:
        solvers()
    if "align" in which:
        align()
