"""Projection command of the B200 build, mirroring ``adamixture-project``
(adamixture/project_entry.py): Q for target samples with a pre-trained P held fixed.

    python -m adamixture_b200.project_entry --data_path target.bed --p_path ref.8.P \\
        --save_dir out --name proj [--algorithm adamem|brqn]

Reads P (whitespace-delimited text, M rows x K columns), clamps it to [1e-5, 1 - 1e-5],
starts Q from ``default_rng(seed).random((N, K))`` with rows normalised, runs the Adam-EM
projection or the SQP + ZAL quasi-Newton projection on the GPU and writes
``{name}.{K}.Q`` with "%.6f" values, as the reference does (project_entry.py:203-291).
Plots are not produced by this package; ``--plot`` is accepted and ignored with a warning.
"""
from __future__ import annotations

import argparse
import logging
import sys
import time
from pathlib import Path

from .cli import add_run_options, check_run_options

log = logging.getLogger(__name__)

MAX_K = 64


def parse_args(argv: list[str]) -> argparse.Namespace:
    """Options of adamixture/project_entry.py:24-113."""
    p = argparse.ArgumentParser(prog="adamixture_b200.project_entry",
                                description="Projection: ancestry proportions Q for target samples "
                                            "with a fixed, pre-trained allele-frequency matrix P.")
    p.add_argument("--data_path", required=True, help="target genotypes (PLINK .bed)")
    p.add_argument("--p_path", required=True, help="pre-trained P matrix (.P text file, M rows x K columns)")
    p.add_argument("--save_dir", required=True)
    p.add_argument("--name", required=True)
    p.add_argument("--labels")
    add_run_options(p)
    a = p.parse_args(argv)
    check_run_options(p, a)
    return a


def run(args: argparse.Namespace, t0: float) -> int:
    import numpy as np
    import torch

    from .src import utils
    from .src.projection import optimize_projection_gpu, optimize_projection_original_gpu

    if args.plot is not None:
        log.warning("    Plotting is not available in this package; --plot is ignored.")
    p_path = Path(args.p_path)
    if not p_path.exists():
        log.error(f"    Error: P matrix file not found: {p_path}")
        return 1
    log.info("    Loading pre-trained P matrix.")
    P = np.loadtxt(str(p_path), dtype=np.float64)
    if P.ndim == 1:
        P = P.reshape(-1, 1)
    M_p, K = P.shape
    P = P.clip(1e-5, 1.0 - 1e-5)
    log.info(f"    P matrix loaded: {M_p} SNPs, K={K} populations.\n")
    if K > MAX_K:
        log.error(f"    Error: K={K} exceeds the GPU limit (MAX_K={MAX_K}).")
        return 1

    device = torch.device("cuda", torch.cuda.current_device())
    G, N, M = utils.read_data(args.data_path, packed=True, chunk_size=args.chunk_size,
                              chrom_mode=args.chrom_mode, autosomes=args.autosomes,
                              specific_chrom=args.specific_chrom, device=device)
    if M != M_p:
        log.error(f"    Error: SNP count mismatch — genotype data has {M} SNPs but P matrix has {M_p} SNPs.")
        return 1
    log.info(f"    Target samples: {N}.\n")

    rng = np.random.default_rng(args.seed)
    Q = rng.random(size=(N, K)).astype(np.float64)
    Q /= Q.sum(axis=1, keepdims=True)
    P_t = torch.tensor(P, dtype=torch.float64, device=device)
    Q_t = torch.tensor(Q, dtype=torch.float64, device=device)
    if args.algorithm == "brqn":
        log.info("    Running SQP + ZAL QN projection (P fixed)...\n")
        Q_opt = optimize_projection_original_gpu(
            G=G, P=P_t, Q=Q_t, max_iter=args.max_iter, K=K, M=M, N=N, tol=args.tol, Q_hist=args.Q_hist,
            patience=args.patience, device=device, chunk_size=args.chunk_size, threads_per_block=0)
    else:
        log.info("    Running Adam-EM projection (P fixed)...\n")
        Q_opt = optimize_projection_gpu(
            G=G, P=P_t, Q=Q_t, lr=args.lr, beta1=args.beta1, beta2=args.beta2, reg_adam=args.reg_adam,
            max_iter=args.max_iter, check=args.check, M=M, lr_decay=args.lr_decay, min_lr=args.min_lr,
            patience=args.patience, tol_adam=args.tol, device=device, chunk_size=args.chunk_size,
            threads_per_block=0, precision=args.precision)
    out_path = Path(args.save_dir)
    out_path.mkdir(parents=True, exist_ok=True)
    utils.write_outputs(Q_opt.cpu().numpy(), args.name, K, out_path, decimals=6)
    log.info(f"\n    Total elapsed time: {time.time() - t0:.2f}s\n")
    return 0


def main(argv: list[str] | None = None) -> int:
    logging.basicConfig(stream=sys.stdout, level=logging.INFO, format="%(message)s")
    t0 = time.time()
    args = parse_args(sys.argv[1:] if argv is None else argv)
    log.info("    Projection Mode\n")
    return run(args, t0)


if __name__ == "__main__":
    sys.exit(main())
