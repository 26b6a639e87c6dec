"""Supervised command of the B200 build, mirroring ``adamixture-supervised``
(adamixture/supervised_entry.py): known population labels for a subset of the samples
anchor P, Q is estimated for every sample and the labelled rows are snapped back to their
one-hot memberships after every update.

    python -m adamixture_b200.supervised_entry --data_path cohort.bed --labels pops.txt \\
        --save_dir out --name sup [--level 1|2|3] [--algorithm adamem|brqn]

The labels file of the chosen level holds one line per sample: a population name, or ``-``
for an unlabelled sample. Names are numbered 1, 2, ... in order of first appearance and K
is the number of distinct names (supervised_entry.py:149-190, 294-304). P starts from the
labelled samples' allele frequencies, Q from ``default_rng(seed).random((N, K))`` with the
labelled rows set near one-hot (supervised_entry.py:309-315); the outputs are
``{name}.{K}.Q`` and ``{name}.{K}.P`` with "%.6f" values (supervised_entry.py:380-391).
Plots are not produced by this package; ``--plot`` is accepted and ignored with a warning.
"""
from __future__ import annotations

import argparse
import logging
import sys
import time
from pathlib import Path

import numpy as np

from .cli import add_run_options, check_run_options

log = logging.getLogger(__name__)

MAX_K = 64


def parse_args(argv: list[str]) -> argparse.Namespace:
    """Options of adamixture/supervised_entry.py:24-128 (K comes from the labels, so -k,
    --k, --min_k and --max_k are refused)."""
    for a in argv:
        if a in ("-k", "--k", "--min_k", "--max_k"):
            raise SystemExit("K, min_k, and max_k are not allowed in supervised mode. "
                             "K is automatically derived from the labels.")
    p = argparse.ArgumentParser(prog="adamixture_b200.supervised_entry",
                                description="Supervised mode: labelled samples anchor the allele "
                                            "frequencies; ancestry proportions for all samples.")
    p.add_argument("--data_path", required=True, help="genotypes (PLINK .bed)")
    p.add_argument("--save_dir", required=True)
    p.add_argument("--name", required=True)
    p.add_argument("--no_freqs", action="store_true", help="do not save the P matrix")
    p.add_argument("--labels", required=True,
                   help="one label per sample: a population name, or '-' for an unlabelled sample")
    p.add_argument("--level", type=int, default=1, choices=[1, 2, 3],
                   help="labels level used for supervision: 1 = --labels, 2 = --labels2, 3 = --labels3")
    add_run_options(p)
    a = p.parse_args(argv)
    level_arg = {1: "labels", 2: "labels2", 3: "labels3"}[a.level]
    if getattr(a, level_arg) is None:
        p.error(f"--{level_arg} is required when --level {a.level} is selected.")
    check_run_options(p, a)
    return a


def parse_labels_file(path: Path) -> list[str]:
    """Non-empty, stripped lines of a labels file (supervised_entry.py:131-146)."""
    with open(path) as f:
        return [line.strip() for line in f if line.strip()]


def labels_to_y(raw_labels: list[str]) -> tuple[np.ndarray, dict[str, int]]:
    """``-`` -> 0; every other name -> 1, 2, ... in order of first appearance
    (supervised_entry.py:149-176). Returns ``(y int32 [N], name -> id)``."""
    pop_to_int: dict[str, int] = {}
    y = np.zeros(len(raw_labels), dtype=np.int32)
    for i, lbl in enumerate(raw_labels):
        if lbl != "-":
            y[i] = pop_to_int.setdefault(lbl, len(pop_to_int) + 1)
    return y, pop_to_int


def run(args: argparse.Namespace, t0: float) -> int:
    import torch

    from .src import utils
    from .src.supervised import (init_p_supervised_gpu, init_q_supervised, optimize_supervised_gpu,
                                 optimize_supervised_original_gpu)

    if args.plot is not None:
        log.warning("    Plotting is not available in this package; --plot is ignored.")
    sup_path = Path(getattr(args, {1: "labels", 2: "labels2", 3: "labels3"}[args.level]))
    if not sup_path.exists():
        log.error(f"    Error: Labels file not found: {sup_path}")
        return 1
    y, _ = labels_to_y(parse_labels_file(sup_path))
    K = int(y.max()) if y.size else 0
    if K < 2:
        log.error(f"    Error: Number of populations K (derived from labels) must be at least 2, but got {K}.")
        return 1
    if K > MAX_K:
        log.error(f"    Error: K={K} exceeds the GPU limit (MAX_K={MAX_K}).")
        return 1

    device = torch.device("cuda", torch.cuda.current_device())
    G, N, M = utils.read_data(args.data_path, packed=True, chunk_size=args.chunk_size,
                              chrom_mode=args.chrom_mode, autosomes=args.autosomes,
                              specific_chrom=args.specific_chrom, device=device)
    if N != len(y):
        log.error(f"    Error: Sample count mismatch — genotype data has {N} samples "
                  f"but labels file has {len(y)}.")
        return 1

    rng = np.random.default_rng(args.seed)
    P = init_p_supervised_gpu(G, y, K, M)
    Q = rng.random(size=(N, K)).astype(np.float64)
    Q /= Q.sum(axis=1, keepdims=True)
    init_q_supervised(Q, y, K)
    Q_t = torch.tensor(Q, dtype=torch.float64, device=device)
    if args.algorithm == "brqn":
        log.info("    Running supervised SQP + ZAL QN...\n")
        P_opt, Q_opt = optimize_supervised_original_gpu(
            G=G, P=P, Q=Q_t, y=y, max_iter=args.max_iter, K=K, M=M, N=N, tol=args.tol, Q_hist=args.Q_hist,
            patience=args.patience, device=device, chunk_size=args.chunk_size, threads_per_block=0)
    else:
        log.info("    Running supervised Adam-EM...\n")
        P_opt, Q_opt = optimize_supervised_gpu(
            G=G, P=P, Q=Q_t, y=y, lr=args.lr, beta1=args.beta1, beta2=args.beta2, reg_adam=args.reg_adam,
            max_iter=args.max_iter, check=args.check, M=M, lr_decay=args.lr_decay, min_lr=args.min_lr,
            patience=args.patience, tol_adam=args.tol, device=device, chunk_size=args.chunk_size,
            threads_per_block=0, precision=args.precision)
    out_path = Path(args.save_dir)
    out_path.mkdir(parents=True, exist_ok=True)
    utils.write_outputs(Q_opt.cpu().numpy(), args.name, K, out_path,
                        P=None if args.no_freqs else P_opt.cpu().numpy(), decimals=6)
    log.info(f"\n    Total elapsed time: {time.time() - t0:.2f}s\n")
    return 0


def main(argv: list[str] | None = None) -> int:
    logging.basicConfig(stream=sys.stdout, level=logging.INFO, format="%(message)s")
    t0 = time.time()
    args = parse_args(sys.argv[1:] if argv is None else argv)
    log.info("    Supervised Mode\n")
    return run(args, t0)


if __name__ == "__main__":
    sys.exit(main())
