"""Run coordinator of the B200 build: ``adamixture/src/main.py`` for ``--device gpu``.

Reads the data once (decoded on the GPU), runs the one-time setup at K_max, trains every
requested K (single K or a min..max sweep, one or several initialisations), aligns each
K's clusters to the previous K's, writes ``{name}.{K}.Q`` / ``.P`` in the reference's text
format and, with ``--cv``, scores every K by cross-validation on the GPU afterwards.
Plots are not produced by this package (no plotting stack); the plot options are accepted
and ignored with a warning.
"""
from __future__ import annotations

import argparse
import logging
import time
from pathlib import Path

import numpy as np
import torch

from . import utils
from .adamixture import initialize_k, setup, train_k
from .align import align_clusters

log = logging.getLogger(__name__)


def main(args: argparse.Namespace, t0: float) -> int:
    try:
        if args.min_k is not None and args.max_k is not None:
            k_values = list(range(args.min_k, args.max_k + 1))
            log.info(f"\n    Running from {args.min_k} to {args.max_k}.\n")
        else:
            k_values = [int(args.k)]
        if getattr(args, "plot", None) is not None or getattr(args, "plot_single", None) is not None:
            log.warning("    Plotting is not available in this package; --plot options are ignored.")
        n_inits = int(args.n_inits)
        K_max = max(k_values)
        Path(args.save_dir).mkdir(parents=True, exist_ok=True)
        device = torch.device("cuda", torch.cuda.current_device())
        G, N, M = utils.read_data(args.data_path, packed=True, chunk_size=args.chunk_size,
                                  chrom_mode=args.chrom_mode, autosomes=args.autosomes,
                                  specific_chrom=getattr(args, "specific_chrom", None), device=device)
        original = args.algorithm == "brqn"
        precision = getattr(args, "precision", None)
        trained: dict[int, tuple] = {}
        previous_Q = None
        device_obj, tpb, f, U, S, V, G = setup(
            G, N, M, K_max, int(args.seed), int(args.power), float(args.tol_svd), int(args.chunk_size),
            "cuda", original=original, init_original=args.init, q_hist=args.Q_hist, compute_svd=n_inits == 1)
        for K in k_values:
            log.info(f"\n    Running on K = {K}.\n")
            t_k = time.time()
            common = dict(original=original, rtol=float(args.tol), Q_hist=args.Q_hist, init_original=args.init,
                          em_init_steps=int(args.em_init_steps), precision=precision)
            hp = (int(args.seed), float(args.lr), float(args.beta1), float(args.beta2), float(args.reg_adam),
                  int(args.max_iter), int(args.check), int(args.max_als), float(args.tol_als),
                  float(args.lr_decay), float(args.min_lr), int(args.chunk_size), int(args.patience),
                  float(args.tol), device_obj, tpb)
            if n_inits == 1:
                P, Q = train_k(G, N, M, K, U, S, V, f, *hp, **common)
            else:
                best = (None, None, -np.inf)
                for init_idx in range(n_inits):
                    s = int(args.seed) + init_idx
                    P0, Q0, logl = initialize_k(G, N, M, K, f, s, int(args.power), float(args.tol_svd),
                                                int(args.max_als), float(args.tol_als), int(args.chunk_size),
                                                device_obj, tpb, original=original, init_original=args.init,
                                                em_init_steps=int(args.em_init_steps))
                    if logl > best[2]:
                        best = (P0, Q0, logl)
                log.info(f"\n    Best initialization log-likelihood for K={K}: {best[2]:.1f}")
                P, Q = train_k(G, N, M, K, None, None, None, f, *hp, P_init=best[0], Q_init=best[1], **common)
            P_np, Q_np = P.cpu().numpy(), Q.cpu().numpy()
            if previous_Q is not None:
                perm = align_clusters(previous_Q, Q_np)
                Q_np, P_np = Q_np[:, perm], P_np[:, perm]
            previous_Q = Q_np
            utils.write_outputs(Q_np, args.name, K, args.save_dir, P=None if args.no_freqs else P_np)
            if args.cv:
                trained[K] = (P, Q)
            log.info(f"\n    K={K} completed in {time.time() - t_k:.2f} seconds.")
        if args.cv and trained:
            from .cv import run_cross_validation

            cv_results = {}
            for K, (P, Q) in sorted(trained.items()):
                log.info(f"\n    Running {int(args.cv)}-fold CV on genotype entries for K={K}...")
                cv_results[K] = run_cross_validation(args, G, N, M, K, P, Q)
            log.info("\n    ---- Cross-validation summary ----")
            for k_val, idx in sorted(cv_results.items()):
                log.info(f"    K={k_val}: CV index = {idx:.4f}")
            log.info("    ----------------------------------")
        log.info(f"\n    Total elapsed time: {time.time() - t0:.2f} seconds.\n")
        return 0
    except Exception as e:  # the reference reports and returns 1 (main.py:288-292)
        log.error(f"    Unexpected error: {e}")
        return 1
