"""Command line of the B200 build, mirroring the reference's ``adamixture`` options
(adamixture/entry.py:18-128) for ``--device gpu``:

    python -m adamixture_b200 --k 8 --data_path cohort.bed --save_dir out --name run --device gpu

Options of the reference that concern other devices or the plotting stack are accepted;
``--precision`` (f64 | f32 | bf16 | f16 | mixed | auto) selects the Adam-EM E-step arithmetic.
"""
from __future__ import annotations

import argparse
import logging
import sys
import time


def add_run_options(p: argparse.ArgumentParser) -> None:
    """The optimiser, data and plot options the projection and supervised commands share
    (adamixture/project_entry.py:69-96, adamixture/supervised_entry.py:77-98)."""
    p.add_argument("--lr", type=float, default=0.005)
    p.add_argument("--beta1", type=float, default=0.80)
    p.add_argument("--beta2", type=float, default=0.88)
    p.add_argument("--reg_adam", type=float, default=1e-8)
    p.add_argument("--lr_decay", type=float, default=0.5)
    p.add_argument("--min_lr", type=float, default=1e-4)
    p.add_argument("--patience", type=int, default=3)
    p.add_argument("--tol", type=float, default=0.1)
    p.add_argument("--max_iter", type=int, default=10000)
    p.add_argument("--check", type=int, default=5)
    p.add_argument("--algorithm", choices=["brqn", "adamem"], default="brqn")
    p.add_argument("--Q_hist", type=int, default=3, help=argparse.SUPPRESS)
    p.add_argument("-s", "--seed", type=int, default=42)
    p.add_argument("-t", "--threads", type=int, default=1)
    p.add_argument("--chunk_size", type=int, default=4096)
    p.add_argument("--device", default="cuda", choices=["cpu", "cuda", "gpu", "mps"])
    p.add_argument("--chrom_mode", choices=["all", "autosomes"], default="autosomes")
    p.add_argument("--autosomes", type=int, default=22)
    p.add_argument("--specific_chrom", nargs="+")
    p.add_argument("--labels2")
    p.add_argument("--labels3")
    p.add_argument("--colors")
    p.add_argument("--plot", nargs="*")
    p.add_argument("--precision", choices=["f64", "f32", "bf16", "f16", "mixed", "auto"], default=None,
                   help="Adam-EM E-step arithmetic (default: auto)")


def check_run_options(p: argparse.ArgumentParser, a: argparse.Namespace) -> None:
    """The reference's parameter checks of these commands (adamixture/project_entry.py:141-158),
    as argument errors."""
    if a.device not in ("cuda", "gpu"):
        p.error("adamixture_b200 runs on the GPU only (--device cuda)")
    checks = ((a.threads >= 1, "--threads must be at least 1"), (a.lr > 0, "--lr must be positive"),
              (0 <= a.beta1 < 1, "--beta1 must be in [0, 1)"), (0 <= a.beta2 < 1, "--beta2 must be in [0, 1)"),
              (0 < a.lr_decay <= 1, "--lr_decay must be in (0, 1]"), (a.min_lr > 0, "--min_lr must be positive"),
              (a.patience >= 1, "--patience must be at least 1"), (a.seed >= 0, "--seed must be non-negative"),
              (a.max_iter >= 1, "--max_iter must be at least 1"), (a.check >= 1, "--check must be at least 1"),
              (a.chunk_size >= 1, "--chunk_size must be at least 1"), (a.tol > 0, "--tol must be positive"),
              (a.reg_adam >= 0, "--reg_adam must be non-negative"), (a.Q_hist >= 1, "--Q_hist must be at least 1"),
              (a.chrom_mode != "autosomes" or a.specific_chrom or a.autosomes >= 1,
               "--autosomes must be at least 1"))
    for ok, msg in checks:
        if not ok:
            p.error(msg)


def parse_args(argv: list[str]) -> argparse.Namespace:
    p = argparse.ArgumentParser(prog="adamixture_b200", description="ADMIXTURE likelihood on one B200.")
    p.add_argument("--lr", type=float, default=0.005)
    p.add_argument("--beta1", type=float, default=0.80)
    p.add_argument("--beta2", type=float, default=0.88)
    p.add_argument("--reg_adam", type=float, default=1e-8)
    p.add_argument("--algorithm", choices=["brqn", "adamem"], default="brqn")
    p.add_argument("--init", choices=["em", "als", "mlp"], default="als",
                   help="initialisation: random + EM priming, SVD + ALS, or the learned warm start "
                        "on top of SVD + ALS (Adam-EM only; kept only if no worse than plain EM)")
    p.add_argument("--em_init_steps", type=int, default=5, help=argparse.SUPPRESS)
    p.add_argument("--Q_hist", type=int, default=3, help=argparse.SUPPRESS)
    p.add_argument("--lr_decay", type=float, default=0.5)
    p.add_argument("--min_lr", type=float, default=1e-4)
    p.add_argument("--patience", type=int, default=3)
    p.add_argument("--tol", type=float, default=0.1)
    p.add_argument("-s", "--seed", type=int, default=42)
    p.add_argument("-k", "--k", type=int)
    p.add_argument("--min_k", type=int)
    p.add_argument("--max_k", type=int)
    p.add_argument("--save_dir", required=True)
    p.add_argument("--data_path", required=True)
    p.add_argument("--name", required=True)
    p.add_argument("-t", "--threads", type=int, default=1)
    p.add_argument("--device", default="gpu", choices=["cpu", "gpu", "mps"])
    p.add_argument("--chrom_mode", choices=["all", "autosomes"], default="autosomes")
    p.add_argument("--autosomes", type=int, default=22)
    p.add_argument("--specific_chrom", nargs="+")
    p.add_argument("--max_iter", type=int, default=10000)
    p.add_argument("--check", type=int, default=5)
    p.add_argument("--no_freqs", action="store_true", default=False)
    p.add_argument("--max_als", type=int, default=1000)
    p.add_argument("--tol_als", type=float, default=1e-4)
    p.add_argument("--power", type=int, default=5)
    p.add_argument("--tol_svd", type=float, default=1e-1)
    p.add_argument("--chunk_size", type=int, default=8192)
    p.add_argument("--n_inits", type=int, default=1)
    p.add_argument("--cv", nargs="?", const=5, default=0, type=int)
    p.add_argument("--plot", nargs="*")
    p.add_argument("--plot_single", nargs="*")
    p.add_argument("--labels")
    p.add_argument("--labels2")
    p.add_argument("--labels3")
    p.add_argument("--colors")
    p.add_argument("--precision", choices=["f64", "f32", "bf16", "f16", "mixed", "auto"], default=None)
    a = p.parse_args(argv)
    if a.device != "gpu":
        p.error("adamixture_b200 runs on the GPU only (--device gpu)")
    if (a.k is None) == (a.min_k is None or a.max_k is None):
        p.error("give either -k or both --min_k and --max_k")
    ks = [a.k] if a.k is not None else list(range(a.min_k, a.max_k + 1))
    if min(ks) < 1 or max(ks) > 64:
        p.error("K must be between 1 and 64 on the GPU")
    return a


def main(argv: list[str] | None = None) -> int:
    logging.basicConfig(stream=sys.stdout, level=logging.INFO, format="%(message)s")
    args = parse_args(sys.argv[1:] if argv is None else argv)
    from .src.main import main as run

    return run(args, time.time())
