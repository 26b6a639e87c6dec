"""Several GPUs, one process each: the ``adamixture`` run for one K with the genotypes sharded
by SNP rows.

    python -m torch.distributed.run --nnodes 1 --nproc-per-node 8 --master-addr 127.0.0.1 \\
        -m adamixture_b200.dist_entry --k 10 --data_path cohort.bed --save_dir out --name run

Every rank reads the .fam and .bim files and only its own rows of the .bed -- a contiguous
range of whole packed rows of the kept SNPs (``em_adam_dist.shard_rows``) -- and decodes
them with the reference's LUT; the ranks agree on the reference's 0<->2 flip from the mean
dosage over all observed entries (one all-reduce of two exact counts;
adamixture/src/snp_reader.py:747-757). Then the sharded randomized SVD + ALS
(``model.init_dist``), the sharded Adam-EM (``model.em_adam_dist``) or SQP + ZAL QN
(``model.br_qn_dist``), and rank 0 gathers the P rows and writes ``{name}.{K}.Q`` and
``.P`` in the reference's text format (adamixture/src/utils.py:252-273). The options are the
single-GPU command's for one K; cross-validation and K sweeps run through the single-GPU
command. The reference has no multi-GPU mode; this is its single-GPU run, sharded.
"""
from __future__ import annotations

import argparse
import logging
import os
import sys
import time
from pathlib import Path

import numpy as np
import torch
import torch.distributed as dist

from .cli import add_run_options, check_run_options
from .src.packing import BED_LUT, _keep, flip, pack

log = logging.getLogger(__name__)


def parse_args(argv: list[str]) -> argparse.Namespace:
    p = argparse.ArgumentParser(prog="adamixture_b200.dist_entry",
                                description="ADMIXTURE likelihood for one K on several GPUs (SNP-sharded).")
    add_run_options(p)
    p.add_argument("-k", "--k", type=int, required=True)
    p.add_argument("--data_path", required=True)
    p.add_argument("--save_dir", required=True)
    p.add_argument("--name", required=True)
    p.add_argument("--max_als", type=int, default=1000)
    p.add_argument("--tol_als", type=float, default=1e-4)
    p.add_argument("--power", type=int, default=5)
    p.add_argument("--tol_svd", type=float, default=1e-1)
    a = p.parse_args(argv)
    check_run_options(p, a)
    if not 1 <= a.k <= 64:
        p.error("K must be between 1 and 64 on the GPU")
    return a


def read_bed_shard(path, rank: int, world: int, chrom_mode: str = "autosomes", autosomes: int = 22,
                   specific_chrom=None, group=None):
    """This rank's rows of the kept SNPs of ``path`` (.bed with .bim/.fam beside it) in the
    packed layout: ``(G rows [ceil((j1-j0)/4), N] uint8 numpy, N, M, j0, j1)``. The flip
    follows the global mean dosage, so the shards concatenate to ``read_bed_packed``'s
    matrix."""
    from .model.em_adam_dist import shard_rows

    path = Path(path)
    base = path.with_suffix("") if path.suffix == ".bed" else path
    fam, bim, bed = (Path(str(base) + s) for s in (".fam", ".bim", ".bed"))
    with open(fam) as fh:
        N = sum(1 for _ in fh)
    nb = (N + 3) // 4
    keep = []
    with open(bim) as fh:
        for line in fh:
            parts = line.split()
            if parts:
                keep.append(_keep(parts[0], chrom_mode, autosomes, specific_chrom))
    kept = np.flatnonzero(np.array(keep, dtype=bool))
    M = int(kept.size)
    if M == 0:
        raise ValueError("genotype data contains 0 SNPs after filtering")
    raw = np.memmap(bed, dtype=np.uint8, mode="r", offset=3)
    if raw.size % nb or raw.size // nb != len(keep):
        raise ValueError(f"{bed}: size does not match {N} samples and {len(keep)} variants")
    j0, j1 = shard_rows(M, world, rank)
    rows = np.asarray(raw.reshape(-1, nb)[kept[j0:j1]])
    i = np.arange(N)
    codes = BED_LUT[(rows[:, i >> 2] >> ((i & 3) << 1).astype(np.uint8)) & 3]   # [j1-j0, N], 3 = missing
    obs = codes != 3
    counts = torch.tensor([float(codes[obs].astype(np.int64).sum()), 2.0 * float(obs.sum())], dtype=torch.float64)
    if dist.is_available() and dist.is_initialized():
        dev = torch.device("cuda", torch.cuda.current_device()) if dist.get_backend(group) == "nccl" else None
        if dev is not None:
            counts = counts.to(dev)
        dist.all_reduce(counts, group=group)
        counts = counts.cpu()
    Gp = pack(codes)
    if counts[1] > 0 and float(counts[0] / counts[1]) >= 0.5:
        if rank == 0:
            log.info("    Flipping genotype encoding (packed).")
        Gp = flip(Gp, j1 - j0)
    return Gp, N, M, j0, j1


class CudaShardBackends:
    """The CUDA side of a rank: the packed rows on its GPU and this library's kernels."""

    def __init__(self, device, precision=None):
        from .model.br_qn_dist import CudaBrqnBackend
        from .model.em_adam_dist import CudaBackend
        from .model.init_dist import CudaInitBackend

        self.device = torch.device(device)
        self.init, self.em, self.brqn = CudaInitBackend(), CudaBackend(precision), CudaBrqnBackend()

    def prepare(self, Gp: np.ndarray, M_local: int):
        return torch.from_numpy(np.ascontiguousarray(Gp)).to(self.device)


def run(args: argparse.Namespace, backends=None, group=None) -> tuple[np.ndarray, np.ndarray] | None:
    """One rank's run (inside an initialised process group). Rank 0 writes the outputs and
    returns ``(P, Q)``; the other ranks return None."""
    from .model.br_qn_dist import optimize_original_dist
    from .model.em_adam_dist import optimize_parameters_dist
    from .model.init_dist import initialize_sharded
    from .src.utils import write_outputs

    rank, world = dist.get_rank(group), dist.get_world_size(group)
    t0 = time.time()
    Gp, N, M, j0, j1 = read_bed_shard(args.data_path, rank, world, args.chrom_mode, args.autosomes,
                                      args.specific_chrom, group)
    if rank == 0:
        log.info(f"    Data loaded: {N} samples, {M} SNPs, {world} rank(s) of about {(M + world - 1) // world} SNPs.")
    be = backends or CudaShardBackends(torch.device("cuda", torch.cuda.current_device()), args.precision)
    G = be.prepare(Gp, j1 - j0)
    K, M_loc = args.k, j1 - j0
    P, Q = initialize_sharded(G, N, M, j0, j1, K, args.seed, args.power, args.tol_svd, args.max_als, args.tol_als,
                              backend=be.init, group=group)
    if args.algorithm == "adamem":
        P, Q = optimize_parameters_dist(G, P, Q, args.lr, args.beta1, args.beta2, args.reg_adam, args.max_iter,
                                        args.check, K, M_loc, N, args.lr_decay, args.min_lr, args.patience, args.tol,
                                        group=group, backend=be.em)
    else:
        P, Q = optimize_original_dist(G, P, Q, args.max_iter, K, M_loc, N, args.tol, args.Q_hist, args.patience,
                                      backend=be.brqn, group=group, verbose=rank == 0)
    parts = [None] * world if rank == 0 else None
    dist.gather_object(P.cpu().numpy(), parts, dst=0, group=group)
    if rank != 0:
        return None
    P_all = np.concatenate(parts)
    Q_np = Q.cpu().numpy()
    Path(args.save_dir).mkdir(parents=True, exist_ok=True)
    write_outputs(Q_np, args.name, K, args.save_dir, P_all)
    log.info(f"    Total time: {time.time() - t0:.1f}s")
    return P_all, Q_np


def main(argv: list[str] | None = None) -> int:
    import datetime

    logging.basicConfig(stream=sys.stdout, level=logging.INFO, format="%(message)s")
    args = parse_args(sys.argv[1:] if argv is None else argv)
    if not torch.cuda.is_available():
        raise SystemExit("adamixture_b200 runs on CUDA devices only")
    # run alone (without torchrun) as a one-rank job
    for k, v in (("MASTER_ADDR", "127.0.0.1"), ("MASTER_PORT", "29541"), ("RANK", "0"), ("WORLD_SIZE", "1")):
        os.environ.setdefault(k, v)
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist.init_process_group("nccl", device_id=torch.device("cuda", local), timeout=datetime.timedelta(minutes=30))
    try:
        run(args)
    finally:
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
