"""Data input and result output of the B200 build, mirroring the reference's
``adamixture/src/utils.py`` (``read_data`` for PLINK BED, ``write_outputs``)."""
from __future__ import annotations

import logging
from pathlib import Path

import numpy as np
import torch

from .. import _lib
from .packing import read_bed_packed

log = logging.getLogger(__name__)


def read_data(data_path: str, packed: bool = True, chunk_size: int = 8192, chrom_mode: str = "autosomes",
              autosomes: int = 22, specific_chrom=None, verbose: bool = True, device=None):
    """PLINK BED -> ``(G, N, M)``: the packed uint8 [ceil(M/4), N] tensor (decoded and
    flipped on ``device`` when it is a CUDA device), or the unpacked uint8 [M, N] array when
    ``packed`` is False (adamixture/src/utils.py:read_data, BED branch)."""
    path = Path(data_path)
    if path.suffix not in (".bed", ""):
        raise ValueError(f"{data_path}: only PLINK .bed input is supported by this package")
    G, N, M = read_bed_packed(path, chrom_mode, autosomes, specific_chrom, device=device)
    if verbose:
        log.info(f"    Data loaded: {N} samples, {M} SNPs.")
    if packed:
        return G, N, M
    from .packing import unpack

    return unpack(G.cpu().numpy(), M), N, M


def write_outputs(Q: np.ndarray, run_name: str, K: int, out_path: str | Path, P: np.ndarray = None,
                  decimals: int | None = None) -> None:
    """``{run_name}.{K}.Q`` (and ``.P``): the reference's text format, written natively --
    "%.18e" values (adamixture/src/utils.py:252-273), or "%.{decimals}f" values as the
    projection and supervised commands write them (``decimals=6``)."""
    out_path = Path(out_path)
    for X, ext in ((Q, "Q"), (P, "P")):
        if X is None:
            continue
        X = np.ascontiguousarray(X.detach().cpu().numpy() if isinstance(X, torch.Tensor) else X, dtype=np.float64)
        if X.ndim == 1:
            X = X[:, None]
        fn = str(out_path / f"{run_name}.{K}.{ext}").encode()
        if decimals is None:
            _lib.call("adx_write_text_matrix", fn, X.ctypes.data, X.shape[0], X.shape[1], 0)
        else:
            _lib.call("adx_write_text_matrix_fixed", fn, X.ctypes.data, X.shape[0], X.shape[1], decimals, 0)
    log.info("    Q and P matrices saved." if P is not None else "    Q matrix saved.")
