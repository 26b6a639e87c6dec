"""Host side of the 2-bit packed genotype layout and the PLINK BED reader.

Layout (the reference's GPU layout, adamixture/src/utils_c/cython/snp_reader.pyx:76-120):
packed ``G[ceil(M/4), N]`` uint8, byte ``(j>>2)*N + i`` holds SNP j of sample i in
bits ``2*(j&3)``; values 0/1/2 are allele counts and 3 is missing; unused bits of the
last row are zero.

The reader decodes SNP-major PLINK BED with the LUT [2,3,1,0] and, like the
reference (adamixture/src/snp_reader.py:747-757), swaps 0<->2 everywhere when the
mean dosage/2 over observed entries is >= 0.5. Large files are decoded on the GPU
by ``adx_bed_to_packed`` when a device is given; small ones on the host.
"""
from __future__ import annotations

import logging
from pathlib import Path

import numpy as np

log = logging.getLogger(__name__)

BED_LUT = np.array([2, 3, 1, 0], dtype=np.uint8)
FLIP = np.array([2, 1, 0, 3], dtype=np.uint8)


def pack(G: np.ndarray) -> np.ndarray:
    """Unpacked ``[M, N]`` (values 0..3) -> packed ``[ceil(M/4), N]``."""
    M, N = G.shape
    out = np.zeros(((M + 3) // 4, N), dtype=np.uint8)
    for k in range(4):
        rows = G[k::4].astype(np.uint8) & 3
        out[: rows.shape[0]] |= rows << (2 * k)
    return out


def unpack(Gp: np.ndarray, M: int) -> np.ndarray:
    """Packed ``[ceil(M/4), N]`` -> unpacked ``[M, N]`` uint8."""
    j = np.arange(M)
    return ((Gp[j >> 2] >> ((j & 3) << 1).astype(np.uint8)[:, None]) & 3).astype(np.uint8)


def bed_rows_to_packed(rows: np.ndarray, N: int) -> np.ndarray:
    """SNP-major BED rows ``[M, ceil(N/4)]`` -> packed ``[ceil(M/4), N]``."""
    i = np.arange(N)
    codes = (rows[:, i >> 2] >> ((i & 3) << 1).astype(np.uint8)) & 3
    return pack(BED_LUT[codes])


def packed_mean(Gp: np.ndarray, M: int, block: int = 1 << 14) -> float:
    """Mean of g/2 over observed entries of a packed matrix (0 when none observed)."""
    tot = 0
    cnt = 0
    for s in range(0, M, block):
        g = unpack(Gp[s // 4: (min(M, s + block) + 3) // 4], min(block, M - s))
        obs = g != 3
        tot += int(g[obs].astype(np.int64).sum())
        cnt += 2 * int(obs.sum())
    return 0.0 if cnt == 0 else tot / cnt


def flip(Gp: np.ndarray, M: int) -> np.ndarray:
    """0<->2 swap of every entry of a packed matrix (padding bits stay zero)."""
    lut = np.zeros(256, dtype=np.uint8)
    for b in range(256):
        v = 0
        for k in range(4):
            v |= int(FLIP[(b >> (2 * k)) & 3]) << (2 * k)
        lut[b] = v
    out = lut[Gp]
    rem = M % 4
    if rem:
        out[-1] &= np.uint8((1 << (2 * rem)) - 1)
    return out


def _keep(chrom: str, chrom_mode: str, autosomes: int, specific) -> bool:
    c = chrom.lower().removeprefix("chr")
    if chrom_mode == "all":
        return True
    if specific is not None:
        return c in {str(s).lower().removeprefix("chr") for s in specific}
    return c.isdigit() and 1 <= int(c) <= autosomes


def read_bed_packed(path: str | Path, chrom_mode: str = "autosomes", autosomes: int = 22,
                    specific_chrom=None, device=None):
    """Read ``path`` (.bed with .bim/.fam beside it) into the packed layout.

    Returns ``(G, N, M)`` with ``G`` a torch uint8 tensor ``[ceil(M/4), N]`` on
    ``device`` (host when None). Follows adamixture/src/snp_reader.py:353-443 for the
    packed branch and :747-757 for the flip.
    """
    import torch

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
    keep = np.array(keep, dtype=bool)
    raw = np.fromfile(bed, dtype=np.uint8, offset=3)
    if raw.size % nb:
        raise ValueError(f"{bed}: size does not match {N} samples")
    rows = raw.reshape(-1, nb)
    if rows.shape[0] != keep.size:
        raise ValueError(f"{bim}: {keep.size} variants but {bed} holds {rows.shape[0]}")
    rows = np.ascontiguousarray(rows[keep])
    M = rows.shape[0]
    if M == 0:
        raise ValueError("genotype data contains 0 SNPs after filtering")
    if device is not None and torch.device(device).type == "cuda":
        from .. import ops
        G = ops.bed_to_packed(torch.from_numpy(rows).to(device), N, M)
        return G, N, M
    Gp = bed_rows_to_packed(rows, N)
    if packed_mean(Gp, M) >= 0.5:
        log.info("    Flipping genotype encoding (packed).")
        Gp = flip(Gp, M)
    return torch.from_numpy(Gp), N, M
