"""Autotuner for the tile (shared-memory layout) of the float64 tensor-core E-step sweep.

The float64 sweep (``csrc/em_sweep_dmma.cu``) has two layouts for K <= 8: layout 0, one
8-warp CTA per SM with up to 255 registers a thread (the only layout for 8 < K <= 16),
and layout 1, compact Q/P tiles and reduction buffers in 112 KiB with at most 128
registers a thread, so two CTAs share an SM. A layout moves values in shared memory and
changes the occupancy only -- never the arithmetic or its order -- so both give
bit-identical statistics; which one is faster depends on K, the shape and the GPU.

``tune_dmma`` times every layout of K on the caller's own matrix (a sweep over whole
waves of CTAs, CUDA events on the current stream, after a warm-up launch), selects the
fastest for (device, K) in the library (``adx_dmma_tile_set``), logs the choice and the
timings, and caches them for the process per (GPU name, M, N, K); with ``ADX_TUNE_CACHE``
naming a JSON file the cache also persists across processes. ``ADX_AUTOTUNE=0`` turns
tuning off: layout 0 then runs unless a layout is set by hand (``set_tile``).

The reference has no counterpart: its E-step is torch matmuls over decoded chunks
(adamixture/model/em_adam_gpu.py:46-78), with no tile choice.
"""
from __future__ import annotations

import ctypes
import json
import logging
import os
import threading
from pathlib import Path

import torch

from . import _lib, ops

log = logging.getLogger(__name__)

_CACHE: dict[str, dict] = {}
_LOCK = threading.Lock()
_LOADED = False
# CTAs a timed sweep covers at least: whole waves for either layout (1 or 2 CTAs per SM)
_MIN_WAVES = 4


def enabled() -> bool:
    return os.environ.get("ADX_AUTOTUNE", "1") != "0"


def tiles(K: int) -> int:
    """Number of layouts of the float64 sweep for K (1 <= K <= 16)."""
    n = ctypes.c_int(0)
    _lib.call("adx_dmma_tiles", int(K), ctypes.addressof(n))
    return int(n.value)


def get_tile(K: int, device=None) -> int:
    dev = _device_index(device)
    t = ctypes.c_int(-1)
    _lib.call("adx_dmma_tile_get", dev, int(K), ctypes.addressof(t))
    return int(t.value)


def set_tile(K: int, tile: int, device=None) -> None:
    _lib.call("adx_dmma_tile_set", _device_index(device), int(K), int(tile))


def _device_index(device) -> int:
    if device is None:
        return torch.cuda.current_device()
    if isinstance(device, int):
        return device
    d = torch.device(device)
    return d.index if d.index is not None else torch.cuda.current_device()


def _key(device: int, M: int, N: int, K: int) -> str:
    return f"{torch.cuda.get_device_name(device)}|M={M}|N={N}|K={K}"


def _cache_file() -> Path | None:
    p = os.environ.get("ADX_TUNE_CACHE")
    return Path(p) if p else None


def _load_cache() -> None:
    global _LOADED
    if _LOADED:
        return
    _LOADED = True
    f = _cache_file()
    if f is not None and f.exists():
        try:
            _CACHE.update(json.loads(f.read_text()))
        except (OSError, ValueError) as e:
            log.warning(f"    autotune cache {f} unreadable ({e}); tuning afresh")


def _save_cache() -> None:
    f = _cache_file()
    if f is None:
        return
    try:
        f.parent.mkdir(parents=True, exist_ok=True)
        tmp = f.with_suffix(f.suffix + ".tmp")
        tmp.write_text(json.dumps(_CACHE, indent=1, sort_keys=True))
        os.replace(tmp, f)
    except OSError as e:
        log.warning(f"    autotune cache {f} not written ({e})")


def timed_blocks(M: int, N: int, K: int, sms: int) -> int:
    """SNP blocks a tuning sweep covers: at least ``_MIN_WAVES`` waves of two CTAs per SM
    (the partition's CTAs per block times the blocks), or every block when there are fewer."""
    _, n_blocks, per_block = ops.em_sweep_blocks_info(M, N, K)
    want = _MIN_WAVES * 2 * sms
    return min(n_blocks, max(1, -(-want // max(per_block, 1))))


def pick(timings: dict[int, float]) -> int:
    """The fastest layout; a tie (within 1 %) keeps the lower-numbered one."""
    best = min(timings, key=lambda t: (timings[t], t))
    for t in sorted(timings):
        if timings[t] <= timings[best] * 1.01:
            return t
    return best


def tune_dmma(G: torch.Tensor, P: torch.Tensor, Q: torch.Tensor, M: int, workspace: torch.Tensor | None = None,
              reps: int = 2, force: bool = False) -> int:
    """Select the float64 sweep's layout for this K on G's device (see the module text) and
    return it. P, Q: float64 on the device; nothing of theirs is written. ``workspace``: an
    E-step workspace of this shape (float64) whose partial sums may be overwritten (one of
    its own is allocated otherwise)."""
    N, K = Q.shape
    dev = G.device.index if G.device.index is not None else torch.cuda.current_device()
    if K > 16 or not enabled():
        return get_tile(K, dev) if K <= 16 else 0
    n = tiles(K)
    if n < 2:
        return 0
    with _LOCK:
        _load_cache()
        key = _key(dev, M, N, K)
        hit = _CACHE.get(key)
        if hit is not None and not force and isinstance(hit.get("tile"), int) and 0 <= hit["tile"] < n:
            set_tile(K, hit["tile"], dev)
            return hit["tile"]
        sms = torch.cuda.get_device_properties(dev).multi_processor_count
        nb = timed_blocks(M, N, K, sms)
        ws = workspace if workspace is not None else ops.em_workspace(M, N, K, "f64", G.device)
        stream = torch.cuda.current_stream(G.device)
        timings = {}
        before = get_tile(K, dev)
        try:
            for tile in range(n):
                set_tile(K, tile, dev)
                ops.em_sweep_blocks(G, P, Q, M, 0, nb, ws)   # warm-up (and the kernel's attributes)
                e0 = torch.cuda.Event(enable_timing=True)
                e1 = torch.cuda.Event(enable_timing=True)
                e0.record(stream)
                for _ in range(reps):
                    ops.em_sweep_blocks(G, P, Q, M, 0, nb, ws)
                e1.record(stream)
                e1.synchronize()
                timings[tile] = e0.elapsed_time(e1) / reps
        except Exception:
            set_tile(K, before, dev)
            raise
        best = pick(timings)
        set_tile(K, best, dev)
        _CACHE[key] = {"tile": best, "ms": {str(t): round(v, 4) for t, v in timings.items()}, "blocks": nb}
        _save_cache()
    log.info(f"    autotune: float64 sweep K={K} ({M} x {N}): layout {best} "
             f"({', '.join(f'layout {t} {v:.3f} ms' for t, v in sorted(timings.items()))}, {nb} SNP blocks)")
    return best


def choices() -> dict[str, dict]:
    """The cached choices of this process: key -> {"tile", "ms" per layout, "blocks"}."""
    with _LOCK:
        return {k: dict(v) for k, v in _CACHE.items()}


def batch_groups(Ks, device=None) -> list[list[int]]:
    """Problem indices of a batch grouped by the layout selected for their K: a batched
    sweep launches one layout, so problems whose K runs layout 1 share one launch and the
    rest another (bit-identical either way). One group when all share a layout."""
    dev = _device_index(device)
    groups: dict[int, list[int]] = {}
    for i, k in enumerate(Ks):
        t = get_tile(k, dev) if 1 <= k <= 16 else 0
        groups.setdefault(t, []).append(i)
    return [groups[t] for t in sorted(groups)]
