"""ctypes binding of the C ABI in ``include/adamixture_b200.h``.

The library is built in-tree (``python -m adamixture_b200.csrc.build``) into
``adamixture_b200/_lib/libadamixture_b200.so``. There is no fallback: if the library is
missing or fails to load, every call raises.
"""
from __future__ import annotations

import ctypes
import threading
from ctypes import c_double, c_int, c_int64, c_size_t, c_uint32, c_uint64, c_void_p
from pathlib import Path

LIB_PATH = Path(__file__).resolve().parent / "_lib" / "libadamixture_b200.so"

ADX_OK, ADX_ERR_ARG, ADX_ERR_CUDA, ADX_ERR_WORKSPACE, ADX_ERR_UNSUPPORTED, ADX_ERR_TIMEOUT = 0, 1, 2, 3, 4, 5
ADX_F64, ADX_F32, ADX_BF16, ADX_F16 = 0, 1, 2, 3
MAX_K = 64

P = c_void_p
I64 = c_int64

# name -> argtypes (restype is int unless listed in _RESTYPE)
SIGNATURES: dict[str, list] = {
    "adx_version": [],
    "adx_last_error": [],
    "adx_unpack_u8": [P, I64, I64, I64, I64, I64, I64, P, P],
    "adx_unpack_center_f32": [P, I64, I64, I64, I64, I64, I64, P, P, P],
    "adx_allele_frequency": [P, I64, I64, P, P],
    "adx_sample_counts": [P, I64, I64, P, P],
    "adx_sample_het_counts": [P, I64, I64, P, P],
    "adx_bed_workspace_bytes": [I64, I64, P],
    "adx_bed_to_packed": [P, I64, I64, P, P, P, c_size_t, P],
    "adx_simulate_packed": [P, P, I64, I64, c_int, c_uint64, c_uint64, c_uint32, P, P],
    "adx_em_workspace_bytes": [I64, I64, c_int, c_int, P],
    "adx_em_status": [P, c_size_t, I64, I64, c_int, c_int, P, P],
    "adx_em_stats": [P, I64, I64, c_int, c_int, P, P, P, P, P, P, c_size_t, P],
    "adx_em_sweep": [P, I64, I64, c_int, c_int, P, P, P, c_size_t, P],
    "adx_em_targets": [P, P, P, P, P, P, I64, I64, c_int, P, P, P],
    "adx_adam_step": [P, P, P, P, P, P, P, P, I64, I64, c_int, c_double, c_double, c_double,
                      c_double, c_double, P, P, P],
    "adx_em_adam_iteration": [P, I64, I64, c_int, c_int, P, P, P, P, P, P, P, P, P, c_double,
                              c_double, c_double, c_double, c_double, P, c_size_t, P],
    "adx_em_graph_create": [P, I64, I64, c_int, c_int, P, P, P, P, P, P, P, P, P, c_int, c_double, c_double,
                            c_double, c_double, P, P, c_size_t, P],
    "adx_em_graph_launch": [P, c_double, P],
    "adx_em_graph_iterations": [P, P],
    "adx_em_graph_destroy": [P],
    "adx_em_batch_workspace_bytes": [I64, I64, c_int, P, P],
    "adx_em_sweep_batch": [I64, I64, c_int, P, P, P, P, P, c_size_t, P],
    "adx_em_batch_apply": [I64, I64, c_int, P, c_int, c_int, P, P, P, P, P, P, P, P, P, P, c_double,
                           c_double, c_double, c_double, c_double, P, c_size_t, P],
    "adx_em_sweep_loglik": [P, I64, I64, c_int, c_int, P, P, P, c_size_t, P],
    "adx_em_sweep_blocks_info": [I64, I64, c_int, c_int, P, P, P],
    "adx_em_sweep_blocks": [P, I64, I64, c_int, c_int, P, P, c_int, c_int, P, c_size_t, P],
    "adx_em_loglik_from_sweep": [P, c_size_t, I64, I64, c_int, c_int, P, P],
    "adx_em_adam_update": [I64, I64, c_int, c_int, P, P, P, P, P, P, P, P, P, c_double, c_double, c_double,
                           c_double, c_double, P, c_size_t, P],
    "adx_dmma_tiles": [c_int, P],
    "adx_dmma_tile_set": [c_int, c_int, c_int],
    "adx_dmma_tile_get": [c_int, c_int, P],
    "adx_loglik_workspace_bytes": [I64, I64, c_int, c_int, P],
    "adx_loglik": [P, I64, I64, c_int, c_int, P, P, P, P, c_size_t, P],
    "adx_loglik_noalloc": [P, I64, I64, c_int, c_int, P, P, P, P],
    "adx_rsvd_rows": [P, I64, I64, P, P, c_int, P, P],
    "adx_rsvd_workspace_bytes": [I64, I64, c_int, P],
    "adx_rsvd_cols": [P, I64, I64, P, P, c_int, c_int, P, P, c_size_t, P],
    "adx_bvls": [P, P, I64, c_int, c_double, c_double, P, P],
    "adx_grad_hess_q": [P, I64, I64, c_int, P, P, P, P, P],
    "adx_grad_hess_p": [P, I64, I64, c_int, P, P, P, P, P],
    "adx_sqp_q": [P, P, P, P, I64, c_int, P, P],
    "adx_sqp_p": [P, P, P, I64, c_int, P, P],
    "adx_project_simplex": [P, I64, c_int, P],
    "adx_project_box": [P, I64, c_int, P],
    "adx_cv_workspace_bytes": [P],
    "adx_cv_mask_list": [P, c_size_t, I64, I64, P, I64, P, c_size_t, P],
    "adx_cv_mask_hash": [P, c_size_t, P, I64, I64, c_uint64, c_int, c_int, P],
    "adx_cv_deviance_list": [P, I64, I64, c_int, P, P, P, I64, P, P, c_size_t, P],
    "adx_cv_deviance_hash": [P, I64, I64, c_int, P, P, c_uint64, c_int, c_int, P, P, c_size_t, P],
    "adx_write_text_matrix": [ctypes.c_char_p, P, I64, I64, c_int],
    "adx_tc_wait_selftest": [c_int, c_uint32, P, P],
    "adx_write_text_matrix_fixed": [ctypes.c_char_p, P, I64, I64, c_int, c_int],
    "adx_mlp_workspace_bytes": [I64, c_int, P],
    "adx_mlp_forward": [P, P, P, P, P, P, P, P, I64, c_int, P, P, c_size_t, P],
    "adx_mlp_backward": [P, P, P, P, I64, c_int, P, P, P, P, P, P, P, P, c_size_t, P],
    "adx_mlp_adam": [P, P, P, P, P, I64, ctypes.c_float, ctypes.c_float, ctypes.c_float, ctypes.c_float,
                     c_int, P],
}
_RESTYPE = {"adx_version": ctypes.c_char_p, "adx_last_error": ctypes.c_char_p}

_lock = threading.Lock()
_lib: ctypes.CDLL | None = None


class AdxError(RuntimeError):
    """A library call returned an error status."""


def load() -> ctypes.CDLL:
    """Load the library (once) and declare every entry point's signature."""
    global _lib
    if _lib is not None:
        return _lib
    with _lock:
        if _lib is not None:
            return _lib
        if not LIB_PATH.exists():
            raise AdxError(
                f"{LIB_PATH} is missing; build it with `python -m adamixture_b200.csrc.build`"
            )
        lib = ctypes.CDLL(str(LIB_PATH))
        for name, args in SIGNATURES.items():
            fn = getattr(lib, name)
            fn.argtypes = args
            fn.restype = _RESTYPE.get(name, c_int)
        _lib = lib
        return lib


def call(name: str, *args) -> None:
    """Call entry point ``name``; raise AdxError with the library's message on failure."""
    lib = load()
    rc = getattr(lib, name)(*args)
    if rc != ADX_OK:
        msg = lib.adx_last_error().decode(errors="replace")
        kind = {ADX_ERR_ARG: "invalid argument", ADX_ERR_CUDA: "CUDA error",
                ADX_ERR_WORKSPACE: "workspace too small",
                ADX_ERR_UNSUPPORTED: "unsupported"}.get(rc, f"status {rc}")
        raise AdxError(f"{name}: {kind}: {msg}")


def query_size(name: str, *args) -> int:
    out = c_size_t(0)
    call(name, *args, ctypes.addressof(out))
    return int(out.value)


def version() -> str:
    return load().adx_version().decode()
