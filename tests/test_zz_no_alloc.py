"""The allocation-free log-likelihood entry point (adx_loglik_noalloc).

Some callers of this library cannot allocate device memory themselves: a host whose
device memory belongs to another allocator (a framework's pool, or a language runtime
that must account for every byte), or a code path that cannot accept the device-wide
synchronisation that cudaMalloc/cudaFree imply. For them adx_loglik_noalloc keeps its
per-block partial sums in a fixed 16 KiB device array inside the library instead of a
caller-provided workspace.

This test calls it through the C ABI and checks it against adx_loglik (workspace form,
same arithmetic) on two calls in a row, since the array keeps the previous call's
contents. It lives in a file of its own that sorts last, so that a run stopping at the
first failure has run every other test first; it also passes alone in a fresh process.
"""
import numpy as np
import pytest
import torch

from adamixture_b200 import _lib

pytestmark = pytest.mark.gpu


def _dev(x, dtype):
    return torch.from_numpy(np.ascontiguousarray(x)).cuda().to(dtype)


def _with_workspace(G, P, Q, M, prec):
    N, K = Q.shape
    nbytes = _lib.query_size("adx_loglik_workspace_bytes", M, N, K, prec)
    ws = torch.empty(nbytes, dtype=torch.uint8, device=G.device)
    out = torch.empty((), dtype=torch.float64, device=G.device)
    _lib.call("adx_loglik", G.data_ptr(), M, N, K, prec, P.data_ptr(), Q.data_ptr(),
              out.data_ptr(), ws.data_ptr(), ws.numel(), torch.cuda.current_stream().cuda_stream)
    return float(out.item())


def _no_alloc(G, P, Q, M, prec):
    N, K = Q.shape
    out = torch.full((), float("nan"), dtype=torch.float64, device=G.device)
    _lib.call("adx_loglik_noalloc", G.data_ptr(), M, N, K, prec, P.data_ptr(), Q.data_ptr(),
              out.data_ptr(), torch.cuda.current_stream().cuda_stream)
    return float(out.item())


def _random_cohort(N, M, K, seed):
    rng = np.random.default_rng(seed)
    G = rng.choice(4, size=(M, N), p=[0.3, 0.35, 0.3, 0.05]).astype(np.uint8)
    packed = np.zeros(((M + 3) // 4, N), dtype=np.uint8)
    for s in range(4):
        rows = G[s::4]
        packed[: rows.shape[0]] |= rows << (2 * s)
    P = np.clip(rng.beta(0.8, 0.8, size=(M, K)), 1e-5, 1 - 1e-5)
    Q = rng.dirichlet(np.full(K, 0.5), size=N)
    return {"M": M, "packed": packed, "P0": P, "Q0": Q}


@pytest.mark.parametrize("prec", [_lib.ADX_F64, _lib.ADX_F32])
def test_no_alloc_loglik_matches_workspace_form(cuda, demo, synth, prec):
    dt = torch.float64 if prec == _lib.ADX_F64 else torch.float32
    # a shape whose plan fills many more partial slots comes first, so a later, smaller
    # call that read a stale slot would differ; then two cohorts of different shape, each
    # called twice in a row
    big = _random_cohort(6000, 3000, 8, 5)
    for d in (big, demo, synth, demo):
        M = int(d["M"])
        G = torch.from_numpy(d["packed"]).cuda()
        P, Q = _dev(d["P0"], dt), _dev(d["Q0"], dt)
        ref = _with_workspace(G, P, Q, M, prec)
        for _ in range(2):
            got = _no_alloc(G, P, Q, M, prec)
            # the same plan, kernels and fixed-order sum of the partials: bit-identical
            assert got == ref, (got, ref)
        if "loglik0" in d:
            assert abs(ref - float(d["loglik0"])) <= 1e-6 * abs(float(d["loglik0"]))


def test_no_alloc_rejects_bad_arguments(cuda):
    G = torch.zeros((1, 4), dtype=torch.uint8, device=cuda)
    P = torch.zeros((2, 65), dtype=torch.float64, device=cuda)
    out = torch.zeros((), dtype=torch.float64, device=cuda)
    with pytest.raises(_lib.AdxError, match="invalid argument"):
        _lib.call("adx_loglik_noalloc", G.data_ptr(), 2, 4, 65, _lib.ADX_F64, P.data_ptr(),
                  P.data_ptr(), out.data_ptr(), torch.cuda.current_stream().cuda_stream)
