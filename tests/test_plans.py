"""CPU checks of the launch plans, read back through the workspace-size queries (host code
only; no GPU needed).

* Tensor-core sweep: the sample-split count is the one whose grid, dispatched in blockIdx
  order onto 148 SMs with one CTA per SM, finishes first (the smallest count within 0.2 %
  of the earliest finish), over the counts around the ~8-wave one. The rule is restated
  here as a greedy list schedule and compared with the library's choice.
* Log-likelihood: the grid never exceeds 1776 blocks (148 x 12), so its partial sums
  always fit the allocation-free variant's 2048-entry array.
* Batched float64 E-step: its workspace is every problem's single-problem partials side by
  side (the float64 plan does not depend on K), and it rejects K > 16 and more than 64
  problems.
"""
import heapq

import pytest

from adamixture_b200 import _lib

SMS, R, TILE, OVERHEAD = 148, 7, 128, 3
LL_BLOCKS, NOALLOC_PARTIALS = 1776, 2048


def cdiv(a, b):
    return -(-a // b)


def makespan(M, n_stile, n_split, n_mblk):
    m_tiles = cdiv(M, TILE)
    free_at = [0] * SMS
    end = 0
    for s in range(n_split):
        n_my = (n_stile - s + n_split - 1) // n_split
        for b in range(n_mblk):
            t = heapq.heappop(free_at) + n_my * min(R, m_tiles - b * R) + OVERHEAD
            heapq.heappush(free_at, t)
            end = max(end, t)
    return end


def expected_split(M, N):
    n_stile, n_mblk = cdiv(N, TILE), cdiv(M, R * TILE)
    lo = max(1, min(n_stile, cdiv(8 * SMS, n_mblk)))
    hi = min(n_stile, 2 * lo + 8)
    best_t, best_n = None, lo
    for n in range(max(1, lo // 2), hi + 1):
        t = makespan(M, n_stile, n, n_mblk)
        if best_t is None or 1000 * t < 998 * best_t:
            best_t, best_n = t, n
    return best_n


def library_split(M, N, K, prec):
    """n_split recovered from the tensor-core workspace size: a 256-byte header, the A/B
    partials (n_split x M x 2K floats) and the T partials (n_mblk x N x K floats) rounded up
    to 256 bytes, then one 4 KiB converted-Q tile per 128 samples."""
    nbytes = _lib.query_size("adx_em_workspace_bytes", M, N, K, prec)
    n_stile, n_mblk = cdiv(N, TILE), cdiv(M, R * TILE)
    partial_bytes = nbytes - n_stile * 4096 - 256 - 4 * n_mblk * N * K
    ab = 4 * M * 2 * K
    assert ab > 255
    return partial_bytes // ab


@pytest.mark.parametrize("M,N", [(500_000, 200_000), (50_000, 200_000), (200_000, 10_000),
                                 (13_000, 1_000), (4_000, 300), (2_000_000, 50_000), (896 * 148, 128 * 40),
                                 (33, 200_000), (1_000_000, 129)])
def test_tc_split_count_minimises_the_simulated_dispatch(M, N):
    want = expected_split(M, N)
    for prec in (_lib.ADX_F16, _lib.ADX_BF16):
        assert library_split(M, N, 10, prec) == want
    # independent of K (the plan is a function of M and N)
    assert library_split(M, N, 3, _lib.ADX_F16) == want


def test_tc_split_fills_the_last_wave_at_the_bench_shape():
    # N=200,000 x M=500,000: 559 SNP blocks; the fixed 8-wave rule's 3 splits leave the
    # twelfth wave a third full, the chosen count finishes within 0.5 % of the ideal
    M, N = 500_000, 200_000
    n_stile, n_mblk = cdiv(N, TILE), cdiv(M, R * TILE)
    n = library_split(M, N, 10, _lib.ADX_F16)
    ideal = cdiv(M, TILE) * n_stile / SMS
    assert makespan(M, n_stile, n, n_mblk) <= 1.005 * ideal + 34 * OVERHEAD
    assert makespan(M, n_stile, 3, n_mblk) > 1.05 * ideal


@pytest.mark.parametrize("prec", [_lib.ADX_F64, _lib.ADX_F32])
def test_loglik_grid_stays_within_the_partials_bound(prec):
    worst = 0
    for M in (1, 3, 31, 32, 33, 1_000, 4_099, 77_777, 500_000, 10_000_000):
        for N in (1, 7, 255, 1_024, 1_025, 10_000, 200_000, 1_000_000):
            for K in (1, 3, 10, 16, 40, 64):
                nbytes = _lib.query_size("adx_loglik_workspace_bytes", M, N, K, prec)
                blocks = (nbytes - 256) // 8
                assert 1 <= blocks <= LL_BLOCKS, (M, N, K, blocks)
                worst = max(worst, blocks)
    assert worst <= NOALLOC_PARTIALS


def _batch_bytes(M, N, Ks):
    import ctypes

    arr = (ctypes.c_int * len(Ks))(*Ks)
    return _lib.query_size("adx_em_batch_workspace_bytes", M, N, len(Ks), ctypes.addressof(arr))


def f64_plan(M, N):
    """The float64 tensor-core sweep's partition (K <= 16), restated: 256-sample sub-tiles,
    16-SNP chunks, splits x SNP blocks near 1776 blocks minimising partial traffic."""
    import math

    n_stile = cdiv(N, 256)
    n_split = int(math.floor(math.sqrt(1776 * N / (2.0 * M)) + 0.5))
    n_split = max(1, min(n_split, n_stile, 1776))
    n_mblk = max(1, min(1776 // n_split, cdiv(M, 16)))
    mb = cdiv(cdiv(M, n_mblk), 16) * 16
    return n_split, cdiv(M, mb)


@pytest.mark.parametrize("M,N", [(100_000, 20_000), (3_001, 4_096), (33, 1_000_000), (500_000, 200_000)])
def test_batch_workspace_is_the_single_problem_partials_side_by_side(M, N):
    # the float64 plan does not depend on K, so a batch's workspace is a 256-byte header plus
    # every problem's single-problem partials (each 256-byte aligned); a single problem's
    # workspace also holds one log-likelihood partial per block after its partials
    n_split, n_mblk = f64_plan(M, N)
    Ks = [2, 7, 10, 12, 16, 1]
    total = 256
    for K in Ks:
        part = cdiv((n_split * M * 2 * K + n_mblk * N * K) * 8, 256) * 256
        single = _lib.query_size("adx_em_workspace_bytes", M, N, K, _lib.ADX_F64)
        assert single == 256 + part + n_split * n_mblk * 8, (M, N, K)
        total += part
    assert _batch_bytes(M, N, Ks) == total


def test_batch_rejects_what_it_cannot_run():
    with pytest.raises(_lib.AdxError, match="invalid argument"):
        _batch_bytes(1000, 1000, [17])          # the batched sweep is the K <= 16 float64 form
    with pytest.raises(_lib.AdxError, match="invalid argument"):
        _batch_bytes(1000, 1000, [4] * 65)      # at most 64 problems per launch
    with pytest.raises(_lib.AdxError, match="invalid argument"):
        _batch_bytes(1000, 1000, [0])


def test_float64_plan_stays_within_the_block_bound():
    # the E-step plan's grid (sample splits x SNP blocks) never exceeds 1776 blocks, including
    # a single SNP row against a million samples
    for M in (1, 16, 1_000, 500_000):
        for N in (1, 257, 200_000, 1_000_000):
            for K in (3, 10, 16, 40):
                nbytes = _lib.query_size("adx_loglik_workspace_bytes", M, N, K, _lib.ADX_F64)
                assert (nbytes - 256) // 8 <= LL_BLOCKS, (M, N, K)
