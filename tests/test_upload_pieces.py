"""CPU checks of how a packed matrix in host memory is cut into upload pieces (host logic):
the pieces cover the SNP blocks in order, their sweeps take no more waves than the full
sweep, and at N=200,000 x M=500,000 the float64 partition (19 CTAs per block, 93 blocks)
gives three pieces of 31 blocks (589 CTAs, four waves of 148 SMs each)."""
import ctypes

import pytest

from adamixture_b200 import _lib
from adamixture_b200.model.em_adam_gpu import upload_pieces


def cdiv(a, b):
    return -(-a // b)


@pytest.mark.parametrize("nb", [1, 2, 5, 31, 93, 148, 1000, 1776])
@pytest.mark.parametrize("cpb", [1, 2, 7, 19, 148, 300])
@pytest.mark.parametrize("sms", [148, 132])
def test_pieces_cover_the_blocks_in_whole_waves(nb, cpb, sms):
    pcs = upload_pieces(nb, cpb, sms)
    assert pcs[0][0] == 0 and pcs[-1][1] == nb and 1 <= len(pcs) <= 4
    assert all(a < b for a, b in pcs) and all(x[1] == y[0] for x, y in zip(pcs, pcs[1:]))
    assert sum(cdiv((b - a) * cpb, sms) for a, b in pcs) == cdiv(nb * cpb, sms)


def _info(M, N, K):
    spb, nb, cpb = ctypes.c_int64(0), ctypes.c_int(0), ctypes.c_int(0)
    _lib.call("adx_em_sweep_blocks_info", M, N, K, _lib.ADX_F64, ctypes.addressof(spb), ctypes.addressof(nb),
              ctypes.addressof(cpb))
    return spb.value, nb.value, cpb.value


def test_bench_shape_pieces():
    spb, nb, cpb = _info(500_000, 200_000, 10)
    assert (nb, cpb) == (93, 19) and spb % 16 == 0 and nb == cdiv(500_000, spb)
    assert upload_pieces(nb, cpb, 148) == [(0, 31), (31, 62), (62, 93)]


def test_blocks_info_rejects_other_forms():
    with pytest.raises(_lib.AdxError):
        _info(1000, 1000, 17)
    spb, nb, cpb = ctypes.c_int64(0), ctypes.c_int(0), ctypes.c_int(0)
    with pytest.raises(_lib.AdxError):
        _lib.call("adx_em_sweep_blocks_info", 1000, 1000, 4, _lib.ADX_F32, ctypes.addressof(spb),
                  ctypes.addressof(nb), ctypes.addressof(cpb))
