"""CPU check of the float64 sweep's shared-memory layouts (csrc/em_sweep_dmma.cu).

For both layouts (Lay<0>, Lay<1>) this restates, lane by lane, every fragment access the
chunk loop makes -- the Q-tile fills and loads for h and for A/B, the P-group fills and
loads for h and for T, the transpose-tile stores and loads -- and checks that
  * every index stays inside its region (Q: W x QSTR, P group: GS x PSTR, transpose tile:
    WS x DSTR per warp), and
  * no half-warp of a 64-bit access touches two different addresses in the same bank pair
    (conflict-free; identical addresses are a broadcast).
The constants mirror the kernel's; a change there that breaks either property fails here
before any GPU run.
"""
import pytest

WARPS, WS, CH, DSTR = 8, 32, 16, 20
W = WARPS * WS

LAYOUTS = {
    0: dict(QSTR=24, QC=16, PSTR=20, PC=16, GRP=8, NV=16, KSMAX=4, sw=lambda r: ((r >> 3) & 3) << 2),
    1: dict(QSTR=16, QC=8, PSTR=12, PC=8, GRP=4, NV=8, KSMAX=2, sw=lambda r: (((r >> 3) & 3) << 2) ^ ((r & 1) << 3)),
}


def dsw(r):
    return ((r >> 3) & 3) << 2


def conflict_free(addrs):
    """64-bit accesses of a warp: each half-warp is one wavefront when its distinct
    addresses fall in distinct bank pairs (address mod 16 doubles)."""
    for h in range(2):
        seen = {}
        for a in set(addrs[16 * h:16 * h + 16]):
            if a % 16 in seen:
                return False
            seen[a % 16] = a
    return True


def lanes():
    return [(lane >> 2, lane & 3) for lane in range(32)]


@pytest.mark.parametrize("tl", [0, 1])
def test_q_tile_accesses(tl):
    L = LAYOUTS[tl]
    QSTR, sw = L["QSTR"], L["sw"]
    KS, NK = L["KSMAX"], (L["KSMAX"] + 1) // 2
    # fill: column k of row r (k < QC) at r*QSTR + (k ^ sw(r)); a row's columns distinct
    for r in range(W):
        cols = [k ^ sw(r) for k in range(L["QC"])]
        assert len(set(cols)) == L["QC"] and max(cols) < QSTR
    for warp in range(WARPS):
        for nt in range(4):
            # h: B operand, k-slots 4ks + t (k8 pairs use ks and ks+1), column g of the tile
            for ks in range(KS):
                ad = []
                for g, t in lanes():
                    r = warp * WS + 8 * (g >> 1) + 2 * nt + (g & 1)
                    c = (4 * ks + t) ^ sw(r)
                    assert 0 <= r < W and 0 <= c < QSTR
                    ad.append(r * QSTR + c)
                assert conflict_free(ad), ("h", tl, warp, nt, ks)
            # A/B: B operand rows 8t + 2nt (k-slot t) and 8t + 2nt + 1 (k-slot t + 4)
            for c_ in range(2):
                for n in range(NK):
                    ad = []
                    for g, t in lanes():
                        r = warp * WS + 8 * t + 2 * nt + c_
                        c = (8 * n + g) ^ sw(r)
                        assert 0 <= r < W and 0 <= c < QSTR
                        ad.append(r * QSTR + c)
                    assert conflict_free(ad), ("ab", tl, warp, nt, c_, n)


@pytest.mark.parametrize("tl", [0, 1])
def test_p_group_accesses(tl):
    L = LAYOUTS[tl]
    PSTR, GS = L["PSTR"], CH * L["GRP"]
    KS, NK = L["KSMAX"], (L["KSMAX"] + 1) // 2
    assert L["PC"] <= PSTR
    for ch in range(L["GRP"]):
        base = ch * CH * PSTR
        # h: A operand rows g and g + 8, columns 4ks + t
        for ks in range(KS):
            for hh in range(2):
                ad = []
                for g, t in lanes():
                    a = base + (g + 8 * hh) * PSTR + 4 * ks + t
                    assert a < GS * PSTR and 4 * ks + t < L["PC"]
                    ad.append(a)
                assert conflict_free(ad), ("ph", tl, ch, ks, hh)
        # T: B operand rows (SNPs) 8q + t and 8q + t + 4, column 8n + g
        for q in range(2):
            for off in (0, 4):
                for n in range(NK):
                    ad = []
                    for g, t in lanes():
                        a = base + (8 * q + t + off) * PSTR + 8 * n + g
                        assert a < GS * PSTR and 8 * n + g < L["PC"]
                        ad.append(a)
                    assert conflict_free(ad), ("pb", tl, ch, q, off, n)


def test_transpose_tile_accesses():
    # stores: element e of tile nt -> row 8t + 2nt + e%2, column g + 8(e/2), swizzled
    for nt in range(4):
        for e in range(4):
            ad = []
            for g, t in lanes():
                r = 8 * t + 2 * nt + (e & 1)
                c = (g + 8 * (e >> 1)) ^ dsw(r)
                assert r < WS and c < DSTR
                ad.append(r * DSTR + c)
            assert conflict_free(ad), ("dT store", nt, e)
    # loads: rows 16m + g (+8), columns 8q + t (+4)
    for q in range(2):
        for off in (0, 4):
            for m in range(2):
                for hh in range(2):
                    ad = []
                    for g, t in lanes():
                        r = 16 * m + g + 8 * hh
                        c = (8 * q + t + off) ^ dsw(r)
                        assert r < WS and c < DSTR
                        ad.append(r * DSTR + c)
                    assert conflict_free(ad), ("dT load", q, off, m, hh)


@pytest.mark.parametrize("tl", [0, 1])
def test_reduction_buffer_and_shared_memory_budget(tl):
    L = LAYOUTS[tl]
    NV = L["NV"]
    # stores (warp*NV + v)*32 + lane, sums read (ww*NV + v)*32 + l: inside 8*NV*32 doubles
    assert (WARPS * NV + 0) * 32 == WARPS * NV * 32
    doubles = W * L["QSTR"] + CH * L["GRP"] * L["PSTR"] + WARPS * WS * DSTR + 2 * WARPS * NV * 32 + WARPS * WS
    nbytes = 8 * doubles
    if tl == 0:
        assert nbytes == 178176 and nbytes <= 227 * 1024
    else:
        assert nbytes == 114688 and 2 * (nbytes + 1024) <= 228 * 1024
    # every thread sums NV*32/256 values of the chunk
    assert (NV * 32) % (WARPS * 32) == 0
