"""The tile arithmetic of the tcgen05 step (k_tensor_step in
cat_cpu_b200/csrc/k_tensor.cu), restated in numpy and checked against the
oracle on the CPU.

The kernel reads the packed grid, spreads each 32-cell group to bytes with
(w >> k) & 0x01010101 (byte position 4k+j of a group holds cell pi(4k+j) =
8j+k), and runs product 1 as one MMA of N = Tc per 32-column K step s of the
whole X tile, against rows 32 (ks1 - 1 - s) .. of one Toeplitz band matrix W
whose K index follows pi and whose N index follows sigma (the output cell of
accumulator column n).  Product 2 sums rows with B_v, and the rule runs on
8-bit (R <= 5) or 16-bit lanes with the centre cells taken from the packed
input word.  The result bits are gathered into the output word by one shift
per register.  This test runs that exact sequence (tile geometry, K steps,
torus wrap of rows and words, lane constants with 32-bit wraparound, byte
permutes, gather) on whole small grids and compares every generation with the
oracle, so that the index algebra is settled before the kernel runs on a GPU."""
import numpy as np
import pytest

from oracle import oracle as O

M32 = np.uint64(0xFFFFFFFF)


def pi(q):
    return 8 * (q & 3) + (q >> 2)


def sigma(n, lanes16):
    return 16 * (n & 1) + (n >> 1) if lanes16 else pi(n)


def lane_consts(lo, hi, bits):
    top = 1 << (bits - 1)
    lo = max(lo, 0)
    hi = min(hi, top - 1)
    if hi < lo or lo > top - 1:
        lo, hi = top, 0
    return top - lo, top + hi


def plan(n, R, rule):
    """tensor_geometry + the rule constants of tensor_plan_create."""
    smin, smax, bmin, bmax = rule
    Tc = 128
    PADC = 16 if R <= 16 else 16 + 32 * ((R - 16 + 31) // 32)
    nb = 1 if R <= 32 else (128 + 2 * R + 127) // 128
    Tr = 128 - 2 * R if nb == 1 else min(128, 128 * nb - 2 * R)
    ks1 = (PADC + Tc + R + 31) // 32
    atoms = (ks1 + 3) // 4
    nchunks = Tc // 32
    lanes16 = (2 * R + 1) ** 2 > 127
    bits = 16 if lanes16 else 8
    bc = 0x00010001 if lanes16 else 0x01010101
    nlo_d, hih_d = lane_consts(bmin, bmax, bits)
    nlo_s, hih_s = lane_consts(smin + 1, smax + 1, bits)
    return dict(PADC=PADC, Tc=Tc, Tr=Tr, nb=nb, atoms=atoms, ks1=ks1, nchunks=nchunks, lanes16=lanes16,
                nlo0=(nlo_d * bc) & 0xFFFFFFFF, dlo=(nlo_s - nlo_d) & 0xFFFFFFFF,
                hiH0=(hih_d * bc) & 0xFFFFFFFF, dhi=(hih_s - hih_d) & 0xFFFFFFFF)


def w_matrix(P, R):
    """W[m][k], m < 32 (ks1 + nchunks - 1), k < 32: row m serves chunk offset
    D = ks1 - 1 - m // 32 and accumulator column m % 32; byte k of a group is cell pi(k)."""
    ks1, nch, PADC, lanes16 = P["ks1"], P["nchunks"], P["PADC"], P["lanes16"]
    m = np.arange(32 * (ks1 + nch - 1))[:, None]
    k = np.arange(32)[None, :]
    D = ks1 - 1 - (m >> 5)
    d = 32 * D + pi(k) - PADC - sigma(m & 31, lanes16)
    return ((d >= -R) & (d <= R)).astype(np.int64)


def prmt(a, b, sel):
    """prmt.b32 default mode on uint64 arrays holding 32-bit values."""
    src = [(a >> np.uint64(8 * i)) & np.uint64(0xFF) for i in range(4)] + \
          [(b >> np.uint64(8 * i)) & np.uint64(0xFF) for i in range(4)]
    out = np.zeros_like(a)
    for i in range(4):
        nib = (sel >> (4 * i)) & 0xF
        byte = src[nib & 7]
        if nib & 8:
            byte = np.where(byte & np.uint64(0x80), np.uint64(0xFF), np.uint64(0))
        out |= byte << np.uint64(8 * i)
    return out


def tensor_step(grid, R, rule):
    """One generation exactly as k_tensor_step computes it (numpy, int arithmetic)."""
    n = grid.shape[0]
    P = plan(n, R, rule)
    PADC, Tc, Tr, nb = P["PADC"], P["Tc"], P["Tr"], P["nb"]
    XW = 128 * P["atoms"]
    assert Tr >= 1
    W = w_matrix(P, R)
    ks1 = P["ks1"]
    assert 32 * ks1 <= XW
    m_ = np.arange(128)[:, None]
    k_ = np.arange(128 * nb)[None, :]
    Bv = ((k_ >= m_) & (k_ <= m_ + 2 * R)).astype(np.int64)
    nw = (n + 31) // 32
    words = np.zeros((n, nw * 32), dtype=np.uint64)
    words[:, :n] = grid
    cur_words = (words.reshape(n, nw, 32) << np.arange(32, dtype=np.uint64)).sum(axis=2)  # packed input rows
    out_words = np.zeros((n, nw), dtype=np.uint64)
    tiles_x, tiles_y = -(-n // Tc), -(-n // Tr)
    q = np.arange(32)
    nlo0, dlo, hiH0, dhi = (np.uint64(P[k]) for k in ("nlo0", "dlo", "hiH0", "dhi"))
    for ty in range(tiles_y):
        for tx in range(tiles_x):
            rbase, cbase = ty * Tr - R, tx * Tc - PADC
            # X tile in shared-memory byte order: position 32g + q holds cell pi(q) of group g
            cols = np.concatenate([(cbase + 32 * g + pi(q)) % n for g in range(XW // 32)])
            H = np.zeros((128 * nb, Tc), dtype=np.int64)
            for b in range(nb):  # row blocks: product 1 per block, one MMA per K step
                rows = (rbase + 128 * b + np.arange(128)) % n
                X = grid[np.ix_(rows, cols)].astype(np.int64)
                Hb = np.zeros((128, Tc), dtype=np.int64)
                for st in range(ks1):
                    m0 = 32 * (ks1 - 1 - st)
                    Hb += X[:, 32 * st: 32 * st + 32] @ W[m0: m0 + Tc].T
                H[128 * b: 128 * b + 128] = Hb
            assert H.max() <= 2 * R + 1
            C = Bv @ H  # box counts, centre included (product 2 over all blocks)
            for i in range(P["nchunks"]):
                wi = tx * (Tc // 32) + i
                gi = ty * Tr + np.arange(128)
                ok = (gi < n) & (wi < nw)
                cw = np.where(ok, cur_words[np.minimum(gi, n - 1), min(wi, nw - 1)], np.uint64(0))
                Cc = C[:, 32 * i: 32 * i + 32].astype(np.uint64)
                # tcgen05.ld .pack::16b: register r = column 2r (low 16) | column 2r+1 (high 16)
                v = [(Cc[:, 2 * r] & np.uint64(0xFFFF)) | ((Cc[:, 2 * r + 1] & np.uint64(0xFFFF)) << np.uint64(16))
                     for r in range(16)]
                acc = np.zeros(128, dtype=np.uint64)
                if not P["lanes16"]:
                    for k in range(8):
                        B4 = prmt(v[2 * k], v[2 * k + 1], 0x6420)
                        s4 = (cw >> np.uint64(k)) & np.uint64(0x01010101)
                        ge = (B4 + nlo0 + s4 * dlo) & M32
                        le = (hiH0 + s4 * dhi - B4) & M32
                        acc |= (ge & le & np.uint64(0x80808080)) >> np.uint64(7 - k)
                else:
                    for r in range(16):
                        s2 = (cw >> np.uint64(r)) & np.uint64(0x00010001)
                        ge = (v[r] + nlo0 + s2 * dlo) & M32
                        le = (hiH0 + s2 * dhi - v[r]) & M32
                        acc |= (ge & le & np.uint64(0x80008000)) >> np.uint64(15 - r)
                for mm in range(Tr):
                    gi = ty * Tr + mm
                    if gi < n and wi < nw:
                        out_words[gi, wi] = acc[mm]
    bits = ((out_words[:, :, None] >> np.arange(32, dtype=np.uint64)[None, None, :]) & np.uint64(1))
    return bits.reshape(n, nw * 32)[:, :n].astype(np.uint8)


CASES = [
    # (n, R, rule, density, seed, steps)
    (64, 1, O.CONWAY, 0.35, 1, 3),
    (97, 2, O.sweep_rule(2), 0.5, 2, 2),
    (160, 5, O.BOSCO_R5, 0.5, 3, 2),
    (256, 5, O.BOSCO_R5, 0.5, 4, 1),
    (41, 3, O.sweep_rule(3), 0.4, 5, 2),
    (120, 8, O.scaled_rule(8), 0.45, 6, 2),
    (200, 16, O.scaled_rule(16), 0.45, 7, 1),
    (150, 17, O.scaled_rule(17), 0.45, 8, 1),
    (100, 32, O.scaled_rule(32), 0.44, 9, 1),
    (33, 5, O.BOSCO_R5, 0.5, 10, 2),
    (20, 4, O.sweep_rule(4), 0.5, 11, 2),
    (300, 40, O.scaled_rule(40), 0.45, 12, 1),   # two row blocks
    (300, 64, O.scaled_rule(64), 0.45, 13, 1),   # two row blocks, 9 K steps
    (250, 90, O.scaled_rule(90), 0.45, 14, 1),   # three row blocks, 11 K steps
    (96, 33, O.scaled_rule(33), 0.45, 15, 1),
]


@pytest.mark.parametrize("n,R,rule,density,seed,steps", CASES)
def test_tile_arithmetic_matches_oracle(n, R, rule, density, seed, steps):
    g = O.generate(n, seed, density, 1)
    for s in range(steps):
        want = O.step(g, R, rule)
        got = tensor_step(g, R, rule)
        assert np.array_equal(got, want), f"generation {s + 1}: {int((got != want).sum())} cells differ"
        g = want


def test_rule_lanes_every_count():
    """Every box count and centre against the scalar rule, for rules with empty and
    out-of-range intervals, in both lane widths (through the same constants)."""
    for R in (1, 2, 5, 6, 12, 32, 64, 90):
        N = (2 * R + 1) ** 2
        for rule in [O.scaled_rule(R), (0, N, 0, N), (N, 0, 5, 3), (-3, 2, N + 5, N + 9), (4, 4, 4, 4)]:
            P = plan(64, R, rule)
            B = np.arange(N + 1, dtype=np.uint64)
            smin, smax, bmin, bmax = rule
            top = np.uint64(0x8000 if P["lanes16"] else 0x80)
            mask = np.uint64(0xFFFF if P["lanes16"] else 0xFF)
            nlo0, dlo, hiH0, dhi = (np.uint64(P[k]) for k in ("nlo0", "dlo", "hiH0", "dhi"))
            for s in (0, 1):
                k = B.astype(np.int64) - s
                want = ((k >= smin) & (k <= smax)) if s else ((k >= bmin) & (k <= bmax))
                sw = np.uint64(s)
                # lane 0 only (the other lanes hold the same constants)
                ge = (B + (nlo0 & mask) + sw * dlo) & M32
                le = ((hiH0 & mask) + sw * dhi - B) & M32
                got = (ge & le & top) != 0
                valid = B >= s  # a live centre implies B >= 1
                assert np.array_equal(got[valid], want[valid]), (R, rule, s)
