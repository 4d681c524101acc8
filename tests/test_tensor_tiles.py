"""The tile arithmetic of the tcgen05 step (k_tensor_step in
cat_cpu_b200/csrc/k_tensor.cu), restated in numpy and checked against the
oracle on the CPU.

The kernel reads the packed grid, spreads each 32-cell group to bytes with
(w >> k) & 0x01010101 (byte position 4k+j of a group holds cell pi(4k+j) =
8j+k), and runs product 1 as one MMA of N = Tc per 32-column K step s of the
whole X tile, against rows 32 (ks1 - 1 - s) .. of one Toeplitz band matrix W
whose K index follows pi and whose N index follows sigma (the output cell of
accumulator column n).  Product 2 sums rows with B_v, read as 128-row windows
of its Toeplitz store G, one per 32 bytes of K: row sums as u8 (R <= 127), or
as the f16 of H + 1024 (R = 128), whose bits are the 16-bit H plus 0x6400.
The rule runs on 8-bit (R <= 5), 16-bit (R <= 90) or 32-bit lanes (on the s32
count, or on the bit pattern of the f32 count plus 1024 (2R+1)) with the
centre cells taken from the packed input word.  The result bits are gathered into the output word by one shift
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


LANES8, LANES16, LANES32, F16 = 0, 1, 2, 3
F16_OFFSET = 1024


def sigma(n, mode):
    if mode == LANES8:
        return pi(n)
    if mode == LANES16:
        return 16 * (n & 1) + (n >> 1)
    return n


def tensor_mode(R):
    N = (2 * R + 1) ** 2
    if N <= 127:
        return LANES8
    if N < 1 << 15:
        return LANES16
    return LANES32 if 2 * R + 1 <= 255 else F16


def f32_bits(x):
    return int(np.array([x], dtype=np.float32).view(np.uint32)[0])


def lane_consts32(lo, hi, maxB, fbits, off):
    lo, hi = max(lo, 0), min(hi, maxB)
    if hi < lo:
        return 0, 0x80000000
    lb, hb = (f32_bits(lo + off), f32_bits(hi + off)) if fbits else (lo, hi)
    return (0x80000000 - lb) & 0xFFFFFFFF, (0x80000000 + hb) & 0xFFFFFFFF


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
    mode = tensor_mode(R)
    if mode >= LANES32:
        maxB = (2 * R + 1) ** 2
        fb = mode == F16
        off = F16_OFFSET * (2 * R + 1) if fb else 0
        bc = 1
        nlo_d, hih_d = lane_consts32(bmin, bmax, maxB, fb, off)
        nlo_s, hih_s = lane_consts32(smin + 1, smax + 1, maxB, fb, off)
    else:
        bits = 16 if mode == LANES16 else 8
        bc = 0x00010001 if mode == LANES16 else 0x01010101
        nlo_d, hih_d = lane_consts(bmin, bmax, bits)
        nlo_s, hih_s = lane_consts(smin + 1, smax + 1, bits)
    k2 = 16 if mode == F16 else 32
    return dict(PADC=PADC, Tc=Tc, Tr=Tr, nb=nb, atoms=atoms, ks1=ks1, nchunks=nchunks, mode=mode,
                lanes16=mode == LANES16, k2=k2,
                nlo0=(nlo_d * bc) & 0xFFFFFFFF, dlo=(nlo_s - nlo_d) & 0xFFFFFFFF,
                hiH0=(hih_d * bc) & 0xFFFFFFFF, dhi=(hih_s - hih_d) & 0xFFFFFFFF)


def w_matrix(P, R):
    """W[m][k], m < 32 (ks1 + nchunks - 1), k < 32: row m serves chunk offset
    D = ks1 - 1 - m // 32 and accumulator column m % 32; byte k of a group is cell pi(k)."""
    ks1, nch, PADC, mode = P["ks1"], P["nchunks"], P["PADC"], P["mode"]
    m = np.arange(32 * (ks1 + nch - 1))[:, None]
    k = np.arange(32)[None, :]
    D = ks1 - 1 - (m >> 5)
    d = 32 * D + pi(k) - PADC - sigma(m & 31, mode)
    return ((d >= -R) & (d <= R)).astype(np.int64)


def g_matrix(P, R):
    """G[i][kk], i < 128 + k2 (T2 - 1), kk < k2: the Toeplitz store of B_v.
    Product-2 K step t reads rows k2 (T2 - 1 - t) .. + 127."""
    k2 = P["k2"]
    T2 = 128 * P["nb"] // k2
    i = np.arange(128 + k2 * (T2 - 1))[:, None]
    kk = np.arange(k2)[None, :]
    d = k2 * (T2 - 1) + kk - i
    return ((d >= 0) & (d <= 2 * R)).astype(np.int64)


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
    G = g_matrix(P, R)
    k2, mode = P["k2"], P["mode"]
    T2 = 128 * nb // k2
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
            if mode == F16:
                # the re-quantisation's integer add gives the f16 of H + 1024
                h16 = (H & 0xFFFF) + 0x6400
                assert np.array_equal(h16.astype(np.uint16),
                                      (H + F16_OFFSET).astype(np.float16).view(np.uint16))
                Hq = (H + F16_OFFSET).astype(np.int64)
            else:
                assert H.max() <= 255
                Hq = H
            # product 2: one MMA per k2 rows of K over the Toeplitz windows of G
            C = np.zeros((128, Tc), dtype=np.int64)
            for t in range(T2):
                g0 = k2 * (T2 - 1 - t)
                C += G[g0: g0 + 128] @ Hq[k2 * t: k2 * t + k2]
            if mode == F16:
                assert C.max() < 1 << 24  # exact in the f32 accumulator
                C = np.array(C, dtype=np.float32).view(np.uint32).astype(np.int64)
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
                if mode >= LANES32:
                    # plain 32-bit loads: register k = column k = output cell k
                    for k in range(32):
                        s1 = (cw >> np.uint64(k)) & np.uint64(1)
                        ge = (Cc[:, k] + nlo0 + s1 * dlo) & M32
                        le = (hiH0 + s1 * dhi - Cc[:, k]) & M32
                        acc |= ((ge & le) >> np.uint64(31)) << np.uint64(k)
                elif mode == LANES8:
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
    (300, 91, O.scaled_rule(91), 0.45, 16, 1),   # 32-bit lanes, 11 K steps
    (260, 113, O.scaled_rule(113), 0.45, 17, 1),  # 32-bit lanes, 13 K steps
    (300, 127, O.scaled_rule(127), 0.45, 18, 1),  # largest u8 row sum (255)
    (300, 128, O.scaled_rule(128), 0.45, 19, 1),  # f16 row sums (up to 257)
    (130, 128, O.scaled_rule(128), 0.448, 20, 1),  # f16, n close to R
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
    for R in (1, 2, 5, 6, 12, 32, 64, 90, 91, 127, 128):
        N = (2 * R + 1) ** 2
        for rule in [O.scaled_rule(R), (0, N, 0, N), (N, 0, 5, 3), (-3, 2, N + 5, N + 9), (4, 4, 4, 4)]:
            P = plan(64, R, rule)
            B = np.arange(N + 1, dtype=np.uint64)
            smin, smax, bmin, bmax = rule
            mode = P["mode"]
            top = np.uint64({LANES8: 0x80, LANES16: 0x8000}.get(mode, 0x80000000))
            mask = np.uint64({LANES8: 0xFF, LANES16: 0xFFFF}.get(mode, 0xFFFFFFFF))
            nlo0, dlo, hiH0, dhi = (np.uint64(P[k]) for k in ("nlo0", "dlo", "hiH0", "dhi"))
            # what the lane holds for count B: B itself, or the f32 bits of B + 1024 (2R+1)
            L = B
            if mode == F16:
                L = np.array(B + np.uint64(F16_OFFSET * (2 * R + 1)), dtype=np.float32).view(np.uint32)
                L = L.astype(np.uint64)
            for s in (0, 1):
                k = B.astype(np.int64) - s
                want = ((k >= smin) & (k <= smax)) if s else ((k >= bmin) & (k <= bmax))
                sw = np.uint64(s)
                # lane 0 only (the other lanes hold the same constants)
                ge = (L + (nlo0 & mask) + sw * dlo) & M32
                le = ((hiH0 & mask) + sw * dhi - L) & M32
                got = (ge & le & top) != 0
                valid = B >= s  # a live centre implies B >= 1
                assert np.array_equal(got[valid], want[valid]), (R, rule, s)
