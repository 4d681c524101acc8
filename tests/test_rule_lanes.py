"""The lane arithmetic of the plain prefix-sum kernel (k_plain_wide in
cat_cpu_b200/csrc/k_plain.cu), restated in numpy and checked against the
scalar interval rule for every box count, on the CPU.

Row-pair mode keeps the box counts of rows r and r+1 for one column in the
low and high 16 bits of one 32-bit word.  The kernel forms them as a difference
of 32-bit prefix sums taken modulo 2^32, and then tests both lanes at once:
  - B + (2^15 - lo) has bit 15 set iff B >= lo;
  - (2^15 + hi) - B has bit 15 set iff B <= hi.
lo and hi follow from the centre through one multiply-add on the lane-packed
centres.  This holds while every box count stays below 2^15, which is why the
kernel uses row pairs only for R <= 90 ((2R+1)^2 = 32761).  The 32-bit-lane mode
uses the same test with 2^31.  These tests pin those bounds: exact up to R = 90,
and not exact at R = 91 in 16-bit lanes."""
import numpy as np
import pytest

M32 = 0xFFFFFFFF


def rule_constants(radius, rule, pair):
    """The kernel's RuleScan: nlo0/hih0 for a dead centre, dnlo/dhih for a live one."""
    smin, smax, bmin, bmax = rule
    N = (2 * radius + 1) ** 2
    cl = lambda v, a, b: max(a, min(b, v))
    lo0, hi0 = cl(bmin, 0, N + 1), cl(bmax, -1, N)
    lo1, hi1 = cl(smin + 1, 0, N + 1), cl(smax + 1, -1, N)
    M = 0x8000 if pair else 0x80000000
    nlo0 = ((M - lo0) * 0x10001 if pair else M - lo0) & M32
    hih0 = ((M + hi0) * 0x10001 if pair else M + hi0) & M32
    return nlo0, hih0, (lo0 - lo1) & M32, (hi1 - hi0) & M32


def scalar(B, s, rule):
    smin, smax, bmin, bmax = rule
    k = B - s
    return np.where(s == 1, (k >= smin) & (k <= smax), (k >= bmin) & (k <= bmax)).astype(np.uint32)


def pair_lanes(B0, B1, s0, s1, radius, rule, base):
    """Both rows' results as the kernel computes them, with the box counts formed
    as a difference of prefix sums offset by `base` (any 32-bit value)."""
    nlo0, hih0, dnlo, dhih = (np.uint64(v) for v in rule_constants(radius, rule, True))
    B0 = B0.astype(np.uint64); B1 = B1.astype(np.uint64)
    ps = np.uint64(base) & np.uint64(M32)
    pe = (ps + B0 + (B1 << np.uint64(16))) & np.uint64(M32)
    sw = s0.astype(np.uint64) | (s1.astype(np.uint64) << np.uint64(16))
    mask = np.uint64(M32)
    ge = (pe - ps + ((sw * dnlo + nlo0) & mask)) & mask
    le = (((sw * dhih + hih0) & mask) - pe + ps) & mask
    res = ge & le & np.uint64(0x80008000)
    return ((res >> np.uint64(15)) & np.uint64(1)).astype(np.uint32), ((res >> np.uint64(31)) & np.uint64(1)).astype(np.uint32)


def single_lane(B, s, radius, rule):
    nlo0, hih0, dnlo, dhih = (np.uint64(v) for v in rule_constants(radius, rule, False))
    mask = np.uint64(M32)
    B = B.astype(np.uint64); sw = s.astype(np.uint64)
    ge = (B + ((sw * dnlo + nlo0) & mask)) & mask
    le = (((sw * dhih + hih0) & mask) - B) & mask
    return ((ge & le) >> np.uint64(31)).astype(np.uint32)


def rules_for(radius, rng):
    N = (2 * radius + 1) ** 2
    yield (int(np.ceil(0.33 * N)) - 1, int(0.57 * N) - 1, int(np.ceil(0.34 * N)), int(0.45 * N))
    yield (-5, N + 7, N // 3, N // 3)
    yield (N // 4, N // 5, -3, N)
    yield (0, N - 1, N, N + 5)
    for _ in range(4):
        a, b = sorted(int(x) for x in rng.integers(-2, N + 3, 2))
        c, d = sorted(int(x) for x in rng.integers(-2, N + 3, 2))
        yield (a, b, c, d)


@pytest.mark.parametrize("radius", [6, 13, 32, 64, 89, 90])
def test_pair_lanes_exact_for_every_count(radius):
    rng = np.random.default_rng(radius)
    N = (2 * radius + 1) ** 2
    B = np.arange(N + 1, dtype=np.int64)
    other = rng.integers(0, N + 1, B.size)          # the other row's count
    for rule in rules_for(radius, rng):
        for s0 in (0, 1):
            for s1 in (0, 1):
                base = int(rng.integers(0, 1 << 32))
                S0 = np.full(B.size, s0); S1 = np.full(B.size, s1)
                B0 = np.maximum(B, s0); B1 = np.maximum(other, s1)   # a live centre counts itself
                lo, hi = pair_lanes(B0, B1, S0, S1, radius, rule, base)
                assert np.array_equal(lo, scalar(B0, S0, rule)), (radius, rule, s0, s1)
                assert np.array_equal(hi, scalar(B1, S1, rule)), (radius, rule, s0, s1)


def test_pair_lanes_not_exact_above_r90():
    """At R = 91 a box count reaches 183^2 = 33489 > 2^15 - 1: the 16-bit lane test
    fails for some counts, so the kernel switches to 32-bit lanes there."""
    radius = 91
    N = (2 * radius + 1) ** 2
    rule = (0, N, 0, N)                      # every count inside: all cells alive
    B = np.arange(N + 1)
    lo, _ = pair_lanes(B, B, np.zeros_like(B), np.zeros_like(B), radius, rule, 0)
    assert not np.array_equal(lo, scalar(B, np.zeros_like(B), rule))


@pytest.mark.parametrize("radius", [91, 128, 500, 2038])
def test_single_lane_exact(radius):
    rng = np.random.default_rng(radius)
    N = (2 * radius + 1) ** 2
    B = np.unique(np.concatenate([np.arange(0, min(N, 70000) + 1), rng.integers(0, N + 1, 200000), [N]]))
    for rule in rules_for(radius, rng):
        for s in (0, 1):
            S = np.full(B.size, s)
            Bs = np.maximum(B, s)
            assert np.array_equal(single_lane(Bs, S, radius, rule), scalar(Bs, S, rule)), (radius, rule, s)
