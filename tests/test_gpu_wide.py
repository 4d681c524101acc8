"""The plain variant's fused prefix-sum kernel (k_plain_wide, every R > 5)
against a numpy torus stepper, bit for bit.

It has two forms: row pairs in 16-bit lanes for R <= 90, and one row per 32-bit
lane above that, with 8 window columns per thread up to R = 1018 and 16 beyond.
The cases cover:
  - every R mod 4, which fixes the alignment of the prefix reads;
  - both sides of R = 90;
  - grids narrower and wider than one CTA tile;
  - rectangular (rows != n) and odd row counts, so a row pair can end a band;
  - explicit band heights (even, odd, and longer than the grid);
  - rules with thresholds below 0, above N = (2R+1)^2, and empty intervals.
Marked gpu."""
import numpy as np
import pytest

from oracle import oracle as O
from tests.stripsutil import step_rect

pytestmark = pytest.mark.gpu


def rules_for(radius, rng):
    N = (2 * radius + 1) ** 2
    yield O.scaled_rule(radius)
    a = int(rng.integers(0, N // 2))
    yield (a, a + int(rng.integers(0, N // 2)), int(rng.integers(0, N // 2)), int(rng.integers(N // 3, N)))
    yield (-5, N + 7, N // 3, N // 3)          # survival always; one birth count
    yield (N // 4, N // 5, -3, N // 2)         # empty survival interval
    yield (0, N - 1, N, N + 5)                 # birth only with a full box (never: k <= N - 1)


CASES = [  # rows, n, radius
    (70, 70, 6), (97, 97, 7), (130, 61, 9), (64, 200, 10), (200, 203, 31), (260, 190, 64),
    (181, 181, 89), (190, 181, 90), (200, 200, 91), (133, 300, 94), (260, 260, 127), (300, 257, 128),
    (41, 4200, 6), (101, 4100, 100), (45, 2030, 7),
]


@pytest.mark.parametrize("rows,n,radius", CASES)
def test_wide_kernel_vs_numpy(rows, n, radius):
    import cat_cpu_b200 as C
    rng = np.random.default_rng(rows * 7 + n * 3 + radius)
    for i, rule in enumerate(rules_for(radius, rng)):
        g = (rng.random((rows, n)) < rng.uniform(0.25, 0.65)).astype(np.uint8)
        kw = {} if rows == n else {"rows": rows}
        s = C.CUDASolver(n, radius, rule, variant=C.VARIANT_PLAIN, **kw)
        try:
            band = (0, 16, 17, 30, 4096)[i % 5]
            if band:
                s.set_param("band_rows", band)
            s.setState(g)
            want = g
            for step in range(3):
                s.doStep()
                want = step_rect(want, radius, rule)
                got = s.getCurrentState()
                assert np.array_equal(got, want), \
                    f"rows={rows} n={n} R={radius} rule={rule} band={band} step {step + 1}: " \
                    f"{int((got != want).sum())} cells differ"
        finally:
            s.close()


def test_wide_kernel_16_columns_per_thread():
    """R = 1030 (> 1018): 16 window columns per thread."""
    import cat_cpu_b200 as C
    rows, n, radius = 1031, 1040, 1030
    rng = np.random.default_rng(3)
    g = (rng.random((rows, n)) < 0.5).astype(np.uint8)
    rule = O.scaled_rule(radius)
    s = C.CUDASolver(n, radius, rule, variant=C.VARIANT_PLAIN, rows=rows)
    try:
        s.setState(g)
        want = g
        for step in range(2):
            s.doStep()
            want = step_rect(want, radius, rule)
            assert np.array_equal(s.getCurrentState(), want), f"step {step + 1}"
    finally:
        s.close()


def test_wide_kernel_radius_limit():
    import cat_cpu_b200 as C
    with pytest.raises(C.LtlError):
        C.CUDASolver(2100, 2039, (0, 1, 2, 3), variant=C.VARIANT_PLAIN, rows=2100)
