"""Full-size radius sweeps (32768^2) checked at sampled steps.

Solver 0 cannot run these sizes, so exactness is shown by size-independent
properties: the CPU oracle advances the GPU's own state one generation and must
land on the GPU's next state, and every variant that supports the radius ends
on the same grid.  Marked gpu (and slow: a few minutes on one B200).
"""
import hashlib
import os

import numpy as np
import pytest

from oracle import oracle as O

pytestmark = [pytest.mark.gpu, pytest.mark.slow]

N = 32768


def setup_module(module):
    O.set_threads(os.cpu_count() or 8)


def sha(g):
    return hashlib.sha256(np.ascontiguousarray(g).tobytes()).hexdigest()


def run_variant(C, variant, start, radius, rule, steps):
    s = C.CUDASolver(N, radius, rule, variant=variant)
    try:
        s.setState(start)
        s.doSteps(steps - 1)
        before = s.getCurrentState()
        s.doSteps(1)
        after = s.getCurrentState()
        return before, after
    finally:
        s.close()


@pytest.mark.parametrize("radius", [1, 2, 4, 8, 16, 32])
def test_radius_sweep_32768_200_steps(radius):
    """Seed 2, d = 0.5, scaled interval rule, 200 steps (the radius-sweep workload)."""
    import cat_cpu_b200 as C
    rule = O.scaled_rule(radius)
    start = C.start_grid(N, 2, 0.5, 1)
    variants = [C.VARIANT_PACKED, C.VARIANT_TENSOR, C.VARIANT_PLAIN]
    finals = {}
    for v in variants:
        before, after = run_variant(C, v, start, radius, rule, 200)
        if v == variants[0]:
            assert np.array_equal(O.step(before, radius, rule), after), f"R={radius}: step 200 differs from oracle"
        finals[v] = sha(after)
    assert len(set(finals.values())) == 1, f"R={radius}: variants disagree {finals}"


@pytest.mark.parametrize("radius", [64, 128])
def test_large_radius_32768(radius):
    """Seed 3, d = 0.3 (dies at step 1 under the scaled rule) and d = 0.448 (stays
    mixed for two steps): every step checked against the oracle."""
    import cat_cpu_b200 as C
    rule = O.scaled_rule(radius)
    for seed, d, steps in ((3, 0.3, 2), (3, 0.448, 2)):
        start = C.start_grid(N, seed, d, 1)
        s = C.CUDASolver(N, radius, rule, variant=C.VARIANT_PLAIN)
        try:
            s.setState(start)
            g = start
            for k in range(steps):
                s.doStep()
                want = O.step(g, radius, rule)
                got = s.getCurrentState()
                assert np.array_equal(got, want), f"R={radius} d={d} step {k + 1}"
                g = want
            if d == 0.448:
                assert 0 < int(g.sum()) < N * N or k == 0
        finally:
            s.close()
