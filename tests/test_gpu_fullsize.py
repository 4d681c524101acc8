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
    """Generation 1, generation steps-1 and generation steps of one variant."""
    s = C.CUDASolver(N, radius, rule, variant=variant)
    try:
        s.setState(start)
        s.doSteps(1)
        first = s.getCurrentState()
        s.doSteps(steps - 2)
        before = s.getCurrentState()
        s.doSteps(1)
        after = s.getCurrentState()
        return first, before, after
    finally:
        s.close()


@pytest.mark.parametrize("radius", [1, 2, 4, 8, 16, 32])
def test_radius_sweep_32768_200_steps(radius):
    """Seed 2, d = 0.5, scaled interval rule, 200 steps (the radius-sweep workload).
    Every variant's generation 1 and its step 199 -> 200 are checked against the
    oracle on their own, and all variants must end on the same grid."""
    import cat_cpu_b200 as C
    rule = O.scaled_rule(radius)
    start = C.start_grid(N, 2, 0.5, 1)
    want1 = O.step(start, radius, rule)
    finals = {}
    for v in (C.VARIANT_PACKED, C.VARIANT_TENSOR, C.VARIANT_PLAIN):
        first, before, after = run_variant(C, v, start, radius, rule, 200)
        name = C.VARIANT_NAMES[v]
        assert np.array_equal(first, want1), f"R={radius} {name}: generation 1 differs from the oracle"
        assert np.array_equal(O.step(before, radius, rule), after), f"R={radius} {name}: step 200 differs"
        finals[name] = sha(after)
    assert len(set(finals.values())) == 1, f"R={radius}: variants disagree {finals}"


@pytest.mark.parametrize("radius", [64, 128])
def test_large_radius_32768(radius):
    """Seed 3, d = 0.3 (dies at step 1 under the scaled rule) and d = 0.448 (stays
    mixed for two steps): every step of every variant that takes the radius
    checked against the oracle."""
    import cat_cpu_b200 as C
    rule = O.scaled_rule(radius)
    variants = [C.VARIANT_PLAIN] + ([C.VARIANT_TENSOR] if radius <= 128 else [])
    for seed, d, steps in ((3, 0.3, 2), (3, 0.448, 2)):
        start = C.start_grid(N, seed, d, 1)
        wants = []
        g = start
        for k in range(steps):
            g = O.step(g, radius, rule)
            wants.append(g)
        if d == 0.448:
            assert 0 < int(wants[-1].sum()) < N * N
        for v in variants:
            s = C.CUDASolver(N, radius, rule, variant=v)
            try:
                s.setState(start)
                for k in range(steps):
                    s.doStep()
                    got = s.getCurrentState()
                    assert np.array_equal(got, wants[k]), f"R={radius} d={d} {C.VARIANT_NAMES[v]} step {k + 1}"
            finally:
                s.close()
