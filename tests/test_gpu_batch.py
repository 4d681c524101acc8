"""Batched grids (ltl_batch_*): every grid bit-exact against the CPU oracle.

Marked `gpu`.  The full 4096-grid workload is checked two ways: for every grid
the oracle advances the GPU's state at step 255 one generation and must land on
the GPU's step 256; for a stratified sample (all grids of side <= 96, the 8
largest, 64 random others) the oracle runs the whole 256-step trajectory from
the start grid.
"""
import concurrent.futures as cf
import os

import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu


def setup_module(module):
    O.set_threads(os.cpu_count() or 8)


def start_grids(C, cfg):
    def one(c):
        n, r, rule, d, seed = c
        return C.generate_state(n, seed, d, 1)
    with cf.ThreadPoolExecutor(os.cpu_count() or 8) as ex:
        return list(ex.map(one, cfg))


def flat(grids):
    return np.concatenate([g.ravel() for g in grids])


def split(b, flat_cells):
    return [flat_cells[b.offsets[k]:b.offsets[k + 1]].reshape(b.sizes[k], b.sizes[k]) for k in range(len(b.sizes))]


def small_config(count, nmax, seed=7):
    from cat_cpu_b200.workloads import batch_config
    cfg = []
    for (n, r, rule, d, s) in batch_config(count * 3, seed=seed):
        n = 64 + (n - 64) * (nmax - 64) // (2048 - 64)
        cfg.append((max(n, r), r, rule, d, s))
        if len(cfg) == count:
            break
    return cfg


@pytest.mark.parametrize("flags", [0, 1])
def test_small_batch_every_step_vs_oracle(flags):
    import cat_cpu_b200 as C
    cfg = small_config(40, 600) + [(17, 8, O.scaled_rule(8), 0.45, 11), (5, 3, (1, 20, 5, 18), 0.5, 12),
                                    (97, 5, O.BOSCO_R5, 0.5, 13), (64, 1, O.CONWAY, 0.3, 14)]
    b = C.Batch([(n, r, rule) for (n, r, rule, d, s) in cfg], flags=flags)
    grids = start_grids(C, cfg)
    b.upload_all(flat(grids))
    done = 0
    for target in (1, 2, 7, 20):
        b.step(target - done)
        got = split(b, b.download_all())
        for k, (n, r, rule, d, s) in enumerate(cfg):
            grids[k] = O.run(grids[k], r, rule, target - done)
            assert np.array_equal(got[k], grids[k]), f"grid {k} n={n} r={r} step {target} flags={flags}"
        done = target


def test_batch_modes_and_switches_vs_oracle():
    """The persistent launch (default), per-generation launches with grids kept in
    shared memory, and per-generation launches only, each against the oracle;
    the mode changes between calls on the same batch (the halos a mode leaves
    must serve the next).  Includes narrow grids (one to a few words per row, so
    that warps split into segments) and radii up to 16."""
    import cat_cpu_b200 as C
    cfg = [(40, 2, O.scaled_rule(2), 0.45, 21), (64, 8, O.scaled_rule(8), 0.45, 22), (100, 3, O.sweep_rule(3), 0.5, 23),
           (33, 1, O.CONWAY, 0.35, 24), (257, 5, O.BOSCO_R5, 0.5, 25), (700, 16, O.scaled_rule(16), 0.45, 26),
           (1100, 4, O.scaled_rule(4), 0.45, 27), (16, 12, O.scaled_rule(12), 0.45, 28), (130, 7, O.scaled_rule(7), 0.45, 29)]
    b = C.Batch([(n, r, rule) for (n, r, rule, d, s) in cfg])
    assert b.info()[2] == len(cfg)  # persistent: every grid runs each call in one launch
    grids = start_grids(C, cfg)
    b.upload_all(flat(grids))
    plan = [({}, 3), ({"persistent": 0}, 2), ({"resident_max_bytes": 0}, 3), ({"persistent": 1}, 4),
            ({"persistent": 0, "resident_max_bytes": 225280}, 1), ({"persistent": 1}, 5)]
    for params, steps in plan:
        for k, v in params.items():
            b.set_param(k, v)
        b.step(steps)
        got = split(b, b.download_all())
        for k, (n, r, rule, d, s) in enumerate(cfg):
            grids[k] = O.run(grids[k], r, rule, steps)
            assert np.array_equal(got[k], grids[k]), f"grid {k} n={n} r={r} after {params} + {steps} steps"


def test_single_grid_upload_download():
    import cat_cpu_b200 as C
    cfg = [(300, 5, O.BOSCO_R5, 0.5, 1), (1200, 3, O.scaled_rule(3), 0.4, 2), (64, 8, O.scaled_rule(8), 0.45, 3)]
    b = C.Batch([(n, r, rule) for (n, r, rule, d, s) in cfg])
    grids = start_grids(C, cfg)
    for k, g in enumerate(grids):
        b.upload(k, g)
    b.step(5)
    for k, (n, r, rule, d, s) in enumerate(cfg):
        assert np.array_equal(b.download(k), O.run(grids[k], r, rule, 5)), k


def test_full_batched_workload_sampled():
    """4096 grids, sides log-uniform in [64, 2048], R in 1..8, 256 steps."""
    import cat_cpu_b200 as C
    from cat_cpu_b200.workloads import batch_config
    cfg = batch_config()
    b = C.Batch([(n, r, rule) for (n, r, rule, d, s) in cfg])
    grids = start_grids(C, cfg)
    b.upload_all(flat(grids))
    b.step(255)
    s255 = split(b, b.download_all())
    b.step(1)
    s256 = split(b, b.download_all())

    def check(k):
        n, r, rule, d, s = cfg[k]
        return np.array_equal(O.step(s255[k], r, rule), s256[k])
    with cf.ThreadPoolExecutor(4) as ex:
        ok = list(ex.map(check, range(len(cfg))))
    bad = [k for k, v in enumerate(ok) if not v]
    assert not bad, f"{len(bad)} grids differ at step 256, first {bad[:5]}"
    # whole 256-step trajectories for a stratified sample: every grid of side
    # <= 96, the 8 largest grids (sides near 2048) and 64 others drawn at random
    by_size = sorted(range(len(cfg)), key=lambda k: cfg[k][0])
    small = [k for k in by_size if cfg[k][0] <= 96]
    large = by_size[-8:]
    rest = [k for k in by_size if k not in set(small) | set(large)]
    mid = list(np.random.default_rng(2).choice(rest, size=min(64, len(rest)), replace=False))
    sample = small + large + [int(k) for k in mid]
    assert max(cfg[k][0] for k in sample) >= 1900
    for k in sample:
        n, r, rule, d, s = cfg[k]
        assert np.array_equal(O.run(grids[k], r, rule, 256), s256[k]), f"grid {k} n={n} r={r}: trajectory differs"


def test_batch_errors():
    import cat_cpu_b200 as C
    with pytest.raises(C.LtlError) as e:
        C.Batch([(64, 17, (1, 2, 3, 4))])
    assert e.value.code == C.ltl.EUNSUPPORTED
    with pytest.raises(C.LtlError) as e:
        C.Batch([(4, 5, (1, 2, 3, 4))])
    assert e.value.code == C.ltl.EINVAL
