"""One grid split into row strips (cat_cpu_b200/strips.py), on the CPU: the
partition, the halo exchange schedule and the torus neighbours, with a numpy
stepper per strip, in one process and across 2 and 3 gloo ranks."""
import os

import numpy as np
import pytest
import torch
import torch.multiprocessing as mp

from cat_cpu_b200 import strips as S
from oracle import oracle as O
from tests.stripsutil import NumpyStepper, step_rect


def test_numpy_rect_stepper_matches_oracle_on_squares():
    rng = np.random.default_rng(5)
    for n, r in ((40, 2), (33, 5)):
        rule = O.sweep_rule(r) if r <= 16 else O.scaled_rule(r)
        g = (rng.random((n, n)) < 0.45).astype(np.uint8)
        assert np.array_equal(step_rect(g, r, rule), O.step(g, r, rule))


def test_partition_covers_rows():
    for n, p in ((10, 3), (64, 4), (7, 7)):
        b = S.partition(n, p)
        assert b[0][0] == 0 and b[-1][1] == n and all(b[i][1] == b[i + 1][0] for i in range(p - 1))


@pytest.mark.parametrize("overlap", [True, False])
@pytest.mark.parametrize("parts,k,gens", [(1, 2, 5), (2, 3, 7), (3, 2, 9), (4, 1, 3)])
def test_local_strips_match_full_grid(parts, k, gens, overlap):
    n, r = 48, 2
    rule = O.sweep_rule(r)
    g = (np.random.default_rng(parts * 10 + k).random((n, n)) < 0.45).astype(np.uint8)
    ls = S.LocalStrips(n, r, parts, k, lambda rows, nn: NumpyStepper(rows, nn, r, rule), overlap=overlap)
    ls.set_state(g)
    ls.step(gens)
    assert np.array_equal(ls.get_state().numpy(), O.run(g, r, rule, gens))


def test_strip_thinner_than_halo_is_refused():
    with pytest.raises(ValueError, match="thinner than its halo"):
        S.LocalStrips(20, 3, 4, 2, lambda rows, n: NumpyStepper(rows, n, 3, (1, 2, 3, 4)))


def _dist_worker(rank, world, port, n, r, rule, k, gens, seed, overlap):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        g = (np.random.default_rng(seed).random((n, n)) < 0.45).astype(np.uint8)
        ds = S.DistStrips(n, r, k, lambda rows, nn: NumpyStepper(rows, nn, r, rule), "cpu", overlap=overlap)
        ds.set_state(g)
        ds.step(gens)
        got = ds.get_state().numpy()
        want = O.run(g, r, rule, gens)
        assert np.array_equal(got, want), f"rank {rank}: {int((got != want).sum())} cells differ"
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("overlap", [True, False])
@pytest.mark.parametrize("world,k,gens", [(2, 3, 8), (3, 2, 7)])
def test_dist_strips_gloo(world, k, gens, overlap):
    port = 29500 + 17 * world + k + (100 if overlap else 0)
    n, r = 45, 2
    mp.spawn(_dist_worker, args=(world, port, n, r, O.sweep_rule(r), k, gens, 11, overlap), nprocs=world,
             join=True)
