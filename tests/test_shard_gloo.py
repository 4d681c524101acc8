"""Multi-rank host logic of batch sharding, on CPU with the gloo backend
(world_size 2): disjoint, complete, balanced shards and a gather of per-grid
digests that matches a single-process run.  The per-grid work here is the CPU
oracle; on GPUs each rank would run the same shard through libltl_b200."""
import os
import socket

import pytest


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, q):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        from cat_cpu_b200.shard import partition, digest, gather_digests
        from cat_cpu_b200.workloads import batch_config
        from oracle import oracle as O
        cfg = [(max(16, n // 16), r, rule, d, s) for (n, r, rule, d, s) in batch_config(24, seed=9)]
        parts = partition([n * n for (n, *_rest) in cfg], world)
        local = {}
        for k in parts[rank]:
            n, r, rule, d, s = cfg[k]
            import numpy as np
            import ctypes
            g = np.empty((n, n), dtype=np.uint8)
            O.lib().oracle_generate_from_state_seed(g.ctypes.data_as(ctypes.POINTER(ctypes.c_uint8)), n, s,
                                                    ctypes.c_float(d), 1)
            local[k] = digest(O.run(g, r, rule, 5))
        merged = gather_digests(local)
        q.put((rank, parts, merged))
    finally:
        dist.destroy_process_group()


def test_partition_properties():
    from cat_cpu_b200.shard import partition
    from cat_cpu_b200.workloads import batch_config
    cells = [n * n for (n, *_r) in batch_config()]
    for world in (1, 2, 4, 8):
        parts = partition(cells, world)
        flat = sorted(i for p in parts for i in p)
        assert flat == list(range(len(cells)))
        loads = [sum(cells[i] for i in p) for p in parts]
        assert max(loads) - min(loads) <= max(cells)


def test_two_rank_gloo_gather():
    import multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    results = [q.get(timeout=240) for _ in range(2)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    (r0, parts0, m0), (r1, parts1, m1) = sorted(results, key=lambda x: x[0])
    assert parts0 == parts1
    assert m0 == m1 and len(m0) == 24
    # single-process reference of the same digests
    import ctypes
    import numpy as np
    from cat_cpu_b200.shard import digest
    from cat_cpu_b200.workloads import batch_config
    from oracle import oracle as O
    cfg = [(max(16, n // 16), r, rule, d, s) for (n, r, rule, d, s) in batch_config(24, seed=9)]
    for k, (n, r, rule, d, s) in enumerate(cfg):
        g = np.empty((n, n), dtype=np.uint8)
        O.lib().oracle_generate_from_state_seed(g.ctypes.data_as(ctypes.POINTER(ctypes.c_uint8)), n, s,
                                                ctypes.c_float(d), 1)
        assert m0[k] == digest(O.run(g, r, rule, 5)), k
