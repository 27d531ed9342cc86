"""CPU tests of the data-parallel layout: shard ranges, chunk assignment, and the
all-gather of per-particle results with two gloo ranks (the path NCCL takes on GPUs)."""
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp


def test_shard_ranges_cover_exactly(pkg):
    from simple3_0_b200 import shard
    for n in (0, 1, 7, 20000):
        for world in (1, 2, 3, 8):
            spans = [shard.shard_range(n, r, world) for r in range(world)]
            assert spans[0][0] == 0 and spans[-1][1] == n
            assert all(a[1] == b[0] for a, b in zip(spans, spans[1:]))
            sizes = [hi - lo for lo, hi in spans]
            assert max(sizes) - min(sizes) <= 1
    with pytest.raises(ValueError):
        shard.shard_range(10, 2, 2)


def test_chunk_assignment_balances(pkg):
    from simple3_0_b200 import shard
    rng = np.random.default_rng(0)
    costs = [shard.chunk_cost(rng.integers(500, 5001), rng.integers(50, 301), 1, n, k)
             for n, k in [(128, 19), (360, 39), (600, 59)] * 21 + [(128, 19)]]
    for world in (2, 4, 8):
        a = shard.assign_chunks(costs, world)
        assert sorted(i for lst in a for i in lst) == list(range(len(costs)))
        loads = [sum(costs[i] for i in lst) for lst in a]
        assert max(loads) <= sum(loads) / world + max(costs)


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, n, root, q):
    import sys
    sys.path.insert(0, root)
    import __graft_entry__ as entry
    shard = entry.load_package().shard
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=__import__("datetime").timedelta(seconds=60))
    lo, hi = shard.shard_range(n, rank, world)
    idx = np.arange(lo, hi)
    rec = shard.as_records(idx % 7 + 1, idx % 360 + 1, idx % 81, idx * 0.001)
    full = shard.gather_results(torch.from_numpy(rec), n, world)
    if rank == 0:
        q.put(full.numpy().copy())
    dist.barrier()
    dist.destroy_process_group()


def test_gather_two_ranks_gloo(pkg):
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    n, world = 1001, 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, n, root, q)) for r in range(world)]
    for p in procs:
        p.start()
    full = q.get(timeout=120)
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    idx = np.arange(n)
    from simple3_0_b200 import shard
    assert np.array_equal(full, shard.as_records(idx % 7 + 1, idx % 360 + 1, idx % 81, idx * 0.001))
