"""The multi-rank ensemble path on CPU: member sharding and a world-size-2
gloo run whose ranks each advance their shard (with the CPU oracle) and
reduce only diagnostics."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from chimera_b200.problems import grf_ensemble_sizes
from chimera_b200.shard import shard_loads, shard_members


@pytest.mark.parametrize("world", [1, 2, 3, 4, 8])
def test_every_member_once_and_balanced(world):
    sizes = [n * n for n in grf_ensemble_sizes(1)]
    seen = []
    for r in range(world):
        seen += shard_members(sizes, world, r)
    assert sorted(seen) == list(range(len(sizes)))
    loads = shard_loads(sizes, world)
    assert max(loads) - min(loads) <= max(sizes)
    assert sum(loads) == sum(sizes)


def test_shard_rejects_bad_rank():
    with pytest.raises(ValueError):
        shard_members([1, 2], 2, 2)


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, sizes, nsteps, out):
    import torch
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    from chimera_b200 import problems
    from oracle import oracle
    mine = shard_members([n * n for n in sizes], world, rank)
    mass = torch.zeros(len(sizes), dtype=torch.float64)
    for m in mine:
        cfg, st = problems.grf_member(sizes[m], 500 + m)
        s = oracle.State(st)
        oracle.run(cfg, s, nsteps)
        mass[m] = s.a[0].sum()
    dist.all_reduce(mass)          # diagnostics only
    if rank == 0:
        out.put(mass.numpy().tolist())
    dist.barrier()
    dist.destroy_process_group()


def test_two_gloo_ranks_match_one_process(oracle):
    sizes = [16, 24, 16, 32, 20]
    nsteps = 3
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, sizes, nsteps, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = q.get(timeout=120)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    from chimera_b200 import problems
    ref = []
    for m, n in enumerate(sizes):
        cfg, st = problems.grf_member(n, 500 + m)
        s = oracle.State(st)
        oracle.run(cfg, s, nsteps)
        ref.append(s.a[0].sum())
    assert np.array_equal(np.array(res), np.array(ref))
