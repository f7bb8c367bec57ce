"""The multi-rank ensemble path on CPU: member sharding, and gloo runs of 2
and 3 ranks whose ranks each advance their shard (with the CPU oracle) and
gather only diagnostics (chimera_b200.shard.gather_diagnostics)."""
import os
import socket

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


class OracleBatch:
    """Members advanced by the CPU oracle, answering ``diag(member=k)`` with
    the fields a sharded ensemble gathers (t, steps, mass and energy totals;
    the others zero), in the role of ``gpu.Solver``."""

    def __init__(self, oracle, sizes, members):
        from chimera_b200 import problems
        self.oracle = oracle
        self.members = []
        for m in members:
            cfg, st = problems.grf_member(sizes[m], 500 + m)
            self.members.append((cfg, oracle.State(st), [0]))

    def step(self, n):
        for cfg, s, count in self.members:
            count[0] += len(self.oracle.run(cfg, s, n))

    def diag(self, member=0):
        from chimera_b200.shard import DIAG_FIELDS
        _, s, count = self.members[member]
        d = dict.fromkeys(DIAG_FIELDS, 0.0)
        d.update(t=s.t, steps=count[0], mass=float(s.a[0].sum()), energy=float(s.a[3].sum()))
        return d


def _worker(rank, world, port, sizes, nsteps, out):
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    from chimera_b200.shard import gather_diagnostics
    from oracle import oracle
    mine = shard_members([n * n for n in sizes], world, rank)
    batch = OracleBatch(oracle, sizes, mine)      # members are independent: no exchange
    batch.step(nsteps)
    out.put((rank, gather_diagnostics(batch, mine, len(sizes))))   # diagnostics only
    dist.barrier()
    dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_gloo_ranks_gather_every_members_diagnostics(oracle, world):
    """Each rank advances its shard; after the one all-reduce every rank holds
    every member's diagnostics, equal to a single process's."""
    sizes = [16, 24, 16, 32, 20]
    nsteps = 3
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, sizes, nsteps, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = dict(q.get(timeout=120) for _ in range(world))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    one = OracleBatch(oracle, sizes, range(len(sizes)))
    one.step(nsteps)
    ref = [one.diag(member=m) for m in range(len(sizes))]
    for r in range(world):
        assert len(res[r]) == len(sizes)
        for m in range(len(sizes)):
            for f in ("t", "steps", "mass", "energy", "status"):
                assert res[r][m][f] == ref[m][f], (r, m, f)
            assert res[r][m]["steps"] == nsteps


def test_gather_without_a_process_group_is_local():
    from chimera_b200.shard import gather_member_rows
    t = gather_member_rows({1: [1.0, 2.0], 3: [3.0, 4.0]}, 4, 2)
    assert t.tolist() == [[0.0, 0.0], [1.0, 2.0], [0.0, 0.0], [3.0, 4.0]]
    with pytest.raises(ValueError):
        gather_member_rows({4: [0.0, 0.0]}, 4, 2)


def _leaving_worker(rank, world, port, sizes, out):
    import datetime

    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=10))
    from chimera_b200.shard import gather_diagnostics
    from oracle import oracle
    mine = shard_members([n * n for n in sizes], world, rank)
    batch = OracleBatch(oracle, sizes, mine)
    batch.step(2)
    if rank == 1:                    # leaves after its steps, before the gather
        out.put((rank, "left"))
        out.close()
        out.join_thread()
        os._exit(3)
    try:
        gather_diagnostics(batch, mine, len(sizes))
        out.put((rank, "gathered"))
    except Exception:   # the failure this test expects
        out.put((rank, "error"))
    out.close()
    out.join_thread()
    os._exit(4)


def test_a_rank_that_leaves_ends_the_gather_with_an_error():
    """Failure detection on the host: when a rank of a sharded ensemble exits
    before the diagnostics gather, the other rank's gather ends with an error
    within the process group's timeout instead of waiting for good."""
    sizes = [16, 24, 16, 20]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_leaving_worker, args=(r, 2, port, sizes, q)) for r in range(2)]
    for p in procs:
        p.start()
    try:
        res = dict(q.get(timeout=120) for _ in range(2))
    finally:
        for p in procs:
            p.join(timeout=60)
            if p.is_alive():
                p.kill()
    assert res == {0: "error", 1: "left"}
