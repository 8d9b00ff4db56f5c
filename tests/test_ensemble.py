"""Ensemble host logic: seeded member specs, greedy sharding over ranks, and the
two-rank (gloo, CPU) path that shards members with no data-path collective."""
import os
import socket
import time

import numpy as np
import pytest

from fdd3260_b200 import ensemble as E


def test_specs_are_seeded_and_within_the_configured_sets():
    a, b = E.ensemble_specs(64, seed=3000), E.ensemble_specs(64, seed=3000)
    assert [(s.nxy, s.nz, s.seed, s.amp) for s in a] == [(s.nxy, s.nz, s.seed, s.amp) for s in b]
    assert all(s.nxy in E.NX_CHOICES and s.nz in E.NZ_CHOICES and 1.0 <= s.amp <= 3.0 for s in a)
    assert all(s.centre[2] <= s.nz * 40.0 / 3.0 + 1e-9 for s in a)
    assert len({s.nxy for s in a}) > 2 and len({s.nz for s in a}) > 1


@pytest.mark.parametrize("nranks", [1, 2, 3, 4, 8])
def test_partition_covers_every_member_once_and_balances_cells(nranks):
    specs = E.ensemble_specs(64, seed=3000)
    cells = [s.cells for s in specs]
    parts = E.partition(cells, nranks)
    flat = sorted(i for p in parts for i in p)
    assert flat == list(range(64))
    loads = [sum(cells[i] for i in p) for p in parts]
    # greedy largest-first: the imbalance is at most the largest member
    assert max(loads) - min(loads) <= max(cells)
    assert E.partition(cells, nranks) == parts


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank_main(rank, world, port, q):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    specs = E.ensemble_specs(64, seed=3000)
    mine = E.partition([s.cells for s in specs], world)[rank]
    got = [None] * world
    dist.all_gather_object(got, mine)   # host-side gather of the assignment (metrics path only)
    dist.destroy_process_group()
    q.put((rank, mine, got))


def test_two_rank_sharding_over_gloo():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
    assert all(p.exitcode == 0 for p in procs)
    res.sort()
    (r0, m0, g0), (r1, m1, g1) = res
    assert g0 == g1 == [m0, m1]
    assert set(m0).isdisjoint(m1) and sorted(m0 + m1) == list(range(64))


# ---- the sharded run with work: each of two gloo ranks steps its own members ----
SMALL = dict(nx_choices=(16, 24, 32), nz_choices=(8, 12))


class _OracleShard:
    """CPU stand-in for a rank's Ensemble, with its interface (step, time_steps): every
    member of the rank is stepped by the oracle (the CPU restatement of the reference)."""

    def __init__(self, specs):
        from oracle import oracle as O
        self.items = []
        for sp in specs:
            d, st = E.member_problem(sp, init=O.Init())
            self.items.append([sp.index, O.Oracle(d), st])

    def step(self, n, ntime0=1):
        for it in self.items:
            if n > 0:
                it[2], _, _ = it[1].stepping(it[2], nsteps=n, ntime0=ntime0)

    def time_steps(self, n, ntime0=1):
        t0 = time.perf_counter()
        self.step(n, ntime0)
        return (time.perf_counter() - t0) * 1e3


def _work_rank(rank, world, port, q):
    import torch
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)

    def rmax(x):
        t = torch.tensor([float(x)], dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    def rsum(x):
        t = torch.tensor([float(x)], dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.SUM)
        return float(t.item())

    specs = E.ensemble_specs(6, seed=4000, **SMALL)
    sh = E.shard_and_time(specs, rank, world, _OracleShard, warmup=3, steps=2, barrier=dist.barrier,
                          reduce_max=rmax, reduce_sum=rsum)
    finals = {it[0]: (it[2].u, it[2].w, it[2].scal[0]) for it in sh["stepper"].items}
    dist.destroy_process_group()
    q.put((rank, {k: sh[k] for k in ("t_ms", "rank_ms", "cells", "members", "value")}, finals))


def test_two_ranks_step_their_members_and_gather_only_metrics():
    """The path bench.py's ensemble workload takes (ensemble.shard_and_time), with the
    oracle as each rank's stepper: the ranks' members are disjoint and cover the ensemble,
    the gathered time is the max over ranks and the cells the sum, and every member ends
    bit for bit where it ends when stepped alone: nothing couples the ranks' data."""
    import torch.multiprocessing as mp
    from oracle import oracle as O
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_work_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted([q.get(timeout=300) for _ in procs], key=lambda x: x[0])
    for p in procs:
        p.join(timeout=60)
    assert all(p.exitcode == 0 for p in procs)
    (_, m0, f0), (_, m1, f1) = res
    specs = E.ensemble_specs(6, seed=4000, **SMALL)
    assert set(m0["members"]).isdisjoint(m1["members"])
    assert sorted(m0["members"] + m1["members"]) == list(range(6))
    assert m0["t_ms"] == m1["t_ms"] == max(m0["rank_ms"], m1["rank_ms"])
    assert m0["cells"] == m1["cells"] == sum(s.cells for s in specs)
    assert m0["value"] == m0["cells"] * 2 / (m0["t_ms"] / 1e3) / 1e6
    finals = {**f0, **f1}
    for sp in specs:
        d, st = E.member_problem(sp, init=O.Init())
        alone, _, _ = O.Oracle(d).stepping(st, nsteps=5, ntime0=1)
        u, w, th = finals[sp.index]
        assert np.array_equal(u, alone.u) and np.array_equal(w, alone.w) and np.array_equal(th, alone.scal[0])
