"""Ensemble host logic: seeded member specs, greedy sharding over ranks, and the
two-rank (gloo, CPU) path that shards members with no data-path collective."""
import os
import socket

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
