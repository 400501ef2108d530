"""The multi-rank host logic on CPU ranks (gloo, world size 2): bench.py's
max-over-ranks timing, the library's LPT placement of independent systems
(mdb_place_lpt: each system on exactly one rank, loads balanced, the same on
every rank), and per-rank replica seeds."""
import os
import socket

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

import bench
import md_simulation_cuda_b200 as mdb


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        # timing: every rank gets the slowest rank's time
        t = bench.max_over_ranks(0.5 + rank, dist, "cpu")
        # LPT shards of the 512-system FIRE mix sizes (deterministic on every rank)
        from md_simulation_cuda_b200 import workloads as wl

        sizes = [len(f) for f, _ in wl.fire_mix(512)]
        owner, _ = mdb.place_lpt(sizes, world)
        mine = [k for k, r in enumerate(owner) if r == rank]
        load = torch.tensor([float(sum(sizes[k] for k in mine))])
        loads = [torch.zeros(1) for _ in range(world)]
        dist.all_gather(loads, load)
        count = torch.tensor([len(mine)])
        dist.all_reduce(count)
        # replicas: same N, different seeds per rank
        f, _cfg, _mode, _desc = bench.make_workload("nve_4096", rank)
        first = torch.tensor(f["pos"][:4].reshape(-1))
        firsts = [torch.zeros_like(first) for _ in range(world)]
        dist.all_gather(firsts, first)
        out[rank] = (t, [float(x) for x in loads], int(count), max(sizes),
                     bool(torch.equal(firsts[0], firsts[1])), len(f))
    finally:
        dist.destroy_process_group()


def test_two_cpu_ranks():
    world = 2
    port = _free_port()
    with mp.Manager() as m:
        out = m.dict()
        mp.spawn(_worker, args=(world, port, out), nprocs=world, join=True)
        res = dict(out)
    for r in range(world):
        t, loads, count, biggest, same_start, n = res[r]
        assert t == 1.5                      # max over ranks
        assert count == 512                  # every system on exactly one rank...
        assert abs(loads[0] - loads[1]) <= biggest  # ...and LPT balance within one system
        assert not same_start and n == 4096  # replica seeds differ per rank


def _lpt_reference(costs, nbins):
    """Greedy LPT in Python: largest first (stable), least-loaded bin, ties low."""
    order = sorted(range(len(costs)), key=lambda k: (-costs[k], k))
    load = [0.0] * nbins
    out = [0] * len(costs)
    for k in order:
        b = min(range(nbins), key=lambda d: (load[d], d))
        out[k] = b
        load[b] += costs[k]
    return out, load


def test_lpt_is_a_partition():
    costs = [5, 3, 3, 2, 2, 2, 1, 9]
    owner, load = mdb.place_lpt(costs, 3)
    assert sorted(set(owner.tolist())) == [0, 1, 2]
    loads = [sum(c for c, o in zip(costs, owner) if o == b) for b in range(3)]
    assert loads == load.tolist()
    assert sum(loads) == sum(costs) and max(loads) - min(loads) <= max(costs)


def test_lpt_matches_the_rule_on_the_fire_mix():
    from md_simulation_cuda_b200 import workloads as wl

    costs = [len(f) * 20000.0 for f, _ in wl.fire_mix(512)]
    for nb in (1, 2, 3, 8):
        owner, load = mdb.place_lpt(costs, nb)
        ref_owner, ref_load = _lpt_reference(costs, nb)
        assert owner.tolist() == ref_owner and load.tolist() == ref_load
        assert max(load) <= sum(costs) / nb + max(costs)
