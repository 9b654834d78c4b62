"""Multi-process plumbing of the sharded J/K build, on CPU ranks (gloo).

The GPU engine shards the quartets by bra pair and the ranks sum partial J/K
with one all-reduce (pyscf_b200.dist).  Without GPUs the partial results are
made by the oracle from a split of the density (J/K are linear in D), which
exercises the same reduce path: after reduce_jk every rank must hold the J/K
of the whole density, to the last bits of the sum.
"""
import os
import socket

import numpy
import pytest

from conftest import load_fixture


def _free_port():
    with socket.socket() as s:
        s.bind(('127.0.0.1', 0))
        return s.getsockname()[1]


def _worker(rank, world, port, q):
    import torch
    import torch.distributed as dist
    import oracle
    from pyscf_b200 import dist as b2dist
    os.environ['MASTER_ADDR'] = '127.0.0.1'
    os.environ['MASTER_PORT'] = str(port)
    dist.init_process_group('gloo', rank=rank, world_size=world)
    try:
        f = load_fixture('h2o_631g')
        dm = f['dm_rand']
        # this rank's part of the density: rows assigned round-robin
        part = numpy.zeros_like(dm)
        rows = numpy.arange(dm.shape[0]) % world == rank
        part[rows] = dm[rows]
        vj, vk, _ = oracle.get_jk(part, f['atm'], f['bas'], f['env'], hermi=0, screen=False)
        tj, tk = torch.from_numpy(vj.copy()), torch.from_numpy(vk.copy())
        b2dist.reduce_jk(tj, tk)
        rj, rk, _ = oracle.get_jk(dm, f['atm'], f['bas'], f['env'], hermi=0, screen=False)
        q.put((rank, float(abs(tj.numpy() - rj).max()), float(abs(tk.numpy() - rk).max())))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize('world', [2, 3])
def test_reduce_jk_gloo(world):
    import torch.multiprocessing as mp
    ctx = mp.get_context('spawn')
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    res = [q.get(timeout=10) for _ in range(world)]
    assert sorted(r for r, _, _ in res) == list(range(world))
    for _, ej, ek in res:
        assert ej < 1e-12 and ek < 1e-12


def test_shard_arguments_checked():
    """Shard indices outside [0, count) are rejected by the C ABI without a GPU."""
    from pyscf_b200 import lib
    l = lib.load()
    assert l.b200jk_set_shard(None, 0, 1) == lib.B200JK_EINVAL


def _batch_worker(rank, world, port, q):
    import torch
    import torch.distributed as dist
    from pyscf_b200 import dist as b2dist
    os.environ['MASTER_ADDR'] = '127.0.0.1'
    os.environ['MASTER_PORT'] = str(port)
    dist.init_process_group('gloo', rank=rank, world_size=world)
    try:
        from conftest import GOLDEN
        f = numpy.load(os.path.join(GOLDEN, 'batch_h2o_vdz512.npz'))
        nbas = numpy.diff(f['bas_off'])
        mine = b2dist.my_molecules(list(nbas))
        # every rank's list, gathered only to check the partition here
        n = torch.tensor([len(mine)])
        sizes = [torch.zeros(1, dtype=torch.int64) for _ in range(world)]
        dist.all_gather(sizes, n)
        width = int(max(s.item() for s in sizes))
        pad = torch.full((width,), -1, dtype=torch.int64)
        pad[:len(mine)] = torch.tensor(mine, dtype=torch.int64)
        lists = [torch.zeros(width, dtype=torch.int64) for _ in range(world)]
        dist.all_gather(lists, pad)
        q.put((rank, [[int(x) for x in l if x >= 0] for l in lists], [int(x) for x in nbas]))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize('world', [2, 4])
def test_batch_shards_whole_molecules_gloo(world):
    """The 512-molecule batch split over `world` ranks by whole molecules:
    every rank derives the same partition with no communication, the parts
    are disjoint and cover the batch, and the estimated work of the most
    loaded rank is within one molecule's of the mean."""
    import torch.multiprocessing as mp
    from pyscf_b200 import dist as b2dist
    ctx = mp.get_context('spawn')
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_batch_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    res = sorted(q.get(timeout=10) for _ in range(world))
    parts = res[0][1]
    assert all(r[1] == parts for r in res)
    flat = sorted(m for p in parts for m in p)
    nbas = res[0][2]
    assert flat == list(range(len(nbas)))
    cost = [b2dist.molecule_cost(n) for n in nbas]
    loads = [sum(cost[m] for m in p) for p in parts]
    assert max(loads) - sum(loads) / world <= max(cost)
