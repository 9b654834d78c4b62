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
