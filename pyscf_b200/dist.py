"""Multi-GPU J/K: one process per GPU, quartets sharded by bra shell pair.

Every rank holds the whole molecule (plan tables and density are small next to
the quartet work) and evaluates the bra pairs ij = rank (mod world) of every
quartet class (b200jk_set_shard); J/K are linear in the quartets, so one
all-reduce (sum, float64) of the concatenated [J; K] gives every rank the full
result.  This replaces the reference's OpenMP split of the block loop in
CVHFnr_direct_drv (pyscf/lib/vhf/nr_direct.c:355-476) and its critical-section
merge of the per-thread JKArrays (nr_direct_dot.c:58-138).

The collective goes through torch.distributed (NCCL between GPUs, gloo for the
CPU tests); no kernel waits on another GPU.
"""


def reduce_jk(vj, vk, group=None):
    """Sum partial J/K over the ranks of `group` in one all-reduce; in place."""
    import torch
    import torch.distributed as dist
    parts = [t for t in (vj, vk) if t is not None]
    if not parts:
        return vj, vk
    flat = torch.cat([t.reshape(-1) for t in parts])
    dist.all_reduce(flat, op=dist.ReduceOp.SUM, group=group)
    off = 0
    for t in parts:
        n = t.numel()
        t.copy_(flat[off:off + n].view_as(t))
        off += n
    return vj, vk


def shard_plan(plan, group=None):
    """Point `plan` at this rank's shard of the quartets."""
    import torch.distributed as dist
    plan.set_shard(dist.get_rank(group), dist.get_world_size(group))
    return plan


def get_jk(plan, dm, hermi=1, with_j=True, with_k=True, precision=0, group=None):
    """Full J/K of a CUDA float64 density on every rank: this rank's shard of
    the quartets on its GPU, then one all-reduce of [J; K]."""
    shard_plan(plan, group)
    vj, vk = plan.get_jk_device(dm, hermi=hermi, with_j=with_j, with_k=with_k, precision=precision)
    return reduce_jk(vj, vk, group)


def grad_jk(plan, dm, with_j=True, with_k=True, direct_scf_tol=1e-14, group=None):
    """Sharded grad.rhf.get_jk: (vj, vk) (3, nao, nao) on every rank."""
    shard_plan(plan, group)
    vj, vk = plan.grad_jk_device(dm, with_j=with_j, with_k=with_k, direct_scf_tol=direct_scf_tol)
    return reduce_jk(vj, vk, group)


# ---------------------------------------------------------------------------
# Batches of molecules: whole molecules per GPU, no collective on the data path.

def molecule_cost(nbas):
    """Work estimate of one molecule's J/K build: its s8 shell quartets before
    screening, P(P+1)/2 with P = nbas(nbas+1)/2 shell pairs."""
    p = nbas * (nbas + 1) // 2
    return p * (p + 1) // 2


def shard_molecules(costs, world):
    """Partition of a batch over `world` GPUs: longest processing time first
    (each molecule, largest cost first, to the least loaded rank; ties to the
    lowest rank).  Returns one sorted index list per rank; deterministic, so
    every rank computes the same partition without communicating."""
    import heapq
    order = sorted(range(len(costs)), key=lambda m: (-costs[m], m))
    heap = [(0, r) for r in range(world)]
    heapq.heapify(heap)
    parts = [[] for _ in range(world)]
    for m in order:
        load, r = heapq.heappop(heap)
        parts[r].append(m)
        heapq.heappush(heap, (load + costs[m], r))
    return [sorted(p) for p in parts]


def my_molecules(nbas_list, group=None):
    """This rank's molecules of a batch (indices into nbas_list)."""
    import torch.distributed as dist
    rank, world = dist.get_rank(group), dist.get_world_size(group)
    return shard_molecules([molecule_cost(n) for n in nbas_list], world)[rank]
