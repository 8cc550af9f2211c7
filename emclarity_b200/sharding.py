"""Multi-GPU host logic: one process per GPU, particles sharded across ranks.

Particles are independent in the orientation search (each one's best orientation depends only on
its own spectrum and the shared reference / grid), so the path shards with no collective on the
data path: every rank searches a contiguous slice of the particle list on its own GPU and the
result rows are gathered to rank 0 on the host at the end -- the same split the reference makes
with MATLAB parfor workers bound to one GPU each (alignment/BH_alignRaw3d_v2.m:764-776) and its
tomogram list partitioning (logicals/BH_multi_parallelJobs.m:32-79).
"""
import numpy as np


def shard_range(n_items, rank, world):
    """Contiguous [begin, end) slice of n_items for `rank` of `world`; sizes differ by at most one."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("bad rank %d / world %d" % (rank, world))
    base, extra = divmod(n_items, world)
    begin = rank * base + min(rank, extra)
    return begin, begin + base + (1 if rank < extra else 0)


def gather_rows(rows, world, dst=0):
    """Gathers each rank's result rows (an (k_i, m) float64 array) to rank `dst` in rank order over the
    default process group; returns the concatenation on dst and None elsewhere."""
    import torch
    import torch.distributed as dist
    rows = np.ascontiguousarray(rows, dtype=np.float64)
    if world == 1:
        return rows
    rank = dist.get_rank()
    m = rows.shape[1] if rows.ndim == 2 else 1
    counts = torch.zeros(world, dtype=torch.int64)
    counts[rank] = rows.shape[0]
    dist.all_reduce(counts)
    cap = int(counts.max())
    buf = torch.zeros((cap, m), dtype=torch.float64)
    buf[:rows.shape[0]] = torch.from_numpy(rows.reshape(-1, m))
    out = [torch.zeros_like(buf) for _ in range(world)] if rank == dst else None
    dist.gather(buf, gather_list=out, dst=dst)
    if rank != dst:
        return None
    return np.concatenate([o[:int(c)].numpy() for o, c in zip(out, counts)], axis=0)


def max_over_ranks(value, world, device=None):
    """Max of a per-rank scalar (e.g. a step time) over all ranks."""
    if world == 1:
        return float(value)
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())
