"""Several GPUs, one process each: the evaluation path has no exchange step.

Models, MCMC chains and Jacobian columns are independent units, so a job
over N ranks gives each rank a contiguous share of the units, every rank
evaluates its share on its own GPU with its own engine context, and results
are gathered once at the end (one all-gather of a few doubles per unit).
Timings are the maximum over ranks. torch.distributed is the plumbing (NCCL
on GPUs, gloo on CPU in the tests); no collective runs on the data path.
"""
import numpy as np


def shard(n, rank, world):
    """The [lo, hi) range of n units that rank owns: contiguous, sizes
    differing by at most one, earlier ranks taking the remainder."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("rank %d outside a world of %d" % (rank, world))
    base, extra = divmod(n, world)
    lo = rank * base + min(rank, extra)
    return lo, lo + base + (1 if rank < extra else 0)


def max_over_ranks(value, dist=None, device="cpu"):
    """The largest value of all ranks (the job's time is the slowest rank's)."""
    if dist is None or not dist.is_initialized() or dist.get_world_size() == 1:
        return float(value)
    import torch
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def gather_rows(rows, n, dist=None, device="cpu"):
    """Every rank's rows ([hi - lo, ...] float64 for its shard of n units)
    assembled into the full [n, ...] array on every rank."""
    rows = np.ascontiguousarray(rows, np.float64)
    if dist is None or not dist.is_initialized() or dist.get_world_size() == 1:
        return rows
    import torch
    world = dist.get_world_size()
    width = int(np.prod(rows.shape[1:])) if rows.ndim > 1 else 1
    most = shard(n, 0, world)[1]  # rank 0 has the largest share
    buf = torch.zeros(most, width, dtype=torch.float64, device=device)
    buf[:rows.shape[0]] = torch.as_tensor(rows.reshape(rows.shape[0], width), device=device)
    parts = [torch.zeros_like(buf) for _ in range(world)]
    dist.all_gather(parts, buf)
    out = []
    for r in range(world):
        lo, hi = shard(n, r, world)
        out.append(parts[r][:hi - lo].cpu().numpy())
    full = np.concatenate(out)
    return full.reshape((n,) + rows.shape[1:])
