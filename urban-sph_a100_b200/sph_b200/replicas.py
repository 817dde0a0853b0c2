"""Whole-job numbers of replica runs (one independent case per rank).

The ISPH path has no exchange between ranks: each rank steps its own deck.
A job's throughput is the work of all ranks divided by the slowest rank's
device time, so the only collectives are two scalar reductions after the
timed region.
"""
import torch
import torch.distributed as dist


def reduce_job(units, ms, device="cpu"):
    """(sum of `units` over ranks, max of `ms` over ranks); one process: unchanged."""
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(units), float(ms)
    u = torch.tensor([float(units)], dtype=torch.float64, device=device)
    m = torch.tensor([float(ms)], dtype=torch.float64, device=device)
    dist.all_reduce(u, op=dist.ReduceOp.SUM)
    dist.all_reduce(m, op=dist.ReduceOp.MAX)
    return float(u.item()), float(m.item())


def throughput(units_per_step, steps, ms, device="cpu"):
    """Whole-job particle-steps/s: all ranks' units x steps / the slowest rank's time."""
    units, ms = reduce_job(units_per_step * steps, ms, device)
    return units / (ms / 1e3), ms
