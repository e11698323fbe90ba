"""Independent replicas, one lattice per rank (one process per GPU).

The Langevin step does not shard: every rank advances its own lattice with
its own noise stream and no exchange during a step.  Ranks meet only to
time the job (a barrier, then the max of the per-rank device times) and to
gather per-replica observables at the end.  These helpers work on any
process group: NCCL with CUDA tensors on GPUs, gloo with CPU tensors.
"""
from __future__ import annotations

import os


def world_info():
    """(world_size, rank, local_rank) from the torchrun environment."""
    return (int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("RANK", "0")),
            int(os.environ.get("LOCAL_RANK", "0")))


_MASK64 = (1 << 64) - 1


def _splitmix64(x: int) -> int:
    """SplitMix64 finaliser (Steele, Lea and Flood, OOPSLA 2014): a
    bijection of 64-bit integers that spreads nearby inputs far apart."""
    x = (x + 0x9E3779B97F4A7C15) & _MASK64
    x = ((x ^ (x >> 30)) * 0xBF58476D1CE4E5B9) & _MASK64
    x = ((x ^ (x >> 27)) * 0x94D049BB133111EB) & _MASK64
    return x ^ (x >> 31)


def replica_seed(base: int, rank: int) -> int:
    """Noise seed of replica `rank`: the base itself on rank 0 (a one-GPU run
    keeps its plain seed), otherwise a 64-bit hash of (base, rank).  For one
    base the ranks' seeds are distinct (the hash is a bijection in its
    argument, and that argument differs per rank), and jobs with nearby bases
    do not share a stream, as base + c * rank would for bases c apart."""
    if rank < 0:
        raise ValueError("rank must be >= 0")
    base = int(base) & _MASK64
    if rank == 0:
        return base
    return _splitmix64(_splitmix64(base) ^ int(rank))


def _device():
    import torch
    import torch.distributed as dist
    if dist.is_initialized() and dist.get_backend() == "nccl":
        return torch.device("cuda", torch.cuda.current_device())
    return torch.device("cpu")


def max_over_ranks(x: float) -> float:
    """Max of a scalar over all ranks (identity without a process group)."""
    import torch
    import torch.distributed as dist
    if not dist.is_initialized() or dist.get_world_size() == 1:
        return float(x)
    t = torch.tensor([float(x)], dtype=torch.float64, device=_device())
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def gather_series(values) -> list:
    """All ranks' per-replica series (e.g. plaquette per order), rank order."""
    import torch
    import torch.distributed as dist
    t = torch.as_tensor(values, dtype=torch.float64).reshape(-1).to(_device())
    if not dist.is_initialized() or dist.get_world_size() == 1:
        return [t.cpu().tolist()]
    out = [torch.empty_like(t) for _ in range(dist.get_world_size())]
    dist.all_gather(out, t)
    return [o.cpu().tolist() for o in out]


def whole_job_rate(units_per_rank: float, world: int, seconds_max: float) -> float:
    """Units per second of the whole job: every rank processed
    `units_per_rank` units and the slowest rank took `seconds_max`."""
    if seconds_max <= 0:
        raise ValueError("seconds_max must be > 0")
    return world * units_per_rank / seconds_max
