"""Multi-GPU runs: independent replicas, one per rank, no collective on the data path.

A single conductor system does not shard (the 3D FFT would need a global transpose and
the real-space sum a halo exchange), so N GPUs solve N independent systems.  The only
collectives are host-side bookkeeping: a barrier around the timed region and the maximum
of the per-rank times, from which the whole-job throughput follows.
"""
from __future__ import annotations

import os


def env_int(name: str, default: int) -> int:
    try:
        return int(os.environ.get(name, default))
    except ValueError:
        return default


def rank_info() -> tuple[int, int, int]:
    """(rank, local rank, world size) from the launcher's environment (1 process: 0, 0, 1)."""
    return env_int("RANK", 0), env_int("LOCAL_RANK", 0), env_int("WORLD_SIZE", 1)


def replica_seed(base_seed: int, rank: int) -> int:
    """Seed of this rank's system: every rank solves a different replica."""
    return base_seed + rank


def max_over_ranks(value: float, world: int, device="cpu") -> float:
    """Maximum of a per-rank time over all ranks (the job ends with its slowest rank)."""
    if world == 1:
        return float(value)
    import torch
    import torch.distributed as dist

    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(world: int) -> None:
    if world > 1:
        import torch.distributed as dist

        dist.barrier()


def job_throughput(units_per_rank: float, max_ms_per_step: float, world: int) -> float:
    """Whole-job throughput (units per second) of `world` ranks that each processed
    `units_per_rank` units per step, the step timed as the maximum over ranks."""
    return world * units_per_rank * 1e3 / max_ms_per_step
