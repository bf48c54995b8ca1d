"""Independent replicas, one process per GPU.

A state vector of one circuit does not shard without exchanging global
qubits, and every workload here fits one B200, so N GPUs run N independent
replicas (each rank its own seeded circuit).  The job's time is the slowest
rank's device time; throughput = all ranks' units / that time (weak
scaling).  The only collectives are this timing reduction and barriers.
"""
from __future__ import annotations


def replica_seed(seed: int, rank: int) -> int:
    """Seed of rank ``rank``'s circuit: distinct circuits, same shape."""
    return seed + rank


def job_time_ms(ms: float, dist=None, device="cpu") -> float:
    """Max of ``ms`` over all ranks (the local value without a process
    group).  Every rank must call it, in the same order as its other
    collectives."""
    if dist is None or not dist.is_initialized() or dist.get_world_size() == 1:
        return float(ms)
    import torch
    t = torch.tensor([float(ms)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_throughput(units_per_rank: float, steps: int, job_ms: float, world: int) -> float:
    """Units per second of the whole job."""
    if job_ms <= 0:
        raise ValueError("job time must be positive")
    return world * units_per_rank * steps / (job_ms / 1e3)
