"""Multi-GPU plumbing of the benchmark: the path shards by sensor, so N GPUs run N independent replicas of a
workload (one process per GPU, torch.distributed for the plumbing only; no collective on the data path).

- replica(workload, rank): rank r's copy: the same sizes and laws, fields and maps drawn from seeds offset by r.
- reduce_step(...): the whole job's figures: the slowest rank's device time and the sum of every rank's work.
- reduce_max(...): the slowest rank's value of any time.
The reductions run over whatever process group is initialized (NCCL on the GPUs; gloo in the CPU tests).
"""
from __future__ import annotations

from . import fields as F
from . import workloads as W


def replica(wl: W.Workload, rank: int) -> W.Workload:
    """Rank r's replica of a workload (rank 0's is the workload itself)."""
    if rank == 0:
        return wl
    sensors = []
    for s in wl.sensors:
        seed = s.seed + 1000 * rank
        f = (F.blobs(s.width, s.height, seed, s.field.n_blobs) if s.field.kind == F.KIND_BLOBS
             else F.tanh_edge(s.width, s.height, seed))
        sensors.append(W.SensorSpec(s.width, s.height, seed, s.camera, dict(s.overrides), f, s.preset))
    return W.Workload(wl.name, sensors, wl.windows, wl.rules)


def reduce_step(total_ms: float, samples: float, events: float, world: int, device: str = "cuda"):
    """(max over ranks of total_ms, sum of samples, sum of events)."""
    if world <= 1:
        return float(total_ms), float(samples), float(events)
    import torch
    import torch.distributed as dist

    t = torch.tensor([total_ms, samples, events], dtype=torch.float64, device=device)
    mx, sm = t.clone(), t.clone()
    dist.all_reduce(mx, op=dist.ReduceOp.MAX)
    dist.all_reduce(sm, op=dist.ReduceOp.SUM)
    return float(mx[0]), float(sm[1]), float(sm[2])


def reduce_max(value: float, world: int, device: str = "cuda") -> float:
    if world <= 1:
        return float(value)
    import torch
    import torch.distributed as dist

    t = torch.tensor([value], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t[0])
