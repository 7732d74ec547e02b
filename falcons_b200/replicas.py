"""Whole-job throughput of independent replicas (one field per rank, no exchange step).

A single field's stream is one global code sequence, so the path does not shard: N GPUs run N
independent compress/decompress replicas, and the job's throughput is the bytes all ranks
processed divided by the slowest rank's time.  The only collectives are these two reductions,
made after the timed region.
"""
from __future__ import annotations

import torch


def job_throughput(local_bytes: float, local_ms: float, group=None, device=None):
    """Returns (GB/s over all ranks, max ms over ranks, total bytes over ranks).

    Without an initialized process group (a single process) the local figures are returned.
    `device` is where the reduction tensors live (a CUDA device for NCCL, CPU for gloo).
    """
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()):
        return local_bytes / (local_ms / 1e3) / 1e9, float(local_ms), float(local_bytes)
    dev = device if device is not None else torch.device("cpu")
    t = torch.tensor([float(local_ms)], dtype=torch.float64, device=dev)
    b = torch.tensor([float(local_bytes)], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX, group=group)
    dist.all_reduce(b, op=dist.ReduceOp.SUM, group=group)
    ms, total = float(t.item()), float(b.item())
    return total / (ms / 1e3) / 1e9, ms, total


def job_sum(value: float, group=None, device=None) -> float:
    """Sum of a per-rank figure over all ranks (the local value without a process group)."""
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()):
        return float(value)
    dev = device if device is not None else torch.device("cpu")
    v = torch.tensor([float(value)], dtype=torch.float64, device=dev)
    dist.all_reduce(v, op=dist.ReduceOp.SUM, group=group)
    return float(v.item())
