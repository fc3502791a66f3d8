"""Multi-GPU host logic (one process per GPU).

Rods are independent in the step, so a batch shards with no collective on the
data path: every rank generates the same global batch description, the
largest differencing (Karmarkar-Karp) partition of the rods by element count
(``eb_partition_rods``) gives each rank an element-balanced share, and each
rank builds and steps only its share.  The only collectives are the barrier
and the reductions of timings and counters (``max_over_ranks``,
``sum_over_ranks``) on whatever backend the process group uses (NCCL on GPUs,
gloo on CPU).
"""
from __future__ import annotations

import copy
import ctypes

import numpy as np

from . import _lib as L


def partition(weights, n_parts: int) -> np.ndarray:
    """Part index of every item (int32), balanced by weight."""
    w = np.ascontiguousarray(weights, dtype=np.int64)
    out = np.zeros(len(w), dtype=np.int32)
    if len(w):
        L.call("eb_partition_rods", w.ctypes.data_as(ctypes.POINTER(ctypes.c_int64)), len(w), int(n_parts),
               out.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)))
    return out


def shard(workload, rank: int, world: int, parts: np.ndarray | None = None):
    """The rods of `workload` that rank `rank` of `world` owns (a copy of the
    workload restricted to its part, per-rod data kept aligned)."""
    if world == 1:
        return workload
    if parts is None:
        parts = partition(workload.n_elements, world)
    idx = np.flatnonzero(parts == rank)
    sub = copy.copy(workload)
    sub.rods = [workload.rods[i] for i in idx]
    for key in ("velocities", "rest_curvature", "contact_rod_material"):
        val = getattr(workload, key)
        if val is not None:
            setattr(sub, key, [val[i] for i in idx])
    if workload.end_torque is not None:
        sub.end_torque = np.asarray(workload.end_torque)[idx]
    return sub


def _reduce(value: float, op, group=None) -> float:
    import torch
    import torch.distributed as dist

    if not dist.is_initialized():
        return float(value)
    device = torch.device("cuda", torch.cuda.current_device()) if dist.get_backend(group) == "nccl" \
        else torch.device("cpu")
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=op, group=group)
    return float(t.item())


def max_over_ranks(value: float, group=None) -> float:
    import torch.distributed as dist
    return _reduce(value, dist.ReduceOp.MAX, group)


def sum_over_ranks(value: float, group=None) -> float:
    import torch.distributed as dist
    return _reduce(value, dist.ReduceOp.SUM, group)
