"""Multi-GPU sharding of the fit path: one process per GPU, frames split
into contiguous ranges, no collective on the data path.

Every candidate's fit is independent (the reference farms frames out to host
threads the same way, source/PALMAnalysis.cpp:96-130), so a stack is split by
frame ranges, each rank fits the candidates of its frames on its own GPU, and
the only exchanges are the job's bookkeeping: the total count and the
slowest rank's time (for throughput), and, if the caller wants every row on
one rank, a gather of the per-rank rows in frame order.
"""
from __future__ import annotations

import numpy as np


def frame_shard(n_frames: int, rank: int, world: int) -> tuple[int, int]:
    """Contiguous, balanced frame range [start, stop) of a rank."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("rank out of range")
    base, extra = divmod(n_frames, world)
    start = rank * base + min(rank, extra)
    return start, start + base + (1 if rank < extra else 0)


def candidate_shard(cands: np.ndarray, rank: int, world: int, n_frames: int) -> np.ndarray:
    """Indices (ascending) of the candidates whose frame lies in the rank's range."""
    start, stop = frame_shard(n_frames, rank, world)
    f = cands["frame"]
    return np.nonzero((f >= start) & (f < stop))[0]


def job_throughput(n_local: int, ms_local: float, group=None):
    """(units over all ranks, slowest rank's ms, units/s of the whole job).
    The time is the maximum over ranks, so the job's throughput is the total
    work over the time the last rank finished."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()):
        return float(n_local), float(ms_local), float(n_local) / (ms_local / 1e3)
    dev = "cuda" if dist.get_backend(group) == "nccl" else "cpu"
    t = torch.tensor([float(ms_local)], dtype=torch.float64, device=dev)
    c = torch.tensor([float(n_local)], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX, group=group)
    dist.all_reduce(c, op=dist.ReduceOp.SUM, group=group)
    return c.item(), t.item(), c.item() / (t.item() / 1e3)


def gather_rows(rows_local: np.ndarray, flags_local: np.ndarray, dst: int = 0, group=None):
    """Rows and flags of every rank on rank dst, concatenated in rank order
    (= frame order for frame_shard); None on the other ranks."""
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()):
        return rows_local, flags_local
    obj = (np.ascontiguousarray(rows_local), np.ascontiguousarray(flags_local))
    parts = [None] * dist.get_world_size(group) if dist.get_rank(group) == dst else None
    dist.gather_object(obj, parts, dst=dst, group=group)
    if parts is None:
        return None
    return np.concatenate([p[0] for p in parts]), np.concatenate([p[1] for p in parts])
