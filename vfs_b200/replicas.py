"""Multi-GPU replicas of the solver: one process per GPU, no exchange between them.

The solve has no cross-GPU step: every stereo pair, and every camera stream with the state
it carries between frames, is independent. N GPUs therefore run N replicas. The host
assigns camera streams to ranks, and a job's throughput is all frames over the slowest
rank's time. Only the timing reduction uses torch.distributed; the data path has no
collective.
"""
from __future__ import annotations

from typing import Dict, List, Tuple


def assign_streams(streams: Dict[int, Tuple[int, int]], world: int) -> Dict[int, int]:
    """Map camera stream id -> rank, balancing per-frame work (pixels).

    Largest streams first, each to the least-loaded rank (ties: lower rank); deterministic, so
    every rank computes the same assignment without communicating.
    """
    if world < 1:
        raise ValueError("world must be >= 1")
    load = [0] * world
    out: Dict[int, int] = {}
    for sid in sorted(streams, key=lambda k: (-streams[k][0] * streams[k][1], k)):
        r = min(range(world), key=lambda i: (load[i], i))
        out[sid] = r
        load[r] += streams[sid][0] * streams[sid][1]
    return out


def my_streams(streams: Dict[int, Tuple[int, int]], world: int, rank: int) -> List[int]:
    """The stream ids this rank serves, in id order."""
    a = assign_streams(streams, world)
    return sorted(k for k, r in a.items() if r == rank)


def job_rate(frames_local: float, ms_local: float, device=None):
    """Job-wide (frames, ms, frames per second): frames summed over ranks, time the maximum
    over ranks (every rank times the same region between barriers). Without an initialized
    process group this is the local figure."""
    import torch
    import torch.distributed as dist

    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        frames, ms = float(frames_local), float(ms_local)
    else:
        t = torch.tensor([float(frames_local), float(ms_local)], dtype=torch.float64,
                         device=device if device is not None else "cpu")
        f = t[:1].clone()
        m = t[1:].clone()
        dist.all_reduce(f, op=dist.ReduceOp.SUM)
        dist.all_reduce(m, op=dist.ReduceOp.MAX)
        frames, ms = float(f.item()), float(m.item())
    return frames, ms, (frames / (ms / 1000.0) if ms > 0 else 0.0)


def merge_serving(latencies_ms: List[float], t_first: float, t_last: float) -> dict:
    """Job-wide serving figures over ranks: every rank's request latencies (ms) and the span
    from the earliest arrival to the latest completion on any rank (time.perf_counter seconds:
    one host's monotonic clock, so comparable between its processes).  Without an initialized
    process group these are the local figures."""
    import numpy as np
    import torch.distributed as dist

    parts = [(list(latencies_ms), float(t_first), float(t_last))]
    if dist.is_available() and dist.is_initialized() and dist.get_world_size() > 1:
        parts = [None] * dist.get_world_size()
        dist.all_gather_object(parts, (list(latencies_ms), float(t_first), float(t_last)))
    lat = np.array([x for p in parts for x in p[0]], dtype=np.float64)
    if lat.size == 0:
        return {"frames": 0}
    busy = [p for p in parts if p[0]]
    span = max(p[2] for p in busy) - min(p[1] for p in busy)
    return {"frames": int(lat.size), "frames_per_s": float(lat.size / span) if span > 0 else None,
            "p50_ms": float(np.percentile(lat, 50)), "p99_ms": float(np.percentile(lat, 99)),
            "mean_ms": float(lat.mean())}
