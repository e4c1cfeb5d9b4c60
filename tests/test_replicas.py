"""Multi-GPU replicas: host-side stream assignment and the job-wide rate over ranks, run as
two gloo processes on the CPU (the solve itself has no cross-GPU exchange)."""
import os
import socket

import pytest

from vfs_b200.replicas import assign_streams, job_rate, my_streams

STREAMS = {0: (848, 800), 1: (848, 800), 2: (848, 800), 3: (848, 800), 4: (424, 400), 5: (424, 400)}


def test_assignment_is_complete_balanced_and_deterministic():
    for world in (1, 2, 3, 4, 8):
        a = assign_streams(STREAMS, world)
        assert sorted(a) == sorted(STREAMS) and all(0 <= r < world for r in a.values())
        assert a == assign_streams(dict(reversed(list(STREAMS.items()))), world)
        load = [0] * world
        for sid, r in a.items():
            load[r] += STREAMS[sid][0] * STREAMS[sid][1]
        biggest = max(w * h for w, h in STREAMS.values())
        assert max(load) - min(load) <= biggest  # greedy bound
        got = sorted(s for r in range(world) for s in my_streams(STREAMS, world, r))
        assert got == sorted(STREAMS)  # every stream on exactly one rank
    assert assign_streams(STREAMS, 2) == {0: 0, 1: 1, 2: 0, 3: 1, 4: 0, 5: 1}


def test_job_rate_without_process_group_is_local():
    frames, ms, rate = job_rate(8, 16.0)
    assert frames == 8 and ms == 16.0 and abs(rate - 500.0) < 1e-9


def _free_port():
    with socket.socket(socket.AF_INET, socket.SOCK_STREAM) as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, q):
    import datetime

    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        # rank r solved 8 frames in 10 + 5 r ms; its streams come from the shared assignment
        frames, ms, rate = job_rate(8, 10.0 + 5.0 * rank)
        q.put((rank, frames, ms, rate, my_streams(STREAMS, world, rank)))
        dist.barrier()
    finally:
        dist.destroy_process_group()


@pytest.mark.timeout(120)
def test_job_rate_over_two_gloo_ranks():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=90) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    res.sort()
    for rank, frames, ms, rate, streams in res:
        assert frames == 16 and ms == 15.0  # frames summed, the slowest rank's time
        assert abs(rate - 16 / 0.015) < 1e-6
    assert sorted(res[0][4] + res[1][4]) == sorted(STREAMS)
    assert not set(res[0][4]) & set(res[1][4])


def _serving_rank(rank, world, port, q):
    import datetime

    import torch.distributed as dist

    from vfs_b200.replicas import merge_serving
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        # rank 0 served 3 requests from t = 1.0 s to 2.0 s, rank 1 one request from 1.5 s to 3.0 s
        lat = [10.0, 20.0, 30.0] if rank == 0 else [40.0]
        span = (1.0, 2.0) if rank == 0 else (1.5, 3.0)
        q.put((rank, merge_serving(lat, *span)))
        dist.barrier()
    finally:
        dist.destroy_process_group()


@pytest.mark.timeout(120)
def test_serving_figures_merge_over_two_gloo_ranks():
    """Multi-GPU serving: every rank reports the job's figures over all ranks' requests."""
    import numpy as np
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_serving_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=90) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for _, st in res:
        assert st["frames"] == 4
        assert abs(st["frames_per_s"] - 4 / 2.0) < 1e-9  # first arrival 1.0 s, last completion 3.0 s
        assert abs(st["p50_ms"] - float(np.percentile([10, 20, 30, 40], 50))) < 1e-9
        assert abs(st["p99_ms"] - float(np.percentile([10, 20, 30, 40], 99))) < 1e-9
    assert res[0][1] == res[1][1]


def test_serving_merge_without_process_group_is_local():
    from vfs_b200.replicas import merge_serving
    st = merge_serving([5.0, 7.0], 0.0, 0.5)
    assert st["frames"] == 2 and abs(st["frames_per_s"] - 4.0) < 1e-9 and st["mean_ms"] == 6.0
    assert merge_serving([], 0.0, 0.0) == {"frames": 0}
