"""Serving loop on the GPU: every stream's results are the same served alone and in a mix
(batches of changing composition, two overlapping slots); admission by free memory."""
import numpy as np
import pytest

from tests.helpers import params, random_case, run_gpu

pytestmark = pytest.mark.gpu

CAMS = [(0, 96, 80, 2), (1, 130, 101, 3), (2, 96, 80, 2)]
P = dict(beta=10.0, gamma=0.8, alpha0=17.0, alpha1=1.2, timestep_lambda=1.0, lambda_=5.0, fScale=2.0,
         nWarpIters=2, nSolverIters=6, limitRange=0.1)


def _frames(sid, w, h, n=4):
    out = []
    for k in range(n):
        i0, i1, mask, tv, cv = random_case(w, h, seed=1000 * sid + k)
        out.append((i0, i1))
    _, _, mask, tv, cv = random_case(w, h, seed=1000 * sid)
    return out, mask, tv, cv


@pytest.mark.parametrize("half", [True, False])
def test_alone_and_in_the_mix_are_identical(gpu, half):
    from vfs_b200.serving import StereoServer, poisson_schedule, replay
    data = {sid: _frames(sid, w, h) for sid, w, h, _ in CAMS}
    alone = {}
    for sid, w, h, L in CAMS:
        srv = StereoServer(max_batch=1, lanes=1, half_storage=half, reserve_bytes=0)
        fr, mask, tv, cv = data[sid]
        srv.open_stream(sid, w, h, mask, tv, cv, L, P)
        reqs = [srv.submit(sid, a, b) for a, b in fr]
        srv.run_until_idle()
        alone[sid] = [r.u for r in reqs]
    srv = StereoServer(max_batch=2, lanes=2, half_storage=half, reserve_bytes=0)
    for sid, w, h, L in CAMS:
        fr, mask, tv, cv = data[sid]
        srv.open_stream(sid, w, h, mask, tv, cv, L, P)
    sched = poisson_schedule({0: 100.0, 1: 100.0, 2: 100.0}, {0: 4, 1: 4, 2: 4}, seed=5)
    frames = {sid: data[sid][0] for sid, _, _, _ in CAMS}
    reqs = replay(srv, sched, frames, realtime=False)
    per = {sid: [r for r in reqs if r.stream_id == sid] for sid, _, _, _ in CAMS}
    for sid in per:
        assert len(per[sid]) == 4
        for k, r in enumerate(per[sid]):
            assert np.array_equal(r.u, alone[sid][k]), (sid, k)
    st = srv.stats()
    assert st["frames"] == 12 and st["p99_ms"] >= st["p50_ms"] > 0


def test_serving_float_storage_matches_dropin_path(gpu):
    from vfs_b200.serving import StereoServer
    sid, w, h, L = CAMS[1]
    fr, mask, tv, cv = _frames(sid, w, h, n=3)
    srv = StereoServer(max_batch=2, lanes=2, half_storage=False, reserve_bytes=0)
    srv.open_stream(sid, w, h, mask, tv, cv, L, P)
    reqs = [srv.submit(sid, a, b) for a, b in fr]
    srv.run_until_idle()
    p = params(beta=P["beta"], gamma=P["gamma"], n_levels=L, n_warp=P["nWarpIters"], n_iter=P["nSolverIters"],
               limit_range=P["limitRange"])
    s = run_gpu(fr[0][0], fr[0][1], mask, tv, cv, p, True)  # drop-in path, frame 0
    for k, (a, b) in enumerate(fr):
        if k > 0:  # later frames continue from the same handle state
            s.copyImagesToDevice(a, b)
            s.solveStereoForwardMasked()
        assert np.array_equal(reqs[k].u, s.copy1DDisparityToHost()), k


def test_admission_refuses_streams_that_do_not_fit(gpu):
    import torch
    from vfs_b200.serving import AdmissionError, StereoServer
    _, total = torch.cuda.mem_get_info()
    srv = StereoServer(max_batch=2, lanes=1, reserve_bytes=total)  # nothing fits beside the reserve
    fr, mask, tv, cv = _frames(0, 96, 80, n=1)
    with pytest.raises(AdmissionError):
        srv.open_stream(0, 96, 80, mask, tv, cv, 2, P)
    assert 0 not in srv.cameras
    srv.reserve = 0
    with pytest.raises(AdmissionError):  # a geometry the solver cannot hold
        srv.open_stream(9, 20000, 20000, None, None, None, 8)
    srv.open_stream(0, 96, 80, mask, tv, cv, 2, P)  # admitted once memory is available
    assert 0 in srv.cameras


def _alone(sid, w, h, L, frames, mask, tv, cv, half=True):
    from vfs_b200.serving import StereoServer
    srv = StereoServer(max_batch=1, lanes=1, half_storage=half, reserve_bytes=0)
    srv.open_stream(sid, w, h, mask, tv, cv, L, P)
    reqs = [srv.submit(sid, a, b) for a, b in frames]
    srv.run_until_idle()
    return [r.u for r in reqs]


def test_parked_stream_continues_bit_for_bit(gpu):
    """A stream parked to host memory between frames (state exported, device memory freed) and
    brought back continues exactly where it stopped."""
    from vfs_b200.serving import StereoServer
    sid, w, h, L = CAMS[1]
    fr, mask, tv, cv = _frames(sid, w, h, n=4)
    want = _alone(sid, w, h, L, fr, mask, tv, cv)
    srv = StereoServer(max_batch=2, lanes=1, reserve_bytes=0)
    srv.open_stream(sid, w, h, mask, tv, cv, L, P)
    got = []
    for k, (a, b) in enumerate(fr):
        r = srv.submit(sid, a, b)
        srv.run_until_idle()
        got.append(r.u)
        if k in (1, 2):
            srv.park_stream(sid)
            assert srv.cameras[sid].solver is None
    assert srv.counters["parks"] == 2 and srv.counters["unparks"] == 2
    for k in range(4):
        assert np.array_equal(got[k], want[k]), k


def test_requests_are_admitted_by_free_memory(gpu):
    """With room for about one and a half stream states beside the reserve, opening three
    streams parks the idle ones, and serving their frames parks and brings back states as
    requests are admitted; every result equals the stream served alone."""
    import torch
    from vfs_b200.serving import StereoServer
    cams = [(10 + k, 256, 200, 3) for k in range(3)]
    data = {sid: _frames(sid, w, h, n=2) for sid, w, h, _ in cams}
    alone = {sid: _alone(sid, w, h, L, data[sid][0], *data[sid][1:]) for sid, w, h, L in cams}
    srv = StereoServer(max_batch=3, lanes=1, reserve_bytes=0)
    state = srv.footprint(256, 200, 3)
    torch.cuda.synchronize()
    torch.cuda.empty_cache()
    free, _ = torch.cuda.mem_get_info()
    srv.reserve = free - int(1.5 * state)
    for sid, w, h, L in cams:
        fr, mask, tv, cv = data[sid]
        srv.open_stream(sid, w, h, mask, tv, cv, L, P)
    assert srv.counters["parks"] >= 1
    reqs = []
    for k in range(2):
        for sid, _, _, _ in cams:
            reqs.append(srv.submit(sid, *data[sid][0][k]))
    srv.run_until_idle()
    assert srv.counters["unparks"] >= 1 and srv.counters["deferred"] >= 1
    for r in reqs:
        k = [q for q in reqs if q.stream_id == r.stream_id].index(r)
        assert np.array_equal(r.u, alone[r.stream_id][k]), (r.stream_id, k)


def test_cancel_and_close_between_frames(gpu):
    """A queued request can be withdrawn; a stream closed between its frames leaves the other
    streams' results unchanged."""
    from vfs_b200.serving import StereoServer
    (s0, w0, h0, L0), (s1, w1, h1, L1) = CAMS[0], CAMS[1]
    f0, m0, tv0, cv0 = _frames(s0, w0, h0, n=3)
    f1, m1, tv1, cv1 = _frames(s1, w1, h1, n=3)
    want0 = _alone(s0, w0, h0, L0, f0, m0, tv0, cv0)
    srv = StereoServer(max_batch=2, lanes=2, reserve_bytes=0)
    srv.open_stream(s0, w0, h0, m0, tv0, cv0, L0, P)
    srv.open_stream(s1, w1, h1, m1, tv1, cv1, L1, P)
    r0 = [srv.submit(s0, *f0[0])]
    r1 = srv.submit(s1, *f1[0])
    extra = srv.submit(s1, *f1[1])
    assert srv.cancel(extra) and extra.cancelled and not srv.cancel(extra)
    srv.run_until_idle()
    assert r1.u is not None and extra.u is None
    srv.close_stream(s1)
    assert s1 not in srv.cameras
    for a, b in f0[1:]:
        r0.append(srv.submit(s0, a, b))
    srv.run_until_idle()
    for k in range(3):
        assert np.array_equal(r0[k].u, want0[k]), k
    assert srv.stats()["cancelled"] == 1
