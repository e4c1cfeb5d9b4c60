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
    free, _ = torch.cuda.mem_get_info()
    srv = StereoServer(max_batch=2, lanes=1, reserve_bytes=free)  # nothing fits beside the reserve
    fr, mask, tv, cv = _frames(0, 96, 80, n=1)
    with pytest.raises(AdmissionError):
        srv.open_stream(0, 96, 80, mask, tv, cv, 2, P)
    assert 0 not in srv.cameras
    srv.reserve = 0
    with pytest.raises(AdmissionError):  # a geometry the solver cannot hold
        srv.open_stream(9, 20000, 20000, None, None, None, 8)
    srv.open_stream(0, 96, 80, mask, tv, cv, 2, P)  # admitted once memory is available
    assert 0 in srv.cameras
