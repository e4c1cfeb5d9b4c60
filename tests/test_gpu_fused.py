"""Fused path (one kernel per primal-dual iteration, batched launches, CUDA graphs).

With float storage the fused path performs the drop-in path's operations in the same
order on the same physical buffers, so the results must be bit-identical, also across
frames (masked-out pixels keep stale state) and inside batches of uneven sizes.  With half
storage of p, q and v-bar the bar is the accuracy one: mean |u - u_fp64| <= 0.05 px.
"""
import numpy as np
import pytest

from tests.helpers import diff_stats, params, random_case, run_gpu, run_oracle

pytestmark = pytest.mark.gpu

OUT = (("u", 1), ("u_", 1), ("warpUV", 2), ("i1warp", 1), ("Iu", 1), ("Iz", 1), ("Tp", 2), ("a", 1))


# the iteration-kernel variants that exist (3-5, 10-11 and 16-17 were removed)
VARIANTS = (0, 1, 2, 6, 7, 8, 9, 12, 13, 14, 15, 18, 19)

def make(i0, i1, mask, tv, cv, p, fused, half=False, graph=True):
    from vfs_b200.stereotgv import StereoTgv
    s = StereoTgv()
    s.set_solve_path(fused, half)
    s.set_graph(graph)
    h, w = i0.shape
    s.limitRange = p["limit_range"]
    s.initialize(w, h, p["beta"], p["gamma"], p["alpha0"], p["alpha1"], p["tsl"], p["lam"], p["n_levels"],
                 p["f_scale"], p["n_warp"], p["n_iter"])
    s.copyMaskToDevice(mask)
    s.loadVectorFields(tv, cv)
    return s


def solve_frames(s, i0, i1, masked, frames):
    for _ in range(frames):
        s.copyImagesToDevice(i0, i1)
        (s.solveStereoForwardMasked if masked else s.solveStereoForward)()
    s.synchronize()


@pytest.mark.parametrize("graph", [False, True])
@pytest.mark.parametrize("masked", [True, False])
@pytest.mark.parametrize("size", [(67, 53), (130, 101)])
def test_fused_bit_identical_to_dropin(gpu, graph, masked, size):
    w, h = size
    i0, i1, mask, tv, cv = random_case(w, h, seed=w + 3 * h)
    p = params(n_levels=2, n_warp=2, n_iter=7)
    a = make(i0, i1, mask, tv, cv, p, fused=False)
    b = make(i0, i1, mask, tv, cv, p, fused=True, graph=graph)
    for frame in range(3):
        solve_frames(a, i0, i1, masked, 1)
        solve_frames(b, i0, i1, masked, 1)
        for name, comps in OUT:
            x, y = a.debug_buffer(name, comps), b.debug_buffer(name, comps)
            assert np.array_equal(x, y), (frame, name, diff_stats(x, y))


def test_fused_odd_iteration_count(gpu):
    # an odd number of inner iterations leaves u in the other ping-pong buffer
    i0, i1, mask, tv, cv = random_case(90, 70, seed=4)
    p = params(n_levels=3, n_warp=3, n_iter=5)
    a = make(i0, i1, mask, tv, cv, p, fused=False)
    b = make(i0, i1, mask, tv, cv, p, fused=True)
    solve_frames(a, i0, i1, True, 2)
    solve_frames(b, i0, i1, True, 2)
    for name, comps in OUT:
        assert np.array_equal(a.debug_buffer(name, comps), b.debug_buffer(name, comps)), name


@pytest.mark.parametrize("one_launch", [False, True])
def test_batch_uneven_sizes_bit_identical(gpu, one_launch):
    from vfs_b200.stereotgv import StereoBatch
    cases = [(96, 64, 2), (130, 101, 3), (67, 53, 2), (200, 120, 3)]
    p0 = params(n_warp=2, n_iter=6)
    singles, members, data = [], [], []
    batch = StereoBatch()
    batch.set_mode(one_launch)
    for k, (w, h, L) in enumerate(cases):
        i0, i1, mask, tv, cv = random_case(w, h, seed=100 + k)
        p = dict(p0, n_levels=L, alpha0=17.0 + k, limit_range=0.1 + 0.05 * k)
        data.append((i0, i1))
        singles.append(make(i0, i1, mask, tv, cv, p, fused=False))
        m = make(i0, i1, mask, tv, cv, p, fused=True)
        batch.add(m)
        members.append(m)
    for frame in range(2):
        for s, (i0, i1) in zip(singles, data):
            solve_frames(s, i0, i1, True, 1)
        for m, (i0, i1) in zip(members, data):
            m.copyImagesToDevice(i0, i1)
        batch.solve(True)
        for s, m in zip(singles, members):
            m.synchronize()
            for name, comps in (("u", 1), ("warpUV", 2)):
                assert np.array_equal(s.debug_buffer(name, comps), m.debug_buffer(name, comps)), (frame, name)


def test_half_storage_accuracy(gpu):
    from vfs_b200 import synth
    pair = synth.make_pair(424, 400, seed=77)
    sp = synth.SOLVER_PARAMS
    p = params(beta=sp["beta"], gamma=sp["gamma"], n_levels=synth.n_levels_for(424), n_warp=sp["nWarpIters"],
               n_iter=sp["nSolverIters"], limit_range=synth.LIMIT_RANGE)
    s = make(pair.i0, pair.i1, pair.mask, pair.tv, pair.cv, p, fused=True, half=True)
    solve_frames(s, pair.i0, pair.i1, True, 1)
    u = s.copy1DDisparityToHost()
    o = run_oracle(pair.i0, pair.i1, pair.mask, pair.tv, pair.cv, p, True, precision=64)
    m = pair.mask > 0
    d = np.abs(u.astype(np.float64) - o.get("u"))[m]
    assert d.mean() <= 0.05, d.mean()
    assert (d > 1.0).mean() < 0.01
    # the warped image is stored in half: copyWarpedImageToHost widens exactly representable
    # half values, close to the float form's warped image of the same frame
    w16 = s.copyWarpedImageToHost()
    assert np.isfinite(w16).all()
    assert np.array_equal(w16.astype(np.float16).astype(np.float32), w16)
    assert np.array_equal(s.debug_buffer("i1warp", 1), w16)
    f = make(pair.i0, pair.i1, pair.mask, pair.tv, pair.cv, p, fused=True, half=False)
    solve_frames(f, pair.i0, pair.i1, True, 1)
    dw = np.abs(w16 - f.copyWarpedImageToHost())[m]
    assert dw.mean() <= 2e-3, dw.mean()


@pytest.mark.parametrize("one_launch", [False, True])
def test_batch_solve_host_matches_device_path(gpu, one_launch):
    """vfs_batch_solve_host (upload, solve and download per pair in one call) gives the same
    disparities as the device-resident sequence copyImagesToDevice -> vfs_batch_solve ->
    copy1DDisparityToHost, over two frames, from pageable and from page-locked buffers."""
    import torch
    from vfs_b200.stereotgv import StereoBatch
    cases = [(96, 64, 2), (130, 101, 3), (67, 53, 2)]
    p0 = params(n_warp=2, n_iter=6)
    ref_batch, host_batch = StereoBatch(half_storage=True), StereoBatch(half_storage=True)
    ref_batch.set_mode(one_launch)
    host_batch.set_mode(one_launch)
    data = []
    for k, (w, h, L) in enumerate(cases):
        i0, i1, mask, tv, cv = random_case(w, h, seed=300 + k)
        p = dict(p0, n_levels=L)
        ref_batch.add(make(i0, i1, mask, tv, cv, p, fused=True, half=True))
        host_batch.add(make(i0, i1, mask, tv, cv, p, fused=True, half=True))
        data.append((i0, i1))
    pinned = [(torch.from_numpy(a).pin_memory(), torch.from_numpy(b).pin_memory()) for a, b in data]
    outs = [torch.full((h, w), -1.0).pin_memory() for (w, h, _) in cases]
    for frame in range(2):
        for m, (i0, i1) in zip(ref_batch.members, data):
            m.copyImagesToDevice(i0, i1)
        ref_batch.solve(True)
        want = [m.copy1DDisparityToHost() for m in ref_batch.members]
        if frame == 0:
            got = host_batch.solve_host(data)
        else:
            got = host_batch.solve_host([(a.numpy(), b.numpy()) for a, b in pinned], [o.numpy() for o in outs])
        for k, (g, w_) in enumerate(zip(got, want)):
            assert np.array_equal(np.asarray(g), w_), (frame, k)


@pytest.mark.parametrize("masked", [True, False])
def test_every_iteration_variant_bit_identical(gpu, masked):
    """All variants of the fused iteration kernel (shared-memory tiles of 4 / 8 / 16 rows,
    3 to 9 iterations per launch on tiles held in shared memory, the whole level in the shared
    memory of a 16- or 8-CTA cluster, 8-row tiles staged by TMA) give the drop-in path's bits
    with float storage and one another's bits with half storage, on sizes that cut tiles
    unevenly.  11 iterations per warp leave a remainder after the multi-iteration launches
    of every K (3, 5, 7, 9).  The 64 x 48 case has no row padding at
    level 0 and an all-on mask, where the multi-iteration kernel must fall back."""
    from vfs_b200.stereotgv import StereoBatch
    cases = [(97, 71, 2), (131, 45, 3), (40, 100, 2), (64, 48, 2)]
    p0 = params(n_warp=2, n_iter=11)
    for k, (w, h, L) in enumerate(cases):
        i0, i1, mask, tv, cv = random_case(w, h, seed=500 + k, circle=(w, h) != (64, 48))
        p = dict(p0, n_levels=L)
        ref = make(i0, i1, mask, tv, cv, p, fused=False)
        solve_frames(ref, i0, i1, masked, 2)
        want = {n: ref.debug_buffer(n, c) for n, c in (("u", 1), ("u_", 1), ("warpUV", 2), ("Tp", 2))}
        half_ref = None
        for variant in VARIANTS:
            s = make(i0, i1, mask, tv, cv, p, fused=True)
            s.set_iteration_variant(variant)
            solve_frames(s, i0, i1, masked, 2)
            for n, c in (("u", 1), ("u_", 1), ("warpUV", 2), ("Tp", 2)):
                assert np.array_equal(s.debug_buffer(n, c), want[n]), (w, h, variant, n)
            sh = make(i0, i1, mask, tv, cv, p, fused=True, half=True)
            sh.set_iteration_variant(variant)
            solve_frames(sh, i0, i1, masked, 2)
            u = sh.copy1DDisparityToHost()
            if half_ref is None:
                half_ref = u
            assert np.array_equal(u, half_ref), (w, h, variant, "half")
    # batched one-launch form with a forced 16-row variant
    b = StereoBatch(half_storage=False)
    b.set_mode(True)
    b.set_iteration_variant(2)
    members, singles, data = [], [], []
    for k, (w, h, L) in enumerate(cases):
        i0, i1, mask, tv, cv = random_case(w, h, seed=600 + k)
        p = dict(p0, n_levels=L)
        m = make(i0, i1, mask, tv, cv, p, fused=True)
        b.add(m)
        members.append(m)
        singles.append(make(i0, i1, mask, tv, cv, p, fused=False))
        data.append((i0, i1))
    for m, (i0, i1) in zip(members, data):
        m.copyImagesToDevice(i0, i1)
    b.solve(masked)
    for s, m, (i0, i1) in zip(singles, members, data):
        solve_frames(s, i0, i1, masked, 1)
        m.synchronize()
        assert np.array_equal(s.debug_buffer("u", 1), m.debug_buffer("u", 1))


@pytest.mark.parametrize("masked", [True, False])
@pytest.mark.parametrize("n_iter", [10, 67])
def test_cluster_resident_iteration_counts(gpu, masked, n_iter):
    """The cluster-resident variants (14: 16 CTAs, 15: 8 CTAs) with an even number of
    iterations per warp (the results stay in the launch's input buffers) and with more
    iterations than one launch takes (64 + 3), over two frames and with CUDA graphs: the
    drop-in path's bits with float storage, variant 1's bits with half storage.  Heights of
    45 and 22 rows leave trailing CTAs without rows; 200 x 90 with 8 CTAs gives each thread
    three pixels."""
    for (w, h, L) in [(97, 71, 2), (131, 45, 2), (200, 90, 2)]:
        i0, i1, mask, tv, cv = random_case(w, h, seed=w * h + n_iter)
        p = params(n_levels=L, n_warp=2, n_iter=n_iter)
        ref = make(i0, i1, mask, tv, cv, p, fused=False)
        solve_frames(ref, i0, i1, masked, 2)
        href = make(i0, i1, mask, tv, cv, p, fused=True, half=True)
        href.set_iteration_variant(1)
        solve_frames(href, i0, i1, masked, 2)
        hu = href.copy1DDisparityToHost()
        for variant in (14, 15):
            s = make(i0, i1, mask, tv, cv, p, fused=True)
            s.set_iteration_variant(variant)
            solve_frames(s, i0, i1, masked, 2)
            for n, c in (("u", 1), ("u_", 1), ("warpUV", 2), ("Tp", 2)):
                assert np.array_equal(s.debug_buffer(n, c), ref.debug_buffer(n, c)), (w, h, variant, n)
            sh = make(i0, i1, mask, tv, cv, p, fused=True, half=True)
            sh.set_iteration_variant(variant)
            solve_frames(sh, i0, i1, masked, 2)
            assert np.array_equal(sh.copy1DDisparityToHost(), hu), (w, h, variant, "half")


def test_launch_overlap_does_not_change_results(gpu):
    """Programmatic dependent launch of the iteration kernels (the default) and plain
    stream-ordered launches give the same bits."""
    from vfs_b200._native import lib
    i0, i1, mask, tv, cv = random_case(150, 90, seed=77)
    p = params(n_levels=3, n_warp=2, n_iter=9)
    out = []
    try:
        for on in (1, 0):
            assert lib().vfs_set_launch_overlap(on) == 0
            for half in (False, True):
                s = make(i0, i1, mask, tv, cv, p, fused=True, half=half)
                solve_frames(s, i0, i1, True, 2)
                out.append(s.copy1DDisparityToHost())
    finally:
        lib().vfs_set_launch_overlap(1)
    assert np.array_equal(out[0], out[2]) and np.array_equal(out[1], out[3])


def test_per_level_variants_and_tuned_choice_reported(gpu):
    """A per-level variant list (here one-iteration at full resolution, nine and seven
    iterations per launch below) gives the drop-in path's bits, and the handle reports what
    it ran; the tuner picks only variants that exist."""
    i0, i1, mask, tv, cv = random_case(120, 90, seed=808)
    p = params(n_levels=3, n_warp=2, n_iter=11)
    ref = make(i0, i1, mask, tv, cv, p, fused=False)
    solve_frames(ref, i0, i1, True, 2)
    s = make(i0, i1, mask, tv, cv, p, fused=True)
    s.set_iteration_variants([1, 13, 12])  # 9 and 7 iterations per launch, remainders single
    solve_frames(s, i0, i1, True, 2)
    assert s.iteration_variants() == [1, 13, 12]
    for n, c in (("u", 1), ("warpUV", 2), ("Tp", 2)):
        assert np.array_equal(s.debug_buffer(n, c), ref.debug_buffer(n, c)), n
    t = make(i0, i1, mask, tv, cv, p, fused=True)
    solve_frames(t, i0, i1, True, 1)  # autotuned
    v = t.iteration_variants()
    assert len(v) == 3 and all(x in VARIANTS for x in v)


def test_new_batch_compositions_reuse_tuned_levels(gpu):
    """Each pair of a concurrent batch is tuned per pyramid level: a batch of a new composition
    (here two of the three pairs) reuses the levels tuned with other pairs in flight, and so does
    a pair solved alone once its level sizes were tuned in a batch; no tuning solve runs again.
    Results are the drop-in path's."""
    from vfs_b200._native import lib
    from vfs_b200.stereotgv import StereoBatch
    count = lambda: lib().vfs_tuning_solves()
    p = params(n_levels=3, n_warp=2, n_iter=9)
    cases = [random_case(152, 136, seed=4100 + k) for k in range(4)]
    pairs = [make(*c, p, fused=True) for c in cases]
    for s in pairs:
        s.set_autotune(True)

    def batch_solve(members):
        b = StereoBatch(half_storage=False)
        for m in members:
            b.add(m)
        for m, c in zip(members, cases):
            m.copyImagesToDevice(c[0], c[1])
        b.solve(True)
        for m in members:
            m.synchronize()

    batch_solve(pairs[:3])  # tunes (unless an earlier test tuned these level sizes)
    n0 = count()
    batch_solve(pairs[:2])  # a new composition, pairs still in flight together
    batch_solve([pairs[0], pairs[3]])
    assert count() == n0
    solve_frames(pairs[1], cases[1][0], cases[1][1], True, 1)  # alone
    solve_frames(pairs[2], cases[2][0], cases[2][1], True, 2)
    assert count() == n0
    ref = make(*cases[2], p, fused=False)
    solve_frames(ref, cases[2][0], cases[2][1], True, 1)
    one = make(*cases[2], p, fused=True)
    solve_frames(one, cases[2][0], cases[2][1], True, 1)
    assert np.array_equal(one.debug_buffer("u", 1), ref.debug_buffer("u", 1))


def test_retired_variants_are_rejected(gpu):
    """Numbers of the removed forms (3-5, 10-11, 16-17) and out-of-range numbers are refused."""
    from vfs_b200.stereotgv import VfsError
    i0, i1, mask, tv, cv = random_case(64, 48, seed=9)
    s = make(i0, i1, mask, tv, cv, params(n_levels=1, n_warp=1, n_iter=1), fused=True)
    for v in (3, 4, 5, 10, 11, 16, 17, 20, -2):
        with pytest.raises(VfsError):
            s.set_iteration_variant(v)
    s.set_iteration_variant(-1)  # back to the tuner


@pytest.mark.parametrize("fine,stagger,prio", [(1, 0, 0), (2, 0, 2), (2, 1, 1), (3, 1, 0), (2, 0, 3), (1, 0, 3), (2, 0, 4)])
def test_fine_concurrency_limit_keeps_results(gpu, fine, stagger, prio):
    """Splitting each pair's solve into coarse levels and a full-resolution part, with at most
    `fine` pairs at full resolution at a time (optionally with the coarse parts staggered the
    same way, the full-resolution parts on high-priority streams, or every part at the priority
    of its full-resolution round), gives the same bits as
    the unsplit batch, over two frames and from host buffers too."""
    from vfs_b200.stereotgv import StereoBatch
    cases = [(96, 64, 2), (130, 101, 3), (67, 53, 2), (200, 120, 3)]
    p0 = params(n_warp=2, n_iter=6)
    ref_b, lim_b = StereoBatch(half_storage=True), StereoBatch(half_storage=True)
    lim_b.set_fine_concurrency(fine)
    lim_b.set_pipeline(bool(stagger), prio)
    data = []
    for k, (w, h, L) in enumerate(cases):
        i0, i1, mask, tv, cv = random_case(w, h, seed=900 + k)
        p = dict(p0, n_levels=L)
        ref_b.add(make(i0, i1, mask, tv, cv, p, fused=True, half=True))
        lim_b.add(make(i0, i1, mask, tv, cv, p, fused=True, half=True))
        data.append((i0, i1))
    for frame in range(2):
        want = ref_b.solve_host(data)
        if frame == 0:
            for m, (i0, i1) in zip(lim_b.members, data):
                m.copyImagesToDevice(i0, i1)
            lim_b.solve(True)
            got = [m.copy1DDisparityToHost() for m in lim_b.members]
        else:
            got = lim_b.solve_host(data)
        for k, (g, w_) in enumerate(zip(got, want)):
            assert np.array_equal(g, w_), (frame, k)


def test_fp16_batch_accuracy_at_full_size(gpu):
    """The batched FP16-storage form at 848 x 800 (two seeded pairs, autotuned kernels, the
    default full-resolution schedule) against the FP64 oracle: mean |du| <= 0.05 px and fewer
    than 1 % of in-mask pixels off by more than 1 px."""
    from vfs_b200 import synth
    from vfs_b200.stereotgv import StereoBatch
    sp = synth.SOLVER_PARAMS
    p = params(beta=sp["beta"], gamma=sp["gamma"], n_levels=synth.n_levels_for(848), n_warp=sp["nWarpIters"],
               n_iter=sp["nSolverIters"], limit_range=synth.LIMIT_RANGE)
    pairs = [synth.make_pair(848, 800, seed=4242 + k) for k in range(2)]
    b = StereoBatch(half_storage=True)
    for pr in pairs:
        b.add(make(pr.i0, pr.i1, pr.mask, pr.tv, pr.cv, p, fused=True, half=True))
    outs = b.solve_host([(pr.i0, pr.i1) for pr in pairs])
    for pr, u in zip(pairs, outs):
        o = run_oracle(pr.i0, pr.i1, pr.mask, pr.tv, pr.cv, p, True, precision=64)
        m = pr.mask > 0
        d = np.abs(np.asarray(u, np.float64) - o.get("u"))[m]
        assert d.mean() <= 0.05, d.mean()
        assert (d > 1.0).mean() < 0.01


def test_mask_change_between_frames_rebuilds_the_launches(gpu):
    """A new mask between frames (graphs already captured under the old one) gives the same
    bits as a handle that saw the same mask sequence on the drop-in path: the tile spans and
    multi-iteration levels derived from the mask are not reused from stale graphs."""
    w, h = 150, 110
    i0, i1, mask, tv, cv = random_case(w, h, seed=1212)
    yy, xx = np.mgrid[0:h, 0:w]
    mask2 = ((xx - 40) ** 2 + (yy - 55) ** 2 < 45 ** 2).astype(np.float32)  # a different disc
    p = params(n_levels=3, n_warp=2, n_iter=7)
    ref = make(i0, i1, mask, tv, cv, p, fused=False)
    f = make(i0, i1, mask, tv, cv, p, fused=True, half=False)
    for frame in range(5):
        if frame == 3:
            ref.copyMaskToDevice(mask2)
            f.copyMaskToDevice(mask2)
        solve_frames(ref, i0, i1, True, 1)
        solve_frames(f, i0, i1, True, 1)
        assert np.array_equal(ref.debug_buffer("u", 1), f.debug_buffer("u", 1)), frame


def test_batch_solve_device_matches_host_buffers(gpu):
    """vfs_batch_solve_device (images and disparities in device memory, copies on each pair's
    lane) gives the bits of vfs_batch_solve_host, over two frames, split schedule included."""
    import torch
    from vfs_b200.stereotgv import StereoBatch
    cases = [(96, 64, 2), (130, 101, 3), (67, 53, 2)]
    p0 = params(n_warp=2, n_iter=6)
    hb, db = StereoBatch(half_storage=True), StereoBatch(half_storage=True)
    db.set_fine_concurrency(1)
    data = []
    for k, (w, h, L) in enumerate(cases):
        i0, i1, mask, tv, cv = random_case(w, h, seed=1400 + k)
        p = dict(p0, n_levels=L)
        hb.add(make(i0, i1, mask, tv, cv, p, fused=True, half=True))
        db.add(make(i0, i1, mask, tv, cv, p, fused=True, half=True))
        data.append((i0, i1))
    d_in = [(torch.from_numpy(a).cuda(), torch.from_numpy(b).cuda()) for a, b in data]
    d_out = [torch.full((h, w), -1.0, device="cuda") for (w, h, _) in cases]
    torch.cuda.synchronize()  # the batch's streams do not wait for the default stream
    for frame in range(2):
        want = hb.solve_host(data)
        db.solve_device(d_in, d_out)
        torch.cuda.synchronize()
        for k, (g, w_) in enumerate(zip(d_out, want)):
            assert np.array_equal(g.cpu().numpy(), w_), (frame, k)


@pytest.mark.parametrize("half", [False, True], ids=["fp32", "fp16"])
def test_tma_and_15_row_iterations_match_default_at_full_size(gpu, half):
    """The TMA-staged iteration kernel (variant 18) and the 15-row tiles (variant 19) on a
    synthetic 848 x 800 fisheye pair, every level, with their per-row tile spans: the bits of
    the default variant (and, with float storage, of the drop-in path); the TMA kernel's
    bounded copy waits never ran out."""
    import ctypes
    from vfs_b200 import synth
    from vfs_b200._native import lib
    pair = synth.make_pair(848, 800, seed=4242)
    sp = synth.SOLVER_PARAMS
    p = params(beta=sp["beta"], gamma=sp["gamma"], n_levels=synth.n_levels_for(848), n_warp=sp["nWarpIters"],
               n_iter=sp["nSolverIters"], limit_range=synth.LIMIT_RANGE)
    out = {}
    for v in (1, 18, 19):
        s = make(pair.i0, pair.i1, pair.mask, pair.tv, pair.cv, p, fused=True, half=half)
        s.set_iteration_variant(v)
        solve_frames(s, pair.i0, pair.i1, True, 2)
        out[v] = (s.copy1DDisparityToHost(), s.debug_buffer("warpUV", 2))
        assert s.iteration_variants() == [v] * synth.n_levels_for(848)
    for v in (18, 19):
        assert np.array_equal(out[1][0], out[v][0]) and np.array_equal(out[1][1], out[v][1]), v
    st = ctypes.c_int(-1)
    assert lib().vfs_device_status(ctypes.byref(st)) == 0 and st.value == 0
