"""The drop-in path against the reference's OWN CUDA solver, built from its unmodified sources.

oracle/Makefile.ref compiles menandro/vfs stereotgv/*.cu (with the stand-ins of
oracle/refcompat/ for the texture-reference API CUDA 12 removed, helper_cuda.h and the few
OpenCV calls) into oracle/_ref/.  These tests run that build and the vfs_b200 drop-in path on
the same inputs and compare their outputs.

Two builds of the reference are used:
* ``nofma``: compiled with -fmad=false, the contraction rule of the vfs_b200 library.  The
  drop-in path (tensor weight through CUDA's expf / powf, its default) evaluates the same float
  operations in the same order through the same texture unit, and its results are required to
  be BIT-IDENTICAL to this build's: every plane, at every size, masked and plain.
* ``stock``: nvcc's default flags (multiply-add contraction on), as the reference ships.  Every
  a*b+c the compiler contracts rounds once instead of twice; over 150 iterations per level that
  changes the reference's own result (by up to 0.1 px at 848x800 and 0.5 px on the Wang case).
  No float32 reimplementation can be closer to it than its own -fmad=false build is, so the
  tests hold the drop-in path to exactly that distance.

The CPU float32 oracle (oracle/tgv_oracle.cpp) is pinned to the reference build here as well.
"""
import os

import numpy as np
import pytest

from tests.helpers import diff_stats, params, random_case, run_gpu, run_oracle

pytestmark = pytest.mark.gpu

TOL_MAX = 1e-3  # px: the drop-in bar


@pytest.fixture(scope="module")
def ref():
    from oracle import ref as R
    if not R.available():
        pytest.skip("reference build missing (oracle/Makefile.ref needs the reference sources)")
    return R


def _exact(got, want, what):
    st = diff_stats(got, want)
    assert st["max"] == 0.0, (what, st)


@pytest.mark.parametrize("masked", [True, False], ids=["masked", "plain"])
@pytest.mark.parametrize("size", [(67, 53), (96, 64), (130, 101)])
def test_small_cases_match_reference_build(gpu, ref, size, masked):
    w, h = size
    i0, i1, mask, tv, cv = random_case(w, h, seed=w * 7 + h)
    p = params(n_levels=2, n_warp=2, n_iter=7)
    s = run_gpu(i0, i1, mask, tv, cv, p, masked)
    r = ref.run_ref(i0, i1, mask, tv, cv, p, masked, fma=False)
    _exact(s.copy1DDisparityToHost(), r.copy1DDisparityToHost(), "u")
    _exact(s.copyDisparityToHost(), r.copyDisparityToHost(), "warpUV")
    for name, comps in (("u_", 1), ("a", 1), ("b", 1), ("c", 1), ("Iu", 1), ("Iz", 1), ("i1warp", 1),
                        ("tv2", 2), ("p", 2), ("q", 4)):
        _exact(s.debug_buffer(name, comps), r.plane(name, comps), name)
    r.close()
    # the shipped build (multiply-add contraction on) differs from it by float32 rounding only
    rs = ref.run_ref(i0, i1, mask, tv, cv, p, masked, fma=True)
    assert diff_stats(s.copy1DDisparityToHost(), rs.copy1DDisparityToHost())["max"] <= TOL_MAX
    rs.close()


@pytest.mark.parametrize("masked", [True, False], ids=["masked", "plain"])
@pytest.mark.parametrize("wh", [(424, 400), (848, 800)])
def test_benchmark_sizes_match_reference_build(gpu, ref, wh, masked):
    """The synthetic fisheye workloads at 424x400 and 848x800 with the benchmark's solver
    settings (4 / 5 levels x 3 warps x 50 iterations), every pixel."""
    from vfs_b200 import synth
    w, h = wh
    pair = synth.make_pair(w, h, seed=1000 + w)
    sp = synth.SOLVER_PARAMS
    p = params(beta=sp["beta"], gamma=sp["gamma"], n_levels=synth.n_levels_for(w), n_warp=sp["nWarpIters"],
               n_iter=sp["nSolverIters"], limit_range=synth.LIMIT_RANGE)
    s = run_gpu(pair.i0, pair.i1, pair.mask, pair.tv, pair.cv, p, masked)
    u = s.copy1DDisparityToHost()
    rn = ref.run_ref(pair.i0, pair.i1, pair.mask, pair.tv, pair.cv, p, masked, fma=False)
    un = rn.copy1DDisparityToHost()
    _exact(u, un, "u")
    _exact(s.copyDisparityToHost(), rn.copyDisparityToHost(), "warpUV")
    rn.close()
    rs = ref.run_ref(pair.i0, pair.i1, pair.mask, pair.tv, pair.cv, p, masked, fma=True)
    us = rs.copy1DDisparityToHost()
    rs.close()
    # distance to the shipped build == the reference's own build-to-build spread
    assert diff_stats(u, us)["max"] <= diff_stats(un, us)["max"]


def test_wang_config_matches_reference_build(gpu, ref):
    """The reference's own Wang fixture and parameters (test_vfs/main.cpp:270-281).  Its mask
    reaches the image border at the coarsest level, where the reference's masked kernels read
    before their buffers' start (zeros in this build, as in vfs_b200)."""
    d = np.load(os.path.join(os.path.dirname(__file__), "golden", "wang_half", "wang_half.npz"))
    p = params(beta=9.0, gamma=0.85, n_levels=5, n_warp=20, n_iter=10, limit_range=0.1)
    mask = d["mask_u8"].astype(np.float32) / 255.0
    u = run_gpu(d["i0"], d["i1"], mask, d["tv"], d["cv"], p, True).copy1DDisparityToHost()
    r = ref.run_ref(d["i0"], d["i1"], mask, d["tv"], d["cv"], p, True, fma=False)
    _exact(u, r.copy1DDisparityToHost(), "u")
    r.close()


def test_state_across_frames_matches_reference_build(gpu, ref):
    """Three frames through one instance: stale masked-out values carry over in both."""
    i0, i1, mask, tv, cv = random_case(72, 60, seed=11)
    p = params(n_levels=2, n_warp=2, n_iter=4)
    s = run_gpu(i0, i1, mask, tv, cv, p, True, frames=3)
    r = ref.run_ref(i0, i1, mask, tv, cv, p, True, frames=3, fma=False)
    _exact(s.copy1DDisparityToHost(), r.copy1DDisparityToHost(), "u")
    r.close()


def test_output_copies_match_reference_build(gpu, ref):
    """copyDisparityToHost, copyWarpedImageToHost, copyDisparityVisToHost (FlowToHSV) and
    copyStereoToHost (ConvertKB) against the reference's own kernels."""
    i0, i1, mask, tv, cv = random_case(96, 64, seed=21)
    p = params(n_levels=2, n_warp=2, n_iter=6)
    s = run_gpu(i0, i1, mask, tv, cv, p, True)
    r = ref.run_ref(i0, i1, mask, tv, cv, p, True, fma=False)
    flow = s.copyDisparityToHost()
    _exact(flow, r.copyDisparityToHost(), "warpUV")
    _exact(s.copyWarpedImageToHost(), r.copyWarpedImageToHost(), "warped image")
    # The output kernels are compared on identical input: the reference instance is given the
    # drop-in path's flow before its FlowToHSV and ConvertKB run.
    r.set_plane("warpUV", flow)
    for scale in (1.0, 4.0, 20.0):
        vs, vr = s.copyDisparityVisToHost(scale), r.copyDisparityVisToHost(scale)
        # flowToHsv.cu:14-21 indexes its 55-entry colour tables with k0, k1 in 1..55: index 55
        # (flow angles in the last 1/54 of the wheel) reads past the tables, which is undefined;
        # vfs_b200 takes the last entry there.  Everywhere else the colours must be identical.
        du = flow[..., 0].astype(np.float64) / scale
        dv = flow[..., 1].astype(np.float64) / scale
        fk = (np.arctan2(-dv, -du) / 3.14159 + 1) / 2 * 54 + 1
        defined = fk < 54.0 - 1e-4
        assert defined.mean() > 0.5
        _exact(vs[defined], vr[defined], f"colour map, flow scale {scale}")
    kb = (45.0, 45.0, 48.0, 32.0, 0.3, -0.1, 0.05, -0.01, 0.064, 0.0, 0.0)
    d_s, X_s = s.copyStereoToHost(*kb)
    d_r, X_r = r.copyStereoToHost(*kb)
    fin = np.isfinite(d_r)
    assert np.array_equal(fin, np.isfinite(d_s)) and fin.any()
    _exact(d_s[fin], d_r[fin], "depth")
    _exact(X_s[fin], X_r[fin], "X")
    r.close()


@pytest.mark.parametrize("kind", ["f32", "u8c3"])
def test_image_overloads_match_reference_build(gpu, ref, kind):
    """The cv::Mat overload of copyImagesToDevice (CV_32F and CV_8UC3 inputs)."""
    i0, i1, mask, tv, cv = random_case(80, 61, seed=5)
    if kind == "f32":
        a, b = i0.astype(np.float32) / 256.0, i1.astype(np.float32) / 256.0
    else:
        rng = np.random.default_rng(3)
        a = np.stack([i0, np.roll(i0, 1, 1), rng.integers(0, 256, i0.shape, dtype=np.uint8)], -1)
        b = np.stack([i1, np.roll(i1, 1, 1), rng.integers(0, 256, i1.shape, dtype=np.uint8)], -1)
    p = params(n_levels=2, n_warp=2, n_iter=5)
    s = run_gpu(a, b, mask, tv, cv, p, True)
    r = ref.run_ref(a, b, mask, tv, cv, p, True, fma=False)
    _exact(s.copy1DDisparityToHost(), r.copy1DDisparityToHost(), "u")
    r.close()


@pytest.mark.parametrize("masked", [True, False], ids=["masked", "plain"])
def test_cpu_oracle_matches_reference_build(gpu, ref, masked):
    """Pins the CPU float32 oracle (the checker of every other test) to the reference itself."""
    i0, i1, mask, tv, cv = random_case(130, 101, seed=130 * 7 + 101)
    p = params(n_levels=2, n_warp=2, n_iter=7)
    o = run_oracle(i0, i1, mask, tv, cv, p, masked, precision=32)
    r = ref.run_ref(i0, i1, mask, tv, cv, p, masked, fma=False)
    st = diff_stats(o.get("u"), r.copy1DDisparityToHost())
    r.close()
    assert st["max"] <= TOL_MAX, st
