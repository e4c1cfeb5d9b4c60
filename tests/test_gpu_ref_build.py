"""The drop-in path against the reference's OWN CUDA solver, built from its unmodified sources.

oracle/Makefile.ref compiles menandro/vfs stereotgv/*.cu (with the stand-ins of
oracle/refcompat/ for the texture-reference API CUDA 12 removed, helper_cuda.h and the few
OpenCV calls) into oracle/_ref/.  These tests run that build and the vfs_b200 drop-in path on
the same inputs and compare their outputs.

Two builds of the reference are compared:
* ``nofma``: compiled with -fmad=false, the contraction rule of the vfs_b200 library.  The two
  then evaluate the same float operations in the same order, and the only arithmetic that
  differs is the tensor weight exp(-beta |grad I|^gamma), where the reference calls CUDA's
  expf / powf and vfs_b200 uses its own exp / log construction.  Bar: max |du| <= 1e-3 px.
* ``stock``: nvcc's default flags, multiply-add contraction on, as the reference ships.  Every
  a*b+c the compiler contracts rounds once instead of twice, so this build differs from the
  ``nofma`` build of the same sources by float32 rounding that 150 iterations per level
  amplify.

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


@pytest.mark.parametrize("fma", [False, True], ids=["nofma", "stock"])
@pytest.mark.parametrize("masked", [True, False], ids=["masked", "plain"])
@pytest.mark.parametrize("size", [(67, 53), (96, 64), (130, 101)])
def test_small_cases_match_reference_build(gpu, ref, size, masked, fma):
    w, h = size
    i0, i1, mask, tv, cv = random_case(w, h, seed=w * 7 + h)
    p = params(n_levels=2, n_warp=2, n_iter=7)
    s = run_gpu(i0, i1, mask, tv, cv, p, masked)
    r = ref.run_ref(i0, i1, mask, tv, cv, p, masked, fma=fma)
    for name, got, want in (("u", s.copy1DDisparityToHost(), r.copy1DDisparityToHost()),
                            ("warpUV", s.copyDisparityToHost(), r.copyDisparityToHost())):
        st = diff_stats(got, want)
        assert st["max"] <= TOL_MAX, (name, st)
    r.close()


@pytest.mark.parametrize("masked", [True, False], ids=["masked", "plain"])
@pytest.mark.parametrize("wh", [(424, 400), (848, 800)])
def test_benchmark_sizes_match_reference_build(gpu, ref, wh, masked):
    """The synthetic fisheye workloads at 424x400 and 848x800 with the benchmark's solver
    settings (4 / 5 levels x 3 warps x 50 iterations): max |du| over every pixel."""
    from vfs_b200 import synth
    w, h = wh
    pair = synth.make_pair(w, h, seed=1000 + w)
    sp = synth.SOLVER_PARAMS
    p = params(beta=sp["beta"], gamma=sp["gamma"], n_levels=synth.n_levels_for(w), n_warp=sp["nWarpIters"],
               n_iter=sp["nSolverIters"], limit_range=synth.LIMIT_RANGE)
    u = run_gpu(pair.i0, pair.i1, pair.mask, pair.tv, pair.cv, p, masked).copy1DDisparityToHost()
    r = ref.run_ref(pair.i0, pair.i1, pair.mask, pair.tv, pair.cv, p, masked, fma=False)
    st = diff_stats(u, r.copy1DDisparityToHost())
    r.close()
    assert st["max"] <= TOL_MAX, st


def test_wang_config_matches_reference_build(gpu, ref):
    """The reference's own Wang fixture and parameters (test_vfs/main.cpp:270-281)."""
    d = np.load(os.path.join(os.path.dirname(__file__), "golden", "wang_half", "wang_half.npz"))
    p = params(beta=9.0, gamma=0.85, n_levels=5, n_warp=20, n_iter=10, limit_range=0.1)
    mask = d["mask_u8"].astype(np.float32) / 255.0
    u = run_gpu(d["i0"], d["i1"], mask, d["tv"], d["cv"], p, True).copy1DDisparityToHost()
    r = ref.run_ref(d["i0"], d["i1"], mask, d["tv"], d["cv"], p, True, fma=False)
    st = diff_stats(u, r.copy1DDisparityToHost())
    r.close()
    assert st["max"] <= TOL_MAX, st


def test_state_across_frames_matches_reference_build(gpu, ref):
    """Three frames through one instance: stale masked-out values carry over in both."""
    i0, i1, mask, tv, cv = random_case(72, 60, seed=11)
    p = params(n_levels=2, n_warp=2, n_iter=4)
    s = run_gpu(i0, i1, mask, tv, cv, p, True, frames=3)
    r = ref.run_ref(i0, i1, mask, tv, cv, p, True, frames=3, fma=False)
    st = diff_stats(s.copy1DDisparityToHost(), r.copy1DDisparityToHost())
    r.close()
    assert st["max"] <= TOL_MAX, st


def test_output_copies_match_reference_build(gpu, ref):
    """copyDisparityToHost, copyWarpedImageToHost, copyDisparityVisToHost (FlowToHSV) and
    copyStereoToHost (ConvertKB) against the reference's own kernels."""
    i0, i1, mask, tv, cv = random_case(96, 64, seed=21)
    p = params(n_levels=2, n_warp=2, n_iter=6)
    s = run_gpu(i0, i1, mask, tv, cv, p, True)
    r = ref.run_ref(i0, i1, mask, tv, cv, p, True, fma=False)
    flow = s.copyDisparityToHost()
    assert diff_stats(flow, r.copyDisparityToHost())["max"] <= TOL_MAX
    assert diff_stats(s.copyWarpedImageToHost(), r.copyWarpedImageToHost())["max"] <= 1e-5
    # The output kernels are compared on identical input: the reference instance is given the
    # drop-in path's flow before its FlowToHSV and ConvertKB run.
    r.set_plane("warpUV", flow)
    for scale in (1.0, 4.0, 20.0):
        st = diff_stats(s.copyDisparityVisToHost(scale), r.copyDisparityVisToHost(scale))
        assert st["max"] <= 1e-6, (scale, st)
    kb = (45.0, 45.0, 48.0, 32.0, 0.3, -0.1, 0.05, -0.01, 0.064, 0.0, 0.0)
    d_s, X_s = s.copyStereoToHost(*kb)
    d_r, X_r = r.copyStereoToHost(*kb)
    fin = np.isfinite(d_r)
    assert np.array_equal(fin, np.isfinite(d_s))
    rel = np.abs(d_s - d_r)[fin] / np.maximum(np.abs(d_r[fin]), 1e-6)
    assert rel.max() < 1e-5, rel.max()
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
    st = diff_stats(s.copy1DDisparityToHost(), r.copy1DDisparityToHost())
    r.close()
    assert st["max"] <= TOL_MAX, st


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
