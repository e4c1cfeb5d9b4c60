"""Warm starts, whole-state export / import, and allocation failures, on the GPU."""
import ctypes

import numpy as np
import pytest

from tests.helpers import params, random_case

pytestmark = pytest.mark.gpu


def _solver(i0, mask, tv, cv, p, fused, half=False):
    from vfs_b200.stereotgv import StereoTgv
    s = StereoTgv()
    s.set_solve_path(fused, half)
    s.limitRange = p["limit_range"]
    h, w = i0.shape
    s.initialize(w, h, p["beta"], p["gamma"], p["alpha0"], p["alpha1"], p["tsl"], p["lam"], p["n_levels"],
                 p["f_scale"], p["n_warp"], p["n_iter"])
    s.copyMaskToDevice(mask)
    s.loadVectorFields(tv, cv)
    return s


def _frames(w, h, n, seed):
    return [random_case(w, h, seed=seed + k)[:2] for k in range(n)]


@pytest.mark.parametrize("masked", [True, False], ids=["masked", "plain"])
@pytest.mark.parametrize("level", [0, 1, 2])
def test_warm_start_fused_matches_dropin(gpu, masked, level):
    """Warm starts from level 0, 1 and 2 (of 3): the fused FP32 path (with CUDA graphs) gives
    the drop-in path's bits over four frames; the first frame is a cold solve."""
    w, h = 130, 101
    _, _, mask, tv, cv = random_case(w, h, seed=71)
    p = params(n_levels=3, n_warp=2, n_iter=7)
    frames = _frames(w, h, 4, seed=300)
    a = _solver(frames[0][0], mask, tv, cv, p, fused=False)
    b = _solver(frames[0][0], mask, tv, cv, p, fused=True)
    c = _solver(frames[0][0], mask, tv, cv, p, fused=False)  # cold reference
    a.set_warm_start(level)
    b.set_warm_start(level)
    for k, (i0, i1) in enumerate(frames):
        for s in (a, b, c):
            s.copyImagesToDevice(i0, i1)
            (s.solveStereoForwardMasked if masked else s.solveStereoForward)()
        ua, ub, uc = a.copy1DDisparityToHost(), b.copy1DDisparityToHost(), c.copy1DDisparityToHost()
        assert np.array_equal(ua, ub), k
        if k == 0:
            assert np.array_equal(ua, uc)  # nothing to start from yet
        assert np.isfinite(ua).all()


def test_warm_start_continues_from_the_previous_disparity(gpu):
    """The same frame solved again and again with a warm start from the coarsest level: each
    solve continues from the last one, so the change from one solve to the next shrinks."""
    from vfs_b200 import synth
    w, h = 424, 400
    pair = synth.make_pair(w, h, seed=6)
    sp = synth.SOLVER_PARAMS
    L = synth.n_levels_for(w)
    p = params(beta=sp["beta"], gamma=sp["gamma"], n_levels=L, n_warp=sp["nWarpIters"], n_iter=sp["nSolverIters"],
               limit_range=synth.LIMIT_RANGE)
    s = _solver(pair.i0, pair.mask, pair.tv, pair.cv, p, fused=True, half=True)
    s.set_warm_start(L - 1)
    m = pair.mask > 0
    us = []
    for _ in range(4):
        s.copyImagesToDevice(pair.i0, pair.i1)
        s.solveStereoForwardMasked()
        us.append(s.copy1DDisparityToHost())
    steps = [float(np.abs(us[k + 1] - us[k])[m].mean()) for k in range(3)]
    assert all(np.isfinite(steps)) and steps[2] < steps[0], steps


@pytest.mark.parametrize("fused,half", [(False, False), (True, False), (True, True)], ids=["plain", "fp32", "fp16"])
def test_export_import_continues_bit_for_bit(gpu, fused, half):
    """Two frames on handle A, its state exported and imported into a fresh handle B (same
    size and levels, nothing else uploaded): B's third frame equals A's."""
    from vfs_b200.stereotgv import StereoTgv
    w, h = 97, 71
    _, _, mask, tv, cv = random_case(w, h, seed=81)
    p = params(n_levels=2, n_warp=2, n_iter=5)
    frames = _frames(w, h, 3, seed=400)
    a = _solver(frames[0][0], mask, tv, cv, p, fused=fused, half=half)
    a.set_warm_start(1)
    for i0, i1 in frames[:2]:
        a.copyImagesToDevice(i0, i1)
        a.solveStereoForwardMasked()
    st = a.export_state()
    b = StereoTgv()
    b.set_solve_path(fused, half)
    b.limitRange = p["limit_range"]
    b.initialize(w, h, p["beta"], p["gamma"], p["alpha0"], p["alpha1"], p["tsl"], p["lam"], p["n_levels"],
                 p["f_scale"], p["n_warp"], p["n_iter"])
    b.set_warm_start(1)
    b.import_state(st)
    # the imported warped image reads back as exported (half values widened in the FP16 form)
    assert np.array_equal(a.copyWarpedImageToHost(), b.copyWarpedImageToHost())
    for s in (a, b):
        s.copyImagesToDevice(*frames[2])
        s.solveStereoForwardMasked()
    assert np.array_equal(a.copy1DDisparityToHost(), b.copy1DDisparityToHost())
    assert np.array_equal(a.copyDisparityToHost(), b.copyDisparityToHost())


def test_import_refuses_another_geometry(gpu):
    from vfs_b200.stereotgv import StereoTgv, VfsError
    _, _, mask, tv, cv = random_case(64, 48, seed=1)
    p = params(n_levels=2, n_warp=1, n_iter=2)
    a = _solver(np.zeros((48, 64), np.uint8), mask, tv, cv, p, fused=False)
    st = a.export_state()
    b = StereoTgv()
    b.initialize(64, 50, p["beta"], p["gamma"], p["alpha0"], p["alpha1"], p["tsl"], p["lam"], 2, 2.0, 1, 2)
    with pytest.raises(VfsError):
        b.import_state(st)
    with pytest.raises(VfsError):
        b.import_state(st[:100])


def test_allocation_failure_is_reported_and_leaks_nothing(gpu):
    """An injected device-pool allocation failure makes initialize return VFS_ERR_NOMEM with
    nothing left allocated, and the handle initialises normally afterwards."""
    import torch
    from vfs_b200._native import lib
    from vfs_b200.stereotgv import StereoTgv, VfsError
    L = lib()
    s = StereoTgv()
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    assert L.vfs_debug_fail_allocation(1) == 0
    with pytest.raises(VfsError) as e:
        s.initialize(424, 400, 10.0, 0.8, 17.0, 1.2, 1.0, 5.0, 4, 2.0, 1, 1)
    assert e.value.status == -4
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert free1 >= free0 - (2 << 20)  # nothing of the failed pool stays allocated
    s.initialize(424, 400, 10.0, 0.8, 17.0, 1.2, 1.0, 5.0, 4, 2.0, 1, 1)
    # the fused pool's allocation fails the same way on the first fused solve
    s.set_solve_path(True, True)
    _, _, mask, tv, cv = random_case(424, 400, seed=2)
    s.copyMaskToDevice(mask)
    s.loadVectorFields(tv, cv)
    s.copyImagesToDevice(np.zeros((400, 424), np.uint8), np.zeros((400, 424), np.uint8))
    assert L.vfs_debug_fail_allocation(1) == 0
    with pytest.raises(VfsError) as e:
        s.solveStereoForwardMasked()
    assert e.value.status == -4
    s.solveStereoForwardMasked()  # the retry allocates and solves
    assert np.isfinite(s.copy1DDisparityToHost()).all()
    assert L.vfs_debug_fail_allocation(0) == 0


def test_graph_cache_drops_graphs_of_old_masks(gpu):
    """Every new mask renews the handle's generation; the graphs captured under the old one are
    destroyed on the next solve instead of accumulating."""
    from vfs_b200._native import lib
    w, h = 96, 64
    i0, i1, mask, tv, cv = random_case(w, h, seed=90)
    p = params(n_levels=2, n_warp=1, n_iter=3)
    s = _solver(i0, mask, tv, cv, p, fused=True, half=True)
    counts = []
    for k in range(6):
        m = mask.copy()
        m[:, : 2 + k] = 0  # a different mask each time
        s.copyMaskToDevice(m)
        for _ in range(2):  # both pointer states of the solve
            s.copyImagesToDevice(i0, i1)
            s.solveStereoForwardMasked()
        counts.append(lib().vfs_cached_graphs(s.handle))
    assert max(counts) <= 4, counts


def test_cpp_dropin_header_solves_on_the_gpu(gpu, tmp_path):
    """A program written against include/stereotgv.h (the reference's class) solves a pair on
    the GPU and gets the same disparity as the Python binding of the same library."""
    import os
    import subprocess
    from vfs_b200.build import LIB
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    w, h = 96, 64
    i0, i1, mask, tv, cv = random_case(w, h, seed=77)
    p = params(n_levels=2, n_warp=2, n_iter=6)
    for name, arr in (("i0", i0), ("i1", i1), ("mask", mask.astype(np.float32)), ("tv", tv.astype(np.float32)),
                      ("cv", cv.astype(np.float32))):
        arr.tofile(str(tmp_path / f"{name}.bin"))
    src = tmp_path / "solve.cpp"
    src.write_text(r"""
#include "stereotgv.h"
#include <cstdio>
#include <cstdlib>
#include <vector>
template <class T> static std::vector<T> load(const char* dir, const char* name, size_t n) {
  std::vector<T> v(n);
  char path[512];
  std::snprintf(path, sizeof(path), "%s/%s.bin", dir, name);
  FILE* f = std::fopen(path, "rb");
  if (!f || std::fread(v.data(), sizeof(T), n, f) != n) { std::printf("read %s failed\n", path); std::exit(3); }
  std::fclose(f);
  return v;
}
int main(int argc, char** argv) {
  const int W = 96, H = 64;
  const char* dir = argv[1];
  auto i0 = load<unsigned char>(dir, "i0", W * H), i1 = load<unsigned char>(dir, "i1", W * H);
  auto mask = load<float>(dir, "mask", W * H);
  auto tv = load<float>(dir, "tv", 2 * W * H), cv = load<float>(dir, "cv", 2 * W * H);
  StereoTgv s;                      // the reference's class and call sequence
  s.limitRange = 0.1f;
  int st = s.initialize(W, H, 10.0f, 0.8f, 17.0f, 1.2f, 1.0f, 5.0f, 2, 2.0f, 2, 6);
  if (!st) st = s.copyMaskToDevice(mask.data());
  if (!st) st = s.loadVectorFields(tv.data(), cv.data());
  if (!st) st = s.copyImagesToDevice(i0.data(), i1.data());
  if (!st) st = s.solveStereoForwardMasked();
  std::vector<float> u(W * H);
  if (!st) st = s.copy1DDisparityToHost(u.data());
  if (st) { std::printf("status %d\n", st); return 2; }
  char path[512];
  std::snprintf(path, sizeof(path), "%s/u.bin", dir);
  FILE* f = std::fopen(path, "wb");
  std::fwrite(u.data(), sizeof(float), u.size(), f);
  std::fclose(f);
  return 0;
}
""")
    exe = tmp_path / "solve"
    libdir = os.path.dirname(LIB)
    r = subprocess.run(["g++", "-std=c++17", f"-I{os.path.join(root, 'include')}", str(src), "-o", str(exe),
                        f"-L{libdir}", "-lvfs_b200", f"-Wl,-rpath,{libdir}"], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    r = subprocess.run([str(exe), str(tmp_path)], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stdout + r.stderr
    u_cpp = np.fromfile(str(tmp_path / "u.bin"), np.float32).reshape(h, w)
    from tests.helpers import run_gpu
    u_py = run_gpu(i0, i1, mask, tv, cv, p, True).copy1DDisparityToHost()
    assert np.array_equal(u_cpp, u_py)
