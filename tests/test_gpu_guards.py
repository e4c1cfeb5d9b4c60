"""Out-of-bounds stores: every device plane of a handle is followed by a guard zone of a known
byte pattern (vfs_debug_check_guards).  Solves of odd and tall sizes, masked and plain, on the
drop-in path and every fused kernel variant, with warm starts, batches and every output kernel,
must leave all guard zones intact.  (compute-sanitizer is not available on this pool; these
zones, checked after small cases, stand in for its out-of-bounds store check.)"""
import numpy as np
import pytest

from tests.helpers import params, random_case

pytestmark = pytest.mark.gpu

VARIANTS = (0, 1, 2, 6, 7, 8, 9, 12, 13, 14, 15, 18, 19)
# odd sizes, a tall image (the masked tensor kernel's h > w case) and a level without row
# padding (stride = width) with an all-on mask
CASES = [(67, 53, 2, True), (130, 101, 3, True), (53, 97, 2, True), (64, 48, 2, False)]


def _make(i0, i1, mask, tv, cv, p, fused=False, half=False):
    from vfs_b200.stereotgv import StereoTgv
    s = StereoTgv()
    s.set_solve_path(fused, half)
    h, w = i0.shape
    s.limitRange = p["limit_range"]
    s.initialize(w, h, p["beta"], p["gamma"], p["alpha0"], p["alpha1"], p["tsl"], p["lam"], p["n_levels"],
                 p["f_scale"], p["n_warp"], p["n_iter"])
    s.copyMaskToDevice(mask)
    s.loadVectorFields(tv, cv)
    return s


def _solve(s, i0, i1, masked, frames=2):
    for _ in range(frames):
        s.copyImagesToDevice(i0, i1)
        (s.solveStereoForwardMasked if masked else s.solveStereoForward)()
    s.synchronize()


@pytest.mark.parametrize("masked", [True, False])
def test_dropin_path_stays_in_bounds(gpu, masked):
    for k, (w, h, L, circle) in enumerate(CASES):
        i0, i1, mask, tv, cv = random_case(w, h, seed=1300 + k, circle=circle)
        s = _make(i0, i1, mask, tv, cv, params(n_levels=L, n_warp=2, n_iter=5))
        _solve(s, i0, i1, masked)
        # every output kernel of the drop-in boundary
        s.copy1DDisparityToHost()
        s.copyDisparityToHost()
        s.copyWarpedImageToHost()
        s.copyDisparityVisToHost(40.0)
        s.copyStereoToHost(300.0, 300.0, w / 2.0, h / 2.0, 0.01, -0.002, 0.001, 0.0, -0.064, 0.0, 0.0)
        assert s.check_guards() == 0, (w, h, masked)


@pytest.mark.parametrize("half", [False, True])
def test_every_fused_variant_stays_in_bounds(gpu, half):
    for k, (w, h, L, circle) in enumerate(CASES):
        i0, i1, mask, tv, cv = random_case(w, h, seed=1400 + k, circle=circle)
        p = params(n_levels=L, n_warp=2, n_iter=11)
        for variant in VARIANTS:
            for masked in (True, False):
                s = _make(i0, i1, mask, tv, cv, p, fused=True, half=half)
                s.set_iteration_variant(variant)
                _solve(s, i0, i1, masked)
                assert s.check_guards() == 0, (w, h, variant, masked)


def test_warm_starts_and_batches_stay_in_bounds(gpu):
    from vfs_b200.stereotgv import StereoBatch
    members = []
    for half in (False, True):
        b = StereoBatch(half_storage=half)
        b.set_fine_concurrency(2)
        data = []
        for k, (w, h, L, circle) in enumerate(CASES):
            i0, i1, mask, tv, cv = random_case(w, h, seed=1500 + k, circle=circle)
            s = _make(i0, i1, mask, tv, cv, params(n_levels=L, n_warp=2, n_iter=6), fused=True, half=half)
            s.set_warm_start(0 if k % 2 else L - 1)
            b.add(s)
            members.append(s)
            data.append((i0, i1))
        for _ in range(3):
            b.solve_host(data)
    for s in members:
        assert s.check_guards() == 0
