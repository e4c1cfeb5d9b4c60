"""Host-side helpers of bench.py (no GPU): the accuracy summary every configuration reports."""
import importlib.util
import os

import numpy as np


def _bench():
    path = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "bench.py")
    spec = importlib.util.spec_from_file_location("bench_under_test", path)
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def test_error_stats_counts_only_pixels_inside_the_masks():
    b = _bench()
    ref = [np.zeros((4, 5)), np.ones((2, 3))]
    u = [np.zeros((4, 5), np.float32), np.ones((2, 3), np.float32)]
    u[0][0, 0] = 2.5     # inside mask 0: one pixel beyond 1 px
    u[0][3, 4] = 100.0   # outside mask 0: ignored
    u[1][1, 2] = 1.25    # inside mask 1
    masks = [np.ones((4, 5), np.float32), np.ones((2, 3), np.float32)]
    masks[0][3, 4] = 0.0
    st = b.error_stats(u, ref, masks)
    n = 19 + 6
    assert st["frames"] == 2
    assert st["max_abs_px"] == 2.5
    assert abs(st["mean_abs_px"] - (2.5 + 0.25) / n) < 1e-12
    assert abs(st["bad_1px_rate"] - 1.0 / n) < 1e-12


def test_oracle_thread_count_is_set_and_restored():
    """The CPU baseline's single-thread frame limits the oracle to one OpenMP thread and puts
    the previous count back."""
    from oracle.oracle import build, set_threads
    build()
    prev = set_threads(1)
    assert prev >= 1
    assert set_threads(prev) == 1
    assert set_threads(0) == prev  # 0 leaves the count as it is
