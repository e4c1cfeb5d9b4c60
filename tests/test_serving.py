"""Host-side logic of the serving loop (no GPU)."""
import numpy as np

from vfs_b200.serving import poisson_schedule


def test_poisson_schedule_is_seeded_ordered_and_complete():
    rates = {0: 30.0, 1: 30.0, 2: 15.0}
    n = {0: 20, 1: 20, 2: 10}
    a = poisson_schedule(rates, n, seed=3)
    b = poisson_schedule(rates, n, seed=3)
    assert a == b
    assert [t for t, _, _ in a] == sorted(t for t, _, _ in a)
    for sid in rates:
        ks = [k for _, s, k in a if s == sid]
        assert ks == list(range(n[sid]))  # each stream's frames arrive in order
    # mean inter-arrival close to 1 / rate
    t0 = [t for t, s, _ in a if s == 0]
    assert 0.5 / 30 < np.mean(np.diff(t0)) < 2.0 / 30


def test_footprint_estimate_without_gpu():
    from vfs_b200._native import lib
    L = lib()
    big = L.vfs_estimate_device_bytes(848, 800, 5, 2.0, 32, 1)
    small = L.vfs_estimate_device_bytes(424, 400, 4, 2.0, 32, 1)
    plain = L.vfs_estimate_device_bytes(848, 800, 5, 2.0, 32, 0)
    assert big > plain > small > 0
    assert 3.5 < big / small < 4.5
    assert L.vfs_estimate_device_bytes(0, 800, 5, 2.0, 32, 1) == 0
