"""Pin the oracle to the reference's own known-answer outputs.

test_vfs/z16.png and depth16.png were written by the reference demo's Wang test
(test_vfs/main.cpp:233-347): masked solve at 424x400 (5 levels, scale 2, 20 warps x 10
iterations, lambda 5, beta 9, gamma 0.85, alpha0 17, alpha1 1.2, limitRange 0.1) followed by
ConvertKB with the camera parameters at main.cpp:238-250 divided by the stereo scaling 2.
The oracle repeats that pipeline from the same inputs (tests/golden/wang_half).
"""
import os

import numpy as np
import pytest

from oracle.oracle import OracleStereoTgv

FIX = os.path.join(os.path.dirname(__file__), "golden", "wang_half", "wang_half.npz")
KB = dict(fx=286.518 / 2, fy=286.602 / 2, cx=423.142 / 2, cy=393.321 / 2, d1=-0.00727452, d2=0.05200624,
          d3=-0.05105740, d4=0.01108238, t1=-0.0639505, t2=0.000184912, t3=-0.0000766807)


def run_wang(precision):
    d = np.load(FIX)
    o = OracleStereoTgv(precision)
    o.set_limit_range(0.1)
    o.initialize(424, 400, 9.0, 0.85, 17.0, 1.2, 1.0, 5.0, 5, 2.0, 20, 10)
    o.copy_mask_to_device(d["mask_u8"].astype(np.float32) / 255.0)
    o.load_vector_fields(d["tv"], d["cv"])
    o.copy_images_to_device(d["i0"], d["i1"])
    o.solve_stereo_forward_masked()
    depth, X = o.convert_kb(*KB.values())
    return d, depth, X, o


def to16(a):
    a = np.nan_to_num(a * 256.0, nan=0.0, posinf=65535, neginf=0)
    return np.clip(np.round(a), 0, 65535).astype(np.uint16)


@pytest.mark.parametrize("precision", [32, 64])
def test_wang_known_answer(precision):
    d, depth, X, _ = run_wang(precision)
    m = d["mask_u8"] > 0
    for mine, ref in ((to16(X[:, :, 2]), d["z16"]), (to16(depth), d["depth16"])):
        a = mine[m].astype(np.float64) / 256
        b = ref[m].astype(np.float64) / 256
        both = (a > 0) & (b > 0) & (a < 255) & (b < 255)
        assert both.mean() > 0.99
        rel = np.abs(a[both] - b[both]) / b[both]
        assert np.median(rel) < 2e-3
        assert np.percentile(rel, 90) < 2e-2
        assert (mine[m] == ref[m]).mean() > 0.40
        assert ((a == 0) == (b == 0)).mean() > 0.999
