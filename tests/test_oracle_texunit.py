"""The oracle's texture-unit model against samples recorded from B200 texture hardware."""
import os

import numpy as np

from oracle import oracle as O

FIX = os.path.join(os.path.dirname(__file__), "golden", "texunit", "texunit.npz")


def test_texture_model_matches_hardware_samples():
    d = np.load(FIX)
    total = mismatch = 0
    worst = 0.0
    for k in range(int(d["ncases"])):
        w, h, f2, lin = (int(x) for x in d[f"c{k}_meta"])
        r = O.tex_sample(d[f"c{k}_tex"], d[f"c{k}_xy"], bool(lin))
        o = d[f"c{k}_out"]
        assert r.shape == o.shape
        total += o.size
        mismatch += int((r != o).sum())
        # tolerance: one float32 ulp at the scale of the texels (results near zero come from
        # cancellation, so their own ulp is smaller than the accumulator's rounding step)
        scale = max(float(np.abs(d[f"c{k}_tex"]).max()), 1e-30)
        ulp = np.maximum(np.spacing(np.abs(o).astype(np.float32)), np.spacing(np.float32(scale))).astype(np.float64)
        err = np.abs(r.astype(np.float64) - o)
        assert np.all(err <= ulp + 1e-12), f"case {k}: error above 1 ulp"
        worst = max(worst, float(err.max()))
        if not lin:  # point sampling is index work: bit-exact
            assert np.array_equal(r, o), f"case {k}: point sampling differs"
    # addressing and weights are exact; only the final rounding of rare ties differs
    assert mismatch / total < 2e-4, (mismatch, total)


def test_texture_weights_grid_exact():
    # the one-hot parity textures give the four bilinear weights directly
    d = np.load(FIX)
    n = int(d["ncases"])
    for k in range(n - 7, n - 3):
        r = O.tex_sample(d[f"c{k}_tex"], d[f"c{k}_xy"], True)
        assert np.array_equal(r, d[f"c{k}_out"])
