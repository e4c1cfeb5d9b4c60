"""Shared runners: the CUDA solver (through the C ABI) and the oracle on the same inputs."""
import numpy as np

from oracle.oracle import OracleStereoTgv


def random_case(w, h, seed, n_levels=2, circle=True):
    """Random smooth-ish textures, a circular mask and unit translation field for small parity cases."""
    rng = np.random.default_rng(seed)
    from scipy.ndimage import gaussian_filter
    base = gaussian_filter(rng.uniform(0, 255, (h + 8, w + 8)), 1.2)
    i0 = np.clip(base[4:4 + h, 4:4 + w], 0, 255).astype(np.uint8)
    i1 = np.clip(np.roll(base, 2, axis=1)[4:4 + h, 3:3 + w] + rng.normal(0, 2, (h, w)), 0, 255).astype(np.uint8)
    yy, xx = np.mgrid[0:h, 0:w]
    r = np.hypot(xx - (w - 1) / 2, yy - (h - 1) / 2)
    mask = (r < 0.45 * min(w, h)).astype(np.float32) if circle else np.ones((h, w), np.float32)
    ang = rng.uniform(-0.2, 0.2, (h, w))
    tv = np.stack([-np.cos(ang), np.sin(ang)], -1).astype(np.float32)
    cv = rng.normal(0, 0.7, (h, w, 2)).astype(np.float32)
    return i0, i1, mask, tv, cv


def params(beta=10.0, gamma=0.8, alpha0=17.0, alpha1=1.2, tsl=1.0, lam=5.0, n_levels=2, f_scale=2.0,
           n_warp=2, n_iter=5, limit_range=0.1):
    return dict(beta=beta, gamma=gamma, alpha0=alpha0, alpha1=alpha1, tsl=tsl, lam=lam, n_levels=n_levels,
                f_scale=f_scale, n_warp=n_warp, n_iter=n_iter, limit_range=limit_range)


def run_gpu(i0, i1, mask, tv, cv, p, masked=True, frames=1, solver=None, portable=False):
    """The drop-in solve through the C ABI.  portable=True computes the tensor weight with the
    portable exp / log that the CPU oracle restates bit for bit (the comparisons with the
    oracle use it); the default calls CUDA's expf / powf as the reference does."""
    from vfs_b200.stereotgv import StereoTgv
    h, w = i0.shape[:2]
    s = solver or StereoTgv()
    s.set_tensor_math(portable)
    s.limitRange = p["limit_range"]
    s.initialize(w, h, p["beta"], p["gamma"], p["alpha0"], p["alpha1"], p["tsl"], p["lam"], p["n_levels"],
                 p["f_scale"], p["n_warp"], p["n_iter"])
    s.copyMaskToDevice(mask)
    s.loadVectorFields(tv, cv)
    for _ in range(frames):
        s.copyImagesToDevice(i0, i1)
        (s.solveStereoForwardMasked if masked else s.solveStereoForward)()
    return s


def run_oracle(i0, i1, mask, tv, cv, p, masked=True, precision=32, frames=1):
    h, w = i0.shape
    o = OracleStereoTgv(precision)
    o.set_limit_range(p["limit_range"])
    o.initialize(w, h, p["beta"], p["gamma"], p["alpha0"], p["alpha1"], p["tsl"], p["lam"], p["n_levels"],
                 p["f_scale"], p["n_warp"], p["n_iter"])
    o.copy_mask_to_device(mask)
    o.load_vector_fields(tv, cv)
    for _ in range(frames):
        o.copy_images_to_device(i0, i1)
        (o.solve_stereo_forward_masked if masked else o.solve_stereo_forward)()
    return o


def diff_stats(a, b, m=None):
    d = np.abs(np.asarray(a, np.float64) - np.asarray(b, np.float64))
    if m is not None:
        d = d[m]
    return dict(max=float(d.max()), mean=float(d.mean()), p99=float(np.percentile(d, 99)))
