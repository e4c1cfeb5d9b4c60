"""GPU tests of the entry points around the solve: histogram equalisation, the
reference-shaped Create / Init / SolveStereo, the f32 and colour image overloads,
ConvertKB (copyStereoToHost) and the disparity colour map."""
import ctypes
import os

import numpy as np
import pytest

from tests.helpers import diff_stats, params, random_case, run_gpu, run_oracle

pytestmark = pytest.mark.gpu
FIX = os.path.join(os.path.dirname(__file__), "golden", "equalize", "equalize.npz")


def test_equalize_hist_matches_cv2(gpu):
    import torch
    from vfs_b200._native import lib
    d = np.load(FIX)
    L = lib()
    for name in d["names"]:
        img = d[f"{name}_in"]
        src = torch.from_numpy(np.ascontiguousarray(img)).cuda()
        dst = torch.empty_like(src)
        st = torch.cuda.current_stream()
        assert L.vfs_equalize_hist_u8(ctypes.c_void_p(src.data_ptr()), ctypes.c_void_p(dst.data_ptr()), img.size,
                                      ctypes.c_void_p(st.cuda_stream)) == 0
        torch.cuda.synchronize()
        assert np.array_equal(dst.cpu().numpy(), d[f"{name}_out"]), name
        # in place
        assert L.vfs_equalize_hist_u8(ctypes.c_void_p(src.data_ptr()), ctypes.c_void_p(src.data_ptr()), img.size,
                                      ctypes.c_void_p(st.cuda_stream)) == 0
        torch.cuda.synchronize()
        assert np.array_equal(src.cpu().numpy(), d[f"{name}_out"]), name


def _write_png_gray(path, img):
    import cv2
    assert cv2.imwrite(str(path), img)


def test_reference_dll_entry_points(gpu, tmp_path):
    """Create / Init (PNG mask, .flo fields) / SolveStereo against the same steps through the
    class interface: equalise (host restatement), copy u8 images, masked solve."""
    from oracle.equalize import equalize_hist
    from vfs_b200 import fields
    from vfs_b200._native import lib
    from vfs_b200.stereotgv import StereoTgv
    i0, i1, mask, tv, cv = random_case(96, 80, seed=21)
    _write_png_gray(tmp_path / "mask.png", (mask * 255).astype(np.uint8))
    fields.write_flo(tmp_path / "tv.flo", tv)
    fields.write_flo(tmp_path / "cv.flo", cv)
    L = lib()
    h = L.Create()
    assert h
    p = params(n_levels=2, n_warp=2, n_iter=6)
    L.Init(h, 96, 80, p["beta"], p["gamma"], p["alpha0"], p["alpha1"], p["tsl"], p["lam"], p["n_levels"],
           p["f_scale"], p["n_warp"], p["n_iter"], 100.0, 0.064, str(tmp_path / "mask.png").encode(),
           str(tmp_path / "tv.flo").encode(), str(tmp_path / "cv.flo").encode())
    assert (L.vfs_last_error(h) or b"") == b"", L.vfs_last_error(h)
    out = np.zeros((80, 96), np.uint8)
    a, b = np.ascontiguousarray(i0), np.ascontiguousarray(i1)
    L.SolveStereo(h, a.ctypes.data_as(ctypes.c_void_p), b.ctypes.data_as(ctypes.c_void_p),
                  out.ctypes.data_as(ctypes.c_void_p), 96, 80, 10.0)
    assert (L.vfs_last_error(h) or b"") == b""
    u_dll = np.zeros((80, 96), np.float32)
    assert L.vfs_copy_1d_disparity_to_host(h, u_dll.ctypes.data_as(ctypes.c_void_p)) == 0
    L.vfs_destroy(h)
    # same steps through the class
    m8 = (mask * 255).astype(np.uint8).astype(np.float32) * np.float32(1.0 / 255.0)
    s = run_gpu(equalize_hist(i0), equalize_hist(i1), m8, tv, cv, dict(p, limit_range=1.0), True)
    assert np.array_equal(u_dll, s.copy1DDisparityToHost())
    # the output depth image is defined: round(255 * Z / maxDepth), Z = focal * |baseline| / u
    z = np.where(u_dll > 0, 100.0 * 0.064 / np.maximum(u_dll, 1e-30), 0.0)
    exp = np.clip(np.rint(255.0 * z / 10.0), 0, 255)
    assert np.abs(exp.astype(int) - out.astype(int)).max() <= 1


def test_init_reports_missing_files(gpu, tmp_path):
    from vfs_b200._native import lib
    L = lib()
    h = L.Create()
    L.Init(h, 64, 48, 10.0, 0.8, 17.0, 1.2, 1.0, 5.0, 2, 2.0, 1, 1, 100.0, 0.064, b"/nonexistent/mask.png",
           b"/nonexistent/tv.flo", b"/nonexistent/cv.flo")
    assert b"mask" in (L.vfs_last_error(h) or b"")
    L.vfs_destroy(h)


@pytest.mark.parametrize("kind", ["f32", "u8c3"])
def test_image_overloads(gpu, kind):
    i0, i1, mask, tv, cv = random_case(72, 60, seed=31)
    p = params(n_levels=2, n_warp=1, n_iter=4)
    if kind == "f32":
        a, b = i0.astype(np.float32) / 255.0, i1.astype(np.float32) / 255.0
        oa, ob = a, b
    else:
        rng = np.random.default_rng(3)
        a = rng.integers(0, 256, (60, 72, 3), dtype=np.uint8)
        b = rng.integers(0, 256, (60, 72, 3), dtype=np.uint8)
        # imageConverter.cu:27-41: ((r + g + b) / 3) / 256 in float
        f = lambda x: ((x[..., 0].astype(np.float32) + x[..., 1].astype(np.float32) + x[..., 2].astype(np.float32))
                       / np.float32(3)) / np.float32(256)
        oa, ob = f(a), f(b)
    s = run_gpu(a, b, mask, tv, cv, p, True, portable=True)
    o = run_oracle(oa, ob, mask, tv, cv, p, True, precision=32)
    assert diff_stats(s.copy1DDisparityToHost(), o.get("u"))["max"] <= 1e-6


def test_convert_kb_and_colour_map(gpu):
    d = np.load(os.path.join(os.path.dirname(__file__), "golden", "wang_half", "wang_half.npz"))
    mask = d["mask_u8"].astype(np.float32) / 255.0
    p = params(beta=9.0, gamma=0.85, n_levels=3, n_warp=2, n_iter=5, limit_range=0.1)
    s = run_gpu(d["i0"], d["i1"], mask, d["tv"], d["cv"], p, True, portable=True)
    o = run_oracle(d["i0"], d["i1"], mask, d["tv"], d["cv"], p, True, precision=32)
    kb = (143.259, 143.301, 211.571, 196.661, -0.00727452, 0.05200624, -0.0510574, 0.01108238, -0.0639505,
          0.000184912, -0.0000766807)
    depth, X = s.copyStereoToHost(*kb)
    od, oX = o.convert_kb(*kb)
    m = (mask > 0) & np.isfinite(od) & (np.abs(od) < 100)
    rel = np.abs(depth[m] - od[m]) / np.maximum(np.abs(od[m]), 1e-6)
    assert np.median(rel) < 1e-5 and np.percentile(rel, 99) < 1e-3
    rgb = s.copyDisparityVisToHost(40.0)
    assert rgb.shape == (400, 424, 3) and np.isfinite(rgb).all() and rgb.min() >= 0 and rgb.max() <= 1.0
