"""ctypes wrapper of the reference's own CUDA solver, built from its unmodified sources.

TEST INFRASTRUCTURE ONLY: imported by tests/ as the reference-build oracle.  The product
package ``vfs_b200`` never imports it.

``oracle/Makefile.ref`` compiles menandro/vfs ``stereotgv/*.cu`` in place (with the stand-ins in
``oracle/refcompat/``) into ``oracle/_ref/libvfs_ref.so`` (nvcc's default flags, multiply-add
contraction on, as the reference ships) and ``oracle/_ref/libvfs_ref_nofma.so`` (``-fmad=false``,
the vfs_b200 library's contraction rule).  The reference sources are needed only to build; the
built libraries run anywhere with a B200.

``RefStereoTgv`` mirrors the reference class (stereotgv/stereotgv.h:107-124) method for method.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_OUT = os.path.join(_HERE, "_ref")
DEFAULT_SOURCE = "/root/reference"
LIB_STOCK = os.path.join(_OUT, "libvfs_ref.so")
LIB_NOFMA = os.path.join(_OUT, "libvfs_ref_nofma.so")
_libs: dict = {}


def source_dir() -> str:
    return os.environ.get("VFS_REFERENCE_SOURCE", DEFAULT_SOURCE)


def build(force: bool = False) -> bool:
    """Build both variants when the reference sources are present.  Returns whether the
    libraries exist afterwards (prebuilt ones are kept when the sources are absent)."""
    src = source_dir()
    if os.path.isdir(os.path.join(src, "stereotgv")):
        if force:
            subprocess.run(["make", "-s", "-C", _HERE, "-f", "Makefile.ref", "clean"], check=True)
        subprocess.run(["make", "-s", "-j8", "-C", _HERE, "-f", "Makefile.ref", f"REF={src}"], check=True)
    return available()


def available() -> bool:
    return os.path.exists(LIB_STOCK) and os.path.exists(LIB_NOFMA)


def lib(fma: bool = True):
    path = LIB_STOCK if fma else LIB_NOFMA
    if path in _libs:
        return _libs[path]
    if not os.path.exists(path):
        raise FileNotFoundError(f"{path} is missing: build it with oracle/Makefile.ref")
    L = ctypes.CDLL(path)
    vp, i, f = ctypes.c_void_p, ctypes.c_int, ctypes.c_float
    L.vref_create.restype = vp
    L.vref_destroy.argtypes = [vp]
    L.vref_last_error.restype = ctypes.c_char_p
    L.vref_initialize.argtypes = [vp, i, i, f, f, f, f, f, f, i, f, i, i]
    L.vref_set_limit_range.argtypes = [vp, f]
    L.vref_stride.argtypes = [vp]
    L.vref_load_vector_fields.argtypes = [vp, vp, vp]
    L.vref_copy_mask.argtypes = [vp, vp]
    L.vref_mask_touches_border.argtypes = [vp]
    L.vref_copy_images_u8.argtypes = [vp, vp, vp]
    L.vref_copy_images_mat.argtypes = [vp, vp, vp, i]
    L.vref_solve.argtypes = [vp, i]
    L.vref_copy_disparity_1d.argtypes = [vp, vp]
    L.vref_copy_disparity_2d.argtypes = [vp, vp]
    L.vref_copy_disparity_vis.argtypes = [vp, vp, f]
    L.vref_copy_warped_image.argtypes = [vp, vp]
    L.vref_copy_stereo.argtypes = [vp, vp, vp] + [f] * 11
    L.vref_get_plane.argtypes = [vp, ctypes.c_char_p, vp, i]
    L.vref_set_plane.argtypes = [vp, ctypes.c_char_p, vp, i]
    _libs[path] = L
    return L


def _p(a: np.ndarray):
    return a.ctypes.data_as(ctypes.c_void_p)


class RefStereoTgv:
    """The reference's StereoTgv, run on the GPU from the reference build."""

    def __init__(self, fma: bool = True):
        self._L = lib(fma)
        self._h = self._L.vref_create()
        if not self._h:
            raise MemoryError("vref_create failed")
        self.width = self.height = 0

    def close(self):
        if self._h:
            self._L.vref_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _ok(self, rc: int):
        if rc != 0:
            raise RuntimeError("reference build: " + self._L.vref_last_error().decode())

    # -- the reference's methods -----------------------------------------------------------
    def initialize(self, w, h, beta, gamma, alpha0, alpha1, tsl, lam, n_levels, f_scale, n_warp, n_iter):
        self.width, self.height = w, h
        self._ok(self._L.vref_initialize(self._h, w, h, beta, gamma, alpha0, alpha1, tsl, lam, n_levels,
                                         f_scale, n_warp, n_iter))

    def set_limit_range(self, v: float):
        self._L.vref_set_limit_range(self._h, float(v))

    @property
    def stride(self) -> int:
        return self._L.vref_stride(self._h)

    def loadVectorFields(self, tv: np.ndarray, cv: np.ndarray):
        tv = np.ascontiguousarray(tv, np.float32)
        cv = np.ascontiguousarray(cv, np.float32)
        assert tv.shape == cv.shape == (self.height, self.width, 2)
        self._ok(self._L.vref_load_vector_fields(self._h, _p(tv), _p(cv)))

    def copyMaskToDevice(self, mask: np.ndarray):
        m = np.ascontiguousarray(mask, np.float32)
        assert m.shape == (self.height, self.width)
        self._ok(self._L.vref_copy_mask(self._h, _p(m)))

    def copyImagesToDevice(self, i0: np.ndarray, i1: np.ndarray):
        """uint8 (h, w) goes through the uchar* overload; float32 (h, w) and uint8 (h, w, 3)
        through the cv::Mat overload."""
        i0 = np.ascontiguousarray(i0)
        i1 = np.ascontiguousarray(i1)
        assert i0.shape == i1.shape and i0.dtype == i1.dtype
        if i0.dtype == np.uint8 and i0.ndim == 2:
            self._ok(self._L.vref_copy_images_u8(self._h, _p(i0), _p(i1)))
        elif i0.dtype == np.float32 and i0.ndim == 2:
            self._ok(self._L.vref_copy_images_mat(self._h, _p(i0), _p(i1), 1))
        elif i0.dtype == np.uint8 and i0.ndim == 3 and i0.shape[2] == 3:
            self._ok(self._L.vref_copy_images_mat(self._h, _p(i0), _p(i1), 2))
        else:
            raise TypeError(f"unsupported image {i0.dtype} {i0.shape}")

    def solveStereoForwardMasked(self):
        self._ok(self._L.vref_solve(self._h, 1))

    def solveStereoForward(self):
        self._ok(self._L.vref_solve(self._h, 0))

    def copy1DDisparityToHost(self) -> np.ndarray:
        out = np.empty((self.height, self.width), np.float32)
        self._ok(self._L.vref_copy_disparity_1d(self._h, _p(out)))
        return out

    def copyDisparityToHost(self) -> np.ndarray:
        out = np.empty((self.height, self.width, 2), np.float32)
        self._ok(self._L.vref_copy_disparity_2d(self._h, _p(out)))
        return out

    def copyDisparityVisToHost(self, flow_scale: float) -> np.ndarray:
        out = np.empty((self.height, self.width, 3), np.float32)
        self._ok(self._L.vref_copy_disparity_vis(self._h, _p(out), float(flow_scale)))
        return out

    def copyWarpedImageToHost(self) -> np.ndarray:
        out = np.empty((self.height, self.width), np.float32)
        self._ok(self._L.vref_copy_warped_image(self._h, _p(out)))
        return out

    def copyStereoToHost(self, fx, fy, cx, cy, d1, d2, d3, d4, t1, t2, t3):
        depth = np.empty((self.height, self.width), np.float32)
        X = np.empty((self.height, self.width, 3), np.float32)
        self._ok(self._L.vref_copy_stereo(self._h, _p(depth), _p(X), fx, fy, cx, cy, d1, d2, d3, d4,
                                          t1, t2, t3))
        return depth, X

    def set_plane(self, name: str, data: np.ndarray) -> None:
        """Write a (height, width[, comps]) float32 array into the plane ("warpUV" or "u")."""
        d = np.ascontiguousarray(data, np.float32)
        comps = 1 if d.ndim == 2 else d.shape[2]
        assert d.shape[:2] == (self.height, self.width)
        self._ok(self._L.vref_set_plane(self._h, name.encode(), _p(d), comps))

    def plane(self, name: str, comps: int = 1) -> np.ndarray:
        """A device plane cropped to width x height (x comps)."""
        s = self.stride
        out = np.empty((self.height, s, comps), np.float32)
        self._ok(self._L.vref_get_plane(self._h, name.encode(), _p(out), comps))
        out = out[:, :self.width]
        return out[..., 0] if comps == 1 else out


def run_ref(i0, i1, mask, tv, cv, p, masked=True, frames=1, fma=True) -> RefStereoTgv:
    """Same call sequence as the drop-in runner in tests/helpers.py, on the reference build."""
    h, w = i0.shape[:2]
    r = RefStereoTgv(fma)
    r.set_limit_range(p["limit_range"])
    r.initialize(w, h, p["beta"], p["gamma"], p["alpha0"], p["alpha1"], p["tsl"], p["lam"], p["n_levels"],
                 p["f_scale"], p["n_warp"], p["n_iter"])
    r.copyMaskToDevice(mask)
    r.loadVectorFields(tv, cv)
    for _ in range(frames):
        r.copyImagesToDevice(i0, i1)
        (r.solveStereoForwardMasked if masked else r.solveStereoForward)()
    return r
