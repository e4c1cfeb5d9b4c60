"""ctypes wrapper of the CPU oracle (oracle/tgv_oracle.cpp).

TEST INFRASTRUCTURE ONLY: imported by tests/, by ``__graft_entry__.smoke()`` (to check the
CUDA result) and by ``bench.py``'s CPU-baseline leg.  The product package ``vfs_b200``
never imports it.

The class mirrors the reference ``StereoTgv`` host API (stereotgv/stereotgv.h:107-124):
``initialize`` → ``load_vector_fields`` → ``copy_mask_to_device`` →
``copy_images_to_device`` → ``solve_stereo_forward[_masked]`` → getters.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "_build", "libtgv_oracle.so")
_lib = None


def build(force: bool = False) -> str:
    """Compile the oracle shared library with its Makefile (g++, OpenMP)."""
    src = os.path.join(_HERE, "tgv_oracle.cpp")
    if force or not os.path.exists(_LIB_PATH) or os.path.getmtime(_LIB_PATH) < os.path.getmtime(src):
        subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


def lib():
    global _lib
    if _lib is None:
        build()
        L = ctypes.CDLL(_LIB_PATH)
        vp, i, f = ctypes.c_void_p, ctypes.c_int, ctypes.c_float
        L.oracle_create.restype = vp
        L.oracle_create.argtypes = [i]
        L.oracle_destroy.argtypes = [vp]
        L.oracle_set_hw_texture.argtypes = [i]
        L.oracle_set_threads.argtypes = [i]
        L.oracle_set_threads.restype = i
        L.oracle_initialize.argtypes = [vp, i, i, f, f, f, f, f, f, i, f, i, i, f, i, i]
        L.oracle_set_limit_range.argtypes = [vp, f]
        L.oracle_load_vector_fields.argtypes = [vp, vp, vp]
        L.oracle_copy_mask.argtypes = [vp, vp]
        L.oracle_copy_images_u8.argtypes = [vp, vp, vp]
        L.oracle_copy_images_f32.argtypes = [vp, vp, vp]
        L.oracle_solve.argtypes = [vp, i]
        L.oracle_convert_kb.argtypes = [vp] + [f] * 11
        L.oracle_stride.argtypes = [vp]
        L.oracle_get.argtypes = [vp, ctypes.c_char_p, i, vp]
        L.oracle_get_raw.argtypes = [vp, ctypes.c_char_p, vp, ctypes.c_size_t]
        L.oracle_tex_sample.argtypes = [vp, i, i, i, i, vp, i, vp]
        _lib = L
    return _lib


def _p(a: np.ndarray):
    return a.ctypes.data_as(ctypes.c_void_p)


def tex_sample(tex: np.ndarray, xy: np.ndarray, linear: bool) -> np.ndarray:
    """Texture-unit model: sample tight (h, w, comps) float32 texture at normalized xy."""
    tex = np.ascontiguousarray(tex, np.float32)
    if tex.ndim == 2:
        tex = tex[:, :, None]
    h, w, comps = tex.shape
    xy = np.ascontiguousarray(xy, np.float32)
    n = xy.shape[0]
    out = np.zeros((n, comps), np.float32)
    lib().oracle_tex_sample(_p(tex), w, h, comps, int(linear), _p(xy), n, _p(out))
    return out


def set_hw_texture(on: bool) -> None:
    lib().oracle_set_hw_texture(int(on))


def set_threads(n: int) -> int:
    """OpenMP threads of this thread's later oracle solves (n > 0); returns the previous count."""
    return int(lib().oracle_set_threads(int(n)))


class OracleStereoTgv:
    """CPU restatement of ``StereoTgv`` in float64 (precision=64) or float32 (32)."""

    def __init__(self, precision: int = 64, block_width: int = 32, stride_alignment: int = 32):
        self._L = lib()
        self._h = self._L.oracle_create(precision)
        self.precision = precision
        self.block_width = block_width
        self.stride_alignment = stride_alignment
        self.limit_range = 1.0  # stereotgv.h:45 default

    def __del__(self):
        h = getattr(self, "_h", None)
        if h:
            self._L.oracle_destroy(h)
            self._h = None

    def initialize(self, width, height, beta, gamma, alpha0, alpha1, timestep_lambda, lam,
                   n_levels, f_scale, n_warp_iters, n_solver_iters):
        self.width, self.height = int(width), int(height)
        rc = self._L.oracle_initialize(self._h, self.width, self.height, beta, gamma, alpha0, alpha1,
                                       timestep_lambda, lam, int(n_levels), f_scale, int(n_warp_iters),
                                       int(n_solver_iters), self.limit_range, self.block_width,
                                       self.stride_alignment)
        if rc != 0:
            raise ValueError("oracle initialize rejected its arguments")
        return 0

    def set_limit_range(self, lr: float):
        self.limit_range = float(lr)
        self._L.oracle_set_limit_range(self._h, self.limit_range)

    def load_vector_fields(self, tv: np.ndarray, cv: np.ndarray):
        tv = np.ascontiguousarray(tv, np.float32)
        cv = np.ascontiguousarray(cv, np.float32)
        assert tv.shape == (self.height, self.width, 2) and cv.shape == tv.shape
        self._L.oracle_load_vector_fields(self._h, _p(tv), _p(cv))

    def copy_mask_to_device(self, mask: np.ndarray):
        mask = np.ascontiguousarray(mask, np.float32)
        assert mask.shape == (self.height, self.width)
        self._L.oracle_copy_mask(self._h, _p(mask))

    def copy_images_to_device(self, i0: np.ndarray, i1: np.ndarray):
        assert i0.shape == (self.height, self.width) and i1.shape == i0.shape
        if i0.dtype == np.uint8:
            i0 = np.ascontiguousarray(i0)
            i1 = np.ascontiguousarray(i1, np.uint8)
            self._L.oracle_copy_images_u8(self._h, _p(i0), _p(i1))
        else:
            i0 = np.ascontiguousarray(i0, np.float32)
            i1 = np.ascontiguousarray(i1, np.float32)
            self._L.oracle_copy_images_f32(self._h, _p(i0), _p(i1))

    def solve_stereo_forward_masked(self):
        self._L.oracle_solve(self._h, 1)

    def solve_stereo_forward(self):
        self._L.oracle_solve(self._h, 0)

    def get(self, name: str, comps: int = 1) -> np.ndarray:
        out = np.zeros((self.height, self.width, comps), np.float64)
        rc = self._L.oracle_get(self._h, name.encode(), comps, _p(out))
        if rc != 0:
            raise KeyError(name)
        return out[:, :, 0] if comps == 1 else out

    def disparity_1d(self) -> np.ndarray:
        return self.get("u")

    def disparity_2d(self) -> np.ndarray:
        return self.get("warpUV", 2)

    def convert_kb(self, fx, fy, cx, cy, d1, d2, d3, d4, t1, t2, t3):
        self._L.oracle_convert_kb(self._h, fx, fy, cx, cy, d1, d2, d3, d4, t1, t2, t3)
        return self.get("depth"), self.get("X", 3)
