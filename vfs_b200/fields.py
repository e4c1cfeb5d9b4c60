"""Camera models and the two per-pixel vector fields the solver consumes.

The reference loads both fields from Middlebury ``.flo`` files (dllhook/vfs.cpp:26-27,
test_vfs/main.cpp:157-158) made by external MATLAB scripts that are not part of it.  This
module computes them from a calibration instead:

* the **calibration field** ``cv`` (H x W x 2, pixels): for each pixel x of the first camera,
  cv(x) = x1 - x where x1 is the projection in the second camera of the same viewing
  direction.  ``StereoTgv`` samples the second image at x + cv(x) (stereotgv.cu:392), which
  removes the relative rotation (and any intrinsic difference) between the cameras.
* the **translation field** ``tv`` (H x W x 2, unit vectors): the direction in which the
  image of a point on the ray of pixel x moves in the (rotation-free) second camera as the
  point comes closer, i.e. the tangent at infinity of the epipolar curve of x.  The solver's
  disparity u is measured along it (warpImage.cu:136-150), so u > 0 for points in front.

Pixel coordinates are index coordinates: pixel (ix, iy) is centred at (ix, iy).
"""
from __future__ import annotations

import numpy as np


class EquidistantCamera:
    """Equidistant fisheye r = f * theta about the principal point (cx, cy)."""

    def __init__(self, width: int, height: int, f: float | None = None, cx: float | None = None,
                 cy: float | None = None):
        self.width, self.height = int(width), int(height)
        self.f = float(width) / np.pi if f is None else float(f)
        self.cx = (width - 1) / 2.0 if cx is None else float(cx)
        self.cy = (height - 1) / 2.0 if cy is None else float(cy)

    def unproject(self, u, v):
        x = (np.asarray(u, np.float64) - self.cx) / self.f
        y = (np.asarray(v, np.float64) - self.cy) / self.f
        theta = np.hypot(x, y)
        phi = np.arctan2(y, x)
        s = np.sin(theta)
        return np.stack([s * np.cos(phi), s * np.sin(phi), np.cos(theta)], -1)

    def project(self, d):
        d = np.asarray(d, np.float64)
        n = np.linalg.norm(d, axis=-1)
        theta = np.arccos(np.clip(d[..., 2] / np.maximum(n, 1e-300), -1.0, 1.0))
        phi = np.arctan2(d[..., 1], d[..., 0])
        r = self.f * theta
        return self.cx + r * np.cos(phi), self.cy + r * np.sin(phi)

    def theta_of_radius(self, r):
        return np.asarray(r, np.float64) / self.f


class KannalaBrandtCamera:
    """Kannala-Brandt fisheye (the T265 model): theta_d = theta (1 + k1 t^2 + k2 t^4 + k3 t^6 + k4 t^8),
    u = fx * theta_d * cos(phi) + cx, v = fy * theta_d * sin(phi) + cy."""

    def __init__(self, width, height, fx, fy, cx, cy, k1, k2, k3, k4):
        self.width, self.height = int(width), int(height)
        self.fx, self.fy, self.cx, self.cy = map(float, (fx, fy, cx, cy))
        self.k = tuple(map(float, (k1, k2, k3, k4)))

    def _distort(self, t):
        k1, k2, k3, k4 = self.k
        t2 = t * t
        return t * (1 + t2 * (k1 + t2 * (k2 + t2 * (k3 + t2 * k4))))

    def _ddistort(self, t):
        k1, k2, k3, k4 = self.k
        t2 = t * t
        return 1 + t2 * (3 * k1 + t2 * (5 * k2 + t2 * (7 * k3 + t2 * 9 * k4)))

    def unproject(self, u, v):
        x = (np.asarray(u, np.float64) - self.cx) / self.fx
        y = (np.asarray(v, np.float64) - self.cy) / self.fy
        td = np.hypot(x, y)
        phi = np.arctan2(y, x)
        t = td.copy()
        for _ in range(20):  # Newton on theta_d(t) = td
            t = t - (self._distort(t) - td) / self._ddistort(t)
        s = np.sin(t)
        return np.stack([s * np.cos(phi), s * np.sin(phi), np.cos(t)], -1)

    def project(self, d):
        d = np.asarray(d, np.float64)
        n = np.linalg.norm(d, axis=-1)
        t = np.arccos(np.clip(d[..., 2] / np.maximum(n, 1e-300), -1.0, 1.0))
        phi = np.arctan2(d[..., 1], d[..., 0])
        td = self._distort(t)
        return self.cx + self.fx * td * np.cos(phi), self.cy + self.fy * td * np.sin(phi)


def rotation_matrix(axis, angle_rad) -> np.ndarray:
    """Rodrigues rotation about `axis` by `angle_rad`."""
    a = np.asarray(axis, np.float64)
    a = a / np.linalg.norm(a)
    K = np.array([[0, -a[2], a[1]], [a[2], 0, -a[0]], [-a[1], a[0], 0]])
    return np.eye(3) + np.sin(angle_rad) * K + (1 - np.cos(angle_rad)) * (K @ K)


def _grid(cam):
    v, u = np.mgrid[0:cam.height, 0:cam.width].astype(np.float64)
    return u, v


def calibration_field(cam0, cam1, R01: np.ndarray) -> np.ndarray:
    """cv(x) = project1(R01^T d0(x)) - x, with R01 the rotation of camera 1 in camera 0's frame
    (a direction d in camera 0 coordinates is R01^T d in camera 1 coordinates)."""
    u, v = _grid(cam0)
    d = cam0.unproject(u, v)
    d1 = d @ np.asarray(R01, np.float64)  # (R01^T d) for row vectors
    u1, v1 = cam1.project(d1)
    return np.stack([u1 - u, v1 - v], -1).astype(np.float32)


def translation_field(cam, baseline: np.ndarray, eps: float = 1e-5) -> np.ndarray:
    """Unit tangent at infinity of each pixel's epipolar curve for a second camera with the
    first camera's orientation and intrinsics, displaced by `baseline` (camera 0 frame)."""
    u, v = _grid(cam)
    d = cam.unproject(u, v)
    b = np.asarray(baseline, np.float64)
    bn = b / np.linalg.norm(b)
    u1, v1 = cam.project(d - eps * bn)
    u2, v2 = cam.project(d + eps * bn)
    t = np.stack([u1 - u2, v1 - v2], -1)  # central difference of the motion as 1/depth grows
    n = np.linalg.norm(t, axis=-1, keepdims=True)
    t = np.where(n > 0, t / np.maximum(n, 1e-300), np.array([1.0, 0.0]))
    return t.astype(np.float32)


def fisheye_mask(cam, fov_deg: float) -> np.ndarray:
    """1 inside the circle of the given full field of view, 0 outside (H x W float32)."""
    u, v = _grid(cam)
    d = cam.unproject(u, v)
    theta = np.arccos(np.clip(d[..., 2], -1, 1))
    return (theta <= np.deg2rad(fov_deg) / 2).astype(np.float32)


# ---- Middlebury .flo ------------------------------------------------------------------
FLO_TAG = 202021.25


def read_flo(path) -> np.ndarray:
    """Read a .flo file (float32 tag 202021.25, int32 width, int32 height, H*W*2 float32)."""
    b = open(path, "rb").read()
    if len(b) < 12 or np.frombuffer(b, np.float32, 1, 0)[0] != np.float32(FLO_TAG):
        raise ValueError(f"{path}: not a .flo file")
    w, h = (int(x) for x in np.frombuffer(b, np.int32, 2, 4))
    if len(b) < 12 + w * h * 8:
        raise ValueError(f"{path}: truncated")
    return np.frombuffer(b, np.float32, w * h * 2, 12).reshape(h, w, 2).copy()


def write_flo(path, field: np.ndarray) -> None:
    f = np.ascontiguousarray(field, np.float32)
    h, w, c = f.shape
    if c != 2:
        raise ValueError("a .flo field has 2 channels")
    with open(path, "wb") as fh:
        fh.write(np.array([FLO_TAG], np.float32).tobytes())
        fh.write(np.array([w, h], np.int32).tobytes())
        fh.write(f.tobytes())
