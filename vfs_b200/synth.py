"""Seeded synthetic fisheye stereo pairs (the stand-in for recorded T265 data).

Scene: piecewise-smooth surfaces at 0.5-5 m made of 3 random planes, 8 spherical bumps and
a background sphere; surface texture is 5-octave 3-D value noise plus 40 random box-shaped
patches, rendered as 8-bit grey.  Cameras: equidistant fisheye (r = f * theta, f = W / pi),
163 degree circular mask, second camera displaced by a 64 mm x-baseline and rotated by up to
2 degrees, Gaussian noise sigma = 2/255.  The calibration and translation fields come from
:mod:`vfs_b200.fields`.  Everything is a pure function of the seed.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from .fields import (EquidistantCamera, calibration_field, fisheye_mask, rotation_matrix,
                     translation_field)


@dataclass
class StereoPair:
    i0: np.ndarray      # H x W uint8, first camera
    i1: np.ndarray      # H x W uint8, second camera
    mask: np.ndarray    # H x W float32 {0, 1}
    tv: np.ndarray      # H x W x 2 float32 translation field
    cv: np.ndarray      # H x W x 2 float32 calibration field
    depth: np.ndarray   # H x W float64 radial distance seen by camera 0 (metres)
    seed: int


# the solver settings the synthetic workloads are measured with
SOLVER_PARAMS = dict(beta=10.0, gamma=0.8, alpha0=17.0, alpha1=1.2, timestep_lambda=1.0, lambda_=5.0,
                     fScale=2.0, nWarpIters=3, nSolverIters=50)
LIMIT_RANGE = 0.1


def n_levels_for(width: int, f_scale: float = 2.0, min_width: int = 50) -> int:
    """Pyramid depth: halve while the coarsest width stays >= min_width (test_vfs/main.cpp:136)."""
    n, w = 1, width
    while int(w / f_scale) >= min_width:
        w = int(w / f_scale)
        n += 1
    return n


def _hash3(ix, iy, iz, seed):
    h = (ix.astype(np.uint64) * np.uint64(0x9E3779B1) ^ iy.astype(np.uint64) * np.uint64(0x85EBCA77)
         ^ iz.astype(np.uint64) * np.uint64(0xC2B2AE3D) ^ np.uint64(seed * 0x27D4EB2F + 0x165667B1))
    h &= np.uint64(0xFFFFFFFF)
    h ^= h >> np.uint64(15)
    h = (h * np.uint64(0x2C1B3C6D)) & np.uint64(0xFFFFFFFF)
    h ^= h >> np.uint64(12)
    h = (h * np.uint64(0x297A2D39)) & np.uint64(0xFFFFFFFF)
    h ^= h >> np.uint64(15)
    return h.astype(np.float64) / 4294967296.0


def value_noise3(P: np.ndarray, freq: float, seed: int) -> np.ndarray:
    X = P * freq
    i = np.floor(X)
    f = X - i
    f = f * f * (3 - 2 * f)
    i = i.astype(np.int64)
    out = 0.0
    for dx in (0, 1):
        wx = f[..., 0] if dx else 1 - f[..., 0]
        for dy in (0, 1):
            wy = f[..., 1] if dy else 1 - f[..., 1]
            for dz in (0, 1):
                wz = f[..., 2] if dz else 1 - f[..., 2]
                out = out + wx * wy * wz * _hash3(i[..., 0] + dx, i[..., 1] + dy, i[..., 2] + dz, seed)
    return out


@dataclass
class Scene:
    planes: list       # (unit normal n, offset c): points with n.P = c
    spheres: list      # (centre, radius)
    bg_radius: float
    boxes: list        # (lo, hi, value offset)
    seed: int

    @staticmethod
    def random(rng: np.random.Generator, seed: int) -> "Scene":
        planes = []
        for _ in range(3):
            # planes facing the origin, 1.5-4.5 m away, tilted up to 60 degrees from the view axis
            th = rng.uniform(0, np.deg2rad(60))
            ph = rng.uniform(0, 2 * np.pi)
            n = np.array([np.sin(th) * np.cos(ph), np.sin(th) * np.sin(ph), np.cos(th)])
            planes.append((n, rng.uniform(1.5, 4.5)))
        spheres = []
        for _ in range(8):
            th = rng.uniform(0, np.deg2rad(70))
            ph = rng.uniform(0, 2 * np.pi)
            dist = rng.uniform(0.9, 3.0)
            c = dist * np.array([np.sin(th) * np.cos(ph), np.sin(th) * np.sin(ph), np.cos(th)])
            spheres.append((c, rng.uniform(0.15, 0.45)))
        boxes = []
        for _ in range(40):
            c = rng.uniform([-3, -3, 0.5], [3, 3, 5])
            half = rng.uniform(0.05, 0.6, size=3)
            boxes.append((c - half, c + half, rng.uniform(-0.35, 0.35)))
        return Scene(planes, spheres, 5.0, boxes, seed)

    def trace(self, origin: np.ndarray, dirs: np.ndarray) -> np.ndarray:
        """Distance along unit rays `dirs` from `origin` to the first surface (clipped to 0.5-5 m)."""
        o = np.asarray(origin, np.float64)
        t = np.full(dirs.shape[:-1], np.inf)
        for n, c in self.planes:
            den = dirs @ n
            num = c - o @ n
            with np.errstate(divide="ignore", invalid="ignore"):
                tt = np.where(den > 1e-6, num / den, np.inf)
            tt = np.where(tt > 0.3, tt, np.inf)
            t = np.minimum(t, tt)
        for cen, r in self.spheres:
            oc = o - cen
            b = dirs @ oc
            disc = b * b - (oc @ oc - r * r)
            sq = np.sqrt(np.maximum(disc, 0))
            tt = np.where(disc > 0, -b - sq, np.inf)
            tt = np.where(tt > 0.3, tt, np.inf)
            t = np.minimum(t, tt)
        # background sphere about the world origin
        b = dirs @ o
        disc = b * b - (o @ o - self.bg_radius ** 2)
        tb = -b + np.sqrt(np.maximum(disc, 0))
        t = np.minimum(t, tb)
        return np.clip(t, 0.5, self.bg_radius)

    def texture(self, P: np.ndarray) -> np.ndarray:
        v = 0.0
        amp, tot = 1.0, 0.0
        for k in range(5):
            v = v + amp * value_noise3(P, 3.0 * 2 ** k, self.seed * 7 + k)
            tot += amp
            amp *= 0.5
        v = v / tot
        val = 0.12 + 0.76 * v
        for lo, hi, off in self.boxes:
            inside = np.all((P >= lo) & (P <= hi), axis=-1)
            val = val + off * inside
        return np.clip(val, 0.0, 1.0)


def render(scene: Scene, cam: EquidistantCamera, R_wc: np.ndarray, C: np.ndarray, rng, noise_sigma=2.0 / 255.0):
    """Render camera (rotation R_wc = world-from-camera, centre C) as uint8 and return (image, depth)."""
    v, u = np.mgrid[0:cam.height, 0:cam.width].astype(np.float64)
    d = cam.unproject(u, v) @ np.asarray(R_wc, np.float64).T
    t = scene.trace(C, d)
    P = np.asarray(C, np.float64) + d * t[..., None]
    img = scene.texture(P) + rng.normal(0.0, noise_sigma, size=t.shape)
    return np.clip(np.round(img * 255.0), 0, 255).astype(np.uint8), t


def make_pair(width: int, height: int, seed: int, baseline: float = 0.064, max_rot_deg: float = 2.0,
              fov_deg: float = 163.0) -> StereoPair:
    rng = np.random.default_rng(seed)
    scene = Scene.random(rng, seed)
    cam = EquidistantCamera(width, height)
    axis = rng.normal(size=3)
    R01 = rotation_matrix(axis, np.deg2rad(rng.uniform(0.0, max_rot_deg)))
    b = np.array([baseline, 0.0, 0.0])
    i0, depth = render(scene, cam, np.eye(3), np.zeros(3), rng)
    i1, _ = render(scene, cam, R01, b, rng)
    return StereoPair(i0=i0, i1=i1, mask=fisheye_mask(cam, fov_deg), tv=translation_field(cam, b),
                      cv=calibration_field(cam, cam, R01), depth=depth, seed=seed)


def true_disparity(width: int, height: int, depth: np.ndarray, baseline: float = 0.064) -> np.ndarray:
    """The disparity camera 0's depth map implies along the translation field: pixel p sees the
    point depth(p) * ray(p); the calibrated second camera, displaced by `baseline` along x, sees
    it at p'; the disparity is (p' - p) . tv(p).  NaN where the depth is not finite."""
    cam = EquidistantCamera(width, height)
    b = np.array([baseline, 0.0, 0.0])
    tv = translation_field(cam, b)
    yy, xx = np.mgrid[0:height, 0:width].astype(np.float64)
    X = np.asarray(depth, np.float64)[..., None] * cam.unproject(xx, yy)
    u1, v1 = cam.project(X - b)
    return (u1 - xx) * tv[..., 0] + (v1 - yy) * tv[..., 1]


def make_sequence(width: int, height: int, seed: int, n_frames: int, max_step_m: float = 0.05,
                  max_step_deg: float = 3.0, baseline: float = 0.064, max_rot_deg: float = 2.0,
                  fov_deg: float = 163.0, with_depth: bool = False):
    """A camera stream: a fixed seeded scene and a smooth random rig trajectory (<= max_step_m
    and <= max_step_deg per frame).  Returns (fields dict, generator of (i0, i1) frames, or of
    (i0, i1, depth of camera 0) with with_depth)."""
    rng = np.random.default_rng(seed)
    scene = Scene.random(rng, seed)
    cam = EquidistantCamera(width, height)
    R01 = rotation_matrix(rng.normal(size=3), np.deg2rad(rng.uniform(0.0, max_rot_deg)))
    b = np.array([baseline, 0.0, 0.0])
    fields = dict(mask=fisheye_mask(cam, fov_deg), tv=translation_field(cam, b), cv=calibration_field(cam, cam, R01))

    def frames():
        R = np.eye(3)
        C = np.zeros(3)
        vel = rng.normal(size=3)
        vel *= max_step_m * 0.7 / np.linalg.norm(vel)
        for _ in range(n_frames):
            i0, d0 = render(scene, cam, R, C, rng)
            i1, _ = render(scene, cam, R @ R01, C + R @ b, rng)
            yield (i0, i1, d0) if with_depth else (i0, i1)
            acc = rng.normal(size=3) * max_step_m * 0.2
            vel = vel + acc
            nv = np.linalg.norm(vel)
            if nv > max_step_m:
                vel *= max_step_m / nv
            Cn = C + vel
            if np.linalg.norm(Cn) < 1.0:  # stay inside the room
                C = Cn
            else:
                vel = -vel
            R = R @ rotation_matrix(rng.normal(size=3), np.deg2rad(rng.uniform(0.0, max_step_deg)))

    return fields, frames()


# ---- the same renderer on the GPU (torch), for long frame sequences ---------------------
# Same scene, noise and camera model as `render`; transcendental functions come from torch,
# so pixels can differ from the numpy renderer by one grey level.  Used for the serving
# workload (hundreds of frames), not for test fixtures.
def _hash3_t(ix, iy, iz, seed):
    import torch
    m = 0xFFFFFFFF
    h = (ix * 0x9E3779B1) ^ (iy * 0x85EBCA77) ^ (iz * 0xC2B2AE3D) ^ (seed * 0x27D4EB2F + 0x165667B1)
    h = h & m
    h = h ^ (h >> 15)
    h = (h * 0x2C1B3C6D) & m
    h = h ^ (h >> 12)
    h = (h * 0x297A2D39) & m
    h = h ^ (h >> 15)
    return h.to(torch.float64) / 4294967296.0


def _value_noise3_t(P, freq, seed):
    import torch
    X = P * freq
    i = torch.floor(X)
    f = X - i
    f = f * f * (3 - 2 * f)
    i = i.to(torch.int64)
    out = torch.zeros(P.shape[:-1], dtype=torch.float64, device=P.device)
    for dx in (0, 1):
        wx = f[..., 0] if dx else 1 - f[..., 0]
        for dy in (0, 1):
            wy = f[..., 1] if dy else 1 - f[..., 1]
            for dz in (0, 1):
                wz = f[..., 2] if dz else 1 - f[..., 2]
                out = out + wx * wy * wz * _hash3_t(i[..., 0] + dx, i[..., 1] + dy, i[..., 2] + dz, seed)
    return out


def render_t(scene: Scene, rays_cam, R_wc, C, gen, noise_sigma=2.0 / 255.0):
    """GPU render: rays_cam = unit rays of the camera (H x W x 3 torch float64 on the device)."""
    import torch
    dev = rays_cam.device
    R = torch.as_tensor(np.asarray(R_wc, np.float64), device=dev)
    Ct = torch.as_tensor(np.asarray(C, np.float64), device=dev)
    d = rays_cam @ R.T
    t = torch.full(d.shape[:-1], float("inf"), dtype=torch.float64, device=dev)
    for n, c in scene.planes:
        nt = torch.as_tensor(n, device=dev)
        den = d @ nt
        num = c - float(Ct @ nt)
        tt = torch.where(den > 1e-6, num / den, torch.full_like(den, float("inf")))
        tt = torch.where(tt > 0.3, tt, torch.full_like(tt, float("inf")))
        t = torch.minimum(t, tt)
    for cen, r in scene.spheres:
        oc = Ct - torch.as_tensor(cen, device=dev)
        b = d @ oc
        disc = b * b - (float(oc @ oc) - r * r)
        sq = torch.sqrt(torch.clamp(disc, min=0))
        tt = torch.where(disc > 0, -b - sq, torch.full_like(b, float("inf")))
        tt = torch.where(tt > 0.3, tt, torch.full_like(tt, float("inf")))
        t = torch.minimum(t, tt)
    b = d @ Ct
    disc = b * b - (float(Ct @ Ct) - scene.bg_radius ** 2)
    tb = -b + torch.sqrt(torch.clamp(disc, min=0))
    t = torch.clamp(torch.minimum(t, tb), 0.5, scene.bg_radius)
    P = Ct + d * t[..., None]
    v = torch.zeros_like(t)
    amp, tot = 1.0, 0.0
    for k in range(5):
        v = v + amp * _value_noise3_t(P, 3.0 * 2 ** k, scene.seed * 7 + k)
        tot += amp
        amp *= 0.5
    val = 0.12 + 0.76 * (v / tot)
    for lo, hi, off in scene.boxes:
        lo_t = torch.as_tensor(lo, device=dev)
        hi_t = torch.as_tensor(hi, device=dev)
        inside = torch.all((P >= lo_t) & (P <= hi_t), dim=-1)
        val = val + off * inside.to(torch.float64)
    val = torch.clamp(val, 0.0, 1.0)
    noise = torch.randn(t.shape, generator=gen, dtype=torch.float64, device=dev) * noise_sigma
    img = torch.clamp(torch.round((val + noise) * 255.0), 0, 255).to(torch.uint8)
    return img


def make_sequence_gpu(width: int, height: int, seed: int, n_frames: int, device="cuda", max_step_m: float = 0.05,
                      max_step_deg: float = 3.0, baseline: float = 0.064, max_rot_deg: float = 2.0,
                      fov_deg: float = 163.0):
    """Like make_sequence, rendered on the GPU: returns (fields dict, list of (i0, i1) uint8 numpy)."""
    import torch
    rng = np.random.default_rng(seed)
    scene = Scene.random(rng, seed)
    cam = EquidistantCamera(width, height)
    R01 = rotation_matrix(rng.normal(size=3), np.deg2rad(rng.uniform(0.0, max_rot_deg)))
    b = np.array([baseline, 0.0, 0.0])
    fields = dict(mask=fisheye_mask(cam, fov_deg), tv=translation_field(cam, b), cv=calibration_field(cam, cam, R01))
    v, u = np.mgrid[0:height, 0:width].astype(np.float64)
    rays = torch.as_tensor(cam.unproject(u, v), device=device)
    gen = torch.Generator(device=device)
    gen.manual_seed(seed)
    R = np.eye(3)
    C = np.zeros(3)
    vel = rng.normal(size=3)
    vel *= max_step_m * 0.7 / np.linalg.norm(vel)
    frames = []
    for _ in range(n_frames):
        i0 = render_t(scene, rays, R, C, gen).cpu().numpy()
        i1 = render_t(scene, rays, R @ R01, C + R @ b, gen).cpu().numpy()
        frames.append((i0, i1))
        vel = vel + rng.normal(size=3) * max_step_m * 0.2
        nv = np.linalg.norm(vel)
        if nv > max_step_m:
            vel *= max_step_m / nv
        Cn = C + vel
        if np.linalg.norm(Cn) < 1.0:
            C = Cn
        else:
            vel = -vel
        R = R @ rotation_matrix(rng.normal(size=3), np.deg2rad(rng.uniform(0.0, max_step_deg)))
    return fields, frames


def make_pair_gpu(width: int, height: int, seed: int, device="cuda", baseline: float = 0.064,
                  max_rot_deg: float = 2.0, fov_deg: float = 163.0) -> StereoPair:
    """make_pair's scene, rotation and fields, with the two images rendered on the GPU."""
    import torch
    rng = np.random.default_rng(seed)
    scene = Scene.random(rng, seed)
    cam = EquidistantCamera(width, height)
    axis = rng.normal(size=3)
    R01 = rotation_matrix(axis, np.deg2rad(rng.uniform(0.0, max_rot_deg)))
    b = np.array([baseline, 0.0, 0.0])
    v, u = np.mgrid[0:height, 0:width].astype(np.float64)
    rays = torch.as_tensor(cam.unproject(u, v), device=device)
    gen = torch.Generator(device=device)
    gen.manual_seed(seed)
    i0 = render_t(scene, rays, np.eye(3), np.zeros(3), gen).cpu().numpy()
    i1 = render_t(scene, rays, R01, b, gen).cpu().numpy()
    return StereoPair(i0=i0, i1=i1, mask=fisheye_mask(cam, fov_deg), tv=translation_field(cam, b),
                      cv=calibration_field(cam, cam, R01), depth=None, seed=seed)
