"""Synthetic depth frames and their world-space points.

The reference integrates world-space float32 points with a camera origin
(cpp/include/osn_tsdf/types.hpp:122-135); depth frames, intrinsics and poses
become points in a pre-step that backprojects in FP64 and casts to float32
(crates/tartanair/src/lib.rs:307-340). This module supplies both halves for
seeded synthetic scenes with the shapes of the benchmark workloads:

* ``sphere_frame``: one 320x240 frame of a sphere (R 0.5 m at (0, 0, 2)) seen
  from the origin down +z, pinhole fx=fy=240, cx=160, cy=120, no noise;
* ``room_trajectory``: a 6x6x3 m room with 3 spheres and 2 boxes placed from
  a seed, seen along a 100-frame circular orbit (radius 1.5 m, height 1.4 m,
  yaw step 3.6 deg, small pitch jitter) at 640x480, fx=fy=320, cx=320, cy=240,
  depth noise sigma = 0.0015 z^2, 5 % of pixels invalid, depth kept in
  [0.1, 8] m.

Randomness is numpy's Philox counter-based generator keyed by (seed, frame),
so every frame is reproducible on its own. Camera frames follow the pinhole
convention x right, y down, z forward; poses are camera-to-world (R, t) in
float64 and t is the camera origin passed to the integrate call.
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np


@dataclass(frozen=True)
class Intrinsics:
    width: int
    height: int
    fx: float
    fy: float
    cx: float
    cy: float

    def scaled(self, width: int, height: int) -> "Intrinsics":
        sx, sy = width / self.width, height / self.height
        return Intrinsics(width, height, self.fx * sx, self.fy * sy, self.cx * sx, self.cy * sy)


SPHERE_K = Intrinsics(320, 240, 240.0, 240.0, 160.0, 120.0)
ROOM_K = Intrinsics(640, 480, 320.0, 320.0, 320.0, 240.0)


@dataclass
class Frame:
    depth: np.ndarray            # (H, W) float32 metres along the optical axis; 0 = invalid
    R: np.ndarray                # (3, 3) float64 camera-to-world rotation
    t: np.ndarray                # (3,) float64 camera origin in world
    K: Intrinsics

    @property
    def cam(self) -> tuple:
        return (float(self.t[0]), float(self.t[1]), float(self.t[2]))


def backproject(depth: np.ndarray, K: Intrinsics, R: np.ndarray, t: np.ndarray,
                max_range_m: float = 0.0) -> np.ndarray:
    """World points (n, 3) float32 of the valid pixels, in raster order.

    Follows crates/tartanair/src/lib.rs:307-340: a pixel is skipped when its
    depth is non-finite, <= 0, or beyond max_range_m (if > 0); otherwise
    x = (u - cx) z / fx, y = (v - cy) z / fy and R [x y z] + t, all in FP64,
    then cast to float32.
    """
    z = depth
    valid = np.isfinite(z) & (z > 0)
    if max_range_m > 0:
        valid &= z <= max_range_m
    v, u = np.nonzero(valid)
    zd = z[v, u].astype(np.float64)
    x = (u.astype(np.float64) - K.cx) * zd / K.fx
    y = (v.astype(np.float64) - K.cy) * zd / K.fy
    out = np.empty((zd.shape[0], 3), dtype=np.float32)
    for i in range(3):
        out[:, i] = (R[i, 0] * x + R[i, 1] * y + R[i, 2] * zd + t[i]).astype(np.float32)
    return out


def _pixel_rays(K: Intrinsics):
    """Camera-frame ray per pixel, unnormalised with z = 1 (so hit t == depth)."""
    u = np.arange(K.width, dtype=np.float64)
    v = np.arange(K.height, dtype=np.float64)
    uu, vv = np.meshgrid(u, v)
    return np.stack([(uu - K.cx) / K.fx, (vv - K.cy) / K.fy, np.ones_like(uu)], axis=-1)


def _hit_sphere(o, d, c, r):
    oc = c - o
    a = np.einsum("...k,...k->...", d, d)
    b = d @ oc
    cc = oc @ oc - r * r
    disc = b * b - a * cc
    t = np.full(a.shape, np.inf)
    ok = disc >= 0
    sq = np.sqrt(np.where(ok, disc, 0.0))
    t0 = (b - sq) / a
    t1 = (b + sq) / a
    near = np.where(t0 > 1e-9, t0, np.where(t1 > 1e-9, t1, np.inf))
    t[ok] = near[ok]
    return t


def _hit_box_outside(o, d, lo, hi):
    with np.errstate(divide="ignore", invalid="ignore"):
        inv = 1.0 / d
        t1 = (lo - o) * inv
        t2 = (hi - o) * inv
    tmin = np.nanmax(np.minimum(t1, t2), axis=-1)
    tmax = np.nanmin(np.maximum(t1, t2), axis=-1)
    hit = (tmax >= np.maximum(tmin, 0.0)) & (tmin > 1e-9)
    return np.where(hit, tmin, np.inf)


def _hit_box_inside(o, d, lo, hi):
    with np.errstate(divide="ignore", invalid="ignore"):
        inv = 1.0 / d
        t_hi = (hi - o) * inv
        t_lo = (lo - o) * inv
    t_exit = np.where(d > 0, t_hi, np.where(d < 0, t_lo, np.inf))
    return np.min(t_exit, axis=-1)


def sphere_frame(K: Intrinsics = SPHERE_K, center=(0.0, 0.0, 2.0), radius: float = 0.5) -> Frame:
    """One noiseless frame of a sphere, camera at the origin looking down +z."""
    d = _pixel_rays(K)
    t = _hit_sphere(np.zeros(3), d, np.asarray(center, dtype=np.float64), float(radius))
    depth = np.where(np.isfinite(t), t, 0.0).astype(np.float32)
    return Frame(depth, np.eye(3), np.zeros(3), K)


@dataclass
class RoomScene:
    """6x6x3 m room (inside faces) with seeded spheres and axis-aligned boxes."""

    seed: int
    lo: np.ndarray = field(default_factory=lambda: np.array([-3.0, -3.0, 0.0]))
    hi: np.ndarray = field(default_factory=lambda: np.array([3.0, 3.0, 3.0]))
    spheres: list = field(default_factory=list)   # (center (3,), radius)
    boxes: list = field(default_factory=list)     # (lo (3,), hi (3,))

    @staticmethod
    def make(seed: int, n_spheres: int = 3, n_boxes: int = 2, orbit_radius: float = 1.5) -> "RoomScene":
        rng = np.random.Generator(np.random.Philox(np.random.SeedSequence([seed, 0xC0FFEE])))
        scene = RoomScene(seed)

        def place(extent_xy: float) -> np.ndarray:
            # Keep objects off the camera orbit and inside the walls.
            for _ in range(1000):
                xy = rng.uniform(-3.0 + extent_xy + 0.05, 3.0 - extent_xy - 0.05, size=2)
                if abs(np.hypot(*xy) - orbit_radius) > extent_xy + 0.35:
                    return xy
            return np.zeros(2)

        for _ in range(n_spheres):
            r = float(rng.uniform(0.2, 0.6))
            xy = place(r)
            z = float(rng.uniform(r, 3.0 - r))
            scene.spheres.append((np.array([xy[0], xy[1], z]), r))
        for _ in range(n_boxes):
            size = rng.uniform(0.3, 1.0, size=3)
            xy = place(float(np.hypot(size[0], size[1]) / 2))
            lo = np.array([xy[0] - size[0] / 2, xy[1] - size[1] / 2, 0.0])
            scene.boxes.append((lo, lo + size))
        return scene

    def raycast(self, o: np.ndarray, d: np.ndarray) -> np.ndarray:
        t = _hit_box_inside(o, d, self.lo, self.hi)
        for c, r in self.spheres:
            t = np.minimum(t, _hit_sphere(o, d, c, r))
        for lo, hi in self.boxes:
            t = np.minimum(t, _hit_box_outside(o, d, lo, hi))
        return t


def orbit_pose(k: int, rng: np.random.Generator, radius: float = 1.5, height: float = 1.4,
               yaw_step_deg: float = 3.6, pitch_deg: float = -8.0, jitter_deg: float = 1.5):
    """Camera-to-world pose of orbit frame k, looking at the room's vertical axis."""
    theta = np.deg2rad(yaw_step_deg * k)
    pos = np.array([radius * np.cos(theta), radius * np.sin(theta), height])
    pitch = np.deg2rad(pitch_deg + rng.uniform(-jitter_deg, jitter_deg))
    h = -pos[:2] / np.hypot(*pos[:2])
    fwd = np.array([np.cos(pitch) * h[0], np.cos(pitch) * h[1], np.sin(pitch)])
    right = np.array([fwd[1], -fwd[0], 0.0])
    right /= np.linalg.norm(right)
    down = np.cross(fwd, right)
    R = np.stack([right, down, fwd], axis=1)
    return R, pos


def room_frame(scene: RoomScene, k: int, K: Intrinsics = ROOM_K, noise: bool = True,
               invalid_frac: float = 0.05, z_range=(0.1, 8.0)) -> Frame:
    rng = np.random.Generator(np.random.Philox(np.random.SeedSequence([scene.seed, k + 1])))
    R, pos = orbit_pose(k, rng)
    d_cam = _pixel_rays(K)
    d = d_cam @ R.T
    z = scene.raycast(pos, d)
    z = np.where(np.isfinite(z), z, 0.0)
    if noise:
        z = z + rng.standard_normal(z.shape) * (0.0015 * z * z)
        z = np.where(rng.random(z.shape) < invalid_frac, 0.0, z)
    z = np.where((z >= z_range[0]) & (z <= z_range[1]), z, 0.0)
    return Frame(z.astype(np.float32), R, pos, K)


def room_trajectory(seed: int = 0, n_frames: int = 100, K: Intrinsics = ROOM_K,
                    noise: bool = True) -> list:
    scene = RoomScene.make(seed)
    return [room_frame(scene, k, K, noise=noise) for k in range(n_frames)]


def frame_points(f: Frame, max_range_m: float = 0.0) -> np.ndarray:
    return backproject(f.depth, f.K, f.R, f.t, max_range_m)


def sphere_cloud(radius: float, n_theta: int, n_phi: int) -> np.ndarray:
    """Points on a sphere seen from its centre (the reference's analytic scene,
    cpp/tests/analytic_scenes.hpp:19-33, in numpy float32; the C oracle has a
    float-for-float copy for known-answer tests)."""
    i = np.arange(n_theta, dtype=np.float32)
    j = np.arange(n_phi, dtype=np.float32)
    pi = np.float32(np.pi)
    theta = pi * (i + np.float32(0.5)) / np.float32(n_theta)
    phi = np.float32(2.0) * pi * j / np.float32(n_phi)
    st, ct = np.sin(theta)[:, None], np.cos(theta)[:, None]
    sp, cp = np.sin(phi)[None, :], np.cos(phi)[None, :]
    r = np.float32(radius)
    x = r * st * cp
    y = r * st * sp
    z = np.broadcast_to(r * ct, x.shape)
    return np.stack([x, y, z], axis=-1).reshape(-1, 3).astype(np.float32)
