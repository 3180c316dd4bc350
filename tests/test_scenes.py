"""Synthetic inputs: backprojection formula, frame shapes, determinism."""
import numpy as np

from what_irregularity_costs_b200 import scenes


def test_backprojection_matches_per_pixel_fp64():
    """crates/tartanair/src/lib.rs:324-329, one pixel at a time in FP64."""
    rng = np.random.default_rng(1)
    K = scenes.Intrinsics(16, 12, 11.0, 12.5, 7.5, 5.5)
    depth = rng.uniform(0.2, 5.0, size=(12, 16)).astype(np.float32)
    depth[3, 4] = 0.0
    depth[5, 6] = np.nan
    depth[7, 8] = 9.0
    ang = 0.3
    R = np.array([[np.cos(ang), -np.sin(ang), 0], [np.sin(ang), np.cos(ang), 0], [0, 0, 1.0]])
    t = np.array([0.5, -1.25, 2.0])
    pts = scenes.backproject(depth, K, R, t, max_range_m=8.0)
    expect = []
    for v in range(12):
        for u in range(16):
            z = float(depth[v, u])
            if not np.isfinite(z) or z <= 0 or z > 8.0:
                continue
            x = (u - K.cx) * z / K.fx
            y = (v - K.cy) * z / K.fy
            expect.append([np.float32(R[i, 0] * x + R[i, 1] * y + R[i, 2] * z + t[i]) for i in range(3)])
    assert np.array_equal(pts, np.array(expect, dtype=np.float32))


def test_sphere_frame_shape():
    f = scenes.sphere_frame()
    assert f.depth.shape == (240, 320)
    pts = scenes.frame_points(f)
    # A 0.5 m sphere at 2 m covers a disc of ~62 px radius: ~12k valid rays.
    assert 11000 < pts.shape[0] < 13000
    r = np.linalg.norm(pts - np.float32([0, 0, 2]), axis=1)
    assert np.abs(r - 0.5).max() < 1e-5


def test_room_frame_statistics_and_determinism():
    scene = scenes.RoomScene.make(0)
    K = scenes.ROOM_K.scaled(160, 120)
    a = scenes.room_frame(scene, 7, K)
    b = scenes.room_frame(scenes.RoomScene.make(0), 7, K)
    assert np.array_equal(a.depth, b.depth)
    valid = a.depth > 0
    assert 0.92 < valid.mean() < 0.97
    assert a.depth[valid].min() >= 0.1 and a.depth.max() <= 8.0
    assert np.allclose(a.R.T @ a.R, np.eye(3))
    assert abs(np.hypot(a.t[0], a.t[1]) - 1.5) < 1e-12 and a.t[2] == 1.4


def test_room_objects_inside_walls():
    for seed in range(5):
        s = scenes.RoomScene.make(seed)
        assert len(s.spheres) == 3 and len(s.boxes) == 2
        for c, r in s.spheres:
            assert 0.2 <= r <= 0.6
            assert np.all(c - r >= s.lo - 1e-9) and np.all(c + r <= s.hi + 1e-9)
        for lo, hi in s.boxes:
            assert np.all(lo >= s.lo - 1e-9) and np.all(hi <= s.hi + 1e-9)


def test_intrinsics_scaling():
    K = scenes.ROOM_K.scaled(1280, 720)
    assert K.fx == 640.0 and K.cx == 640.0 and K.cy == 360.0
