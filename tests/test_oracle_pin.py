"""Pin the oracle (the C restatement) against the reference's own CPU arm.

The reference arm is compiled from its unmodified sources into
oracle/_ref/libosn_tsdf_ref.so (oracle/Makefile). With one thread it is
deterministic, and the restatement must reproduce it bit for bit: the hash
table, the block coordinates in pool order, all five voxel arrays and the
mesh. The scenes are the reference's own tests
(cpp/tests/test_analytic.cpp) plus multi-frame room data with weight capping.
"""
import numpy as np
import pytest

import oracle
from what_irregularity_costs_b200 import scenes

pytestmark = pytest.mark.skipif(not oracle.ref_available(),
                                reason="reference CPU arm not built (oracle/_ref)")


def _run_both(batches, voxel, pool, trunc=-1.0, cap=32.0, radius=0.0, split=False, colors=None,
              weights=None):
    o = oracle.OracleVolume(voxel, pool, trunc, cap)
    r = oracle.RefVolume(voxel, pool, trunc, cap, threads=1)
    for pts, cam in batches:
        if split:
            o.allocate(pts, cam, radius)
            o.update(pts, cam, radius, colors, weights)
            r.allocate(pts, cam, radius)
            r.update(pts, cam, radius, colors, weights)
        else:
            o.integrate(pts, cam, radius, colors, weights)
            r.integrate(pts, cam, radius, colors, weights)
    return o, r


def _assert_identical(o, r, rgb=False):
    assert o.block_count() == r.block_count()
    assert o.drop_count() == r.drop_count()
    ko, io = o.table()
    kr, ir = r.table()
    assert np.array_equal(ko, kr) and np.array_equal(io, ir)
    for a, b in zip(o.voxels(), r.voxels()):
        assert np.array_equal(a.view(np.uint32) if a.dtype == np.float32 else a,
                              b.view(np.uint32) if b.dtype == np.float32 else b)
    mo = o.extract(0.5, 0.0, 4 << 20, rgb=rgb)
    mr = r.extract(0.5, 0.0, 4 << 20, rgb=rgb)
    if rgb:
        assert np.array_equal(mo[0].view(np.uint32), mr[0].view(np.uint32))
        assert np.array_equal(mo[1], mr[1])
        return mo[0]
    assert np.array_equal(mo.view(np.uint32), mr.view(np.uint32))
    return mo


def test_sphere_known_answer():
    pts = oracle.sphere_points(0.5, 400, 800)
    o, r = _run_both([(pts, (0, 0, 0))], 0.01, 1 << 14)
    mesh = _assert_identical(o, r)
    assert o.block_count() == 1160
    assert mesh.shape[0] == 846288


def test_plane():
    pts = oracle.plane_points(0.30, 0.25, 500)
    o, r = _run_both([(pts, (0, 0, 0))], 0.01, 1 << 14)
    _assert_identical(o, r)


def test_pool_exhaustion_single_thread():
    pts = oracle.sphere_points(0.5, 200, 400)
    o, r = _run_both([(pts, (0, 0, 0))], 0.005, 16)
    _assert_identical(o, r)
    assert o.drop_count() > 0 and o.block_count() == 16


def test_sphere_frame_and_radius():
    f = scenes.sphere_frame()
    pts = scenes.frame_points(f)
    o, r = _run_both([(pts, f.cam)], 0.01, 1 << 15, 0.04, 64.0, radius=1.9)
    _assert_identical(o, r)


def test_room_frames_with_cap_crossing():
    scene = scenes.RoomScene.make(0)
    K = scenes.ROOM_K.scaled(320, 240)
    batches = [(scenes.frame_points(f), f.cam) for f in
               (scenes.room_frame(scene, k, K) for k in range(4))]
    o, r = _run_both(batches, 0.02, 1 << 16, 0.08, 6.0)
    _assert_identical(o, r)
    _, _, w, *_ = o.voxels()
    assert (w == 6.0).any()


def test_colors_and_weights_split_passes():
    f = scenes.sphere_frame()
    pts = scenes.frame_points(f)
    rng = np.random.default_rng(5)
    colors = rng.integers(0, 256, size=(pts.shape[0], 3), dtype=np.uint8)
    weights = rng.uniform(0.25, 2.0, size=pts.shape[0]).astype(np.float32)
    o, r = _run_both([(pts, f.cam), (pts, f.cam)], 0.01, 1 << 15, 0.04, 5.0, split=True,
                     colors=colors, weights=weights)
    _assert_identical(o, r, rgb=True)


def test_offset_camera_negative_coordinates():
    f = scenes.sphere_frame()
    pts = scenes.frame_points(f) - np.float32([3.3, 5.1, 9.7])
    o, r = _run_both([(pts, (-3.3, -5.1, -9.7))], 0.02, 1 << 14, -1.0, 64.0)
    _assert_identical(o, r)


def test_thread_invariance_of_reference_block_count():
    """cpp/tests/test_analytic.cpp:149-184: block count does not depend on the
    reference's thread count, which is what makes A2 usable as a block-set oracle."""
    pts = oracle.sphere_points(0.4, 200, 400)
    one = oracle.RefVolume(0.02, 1 << 14, threads=1)
    many = oracle.RefVolume(0.02, 1 << 14, threads=8)
    one.integrate(pts, (0, 0, 0))
    many.integrate(pts, (0, 0, 0))
    assert one.block_count() == many.block_count()
    assert one.coord_set() == many.coord_set()
