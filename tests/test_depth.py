"""Integrate from a depth image, unprojected on the GPU (osn_tsdf_cuda_integrate_depth).

The device backprojection restates the host's FP64 one operation for
operation (crates/tartanair/src/lib.rs:307-340, scenes.backproject), and the
pixel index orders records as the compacted raster-order point list does, so
integrating a depth frame must give a volume bit-identical to integrating
the host-backprojected points: same block set, same weights, same sums, same
drops -- with invalid pixels, a range cutoff, and voxels crossing the cap.
"""
import numpy as np
import pytest

import oracle
from helpers import assert_matches_oracle, sorted_voxels
from what_irregularity_costs_b200 import CudaVolume, scenes

pytestmark = pytest.mark.gpu


def _same(a, b):
    va, vb = sorted_voxels(a), sorted_voxels(b)
    for x, y in zip(va, vb):
        assert x.shape == y.shape and np.array_equal(x.view(np.uint8), y.view(np.uint8))
    assert a.drop_count() == b.drop_count()


@pytest.mark.parametrize("res,cap,max_range", [((640, 480), 64.0, 0.0), ((320, 240), 6.0, 0.0),
                                               ((640, 480), 64.0, 3.0)])
def test_depth_frames_equal_backprojected_points(cuda, res, cap, max_range):
    scene = scenes.RoomScene.make(2)
    K = scenes.ROOM_K.scaled(*res)
    pts_vol = CudaVolume(0.02, 1 << 17, 0.08, cap, 1 << 18)
    dep_vol = CudaVolume(0.02, 1 << 17, 0.08, cap, 1 << 18)
    ref = oracle.OracleVolume(0.02, 1 << 17, 0.08, cap, 1 << 18)
    for k in range(3):
        f = scenes.room_frame(scene, k, K)
        pts = scenes.frame_points(f, max_range)
        pts_vol.integrate(cuda.from_numpy(pts).cuda(), f.cam)
        dep_vol.integrate_depth(cuda.from_numpy(f.depth).cuda(), f.K, f.R, f.t, max_range)
        ref.integrate(pts, f.cam)  # the host's FP64 backprojection, fed to the oracle
    pts_vol.synchronize()
    dep_vol.synchronize()
    assert dep_vol.status() == 0
    assert dep_vol.block_count() == pts_vol.block_count() == ref.block_count() > 0
    _same(pts_vol, dep_vol)
    assert dep_vol.drop_count() == ref.drop_count()
    assert_matches_oracle(dep_vol, ref)
    if cap == 6.0:
        assert dep_vol.last_update_stats()["crossing_voxels"] > 0


def test_depth_sphere_frame_and_mesh(cuda):
    f = scenes.sphere_frame()
    a = CudaVolume(0.01, 1 << 15, 0.04, 64.0)
    b = CudaVolume(0.01, 1 << 15, 0.04, 64.0)
    a.integrate(cuda.from_numpy(scenes.frame_points(f)).cuda(), f.cam)
    b.integrate_depth(cuda.from_numpy(f.depth).cuda(), f.K, f.R, f.t)
    _same(a, b)
    ma, mb = a.extract_mesh(1 << 20), b.extract_mesh(1 << 20)
    assert ma.shape == mb.shape and ma.shape[0] > 0
    ref = oracle.OracleVolume(0.01, 1 << 15, 0.04, 64.0)
    ref.integrate(scenes.frame_points(f), f.cam)
    assert_matches_oracle(b, ref)
    assert ref.extract(0.5, 0.0, 1 << 20).shape == mb.shape


def test_depth_argument_checks(cuda):
    v = CudaVolume(0.02, 1 << 10, 0.08, 64.0)
    d = cuda.zeros((4, 4), dtype=cuda.float32, device="cuda")
    with pytest.raises(ValueError):
        v.integrate_depth(d.cpu(), scenes.ROOM_K, np.eye(3), np.zeros(3))
    with pytest.raises(ValueError):
        v.integrate_depth(d.double(), scenes.ROOM_K, np.eye(3), np.zeros(3))
    v.integrate_depth(d, scenes.ROOM_K, np.eye(3), np.zeros(3))  # all invalid: no points
    assert v.block_count() == 0 and v.status() == 0
