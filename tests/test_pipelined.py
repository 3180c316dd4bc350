"""Pipelined updates (osn_tsdf_cuda_set_pipelined): the band walk of the next
call overlaps the update tail of this one.

Results must be those of serial mode bit for bit, and so the oracle's:
the walk's saturation filter may read weights the previous tail is still
writing (weights only grow; finish decides acceptance from the final
weights), and the two alternating scratch sets never meet.
"""
import numpy as np
import pytest

import oracle
from helpers import assert_same_blocks, assert_same_voxels, canonical_triangles, sorted_voxels
from what_irregularity_costs_b200 import STORAGE_FP16_U16, STORAGE_FP64, CudaVolume, precision, scenes

pytestmark = pytest.mark.gpu


def _frames(n, res=(640, 480), seed=0):
    scene = scenes.RoomScene.make(seed)
    K = scenes.ROOM_K.scaled(*res)
    return [scenes.room_frame(scene, k, K) for k in range(n)]


def _bits_equal(a, b):
    for x, y in zip(sorted_voxels(a), sorted_voxels(b)):
        assert x.shape == y.shape and np.array_equal(x.view(np.uint8), y.view(np.uint8))


@pytest.mark.parametrize("cap", [64.0, 6.0, 0.0])
def test_pipelined_matches_oracle_and_serial(cuda, cap):
    frames = _frames(5)
    pipe = CudaVolume(0.02, 1 << 19, 0.08, cap, 1 << 20)
    pipe.set_pipelined(True)
    serial = CudaVolume(0.02, 1 << 19, 0.08, cap, 1 << 20)
    ref = oracle.OracleVolume(0.02, 1 << 19, 0.08, cap, 1 << 20)
    for f in frames:
        pts = scenes.frame_points(f)
        d = cuda.from_numpy(pts).cuda()
        pipe.integrate(d, f.cam)
        serial.integrate(d, f.cam)
        ref.integrate(pts, f.cam)
    # Waiting readers see every queued tail without an explicit synchronize.
    assert pipe.block_count() == serial.block_count() == ref.block_count()
    assert pipe.last_update_stats() == serial.last_update_stats()
    if cap == 6.0:
        assert pipe.last_update_stats()["crossing_voxels"] > 0
    assert_same_blocks(pipe, ref)
    assert_same_voxels(pipe, ref)
    _bits_equal(pipe, serial)
    gm, sm = pipe.extract_mesh(1 << 24), serial.extract_mesh(1 << 24)
    # Same triangles; their order in the soup follows pool order, which
    # depends on insertion timing in either mode.
    assert gm.shape == sm.shape
    assert np.array_equal(canonical_triangles(gm), canonical_triangles(sm))
    assert pipe.status() == 0


def test_pipelined_split_passes_depth_and_fp16(cuda):
    frames = _frames(4, (320, 240), seed=3)
    for storage in (0, STORAGE_FP16_U16):
        a = CudaVolume(0.02, 1 << 16, 0.08, 6.0, 1 << 17, storage=storage)
        b = CudaVolume(0.02, 1 << 16, 0.08, 6.0, 1 << 17, storage=storage)
        a.set_pipelined(True)
        for k, f in enumerate(frames):
            d = cuda.from_numpy(scenes.frame_points(f)).cuda()
            if k % 2:
                a.allocate_blocks(d, f.cam)
                a.update_voxels(d, f.cam)
            else:
                a.integrate_depth(cuda.from_numpy(f.depth).cuda(), f.K, f.R, f.t)
            b.integrate(d, f.cam)
        ca, ma, wa = precision._aligned(a)
        cb, mb, wb = precision._aligned(b)
        assert np.array_equal(ca, cb) and np.array_equal(wa, wb) and np.array_equal(ma, mb)


def test_pipelined_reset_noalloc_and_modes(cuda):
    frames = _frames(3, (320, 240), seed=5)
    dev = [(cuda.from_numpy(scenes.frame_points(f)).cuda(), f.cam) for f in frames]
    a = CudaVolume(0.02, 1 << 16, 0.08, 64.0, 1 << 17)
    a.set_pipelined(True)
    for d, cam in dev:
        a.integrate(d, cam)
    a.reset()
    assert a.block_count() == 0
    b = CudaVolume(0.02, 1 << 16, 0.08, 64.0, 1 << 17)
    for d, cam in dev:
        a.allocate_blocks(d, cam)
        assert a.update_voxels_noalloc(d, cam) == 0
        b.integrate(d, cam)
    _bits_equal(a, b)
    a.set_pipelined(False)  # back to serial, state kept
    a.integrate(*dev[0])
    b.integrate(*dev[0])
    _bits_equal(a, b)
    with pytest.raises(ValueError):
        CudaVolume(0.02, 1 << 12, 0.08, 64.0, storage=STORAGE_FP64).set_pipelined(True)
