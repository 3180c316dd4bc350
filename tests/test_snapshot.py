"""Snapshot / restore through host memory.

A volume restored from a snapshot must continue exactly as the original:
integrate the same later frames into both and the voxels stay bit-identical
(the table is rebuilt, so slot positions may differ, which nothing reads
back). Also: restoring into a volume with a different table size, in every
storage mode, and rejecting snapshots of a different configuration.
"""
import numpy as np
import pytest

from helpers import sorted_voxels
from what_irregularity_costs_b200 import STORAGE_FP16_U16, STORAGE_FP32, STORAGE_FP64, CudaVolume, precision, scenes

pytestmark = pytest.mark.gpu


def _frames(n):
    scene = scenes.RoomScene.make(4)
    K = scenes.ROOM_K.scaled(320, 240)
    return [scenes.room_frame(scene, k, K) for k in range(n)]


@pytest.mark.parametrize("storage", [STORAGE_FP32, STORAGE_FP16_U16, STORAGE_FP64])
def test_restore_continues_bit_identically(cuda, storage):
    frames = _frames(5)
    dev = [(cuda.from_numpy(scenes.frame_points(f)).cuda(), f.cam) for f in frames]
    a = CudaVolume(0.02, 1 << 15, 0.08, 6.0, 1 << 16, storage=storage)
    for p, cam in dev[:3]:
        a.integrate(p, cam)
    snap = a.snapshot()
    b = CudaVolume(0.02, 1 << 15, 0.08, 6.0, 1 << 17, storage=storage)  # a larger table
    b.restore(snap)
    assert b.block_count() == a.block_count() and b.drop_count() == a.drop_count()
    for p, cam in dev[3:]:
        a.integrate(p, cam)
        b.integrate(p, cam)
    if storage == STORAGE_FP32:
        for x, y in zip(sorted_voxels(a), sorted_voxels(b)):
            assert np.array_equal(x.view(np.uint8), y.view(np.uint8))
    else:
        for x, y in zip(precision._aligned(a), precision._aligned(b)):
            assert np.array_equal(x, y)
    ma, mb = a.extract_mesh(1 << 24), b.extract_mesh(1 << 24)
    assert ma.shape == mb.shape and ma.shape[0] > 0
    assert a.status() == 0 and b.status() == 0


def test_restore_rejects_other_configurations(cuda):
    f = _frames(1)[0]
    a = CudaVolume(0.02, 1 << 14, 0.08, 64.0)
    a.integrate(cuda.from_numpy(scenes.frame_points(f)).cuda(), f.cam)
    snap = a.snapshot()
    for other in (CudaVolume(0.03, 1 << 14, 0.08, 64.0), CudaVolume(0.02, 1 << 14, 0.08, 32.0),
                  CudaVolume(0.02, 1 << 14, 0.08, 64.0, storage=STORAGE_FP16_U16),
                  CudaVolume(0.02, 16, 0.08, 64.0)):  # pool too small
        with pytest.raises(ValueError):
            other.restore(snap)
    with pytest.raises(ValueError):
        a.restore(snap[:100])  # truncated
    bad = snap.copy()
    bad[0] ^= 0xFF
    with pytest.raises(ValueError):
        a.restore(bad)
    empty = CudaVolume(0.02, 1 << 14, 0.08, 64.0)
    e_snap = empty.snapshot()
    a.restore(e_snap)  # restoring an empty snapshot empties the volume
    assert a.block_count() == 0
