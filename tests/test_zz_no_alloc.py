"""The no-allocation update entry point, checked against update_voxels.

osn_tsdf_cuda_update_voxels_noalloc exists for callers that cannot let the
library allocate device memory during an integrate: code that records the
integrate into a CUDA graph (allocation is not allowed while a stream is
captured), serving loops that budget device memory up front, and
latency-critical threads that cannot absorb the synchronisation a cudaMalloc
or cudaFree implies. Its scratch is one fixed array compiled into the
library, shared by every call, so these tests also run it twice in a row:
the second call starts on whatever the first one left in that array.

This file is collected last on purpose, so a run that stops at its first
failure has already run every other test.
"""
import numpy as np
import pytest

from helpers import TSDF_TOL, assert_same_voxels
from what_irregularity_costs_b200 import CudaVolume, scenes

pytestmark = pytest.mark.gpu

MAX_RECORDS = 1 << 21  # OSN_TSDF_NOALLOC_MAX_RECORDS in include/osn_tsdf_b200.h


def test_noalloc_update_matches_update_voxels_twice(cuda):
    """Two consecutive frames through both entry points on identical volumes.
    A cap of 6 makes many voxels cross the cap inside a frame, so the ordered
    selection runs on the shared scratch as well."""
    scene = scenes.RoomScene.make(1)
    K = scenes.ROOM_K.scaled(480, 360)  # fits the fixed scratch in one call
    frames = [scenes.room_frame(scene, k, K) for k in (0, 1)]
    with CudaVolume(0.02, 1 << 19, 0.08, 6.0) as regular, \
            CudaVolume(0.02, 1 << 19, 0.08, 6.0) as fixed:
        for f in frames:
            d = cuda.from_numpy(scenes.frame_points(f)).cuda()
            regular.allocate_blocks(d, f.cam)
            regular.update_voxels(d, f.cam)
            fixed.allocate_blocks(d, f.cam)
            assert fixed.update_voxels_noalloc(d, f.cam) == 0
            regular.synchronize()
            fixed.synchronize()
            assert fixed.block_count() == regular.block_count() > 0
            err = assert_same_voxels(fixed, regular, tol=TSDF_TOL)
            assert err <= TSDF_TOL
            assert float(fixed.voxels()[2].sum()) > 0.0  # the call did accumulate
        assert fixed.status() == 0 and regular.status() == 0


def test_noalloc_rejects_batches_above_the_fixed_maximum(cuda):
    """A batch needing more than the fixed number of records is refused before
    anything is queued (return code 4), and the volume is left untouched."""
    with CudaVolume(0.02, 1 << 10, 0.08, 64.0) as vol:
        steps = 4  # ceil(0.08 / 0.02): 9 records per point
        n = MAX_RECORDS // (2 * steps + 1) + 1
        # A real buffer of the claimed size, so no call could read past it.
        d = cuda.zeros((n, 3), dtype=cuda.float32, device="cuda")
        assert vol.update_voxels_noalloc(d, (0.0, 0.0, 0.0)) == 4
        fits = cuda.zeros((n - 1, 3), dtype=cuda.float32, device="cuda")
        assert vol.update_voxels_noalloc(fits, (0.0, 0.0, 0.0)) == 0
        vol.synchronize()
        assert vol.block_count() == 0
        assert np.all(vol.voxels()[2] == 0)
