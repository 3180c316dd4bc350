"""The no-allocation update entry point, checked against update_voxels.

osn_tsdf_cuda_update_voxels_noalloc exists for callers that cannot let the
library allocate device memory during an integrate: serving loops that admit
work against a fixed device-memory budget (memory appearing behind their back
breaks the budget), and latency-critical threads that cannot absorb the
device-wide synchronisation a cudaMalloc or cudaFree implies. Its scratch is
one fixed array compiled into the library, shared by every call, so these
tests also run it twice in a row: the second call starts on whatever the
first one left in that array.

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


def test_noalloc_stats_belong_to_the_volume(cuda):
    """The counters a no-alloc call leaves in the shared array are copied to
    the volume's own control block: a later no-alloc call on another volume
    does not change what the first volume reports."""
    scene = scenes.RoomScene.make(2)
    K = scenes.ROOM_K.scaled(320, 240)
    fa, fb = scenes.room_frame(scene, 0, K), scenes.room_frame(scene, 5, K)
    with CudaVolume(0.02, 1 << 16, 0.08, 64.0) as a, CudaVolume(0.02, 1 << 16, 0.08, 64.0) as b, \
            CudaVolume(0.02, 1 << 16, 0.08, 64.0) as ref:
        da = cuda.from_numpy(scenes.frame_points(fa)).cuda()
        db = cuda.from_numpy(scenes.frame_points(fb)[::2].copy()).cuda()
        for v in (a, ref):
            v.allocate_blocks(da, fa.cam)
        ref.update_voxels(da, fa.cam)
        assert a.update_voxels_noalloc(da, fa.cam) == 0
        want = ref.last_update_stats()
        assert a.last_update_stats() == want and want["records"] > 0
        b.allocate_blocks(db, fb.cam)
        assert b.update_voxels_noalloc(db, fb.cam) == 0
        assert b.last_update_stats()["records"] != want["records"]
        assert a.last_update_stats() == want
