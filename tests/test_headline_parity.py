"""The benchmark's headline run against the oracle, end to end.

bench.py's headline figure integrates the full room trajectory (100 frames
of 640x480, 2 cm voxels, trunc 8 cm, 2^20 table slots, pool 2^19, cap 64)
with four consecutive frames per osn_tsdf_cuda_integrate_frames call
(bench.FRAMES_PER_CALL) and serial updates. This test runs exactly that sequence -- the same frames,
the same grouping (bench.frame_groups) and the same volume settings -- and
compares the result with the CPU oracle fed one frame at a time: block set
bit-exact, weights and colour sums exact, mean TSDF within 1e-5, and the
reference's mesh gates (cpp/tests/test_cuda_analytic.cu:244-283: vertex
count within 1 %, symmetric surface distance mean < voxel/100, Hausdorff
< voxel/10). Many voxels reach the cap only after a dozen frames, so this is
the run in which the ordered cap selection does most of its work.
"""
import numpy as np
import pytest

import bench
import oracle
from helpers import TSDF_TOL, assert_same_blocks, assert_same_voxels, surface_distance
from what_irregularity_costs_b200 import CudaVolume

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def trajectory():
    # Spawned workers: safe after CUDA was initialised by earlier tests.
    pts, cams = bench.make_trajectory(bench.N_FRAMES, bench.SEED)
    return pts, cams


def test_headline_run_matches_oracle(cuda, trajectory):
    pts, cams = trajectory
    assert len(pts) == bench.N_FRAMES == 100
    offsets = np.concatenate([[0], np.cumsum([p.shape[0] for p in pts])])
    d_all = cuda.from_numpy(np.concatenate(pts).astype(np.float32)).cuda()
    vol = CudaVolume(bench.VOXEL, bench.POOL, bench.TRUNC, bench.CAP, bench.HASH_SLOTS)
    groups = bench.frame_groups(offsets, cams, bench.FRAMES_PER_CALL)
    assert len(groups) == -(-bench.N_FRAMES // bench.FRAMES_PER_CALL)
    crossing = 0
    for lo, hi, a, b, begin, gcams in groups:
        vol.integrate_frames(d_all[a:b], begin, gcams)
        crossing += vol.last_update_stats()["crossing_voxels"]
    vol.synchronize()
    assert crossing > 10000, "the run must exercise the ordered cap selection"

    ref = oracle.OracleVolume(bench.VOXEL, bench.POOL, bench.TRUNC, bench.CAP, bench.HASH_SLOTS)
    for p, c in zip(pts, cams):
        ref.integrate(p, c)

    assert vol.status() == 0
    assert vol.drop_count() == ref.drop_count() == 0
    assert vol.block_count() == ref.block_count() == 14257
    assert_same_blocks(vol, ref)
    err = assert_same_voxels(vol, ref, tol=TSDF_TOL)
    assert err <= TSDF_TOL
    w = vol.voxels()[2]
    assert w.max() == bench.CAP and int((w == bench.CAP).sum()) > 100000  # many voxels capped

    gm = vol.extract_mesh(16 << 20, 0.5, 0.0)
    rm = ref.extract(0.5, 0.0, 16 << 20)
    assert gm is not None and rm is not None
    nv_g, nv_r = gm.shape[0], rm.shape[0]
    assert abs(nv_g - nv_r) / max(nv_g, nv_r) < 0.01, f"vertex counts {nv_g} vs {nv_r}"
    mean_d, haus = surface_distance(gm, rm)
    assert mean_d < bench.VOXEL / 100 and haus < bench.VOXEL / 10
