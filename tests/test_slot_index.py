"""The slot-index table layout (OSN_TSDF_LAYOUT_SLOT_INDEX), against the oracle.

In this opt-in layout the pool is the table and a block's pool index is its
table slot (the reference's slot-index variant, cpp/src/volume_cuda.cu:194-257,
made a production layout): a claim publishes the block at once and a thread
that meets the key needs no wait for its index. Only the placement of blocks
in memory changes, so every result must equal the pool layout's and the
oracle's: block sets bit-exact, weights and colour sums exact, mean TSDF
within 1e-5, the reference's sphere known answer, identical meshes -- alone,
in several-frame calls, and as scenes of a batched step.
"""
import numpy as np
import pytest

import oracle
from helpers import (TSDF_TOL, assert_matches_oracle, assert_same_blocks, assert_same_voxels,
                     canonical_triangles)
from what_irregularity_costs_b200 import LAYOUT_SLOT_INDEX, Batch, CudaVolume, scenes

pytestmark = pytest.mark.gpu


def test_room_frames_slot_index_matches_oracle(cuda):
    scene = scenes.RoomScene.make(0)
    frames = [scenes.room_frame(scene, k) for k in range(3)]
    vol = CudaVolume(0.02, 1 << 18, 0.08, 6.0, layout=LAYOUT_SLOT_INDEX)
    pool = CudaVolume(0.02, 1 << 18, 0.08, 6.0)
    ref = oracle.OracleVolume(0.02, 1 << 18, 0.08, 6.0)
    assert vol.device_view().pool_capacity == vol.device_view().hash_mask + 1 == 1 << 19
    for f in frames:
        p = scenes.frame_points(f)
        d = cuda.from_numpy(p).cuda()
        vol.integrate(d, f.cam)
        pool.integrate(d, f.cam)
        ref.integrate(p, f.cam)
    assert vol.status() == 0 and vol.drop_count() == 0
    assert vol.last_update_stats()["crossing_voxels"] > 0  # the ordered selection ran
    assert_same_blocks(vol, ref)
    assert_same_voxels(vol, ref, tol=TSDF_TOL)
    gm, pm = vol.extract_mesh(4 << 20, 0.5, 0.0), pool.extract_mesh(4 << 20, 0.5, 0.0)
    assert gm.shape == pm.shape and gm.shape[0] > 0
    assert np.array_equal(canonical_triangles(gm), canonical_triangles(pm))


def test_sphere_known_answer_and_reset(cuda):
    pts = oracle.sphere_points(0.5, 400, 800)
    vol = CudaVolume(0.01, 1 << 14, -1.0, 32.0, layout=LAYOUT_SLOT_INDEX)
    d = cuda.from_numpy(pts).cuda()
    for _ in range(2):  # the second pass after a reset gives the same
        vol.integrate(d, (0.0, 0.0, 0.0))
        assert vol.block_count() == 1160 and vol.drop_count() == 0
        mesh = vol.extract_mesh(1 << 21, 0.5, 0.0)
        assert mesh.shape[0] == 846288
        vol.reset()
        assert vol.block_count() == 0
        assert float(np.abs(vol.means()[2]).sum()) == 0.0


def test_several_frames_per_call_and_split_passes(cuda):
    scene = scenes.RoomScene.make(1)
    K = scenes.ROOM_K.scaled(320, 240)
    frames = [scenes.room_frame(scene, k, K) for k in range(4)]
    pts = [scenes.frame_points(f) for f in frames]
    begin = [0] + [int(x) for x in np.cumsum([p.shape[0] for p in pts])]
    cams = np.array([f.cam for f in frames], dtype=np.float32)
    d_all = cuda.from_numpy(np.concatenate(pts)).cuda()
    multi = CudaVolume(0.02, 1 << 16, 0.08, 6.0, layout=LAYOUT_SLOT_INDEX)
    multi.set_pipelined(True)
    multi.integrate_frames(d_all, begin, cams)
    split = CudaVolume(0.02, 1 << 16, 0.08, 6.0, layout=LAYOUT_SLOT_INDEX)
    ref = oracle.OracleVolume(0.02, 1 << 16, 0.08, 6.0)
    for k, f in enumerate(frames):
        d = d_all[begin[k]:begin[k + 1]]
        split.allocate_blocks(d, f.cam)
        split.update_voxels(d, f.cam)
        ref.integrate(pts[k], f.cam)
    for v in (multi, split):
        assert v.status() == 0
        assert_same_blocks(v, ref)
        assert_same_voxels(v, ref, tol=TSDF_TOL)


def test_batched_scenes_slot_index_match_oracle(cuda):
    # (seed, voxel, hash slots, resolution, cap): two layouts in one batch.
    mix = [(7, 0.02, 1 << 17, (640, 480), 64.0, LAYOUT_SLOT_INDEX),
           (8, 0.04, 1 << 14, (320, 240), 6.0, LAYOUT_SLOT_INDEX),
           (9, 0.015, 1 << 18, (160, 120), 32.0, 0)]
    batch = Batch(len(mix))
    vols, refs, frames = [], [], []
    for seed, voxel, slots, res, cap, layout in mix:
        v = CudaVolume(voxel, slots // 2, 4 * voxel, cap, slots, layout=layout)
        batch.add(v, res[0] * res[1])
        vols.append(v)
        refs.append(oracle.OracleVolume(voxel, slots // 2, 4 * voxel, cap, slots))
        sc = scenes.RoomScene.make(seed)
        K = scenes.ROOM_K.scaled(*res)
        frames.append([scenes.room_frame(sc, k, K) for k in range(3)])
    for k in range(3):
        for s, fr in enumerate(frames):
            p = scenes.frame_points(fr[k])
            batch.set_frame(s, cuda.from_numpy(p).cuda(), fr[k].cam)
            refs[s].integrate(p, fr[k].cam)
        batch.step()
    batch.synchronize()
    assert batch.status() == 0
    for v, ref in zip(vols, refs):
        assert v.drop_count() == ref.drop_count()
        assert_matches_oracle(v, ref, tol=TSDF_TOL)


def test_pool_order_features_are_refused(cuda):
    vol = CudaVolume(0.02, 1 << 10, 0.08, 64.0, layout=LAYOUT_SLOT_INDEX)
    with pytest.raises(RuntimeError):
        vol.snapshot()
    with pytest.raises(RuntimeError):
        vol.evict_chunks(0, 0)
    with pytest.raises(ValueError):
        CudaVolume(0.02, 1 << 10, 0.08, 64.0, layout=7)
