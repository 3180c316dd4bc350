"""Batched integrate: many scenes per step, through the C ABI (osn_tsdf_batch_*).

Every scene integrated through a batch must end bit-identical to the same
scene integrated alone with osn_tsdf_cuda_integrate (same block set, same
weights, same sums to the last bit): the batched passes run the same walk,
the same exact integer cap selection and the same fixed-point sums, only
scheduled differently. Covered: mixed voxel sizes, resolutions, table sizes
and caps; scenes that sit steps out; CUDA-graph replay; the autotuner
(results identical under every shape); FP16 storage; argument checks.
"""
import numpy as np
import pytest

import oracle
from helpers import FP16_ORACLE_TOL, assert_matches_oracle
from what_irregularity_costs_b200 import (STORAGE_FP16_U16, STORAGE_FP32, Batch, CudaVolume,
                                          precision, scenes)

pytestmark = pytest.mark.gpu

# (seed, voxel, hash slots, resolution, cap)
MIX = [
    (0, 0.02, 1 << 18, (640, 480), 64.0),
    (1, 0.01, 1 << 20, (320, 240), 64.0),
    (2, 0.04, 1 << 14, (160, 120), 6.0),
    (3, 0.03, 1 << 16, (1280, 720), 32.0),
    (4, 0.015, 1 << 19, (320, 240), 0.0),
    (5, 0.02, 1 << 17, (160, 120), 64.0),
]


def _frames(seed, res, n):
    scene = scenes.RoomScene.make(seed)
    K = scenes.ROOM_K.scaled(*res)
    return [scenes.room_frame(scene, k, K) for k in range(n)]


def _make(voxel, slots, cap, storage):
    # Explicit table sizes; pools sized for a few frames (not the full 2x).
    return CudaVolume(voxel, min(slots // 2, 1 << 15), 4 * voxel, cap, slots, storage=storage)


def _snapshot(vol):
    coords, mean, w = precision._aligned(vol)
    if vol.storage == STORAGE_FP32:
        c2, t, w2, *_ = vol.voxels()
        order = np.lexsort(c2.T[::-1])
        return coords, w, t[order]
    return coords, w, mean


def _same(a, b):
    for x, y in zip(_snapshot(a), _snapshot(b)):
        assert x.shape == y.shape and np.array_equal(x.view(np.uint8), y.view(np.uint8))


def _run(torch, storage=STORAGE_FP32, n_frames=3, idle=None, graph=False, tune=0, shape=None):
    """Integrate MIX through one batch and each scene alone; return both."""
    frames = [_frames(seed, res, n_frames) for seed, _, _, res, _ in MIX]
    batch = Batch(len(MIX))
    if graph:
        batch.set_graph(True)
    if shape:
        batch.set_shape(*shape)
    if tune:
        batch.autotune(tune)
    bvols, avols = [], []
    for (seed, voxel, slots, res, cap), fr in zip(MIX, frames):
        bv = _make(voxel, slots, cap, storage)
        av = _make(voxel, slots, cap, storage)
        batch.add(bv, res[0] * res[1])
        bvols.append(bv)
        avols.append(av)
    steps = max(n_frames, 16 * tune if tune else 0)
    dev = [[torch.from_numpy(scenes.frame_points(f)).cuda() for f in fr] for fr in frames]
    for k in range(steps):
        for s, (fr, dv) in enumerate(zip(frames, dev)):
            if k >= n_frames or (idle and (s, k) in idle):
                continue
            batch.set_frame(s, dv[k], fr[k].cam)
            avols[s].integrate(dv[k], fr[k].cam)
        batch.step()
    batch.synchronize()
    assert batch.status() == 0
    return batch, bvols, avols


def _oracles(n_frames=3):
    """Every MIX scene fed to the CPU oracle, frame by frame."""
    out = []
    for seed, voxel, slots, res, cap in MIX:
        ref = oracle.OracleVolume(voxel, min(slots // 2, 1 << 15), 4 * voxel, cap, slots)
        for f in _frames(seed, res, n_frames):
            ref.integrate(scenes.frame_points(f), f.cam)
        out.append(ref)
    return out


def test_batch_equals_each_scene_alone(cuda):
    batch, bvols, avols = _run(cuda)
    for b, a in zip(bvols, avols):
        assert b.block_count() == a.block_count() and b.block_count() > 0
        assert b.drop_count() == a.drop_count() == 0
        _same(b, a)
    # A capped scene crossed its cap inside a frame (ordered selection ran).
    assert any(a.last_update_stats()["crossing_voxels"] > 0 for a in avols)
    # And every scene of the mix -- 1280x720 frames, a 2^14-slot table, caps
    # 64 / 32 / 6 / none, voxels 1-4 cm -- equals the CPU oracle.
    for b, ref in zip(bvols, _oracles()):
        assert b.drop_count() == ref.drop_count()
        assert_matches_oracle(b, ref)


def test_batch_with_idle_scenes(cuda):
    idle = {(1, 0), (2, 1), (3, 1), (3, 2), (5, 0)}
    _, bvols, avols = _run(cuda, idle=idle)
    for b, a in zip(bvols, avols):
        _same(b, a)


def test_batch_graph_replay(cuda):
    batch, bvols, avols = _run(cuda, graph=True, n_frames=4)
    for b, a in zip(bvols, avols):
        _same(b, a)


@pytest.mark.parametrize("shape", [(1, 1, 0), (8, 0, 1), (2, 1, 1)])
def test_batch_shapes_give_identical_results(cuda, shape):
    _, bvols, avols = _run(cuda, shape=shape)
    for b, a in zip(bvols, avols):
        _same(b, a)


def test_batch_autotune(cuda):
    batch, bvols, avols = _run(cuda, n_frames=3, tune=1)
    res = batch.tune_results()
    assert len(res) == 16 and all(r["median_ms"] > 0 for r in res)
    sh = batch.shape()
    assert not sh["tuning"]
    best = min(res, key=lambda r: r["median_ms"])
    assert (sh["tiles_per_item"], sh["probe"], sh["finish_pair"]) == (
        best["tiles_per_item"], best["probe"], best["finish_pair"])
    for b, a in zip(bvols, avols):
        _same(b, a)


def test_batch_fp16_storage(cuda):
    _, bvols, avols = _run(cuda, storage=STORAGE_FP16_U16)
    for b, a in zip(bvols, avols):
        _same(b, a)
    for b, ref in zip(bvols, _oracles()):
        assert_matches_oracle(b, ref, tol=FP16_ORACLE_TOL)


def test_batch_argument_checks(cuda):
    batch = Batch(2)
    v32 = CudaVolume(0.02, 1 << 12, 0.08, 64.0)
    v16 = CudaVolume(0.02, 1 << 12, 0.08, 64.0, storage=STORAGE_FP16_U16)
    assert batch.add(v32, 1000) == 0
    with pytest.raises(ValueError):
        batch.add(v32, 1000)  # already attached
    with pytest.raises(ValueError):
        batch.add(v16, 1000)  # storage differs
    pts = cuda.zeros((2000, 3), dtype=cuda.float32, device="cuda")
    with pytest.raises(ValueError):
        batch.set_frame(0, pts, (0.0, 0.0, 0.0))  # more points than reserved
    with pytest.raises(ValueError):
        batch.set_frame(5, pts[:10], (0.0, 0.0, 0.0))  # no such scene
    with pytest.raises(ValueError):
        Batch(65)
    batch.step()  # no frames: a no-op step
    batch.synchronize()
    assert batch.status() == 0 and len(batch) == 1
