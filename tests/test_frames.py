"""Several frames per integrate call (osn_tsdf_cuda_integrate_frames).

Under the cap rule "accept while the weight before a contribution is below
the cap", taken in (frame, point, step) order, a batch of consecutive frames
keeps exactly the contributions that one call per frame keeps: the block
set, the weights and the colour sums must be identical to per-frame calls
and to the CPU oracle fed frame by frame. A voxel's stored TSDF sum takes one
rounding per call instead of one per frame, so mean TSDFs are held to the
float parity bar (1e-5) against both. Covered: caps 64 / 6 (crossing inside
a batch) / none, uneven and empty frames, one frame per call (bit-identical
to integrate), pipelined calls, FP16 storage against the FP64 oracle, depth
images (osn_tsdf_cuda_integrate_depth_frames: bit-identical to integrate_frames
of the host-backprojected points), and the argument checks.
"""
import numpy as np
import pytest

import oracle
from helpers import assert_same_blocks, assert_same_voxels, sorted_voxels
from what_irregularity_costs_b200 import (MAX_DEPTH_FRAMES, MAX_FRAMES, STORAGE_FP16_U16, STORAGE_FP32,
                                          STORAGE_FP64, CudaVolume, precision, scenes)

pytestmark = pytest.mark.gpu

FP16_TOL = 4 * 2.0 ** -11  # normalised TSDF, as for FP16 storage against the FP64 oracle


def _frames(n, res=(640, 480), seed=0):
    scene = scenes.RoomScene.make(seed)
    K = scenes.ROOM_K.scaled(*res)
    return [scenes.room_frame(scene, k, K) for k in range(n)]


def _packed(cuda, frames):
    pts = [scenes.frame_points(f) for f in frames]
    begin = [0] + [int(x) for x in np.cumsum([p.shape[0] for p in pts])]
    cams = np.array([f.cam for f in frames], dtype=np.float32)
    return pts, cuda.from_numpy(np.concatenate(pts)).cuda(), begin, cams


def _bits_equal(a, b):
    for x, y in zip(sorted_voxels(a), sorted_voxels(b)):
        assert x.shape == y.shape and np.array_equal(x.view(np.uint8), y.view(np.uint8))


@pytest.mark.parametrize("cap", [64.0, 6.0, 0.0])
def test_frames_equal_per_frame_calls_and_oracle(cuda, cap):
    frames = _frames(6)
    pts, d_all, begin, cams = _packed(cuda, frames)
    multi = CudaVolume(0.02, 1 << 19, 0.08, cap, 1 << 20)
    single = CudaVolume(0.02, 1 << 19, 0.08, cap, 1 << 20)
    ref = oracle.OracleVolume(0.02, 1 << 19, 0.08, cap, 1 << 20)
    # Two calls of three frames each.
    for lo in (0, 3):
        sub = [b - begin[lo] for b in begin[lo:lo + 4]]
        multi.integrate_frames(d_all[begin[lo]:begin[lo + 3]], sub, cams[lo:lo + 3])
    for k, f in enumerate(frames):
        single.integrate(d_all[begin[k]:begin[k + 1]], f.cam)
        ref.integrate(pts[k], f.cam)
    assert multi.block_count() == single.block_count() == ref.block_count()
    assert multi.drop_count() == single.drop_count() == 0
    if cap == 6.0:
        assert multi.last_update_stats()["crossing_voxels"] > 0
    assert_same_blocks(multi, ref)
    assert_same_voxels(multi, ref)     # weights and colour exact, mean TSDF within 1e-5
    assert_same_voxels(multi, single)  # the same against one call per frame
    assert multi.status() == 0


def test_uneven_and_empty_frames(cuda):
    """Frames of different sizes, frame boundaries inside a 128-point tile,
    and an empty frame."""
    frames = _frames(5, (320, 240), seed=2)
    pts = [scenes.frame_points(f) for f in frames]
    pts[1] = pts[1][:1000]          # small frame, ends mid-tile
    pts[3] = pts[3][:0]             # empty frame
    pts[4] = pts[4][37:]            # starts mid-tile
    begin = [0] + [int(x) for x in np.cumsum([p.shape[0] for p in pts])]
    cams = np.array([f.cam for f in frames], dtype=np.float32)
    d_all = cuda.from_numpy(np.concatenate(pts)).cuda()
    multi = CudaVolume(0.02, 1 << 16, 0.08, 6.0)
    ref = oracle.OracleVolume(0.02, 1 << 16, 0.08, 6.0)
    multi.integrate_frames(d_all, begin, cams)
    for p, f in zip(pts, frames):
        if p.shape[0]:
            ref.integrate(p, f.cam)
    assert_same_blocks(multi, ref)
    assert_same_voxels(multi, ref)
    assert multi.status() == 0


def test_one_frame_per_call_is_integrate(cuda):
    frames = _frames(3, (320, 240), seed=1)
    pts, d_all, begin, cams = _packed(cuda, frames)
    a = CudaVolume(0.02, 1 << 16, 0.08, 6.0)
    b = CudaVolume(0.02, 1 << 16, 0.08, 6.0)
    for k, f in enumerate(frames):
        a.integrate_frames(d_all[begin[k]:begin[k + 1]], [0, begin[k + 1] - begin[k]], cams[k:k + 1])
        b.integrate(d_all[begin[k]:begin[k + 1]], f.cam)
    _bits_equal(a, b)


def test_pipelined_frames(cuda):
    frames = _frames(8)
    pts, d_all, begin, cams = _packed(cuda, frames)
    pipe = CudaVolume(0.02, 1 << 19, 0.08, 64.0, 1 << 20)
    pipe.set_pipelined(True)
    serial = CudaVolume(0.02, 1 << 19, 0.08, 64.0, 1 << 20)
    for lo in (0, 2, 4, 6):
        sub = [b - begin[lo] for b in begin[lo:lo + 3]]
        for v in (pipe, serial):
            v.integrate_frames(d_all[begin[lo]:begin[lo + 2]], sub, cams[lo:lo + 2])
    assert pipe.block_count() == serial.block_count()
    _bits_equal(pipe, serial)
    assert pipe.status() == 0


@pytest.mark.parametrize("cap", [64.0, 6.0])
def test_fp16_frames_against_fp64_oracle(cuda, cap):
    frames = _frames(4)
    pts, d_all, begin, cams = _packed(cuda, frames)
    h = CudaVolume(0.02, 1 << 19, 0.08, cap, 1 << 20, storage=STORAGE_FP16_U16)
    o = CudaVolume(0.02, 1 << 19, 0.08, cap, 1 << 20, storage=STORAGE_FP64)
    h.integrate_frames(d_all, begin, cams)
    for k, f in enumerate(frames):
        o.integrate(d_all[begin[k]:begin[k + 1]], f.cam)
    ch, _, wh = precision._aligned(h)
    co, _, wo = precision._aligned(o)
    assert np.array_equal(ch, co) and np.array_equal(wh, wo), "blocks or weights differ"
    e = precision.tsdf_errors(h, o, 0.08)
    assert e["max_m"] <= FP16_TOL * 0.08, e


def test_frames_argument_checks(cuda):
    frames = _frames(2, (160, 120))
    _, d_all, begin, cams = _packed(cuda, frames)
    v = CudaVolume(0.02, 1 << 12, 0.08, 64.0)
    with pytest.raises(ValueError):
        v.integrate_frames(d_all, [0, 10, 5], cams)           # decreasing
    with pytest.raises(ValueError):
        v.integrate_frames(d_all, [3, 10, begin[-1]], cams)  # does not start at 0
    with pytest.raises(ValueError):
        v.integrate_frames(d_all, begin[:2], cams)              # one entry short
    n = MAX_FRAMES + 1
    with pytest.raises(ValueError):
        v.integrate_frames(d_all, np.arange(n + 1), np.zeros((n, 3)))  # too many frames
    with pytest.raises(ValueError):
        v.integrate_frames(d_all, [0, 0, 0], cams)              # no points
    o = CudaVolume(0.02, 1 << 12, 0.08, 64.0, storage=STORAGE_FP64)
    with pytest.raises(ValueError):
        o.integrate_frames(d_all, begin, cams)
    assert v.block_count() == 0 and v.status() == 0
    assert v.storage == STORAGE_FP32


@pytest.mark.parametrize("res,cap,max_range", [((640, 480), 64.0, 0.0), ((320, 240), 6.0, 3.0)])
def test_depth_frames_equal_point_frames_and_per_image_calls(cuda, res, cap, max_range):
    scene = scenes.RoomScene.make(2)
    K = scenes.ROOM_K.scaled(*res)
    frames = [scenes.room_frame(scene, k, K) for k in range(4)]
    depth = cuda.from_numpy(np.stack([f.depth for f in frames])).cuda()
    Rs = np.stack([f.R for f in frames])
    ts = np.stack([f.t for f in frames])
    pts = [scenes.frame_points(f, max_range) for f in frames]
    begin = [0] + [int(x) for x in np.cumsum([p.shape[0] for p in pts])]
    cams = np.array([f.cam for f in frames], dtype=np.float32)
    dep = CudaVolume(0.02, 1 << 17, 0.08, cap, 1 << 18)
    pts_vol = CudaVolume(0.02, 1 << 17, 0.08, cap, 1 << 18)
    per_image = CudaVolume(0.02, 1 << 17, 0.08, cap, 1 << 18)
    dep.integrate_depth_frames(depth, K, Rs, ts, max_range)
    pts_vol.integrate_frames(cuda.from_numpy(np.concatenate(pts)).cuda(), begin, cams)
    for k, f in enumerate(frames):
        per_image.integrate_depth(depth[k], K, f.R, f.t, max_range)
    assert dep.status() == 0 and dep.block_count() > 0
    _bits_equal(dep, pts_vol)
    assert dep.drop_count() == pts_vol.drop_count()
    assert_same_voxels(dep, per_image)
    if cap == 6.0:
        assert dep.last_update_stats()["crossing_voxels"] > 0


def test_depth_frames_argument_checks(cuda):
    frames = _frames(2, (160, 120))
    depth = cuda.from_numpy(np.stack([f.depth for f in frames])).cuda()
    Rs = np.stack([f.R for f in frames])
    ts = np.stack([f.t for f in frames])
    K = scenes.ROOM_K.scaled(160, 120)
    v = CudaVolume(0.02, 1 << 12, 0.08, 64.0)
    with pytest.raises(ValueError):
        v.integrate_depth_frames(depth, K, Rs[:1], ts[:1])       # one pose short
    with pytest.raises(ValueError):
        v.integrate_depth_frames(depth[0], K, Rs[:1], ts[:1])    # not (F, H, W)
    n = MAX_DEPTH_FRAMES + 1
    many = depth[:1].expand(n, -1, -1).contiguous()
    with pytest.raises(ValueError):
        v.integrate_depth_frames(many, K, np.repeat(Rs[:1], n, 0), np.repeat(ts[:1], n, 0))
    o = CudaVolume(0.02, 1 << 12, 0.08, 64.0, storage=STORAGE_FP64)
    with pytest.raises(ValueError):
        o.integrate_depth_frames(depth, K, Rs, ts)
    assert v.block_count() == 0 and v.status() == 0
