"""CUDA path vs the oracle, through the C ABI, on seeded inputs.

Mirrors the reference's GPU test (cpp/tests/test_cuda_analytic.cu): the
analytic gates of tier 1 and the cross-arm gates of tier 3, plus the
edge cases of cpp/tests/test_analytic.cpp (pool exhaustion) and this
library's extensions (explicit table size, device extraction, measurement
entry points).
"""
import numpy as np
import pytest

import oracle
from helpers import (TSDF_TOL, assert_same_blocks, assert_same_voxels, canonical_triangles,
                     sphere_errors, surface_distance)
from what_irregularity_costs_b200 import CudaVolume, scenes

pytestmark = pytest.mark.gpu


def _pair(torch, batches, voxel, pool, trunc=-1.0, cap=32.0, hash_slots=0, radius=0.0,
          split=False):
    gpu = CudaVolume(voxel, pool, trunc, cap, hash_slots)
    ref = oracle.OracleVolume(voxel, pool, trunc, cap, hash_slots)
    for pts, cam in batches:
        d = torch.from_numpy(np.ascontiguousarray(pts)).cuda()
        if split:
            gpu.allocate_blocks(d, cam, radius)
            gpu.update_voxels(d, cam, radius)
        else:
            gpu.integrate(d, cam, radius)
        ref.integrate(pts, cam, radius)
    gpu.synchronize()
    return gpu, ref


def _mesh_checks(gpu, ref, voxel, min_w=0.5):
    gm = gpu.extract_mesh(4 << 20, min_w, 0.0)
    rm = ref.extract(min_w, 0.0, 4 << 20)
    assert gm is not None and rm is not None
    nv_g, nv_r = gm.shape[0], rm.shape[0]
    rel = abs(nv_g - nv_r) / max(nv_g, nv_r, 1)
    assert rel < 0.01, f"vertex counts {nv_g} vs {nv_r}"
    if nv_g and nv_r:
        mean_d, haus = surface_distance(gm, rm)
        assert mean_d < voxel * 0.01, f"mean surface distance {mean_d}"
        assert haus < voxel * 0.1, f"hausdorff {haus}"
    return gm, rm


def test_sphere_frame_320x240(cuda):
    """The 320x240 sphere frame: 1 cm voxels, trunc 4 cm, 2^16 slots, cap 64."""
    f = scenes.sphere_frame()
    pts = scenes.frame_points(f)
    gpu, ref = _pair(cuda, [(pts, f.cam)], 0.01, 1 << 15, 0.04, 64.0)
    assert gpu.device_view().hash_mask + 1 == 1 << 16
    assert gpu.status() == 0
    assert gpu.drop_count() == 0 == ref.drop_count()
    assert_same_blocks(gpu, ref)
    assert_same_voxels(gpu, ref)
    gm, rm = _mesh_checks(gpu, ref, 0.01)
    assert gm.shape[0] == rm.shape[0]
    mean_e, max_e = sphere_errors(gm, (0, 0, 2), 0.5)
    assert mean_e < 0.01 / 4 and max_e < 0.01


def test_reference_sphere_known_answer(cuda):
    """The reference's analytic sphere (400x800 points from the centre, 1 cm):
    1160 blocks and 846,288 vertices in every arm of the reference."""
    pts = oracle.sphere_points(0.5, 400, 800)
    gpu, ref = _pair(cuda, [(pts, (0.0, 0.0, 0.0))], 0.01, 1 << 14)
    assert gpu.block_count() == 1160 == ref.block_count()
    assert gpu.drop_count() == 0
    assert_same_blocks(gpu, ref)
    assert_same_voxels(gpu, ref)
    gm, rm = _mesh_checks(gpu, ref, 0.01)
    assert rm.shape[0] == 846288
    mean_e, max_e = sphere_errors(gm, (0, 0, 0), 0.5)
    assert mean_e < 0.01 / 4 and max_e < 0.01


def test_plane(cuda):
    """cpp/tests/test_analytic.cpp:109-141: plane z = 0.3 seen from below."""
    pts = oracle.plane_points(0.30, 0.25, 500)
    gpu, ref = _pair(cuda, [(pts, (0.0, 0.0, 0.0))], 0.01, 1 << 14)
    assert_same_blocks(gpu, ref)
    assert_same_voxels(gpu, ref)
    gm, _ = _mesh_checks(gpu, ref, 0.01)
    dz = np.abs(gm[:, 2] - 0.30)
    assert gm.shape[0] > 1000 and dz.mean() < 0.01 / 4 and dz.max() < 0.01


@pytest.mark.parametrize("cap", [64.0, 6.0, 0.0])
def test_room_frames_capped(cuda, cap):
    """Three 640x480 room frames (2 cm, trunc 8 cm, 2^20 slots). A cap of 6
    forces many voxels to cross the cap inside one frame, which exercises the
    ordered selection; cap 0 disables capping."""
    scene = scenes.RoomScene.make(0)
    frames = [scenes.room_frame(scene, k) for k in range(3)]
    batches = [(scenes.frame_points(f), f.cam) for f in frames]
    gpu, ref = _pair(cuda, batches, 0.02, 1 << 19, 0.08, cap)
    stats = gpu.last_update_stats()
    if cap == 6.0:
        assert stats["crossing_voxels"] > 0
    assert gpu.status() == 0
    assert_same_blocks(gpu, ref)
    assert_same_voxels(gpu, ref)
    _mesh_checks(gpu, ref, 0.02)


@pytest.mark.parametrize("voxel", [0.005, 0.01, 0.02, 0.04])
def test_voxel_sizes(cuda, voxel):
    scene = scenes.RoomScene.make(3)
    K = scenes.ROOM_K.scaled(320, 240)
    f = scenes.room_frame(scene, 5, K)
    pts = scenes.frame_points(f)
    gpu, ref = _pair(cuda, [(pts, f.cam)], voxel, 1 << 18, -1.0, 64.0)
    assert gpu.drop_count() == 0
    assert_same_blocks(gpu, ref)
    assert_same_voxels(gpu, ref)


@pytest.mark.parametrize("load", [0.25, 0.5, 0.75, 0.9])
def test_load_factors(cuda, load):
    """Explicit table sizes (create_ex) at the sweep's load factors."""
    f = scenes.sphere_frame()
    pts = scenes.frame_points(f)
    probe = oracle.OracleVolume(0.01, 1 << 15, 0.04, 64.0)
    probe.allocate(pts, f.cam)
    blocks = probe.block_count()
    slots = 1 << int(np.ceil(np.log2(blocks / load)))
    gpu, ref = _pair(cuda, [(pts, f.cam)], 0.01, blocks, 0.04, 64.0, hash_slots=slots)
    assert gpu.device_view().hash_mask + 1 == slots
    assert gpu.block_count() == blocks
    assert_same_blocks(gpu, ref)
    assert_same_voxels(gpu, ref)


def test_pool_exhaustion(cuda):
    """cpp/tests/test_analytic.cpp:187-203: a pool of 16 blocks reports drops.
    Which 16 blocks win depends on the order of insertion, but every sample
    is accounted for: with no cap, each block that got into the pool holds
    exactly the samples the oracle gives it with an unbounded pool, and the
    samples of every other block are counted as dropped."""
    pts = oracle.sphere_points(0.5, 200, 400)
    gpu, ref = _pair(cuda, [(pts, (0.0, 0.0, 0.0))], 0.005, 16, cap=0.0)
    assert gpu.drop_count() > 0
    assert gpu.block_count() == 16
    assert ref.drop_count() > 0 and ref.block_count() == 16
    assert gpu.status() == 0
    big = oracle.OracleVolume(0.005, 1 << 16, -1.0, 0.0)
    big.integrate(pts, (0.0, 0.0, 0.0))
    assert big.drop_count() == 0
    bc, bt, bw, *_ = big.voxels()
    per_block = {tuple(c): (t, w) for c, t, w in zip(bc.tolist(), bt, bw)}
    gc, gt, gw, *_ = gpu.voxels()
    for c, t, w in zip(gc.tolist(), gt, gw):
        assert tuple(c) in per_block, "an allocated block the scene does not touch"
        rt, rw = per_block[tuple(c)]
        assert np.array_equal(w, rw), f"block {c} lost samples"
        seen = rw > 0
        assert np.max(np.abs(t[seen] / w[seen] - rt[seen] / rw[seen])) <= TSDF_TOL
    assert float(gw.sum()) + gpu.drop_count() == float(bw.sum())


def test_pool_exactly_full(cuda):
    """The pool holds exactly the frame's blocks: the last insertions race with
    lookups of the same keys while the pool fills. Every sample must still be
    counted and binned the same way (no drops, voxels equal)."""
    scene = scenes.RoomScene.make(2)
    f = scenes.room_frame(scene, 0)
    pts = scenes.frame_points(f)
    probe = oracle.OracleVolume(0.02, 1 << 19, 0.08, 64.0)
    probe.allocate(pts, f.cam)
    blocks = probe.block_count()
    gpu, ref = _pair(cuda, [(pts, f.cam)], 0.02, blocks, 0.08, 64.0)
    assert gpu.block_count() == blocks and gpu.drop_count() == 0 == ref.drop_count()
    assert gpu.status() == 0
    assert_same_blocks(gpu, ref)
    assert_same_voxels(gpu, ref)


def test_many_rays_through_one_voxel(cuda):
    """3000 rays through the same voxels plus a sparse frame: voxels with
    thousands of records in one batch cross the cap in the big-block path."""
    rng = np.random.default_rng(7)
    same = np.repeat(np.float32([[0.31, -0.27, 1.93]]), 3000, axis=0)
    jitter = (np.float32([0.31, -0.27, 1.93]) +
              rng.normal(0, 0.01, size=(2000, 3)).astype(np.float32))
    pts = np.concatenate([same, jitter, same[:500]]).astype(np.float32)
    gpu, ref = _pair(cuda, [(pts, (0.0, 0.0, 0.0)), (pts[::3], (0.0, 0.0, 0.0))], 0.01, 1 << 12,
                     0.04, 64.0)
    assert gpu.status() == 0
    assert_same_blocks(gpu, ref)
    assert_same_voxels(gpu, ref)
    _, _, w, *_ = ref.voxels()
    assert w.max() == 64.0


def test_radius_cutoff_and_offset_camera(cuda):
    """Far cutoff and a camera far from the origin (negative block coordinates)."""
    f = scenes.sphere_frame()
    pts = scenes.frame_points(f) + np.float32([-7.3, -2.1, -9.9])
    cam = (-7.3, -2.1, -9.9)
    gpu, ref = _pair(cuda, [(pts, cam)], 0.01, 1 << 15, 0.04, 64.0, radius=1.9)
    assert 0 < gpu.block_count() < 2000
    assert_same_blocks(gpu, ref)
    assert_same_voxels(gpu, ref)


def test_separate_passes_and_repeat(cuda):
    """allocate_blocks then update_voxels as two calls, the same frame twice."""
    f = scenes.sphere_frame()
    pts = scenes.frame_points(f)
    gpu, ref = _pair(cuda, [(pts, f.cam), (pts, f.cam)], 0.01, 1 << 15, 0.04, 3.0, split=True)
    assert_same_blocks(gpu, ref)
    assert_same_voxels(gpu, ref)


def test_update_without_allocation_writes_nothing(cuda):
    f = scenes.sphere_frame()
    d = cuda.from_numpy(scenes.frame_points(f)).cuda()
    gpu = CudaVolume(0.01, 1 << 15, 0.04, 64.0)
    gpu.update_voxels(d, f.cam)
    assert gpu.block_count() == 0
    assert gpu.last_update_stats()["records"] == 0


def test_bad_arguments(cuda):
    gpu = CudaVolume(0.01, 1 << 10)
    d = cuda.zeros((4, 3), dtype=cuda.float32, device="cuda")
    with pytest.raises(ValueError):
        gpu.allocate_blocks(d[:0], (0, 0, 0))
    with pytest.raises(ValueError):
        gpu.update_voxels(0, (0, 0, 0), n=4)
    with pytest.raises(ValueError):
        CudaVolume(0.0, 16)
    with pytest.raises(ValueError):
        CudaVolume(0.01, 0)
    with pytest.raises(ValueError):
        CudaVolume(0.01, 16, hash_slots=48)
    # Points on the camera are gated out, as in the reference.
    gpu.integrate(d, (0, 0, 0))
    assert gpu.block_count() == 0


def test_reset_restores_empty_state(cuda):
    f = scenes.sphere_frame()
    pts = scenes.frame_points(f)
    d = cuda.from_numpy(pts).cuda()
    gpu = CudaVolume(0.01, 1 << 15, 0.04, 64.0)
    gpu.integrate(d, f.cam)
    first = gpu.voxels()
    gpu.reset()
    assert gpu.block_count() == 0 and gpu.drop_count() == 0
    keys, idx = gpu.table()
    assert np.all(keys == -1) and np.all(idx == -1)
    gpu.integrate(d, f.cam)
    again = gpu.voxels()
    o1 = np.lexsort(first[0].T[::-1])
    o2 = np.lexsort(again[0].T[::-1])
    for a, b in zip(first, again):
        assert np.array_equal(a[o1], b[o2])


def test_table_layout_matches_reference(cuda):
    """Keys are packed coordinates at their linear-probe slots; indices are
    published; the scratch region holds -2."""
    f = scenes.sphere_frame()
    pts = scenes.frame_points(f)
    gpu, ref = _pair(cuda, [(pts, f.cam)], 0.01, 1 << 15, 0.04, 64.0)
    keys, idx = gpu.table()
    coords = gpu.coords()
    live = keys >= 0
    assert live.sum() == gpu.block_count()
    bias = 1 << 20
    packed = ((coords[:, 0].astype(np.int64) + bias) << 42) | \
             ((coords[:, 1].astype(np.int64) + bias) << 21) | (coords[:, 2].astype(np.int64) + bias)
    assert np.array_equal(np.sort(keys[live]), np.sort(packed))
    assert np.array_equal(np.sort(idx[live]), np.arange(gpu.block_count()))
    assert np.array_equal(packed[idx[live]], keys[live])
    view = gpu.device_view()
    from what_irregularity_costs_b200 import device_tensor
    scratch = device_tensor(view.table + 16 * view.scratch_base, (4, 4), "<i4").cpu().numpy()
    assert np.all(scratch[:, :2].copy().view(np.int64) == -2)
    assert view.block_dim == 8 and abs(view.voxel_size_m - 0.01) < 1e-9
    assert abs(view.trunc_m - 0.04) < 1e-9 and view.weight_cap == 64.0


def test_measurement_entry_points(cuda):
    f = scenes.sphere_frame()
    pts = scenes.frame_points(f)
    d = cuda.from_numpy(pts).cuda()
    ref = oracle.OracleVolume(0.01, 1 << 15, 0.04, 64.0)
    ref.allocate(pts, f.cam)

    nocas = CudaVolume(0.01, 1 << 15, 0.04, 64.0)
    nocas.allocate_no_cas(d, f.cam)
    assert nocas.block_count() == 0 and nocas.drop_count() == 0

    counting = CudaVolume(0.01, 1 << 15, 0.04, 64.0)
    counting.allocate_counting_cas(d, f.cam)
    assert counting.block_count() == ref.block_count()
    assert counting.drop_count() >= counting.block_count()
    assert_same_blocks(counting, ref)

    slot = CudaVolume(0.01, 1 << 15, 0.04, 64.0)
    slot.allocate_slot_index(d, f.cam)
    assert slot.block_count() == ref.block_count()

    hist_vol = CudaVolume(0.01, 1 << 15, 0.04, 64.0)
    hist = hist_vol.allocate_probe_histogram(d, f.cam, n_bins=16)
    assert hist.sum() >= ref.block_count()
    assert_same_blocks(hist_vol, ref)


def test_extract_device_and_rgb(cuda):
    f = scenes.sphere_frame()
    pts = scenes.frame_points(f)
    gpu, ref = _pair(cuda, [(pts, f.cam)], 0.01, 1 << 15, 0.04, 64.0)
    host_pos, host_rgb = gpu.extract_mesh(1 << 20, 0.5, 0.0, rgb=True)
    ref_pos, ref_rgb = ref.extract(0.5, 0.0, 1 << 20, rgb=True)
    assert host_pos.shape == ref_pos.shape and host_rgb.shape == ref_rgb.shape
    # Through this ABI every contribution is grey, so every vertex of both
    # arms interpolates 128 between two corners of colour 128.
    assert np.all(host_rgb == 128) and np.all(ref_rgb == 128)
    cap = host_pos.shape[0]
    dpos = cuda.empty((cap, 6), dtype=cuda.float32, device="cuda")
    drgb = cuda.empty((cap, 3), dtype=cuda.uint8, device="cuda")
    n = gpu.extract_mesh_device(dpos, drgb, cap, 0.5, 0.0)
    assert n == cap
    assert np.array_equal(canonical_triangles(dpos.cpu().numpy()), canonical_triangles(host_pos))
    # Too small a buffer reports overflow, as the reference does.
    assert gpu.extract_mesh(cap - 1, 0.5, 0.0) is None


def test_mesh_bitwise_when_voxels_bitwise(cuda):
    """Where every voxel receives one contribution the sums have nothing to
    reorder, the voxel arrays are bit-identical, and so is the mesh. A 40x40
    grid of points at voxel centres on the plane z = 0.305, seen from a
    camera 100 m away on the axis: the rays are all but parallel, so each
    band voxel meets exactly one sample, and the band is closed."""
    i = np.arange(40, dtype=np.float32)
    x = (i + np.float32(0.5)) * np.float32(0.01) - np.float32(0.2)
    gx, gy = np.meshgrid(x, x)
    pts = np.stack([gx.ravel(), gy.ravel(), np.full(gx.size, 0.305, np.float32)], 1).astype(np.float32)
    gpu, ref = _pair(cuda, [(pts, (0.0, 0.0, -100.0))], 0.01, 1 << 12)
    _, rt, rw = [a for a in oracle_sorted(ref)[:3]]
    assert rw.max() == 1 and int((rw == 1).sum()) == 12800
    assert_same_voxels(gpu, ref, exact_tsdf=True)
    gm = gpu.extract_mesh(1 << 20, 0.5, 0.0)
    rm = ref.extract(0.5, 0.0, 1 << 20)
    assert gm is not None and gm.shape[0] == rm.shape[0] == 36504
    assert np.array_equal(canonical_triangles(gm).view(np.uint32),
                          canonical_triangles(rm).view(np.uint32))


def oracle_sorted(ref):
    from helpers import sorted_voxels
    return sorted_voxels(ref)


def test_tolerance_is_stated():
    assert TSDF_TOL == 1e-5
