"""Storage modes: FP16 mean TSDF + uint16 weight, and the FP64 on-device oracle.

Through the C ABI (create_ex with OSN_TSDF_STORAGE_*), on the same seeded
room frames as the FP32 parity tests:

* every mode allocates the identical block set and accepts the identical
  contributions (weights equal), because hashing, coordinates and the cap
  selection are integer work shared by all modes;
* the FP64 oracle agrees with the CPU oracle within FP32_VS_FP64_TOL: it
  differs only by evaluating each signed distance in double, so the gap is
  the FP32 rounding of the reference's own arithmetic;
* FP16 storage stays within FP16_TOL of the FP64 oracle (the running
  average is formed in FP32 and rounded to half once per batch, so the
  stored mean carries a few half-precision roundings at most);
* meshes of every mode pass the reference's mesh gate against the FP64
  oracle's mesh.
"""
import numpy as np
import pytest

import oracle
from helpers import assert_same_blocks
from what_irregularity_costs_b200 import (STORAGE_FP16_U16, STORAGE_FP32, STORAGE_FP64, CudaVolume,
                                          precision, scenes)

pytestmark = pytest.mark.gpu

# Mean normalised TSDF, FP16 storage vs the FP64 oracle: four half ulps at 1.
FP16_TOL = 4 * 2.0 ** -11
# Mean normalised TSDF, FP32 (the reference's arithmetic, which the CPU oracle
# and the FP32 path share) vs the FP64 oracle. The signed distance is the
# difference of two distances of up to ~9 m, each carrying a few FP32
# roundings (~1e-6 m); over an 8 cm truncation that is ~1e-5 normalised, so
# the bound leaves a margin above the observed ~2e-5.
FP32_VS_FP64_TOL = 1e-4


def _room_batches(n, seed=0, K=None):
    scene = scenes.RoomScene.make(seed)
    out = []
    for k in range(n):
        f = scenes.room_frame(scene, k, K) if K is not None else scenes.room_frame(scene, k)
        out.append((scenes.frame_points(f), f.cam))
    return out


def _run(torch, batches, storage, voxel=0.02, pool=1 << 19, trunc=0.08, cap=64.0, slots=0,
         split=False):
    vol = CudaVolume(voxel, pool, trunc, cap, slots, storage=storage)
    for pts, cam in batches:
        d = torch.from_numpy(np.ascontiguousarray(pts)).cuda()
        if split:
            vol.allocate_blocks(d, cam)
            vol.update_voxels(d, cam)
        else:
            vol.integrate(d, cam)
    vol.synchronize()
    assert vol.status() == 0
    return vol


def _same_weights(a, b):
    ca, _, wa = precision._aligned(a)
    cb, _, wb = precision._aligned(b)
    assert np.array_equal(ca, cb)
    assert np.array_equal(wa, wb), "weights differ between storage modes"


@pytest.mark.parametrize("cap", [64.0, 6.0])
def test_fp64_oracle_matches_cpu_oracle(cuda, cap):
    batches = _room_batches(3)
    g = _run(cuda, batches, STORAGE_FP64, cap=cap)
    ref = oracle.OracleVolume(0.02, 1 << 19, 0.08, cap)
    for pts, cam in batches:
        ref.integrate(pts, cam)
    assert_same_blocks(g, ref)
    coords, mean, w = precision._aligned(g)
    rc, rt, rw = ref.voxels()[:3]
    order = np.lexsort(rc.T[::-1])
    rc, rt, rw = rc[order], rt[order], rw[order]
    assert np.array_equal(coords, rc)
    assert np.array_equal(w, rw.astype(np.float64)), "FP64 weights differ from the CPU oracle"
    seen = rw > 0
    err = np.max(np.abs(mean[seen] - rt[seen].astype(np.float64) / rw[seen]))
    assert err <= FP32_VS_FP64_TOL, f"FP64 oracle vs CPU oracle: {err:.3e}"


@pytest.mark.parametrize("cap", [64.0, 6.0, 0.0])
def test_fp16_u16_against_fp64_oracle(cuda, cap):
    batches = _room_batches(4)
    h = _run(cuda, batches, STORAGE_FP16_U16, cap=cap)
    o = _run(cuda, batches, STORAGE_FP64, cap=cap)
    f = _run(cuda, batches, STORAGE_FP32, cap=cap)
    assert h.device_view().r is None and h.device_view().tsdf
    assert h.lib.osn_tsdf_cuda_storage(h.h) == STORAGE_FP16_U16
    _same_weights(h, o)
    _same_weights(f, o)
    e16 = precision.tsdf_errors(h, o, 0.08)
    e32 = precision.tsdf_errors(f, o, 0.08)
    assert e16["max_m"] <= FP16_TOL * 0.08, e16
    assert e32["max_m"] <= FP32_VS_FP64_TOL * 0.08, e32
    assert e32["max_m"] <= e16["max_m"]
    assert e16["rms_m"] > 0.0  # half precision is visibly coarser than FP32


def test_fp16_split_passes_equal_integrate(cuda):
    batches = _room_batches(2)
    a = _run(cuda, batches, STORAGE_FP16_U16)
    b = _run(cuda, batches, STORAGE_FP16_U16, split=True)
    ca, ma, wa = precision._aligned(a)
    cb, mb, wb = precision._aligned(b)
    assert np.array_equal(ca, cb) and np.array_equal(wa, wb) and np.array_equal(ma, mb)


def test_fp16_weight_saturates_at_u16_max(cuda):
    """No cap: uint16 weights stop at 65535 (the effective cap), FP32 keeps counting."""
    pts = oracle.plane_points(0.30, 0.25, 120)
    batch = [(pts, (0.0, 0.0, 0.0))]
    vol = CudaVolume(0.01, 1 << 12, -1.0, 0.0, storage=STORAGE_FP16_U16)
    d = cuda.from_numpy(pts).cuda()
    for _ in range(3):
        vol.integrate(d, (0.0, 0.0, 0.0))
    _, _, w = vol.means()
    w1 = w.max()
    assert w1 > 0 and vol.status() == 0
    # Fill towards the limit with repeated frames and check it never exceeds it.
    reps = int(np.ceil(65535 / (w1 / 3))) + 2
    for _ in range(reps):
        vol.integrate(d, (0.0, 0.0, 0.0))
    _, mean, w = vol.means()
    assert w.max() == 65535.0
    ref = _run(cuda, batch, STORAGE_FP64, voxel=0.01, pool=1 << 12, trunc=-1.0, cap=0.0)
    _, m64, w64 = precision._aligned(ref)
    _, m16, _ = precision._aligned(vol)
    seen = w64 > 0
    # Every frame is the same, so the mean stays that of one frame.
    assert np.max(np.abs(m16[seen] - m64[seen])) <= FP16_TOL


@pytest.mark.parametrize("storage", [STORAGE_FP16_U16, STORAGE_FP64])
def test_meshes_pass_the_gate_against_fp64(cuda, storage):
    f = scenes.sphere_frame()
    pts = scenes.frame_points(f)
    batch = [(pts, f.cam)]
    v = _run(cuda, batch, storage, voxel=0.01, pool=1 << 15, trunc=0.04, cap=64.0)
    o = _run(cuda, batch, STORAGE_FP64, voxel=0.01, pool=1 << 15, trunc=0.04, cap=64.0)
    mv, cv = v.extract_mesh(1 << 20, 0.5, 0.0, rgb=True)
    mo = o.extract_mesh(1 << 20, 0.5, 0.0)
    assert mv is not None and mo is not None
    assert abs(len(mv) - len(mo)) <= 0.01 * len(mo)
    e = precision.mesh_errors(mv, mo)
    assert e["chamfer_m"] < 0.01 / 100 and e["hausdorff_m"] < 0.01 / 10, e
    assert np.all(cv == 128)
    # Analytic sphere gate (cpp/tests/test_analytic.cpp:86-104).
    r = np.linalg.norm(mv[:, :3].astype(np.float64) - np.array([0.0, 0.0, 2.0]), axis=1)
    assert np.abs(r - 0.5).mean() < 0.01 / 4 and np.abs(r - 0.5).max() < 0.01


def test_fp16_reset_and_reuse(cuda):
    batches = _room_batches(2)
    vol = _run(cuda, batches, STORAGE_FP16_U16)
    _, m1, w1 = precision._aligned(vol)
    vol.reset()
    assert vol.block_count() == 0
    for pts, cam in batches:
        vol.integrate(cuda.from_numpy(pts).cuda(), cam)
    _, m2, w2 = precision._aligned(vol)
    assert np.array_equal(w1, w2) and np.array_equal(m1, m2)


def test_storage_rejects_unknown_mode(cuda):
    with pytest.raises(ValueError):
        CudaVolume(0.02, 1 << 10, 0.08, 64.0, storage=7)
