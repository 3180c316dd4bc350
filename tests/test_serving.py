"""Serving loop (continuous batching over the batched engine).

Sessions of mixed resolution, voxel size and table size send integrate and
extract requests with interleaved arrivals. Every session's result must be
the same as integrating it alone with osn_tsdf_cuda_integrate (bit-identical
block sets, weights and mean TSDF: the batched passes compute exactly what
the single-volume passes compute), and every extract must return the vertex
count the lone volume gives after the same frames. Admission against a small
memory budget must hold sessions back until earlier ones finish.
"""
import numpy as np
import pytest

import oracle
from helpers import FP16_ORACLE_TOL, assert_matches_oracle
from what_irregularity_costs_b200 import STORAGE_FP16_U16, CudaVolume, precision, scenes
from what_irregularity_costs_b200.serving import Request, Server, footprint_bytes, poisson_schedule
from what_irregularity_costs_b200.workloads import SceneSpec

pytestmark = pytest.mark.gpu


def _specs():
    # index, seed, slots, voxel, width, height, frames
    return [
        SceneSpec(0, 11, 1 << 16, 0.02, 320, 240, 5),
        SceneSpec(1, 12, 1 << 15, 0.03, 160, 120, 7),
        SceneSpec(2, 13, 1 << 17, 0.015, 640, 480, 4),
        SceneSpec(3, 14, 1 << 14, 0.04, 160, 120, 6),
        SceneSpec(4, 15, 1 << 16, 0.025, 320, 240, 3, cap=6.0),
    ]


def _frames(sp, n):
    sc = scenes.RoomScene.make(sp.seed)
    K = scenes.ROOM_K.scaled(sp.width, sp.height)
    out = []
    for k in range(n):
        f = scenes.room_frame(sc, k, K)
        out.append((scenes.frame_points(f), f.cam))
    return out


def _alone(torch, sp, frames, extract_after):
    v = CudaVolume(sp.voxel, sp.pool, sp.trunc, sp.cap, sp.hash_slots, storage=STORAGE_FP16_U16)
    counts = {}
    for k in range(sp.frames):
        p, cam = frames[k % len(frames)]
        v.integrate(torch.from_numpy(p).cuda(), cam)
        if k in extract_after:
            buf = torch.empty((1 << 24, 6), dtype=torch.float32, device="cuda")
            counts[k] = v.extract_mesh_device(buf, None, buf.shape[0], 0.5, 0.0)
    v.synchronize()
    return v, counts


def _check(torch, specs, frames, reqs, server):
    for sp in specs:
        ks = {r.frame for r in reqs if r.kind == "extract" and r.session == sp.index}
        alone, counts = _alone(torch, sp, frames[sp.index], ks)
        served = server.finished[sp.index]
        ca, ma, wa = precision._aligned(alone)
        cs, ms, ws = precision._aligned(served)
        assert np.array_equal(ca, cs), f"session {sp.index}: block sets differ"
        assert np.array_equal(wa, ws), f"session {sp.index}: weights differ"
        assert np.array_equal(ma, ms), f"session {sp.index}: mean TSDF differs"
        for r in reqs:
            if r.kind == "extract" and r.session == sp.index:
                assert r.vertices == counts[r.frame] and r.vertices > 0
        # The served session against the CPU oracle fed the same frames: block
        # set and weights exact, mean TSDF within FP16 storage's bound.
        ref = oracle.OracleVolume(sp.voxel, sp.pool, sp.trunc, sp.cap, sp.hash_slots)
        for k in range(sp.frames):
            p, cam = frames[sp.index][k % len(frames[sp.index])]
            ref.integrate(p, cam)
        assert_matches_oracle(served, ref, tol=FP16_ORACLE_TOL)


def test_served_sessions_equal_alone(cuda):
    """Saturated: every request visible at once, so steps carry several sessions."""
    specs = _specs()
    frames = [_frames(sp, 3) for sp in specs]  # distinct frames, cycled
    reqs = poisson_schedule(specs, rate_fps=500.0, extract_every=2, seed=3)
    server = Server(budget_bytes=60e9, graph=True)
    server.keep_volumes = True
    try:
        stats = server.run(specs, frames, reqs, realtime=False)
        assert stats["frames"] == sum(sp.frames for sp in specs)
        assert stats["frames_per_step"] > 1.0  # requests of different sessions shared steps
        assert server.batch.status() == 0
        _check(cuda, specs, frames, reqs, server)
    finally:
        server.close()


def test_realtime_arrivals(cuda):
    """Poisson arrivals in real time: every request completes after it
    arrived, latencies are reported, results still equal the lone volumes."""
    specs = _specs()
    frames = [_frames(sp, 2) for sp in specs]
    reqs = poisson_schedule(specs, rate_fps=3000.0, extract_every=3, seed=9)
    server = Server(budget_bytes=60e9, graph=True, autotune_steps=1)
    server.keep_volumes = True
    try:
        stats = server.run(specs, frames, reqs, realtime=True)
        assert all(r.done >= r.arrival for r in reqs)
        assert stats["integrate_latency_ms"]["p50"] > 0
        assert stats["integrate_latency_ms"]["p99"] is not None
        _check(cuda, specs, frames, reqs, server)
    finally:
        server.close()


def test_admission_by_memory_budget(cuda):
    specs = _specs()
    frames = [_frames(sp, 2) for sp in specs]
    reqs = poisson_schedule(specs, rate_fps=2000.0, extract_every=0, seed=5)
    fps = [footprint_bytes(sp, STORAGE_FP16_U16) for sp in specs]
    budget = sorted(fps)[-1] + sorted(fps)[-2] + 1  # two of the largest at most
    server = Server(budget_bytes=budget, graph=False)
    server.keep_volumes = True
    try:
        stats = server.run(specs, frames, reqs, realtime=False)
        assert stats["frames"] == sum(sp.frames for sp in specs)
        assert stats["peak_ledger_gb"] * 1e9 <= budget
        assert stats["peak_sessions"] < len(specs)  # later sessions waited for memory
        _check(cuda, specs, frames, reqs, server)
    finally:
        server.close()


def test_eviction_to_host_and_back(cuda):
    """Four sessions taking turns under a budget that holds two: idle
    sessions are snapshotted to host and restored on their next request,
    and every result still equals the lone volume."""
    specs = _specs()[:4]
    frames = [_frames(sp, 2) for sp in specs]
    reqs = []
    t = 0.0
    for turn in range(3):  # each session gets a burst of frames, then waits for the others
        for sp in specs:
            for j in range(2):
                k = 2 * turn + j
                if k < sp.frames:
                    reqs.append(Request("integrate", sp.index, k, t))
                    t += 0.004
            t += 0.02
    fps = sorted(footprint_bytes(sp, STORAGE_FP16_U16) for sp in specs)
    budget = fps[-1] + fps[-2] + 1
    server = Server(budget_bytes=budget, graph=False, evict=True)
    server.keep_volumes = True
    try:
        stats = server.run(specs, frames, reqs, realtime=True)
        assert stats["frames"] == len(reqs)
        assert stats["evictions"] > 0 and stats["restores"] > 0
        assert stats["peak_ledger_gb"] * 1e9 <= budget
        for sp in specs:
            used = [r for r in reqs if r.session == sp.index]
            sp2 = SceneSpec(sp.index, sp.seed, sp.hash_slots, sp.voxel, sp.width, sp.height,
                            len(used), cap=sp.cap)
            alone, _ = _alone(cuda, sp2, frames[sp.index], set())
            ca, ma, wa = precision._aligned(alone)
            cs, ms, ws = precision._aligned(server.finished[sp.index])
            assert np.array_equal(ca, cs) and np.array_equal(wa, ws) and np.array_equal(ma, ms)
    finally:
        server.close()
