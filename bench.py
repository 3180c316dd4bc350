"""Benchmark: 640x480 frames/s of the TSDF integrate path on B200.

Workload (one step): reset the volume, then integrate every frame of the
seeded 100-frame room trajectory (640x480, fx=fy=320, 2 cm voxels, trunc
8 cm, 2^20 table slots, pool 2^19 blocks, weight cap 64), i.e. allocate +
update of every frame through the C ABI. frames/s = frames integrated / time.

  value  device-resident points (uploaded once), CUDA events on the volume's
         stream around exactly K steps, max over ranks; the frames go through
         osn_tsdf_cuda_integrate_frames, 4 consecutive frames per call
         (--frames-per-call), serial updates (value_frames_pipelined: the
         same with pipelined updates). value_per_frame: one
         osn_tsdf_cuda_integrate call per frame, pipelined; value_serial:
         one call per frame, serial;
  e2e    the headline arm from pinned HOST buffers: every call's points are
         copied host->device inside the timed region (double-buffered on a
         copy stream) and the block and drop counters are read back per step
         (e2e_per_frame: the same with one integrate call per frame;
         e2e_depth: per-frame depth images unprojected on the GPU);
  roofline  per-kernel CUDA-event times of one instrumented step; the
         dominant kernel's algorithmic bytes per launch / its mean duration
         against the measured HBM copy bandwidth;
  cpu_baseline  the reference's own CPU arm (oracle/_ref, all host threads)
         on a bounded sample of the same frames.

--impl reference times only the reference CPU arm (rank 0) on the same
workload, each step a bounded sample of frames.

Multi-GPU: one process per GPU under torchrun, each integrating its own
replica of the trajectory (independent volumes, no collective on the data
path): weak scaling.
"""
from __future__ import annotations

import argparse
import atexit
import json
import multiprocessing as mp
import os
import statistics
import subprocess
import sys
import time
from concurrent.futures import ProcessPoolExecutor

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

VOXEL, TRUNC, CAP = 0.02, 0.08, 64.0
SLOTS_PER_POINT = 2 * 4 + 1   # band samples per point: 2 * ceil(trunc / voxel) + 1
HASH_SLOTS, POOL = 1 << 20, 1 << 19
N_FRAMES, SEED = 100, 0
FRAMES_PER_CALL = 4  # frames per osn_tsdf_cuda_integrate_frames call in the headline arm
METRIC = "frames/s (640x480 integrate)"
PROFILES = os.path.join(ROOT, "profiles")


def _frame_points(args):
    seed, k = args
    from what_irregularity_costs_b200 import scenes
    scene = scenes.RoomScene.make(seed)
    f = scenes.room_frame(scene, k)
    return scenes.frame_points(f), f.cam, (f.depth, f.R, f.t)


_DEPTH = []  # depth frames and poses of the last make_trajectory call


def make_trajectory(n_frames=N_FRAMES, seed=SEED, workers=None):
    """Points of every frame (generated in spawned workers, before any CUDA use);
    the depth images and poses they came from are kept in _DEPTH."""
    workers = workers or min(16, os.cpu_count() or 1)
    ctx = mp.get_context("spawn")
    with ProcessPoolExecutor(max_workers=workers, mp_context=ctx) as ex:
        out = list(ex.map(_frame_points, [(seed, k) for k in range(n_frames)]))
    pts = [p for p, _, _ in out]
    cams = [c for _, c, _ in out]
    _DEPTH[:] = [d for _, _, d in out]
    return pts, cams


def measured_peak():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(p) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def profile_traffic(kernel):
    """DRAM bytes per launch of `kernel` on one room frame, from its committed
    ncu summary (profiles/<kernel>_room640.md)."""
    try:
        with open(os.path.join(PROFILES, f"{kernel}_room640.md")) as f:
            for line in f:
                if line.startswith("traffic_bytes_per_launch:"):
                    return float(line.split(":", 1)[1].split()[0])
    except OSError:
        pass
    return None


class ClockSampler:
    """nvidia-smi clocks and throttle reasons while the timed region runs."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.rows = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                 "-lms", "100"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
        return self

    def __exit__(self, *exc):
        if getattr(self, "rows", None) is not None:  # already stopped
            return
        self.rows = []
        if self.proc is None:
            return
        self.proc.terminate()
        try:
            out, _ = self.proc.communicate(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
            out, _ = self.proc.communicate()
        for line in out.splitlines():
            parts = [p.strip() for p in line.split(",")]
            if len(parts) >= 9:
                self.rows.append(parts)

    def summary(self):
        rows = self.rows or []
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": reasons, "samples": len(rows)}


def dist_setup(n_gpus, backend="nccl"):
    """Rank, local rank, world size and the process group module (None alone).
    One process per GPU; the data path has no collective (replicas): the
    group only carries the timing barrier and the max over ranks. The short
    timeout ends a collective with an error when a rank is gone."""
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=120))
        return rank, local, world, dist
    return 0, 0, 1, None


def _device(dist):
    return "cuda" if dist is None or dist.get_backend() == "nccl" else "cpu"


def barrier(dist, torch):
    if torch.cuda.is_available():
        torch.cuda.synchronize()
    if dist is not None:
        dist.barrier()


def max_over_ranks(x, dist, torch):
    """The job's time is the slowest rank's."""
    if dist is None:
        return x
    t = torch.tensor([x], dtype=torch.float64, device=_device(dist))
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def frame_groups(offsets, cams, frames_per_call):
    """Consecutive frames in groups of frames_per_call (the last may be
    shorter): (first frame, end frame, first point, end point, frame_begin
    relative to the group's first point (int32, one entry per frame plus
    one), cameras (float32, one row per frame)) per integrate_frames call."""
    offsets = np.asarray(offsets, dtype=np.int64)
    n = len(offsets) - 1
    out = []
    for lo in range(0, n, frames_per_call):
        hi = min(n, lo + frames_per_call)
        begin = np.asarray(offsets[lo:hi + 1] - offsets[lo], dtype=np.int32)
        out.append((lo, hi, int(offsets[lo]), int(offsets[hi]), begin,
                    np.ascontiguousarray(np.asarray(cams[lo:hi], dtype=np.float32))))
    return out


def replica_work(frames_per_rank, world):
    """Frames the whole job integrates: every rank runs its own replica."""
    return frames_per_rank * world


# ---------------------------------------------------------------------------


def sorted_fp32_voxels(coords, tsdf, weight, r, g, b):
    """The five FP32 voxel arrays with blocks in coordinate order."""
    order = np.lexsort(coords.T[::-1]) if coords.shape[0] else np.zeros(0, dtype=np.int64)
    return coords[order], tsdf[order], weight[order], r[order], g[order], b[order]


def parity_vs_oracle(gpu_arrays, pts, cams, path):
    """The headline run's volume against the CPU oracle fed the same frames one
    at a time (outside every timed region): block set, weights and colour sums
    exact, mean TSDF within the float parity bar of 1e-5."""
    import oracle
    t0 = time.perf_counter()
    ref = oracle.OracleVolume(VOXEL, POOL, TRUNC, CAP, HASH_SLOTS)
    for p, c in zip(pts, cams):
        ref.integrate(p, c)
    rc, rt, rw, rr, rg, rb = sorted_fp32_voxels(*ref.voxels())
    gc, gt, gw, gr, gg, gb = gpu_arrays
    out = {"path": path, "frames": len(pts), "oracle": "oracle/tsdf_oracle.c (single-threaded)",
           "tol_mean_tsdf": 1e-5, "oracle_s": None}
    out["blocks"] = "exact" if gc.shape == rc.shape and np.array_equal(gc, rc) else "differ"
    if out["blocks"] != "exact":
        out.update(weights=None, colour=None, max_mean_tsdf_err=None, ok=False)
        return out
    out["weights"] = "exact" if np.array_equal(gw, rw) else f"{int(np.sum(gw != rw))} differ"
    out["colour"] = "exact" if all(np.array_equal(x, y) for x, y in ((gr, rr), (gg, rg), (gb, rb))) \
        else "differ"
    seen = rw > 0
    err = float(np.max(np.abs(gt[seen] / gw[seen] - rt[seen] / rw[seen]))) if seen.any() else 0.0
    out["max_mean_tsdf_err"] = err
    out["blocks_n"] = int(gc.shape[0])
    out["ok"] = out["weights"] == "exact" and out["colour"] == "exact" and err <= 1e-5
    out["oracle_s"] = round(time.perf_counter() - t0, 1)
    return out


def l2_ceilings(lib, bytes_=32 << 20):
    """Measured L2 ceilings of this GPU (osn_tsdf_cuda_l2_probe on a 32 MiB,
    L2-resident buffer): reductions and atomics in G ops/s, streamed loads in
    GB/s, random 4-byte loads in G loads/s."""
    import ctypes as C
    out = {"buffer_bytes": bytes_}
    for kind, name, iters in ((0, "red_u64_gops", 256), (1, "red_u32_gops", 256), (2, "atom_u32_gops", 128),
                              (3, "load16_gbps", 512), (4, "load4_random_gloads", 256)):
        r = C.c_double(0.0)
        rc = lib.osn_tsdf_cuda_l2_probe(kind, bytes_, iters, C.addressof(r))
        out[name] = r.value if rc == 0 else None
    return out


def cpu_reference_rate(pts, cams, budget_s=15.0, threads=None, max_frames=None):
    """Reference CPU arm (osn_tsdf_create/_integrate, all host threads) on the
    first max_frames frames of the trajectory, each pass from an empty volume,
    passes repeated until budget_s is spent (at least one). Returns (frames/s,
    frames integrated, threads, seconds)."""
    import ctypes as C
    import oracle
    lib = oracle.ref_lib()
    threads = threads or (os.cpu_count() or 1)
    sample = list(zip(pts, cams))[: max_frames or len(pts)]
    done, t_total = 0, 0.0
    while True:
        v = lib.osn_tsdf_create(VOXEL, POOL, TRUNC, CAP)
        lib.osn_tsdf_set_thread_count(v, threads)
        try:
            for p, cam in sample:
                ptr = p.ctypes.data_as(C.POINTER(C.c_float))
                t0 = time.perf_counter()
                rc = lib.osn_tsdf_integrate(v, ptr, None, None, p.shape[0], 0, *cam, 0.0)
                t_total += time.perf_counter() - t0
                if rc != 0:
                    raise RuntimeError(f"reference integrate returned {rc}")
                done += 1
        finally:
            lib.osn_tsdf_destroy(v)
        if t_total > budget_s:
            break
    return done / t_total, done, threads, t_total


def a3_gpu_rate(d_all, offsets, cams, steps, torch):
    """The reference's own CUDA arm (cpp/src/volume_cuda.cu, built for sm_100a
    into oracle/_ref by oracle/Makefile) on the same device-resident frames:
    allocate_blocks + update_voxels per frame through its C ABI, CUDA events
    around each pass over the trajectory; its reset (a full memset of the
    pool) is outside the timed region, as in the reference's own harness
    (cpp/bench/bench_arms.cu:707-753)."""
    import ctypes as C
    path = os.path.join(ROOT, "oracle", "_ref", "libosn_tsdf_a3.so")
    if not os.path.exists(path):
        return None
    lib = C.CDLL(path)
    lib.osn_tsdf_cuda_create.restype = C.c_void_p
    lib.osn_tsdf_cuda_create.argtypes = [C.c_float, C.c_int32, C.c_float, C.c_float]
    for name in ("osn_tsdf_cuda_allocate_blocks", "osn_tsdf_cuda_update_voxels"):
        getattr(lib, name).argtypes = [C.c_void_p, C.c_void_p, C.c_int32] + [C.c_float] * 4
    lib.osn_tsdf_cuda_reset.argtypes = [C.c_void_p]
    lib.osn_tsdf_cuda_synchronize.argtypes = [C.c_void_p]
    lib.osn_tsdf_cuda_block_count.argtypes = [C.c_void_p]
    lib.osn_tsdf_cuda_drop_count.argtypes = [C.c_void_p]
    lib.osn_tsdf_cuda_drop_count.restype = C.c_uint64
    lib.osn_tsdf_cuda_destroy.argtypes = [C.c_void_p]
    v = lib.osn_tsdf_cuda_create(VOXEL, POOL, TRUNC, CAP)
    if not v:
        return None
    total_ms = 0.0
    try:
        for step in range(steps + 1):  # the first pass is a warm-up
            lib.osn_tsdf_cuda_reset(v)
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()  # legacy default stream: ordered with the arm's blocking stream
            for k in range(len(cams)):
                a, b = int(offsets[k]), int(offsets[k + 1])
                ptr = d_all.data_ptr() + a * 12
                lib.osn_tsdf_cuda_allocate_blocks(v, ptr, b - a, *cams[k], 0.0)
                lib.osn_tsdf_cuda_update_voxels(v, ptr, b - a, *cams[k], 0.0)
            lib.osn_tsdf_cuda_synchronize(v)
            e1.record()
            torch.cuda.synchronize()
            if step > 0:
                total_ms += e0.elapsed_time(e1)
        blocks = lib.osn_tsdf_cuda_block_count(v)
        drops = lib.osn_tsdf_cuda_drop_count(v)
    finally:
        lib.osn_tsdf_cuda_destroy(v)
    return {"impl": "reference CUDA arm (A3, cpp/src/volume_cuda.cu) built for sm_100a, same GPU",
            "value": len(cams) * steps / (total_ms / 1e3), "unit": "frames/s",
            "ms_per_step": total_ms / steps, "blocks": blocks, "drops": int(drops)}


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    import oracle
    if not oracle.ref_available():
        print(json.dumps({"impl": "reference", "unavailable":
                          "reference CPU arm not built (oracle/_ref/libosn_tsdf_ref.so missing)"}))
        return 0
    frames = min(args.ref_frames, N_FRAMES)
    all_pts, all_cams = make_trajectory(N_FRAMES)
    pts, cams = all_pts[:frames], all_cams[:frames]
    threads = os.cpu_count() or 1
    rates = []
    for i in range(args.warmup + args.steps):
        rate, done, _, t = cpu_reference_rate(pts, cams, budget_s=0.0, threads=threads)
        if i >= args.warmup:
            rates.append((done, t))
    total_frames = sum(d for d, _ in rates)
    total_t = sum(t for _, t in rates)
    value = total_frames / total_t
    sample = f"first {frames} frames of the room trajectory per step, from an empty volume"
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "frames/s",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1e3 * total_t / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": config_dict(points=int(sum(p.shape[0] for p in all_pts))),
        "cpu_baseline": {"value": value, "unit": "frames/s", "cores": threads,
                         "kind": "reference", "sample": sample},
        "e2e": {"value": value, "unit": "frames/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))
    return 0


def set_workload(frames, pool):
    """Frames per step and pool size (the defaults are the benchmark's workload)."""
    global N_FRAMES, POOL
    N_FRAMES, POOL = int(frames), int(pool)


def config_dict(points):
    return {
        "workload": f"room trajectory, {N_FRAMES} frames 640x480 fx=fy=320, 2 cm voxels, "
                    f"trunc 8 cm, 2^20 table slots, pool {POOL} blocks, weight cap 64; step = "
                    "reset + allocate/update of every frame",
        "frames_per_step": N_FRAMES, "resolution": [640, 480], "voxel_m": VOXEL,
        "trunc_m": TRUNC, "hash_slots": HASH_SLOTS, "pool_blocks": POOL, "weight_cap": CAP,
        "points_per_step": points, "seed": SEED,
        "l2": "inputs larger than L2: %.0f MB of points per step" % (points * 12 / 1e6),
    }


def run_ours(args):
    pts, cams = make_trajectory(N_FRAMES)   # before any CUDA use (spawned workers)
    import torch
    from what_irregularity_costs_b200 import CudaVolume, KERNEL_NAMES

    rank, local, world, dist = dist_setup(args.gpus)
    torch.cuda.set_device(local)
    n_points = int(sum(p.shape[0] for p in pts))
    offsets = np.concatenate([[0], np.cumsum([p.shape[0] for p in pts])])
    all_pts = np.concatenate(pts).astype(np.float32)
    d_all = torch.from_numpy(all_pts).cuda()
    host_pinned = torch.from_numpy(all_pts).pin_memory()

    vol = CudaVolume(VOXEL, POOL, TRUNC, CAP, HASH_SLOTS)
    vstream = torch.cuda.ExternalStream(vol.stream_handle())

    def step_device():
        vol.reset()
        for k in range(N_FRAMES):
            a, b = int(offsets[k]), int(offsets[k + 1])
            vol.integrate(d_all[a:b], cams[k])
        vol.join()  # the last tails are part of the step

    # Several frames per call: consecutive frames of the trajectory in groups.
    fpc = max(1, min(args.frames_per_call, N_FRAMES))
    groups = frame_groups(offsets, cams, fpc)

    def step_frames():
        vol.reset()
        for lo, hi, a, b, begin, gcams in groups:
            vol.integrate_frames(d_all[a:b], begin, gcams)
        vol.join()

    def timed(step, steps):
        """W warm-up steps, then K steps between CUDA events on the volume's
        stream, barriers on both sides; the max over ranks (ms)."""
        for _ in range(args.warmup):
            step()
        barrier(dist, torch)
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        ev0.record(vstream)
        for _ in range(steps):
            step()
        ev1.record(vstream)
        barrier(dist, torch)
        return max_over_ranks(ev0.elapsed_time(ev1), dist, torch)

    # Clocks are sampled over every timed arm below (the headline arm alone
    # is shorter than the sampling interval).
    clocks = ClockSampler(local)
    clocks.__enter__()
    atexit.register(clocks.__exit__, None, None, None)  # never leave the sampler running

    # -- value_serial: one call per frame, one update after the other (the
    # reference's stream order)
    serial_ms = timed(step_device, args.steps)
    # -- value_per_frame: one call per frame, pipelined updates (each call's
    # tail overlaps the next walk)
    vol.set_pipelined(True)
    per_frame_ms = timed(step_device, args.steps)
    # -- value_frames_pipelined: FRAMES_PER_CALL frames per call, pipelined
    frames_pipe_ms = timed(step_frames, args.steps)
    # -- value: FRAMES_PER_CALL frames per integrate_frames call, serial
    # updates (every kernel of a call launched behind its predecessor on the
    # volume's stream; measured faster than the pipelined form at 3-8 frames
    # per call, whose cross-stream waits cost more than the overlap gains)
    vol.set_pipelined(False)
    ms = timed(step_frames, args.steps)
    blocks = vol.block_count()
    drops = vol.drop_count()
    status = vol.status()
    # The headline run's volume, kept for the parity check against the oracle.
    headline_voxels = sorted_fp32_voxels(*vol.voxels()) if rank == 0 else None
    frames_total = replica_work(N_FRAMES * args.steps, world)
    value = frames_total / (ms / 1e3)

    # -- e2e: pinned host buffers, copies inside the timed region ------------
    max_n = max(int(np.max(np.diff(offsets))), max(b - a for _, _, a, b, _, _ in groups))
    stage = [torch.empty((max_n, 3), dtype=torch.float32, device="cuda") for _ in range(2)]
    cstream = torch.cuda.Stream()
    copied = [torch.cuda.Event() for _ in range(2)]
    free = [torch.cuda.Event() for _ in range(2)]
    result = torch.zeros(2, dtype=torch.int64).pin_memory()

    def step_e2e():
        vol.reset()
        for k in range(N_FRAMES):
            a, b = int(offsets[k]), int(offsets[k + 1])
            s = k & 1
            with torch.cuda.stream(cstream):
                cstream.wait_event(free[s])
                stage[s][: b - a].copy_(host_pinned[a:b], non_blocking=True)
                copied[s].record(cstream)
            vstream.wait_event(copied[s])
            vol.integrate(stage[s][: b - a], cams[k])
            free[s].record(vstream)  # the walk has read the frame (the tail never does)
        result[0] = vol.block_count()
        result[1] = vol.drop_count()

    def step_e2e_frames():
        vol.reset()
        for g, (lo, hi, a, b, begin, gcams) in enumerate(groups):
            s = g & 1
            with torch.cuda.stream(cstream):
                cstream.wait_event(free[s])
                stage[s][: b - a].copy_(host_pinned[a:b], non_blocking=True)
                copied[s].record(cstream)
            vstream.wait_event(copied[s])
            vol.integrate_frames(stage[s][: b - a], begin, gcams)
            free[s].record(vstream)
        result[0] = vol.block_count()
        result[1] = vol.drop_count()

    for s in range(2):
        free[s].record(vstream)
    # e2e_per_frame: one integrate call per frame, pipelined updates
    vol.set_pipelined(True)
    e2e_pf_ms = timed(step_e2e, args.steps)
    e2e_per_frame = frames_total / (e2e_pf_ms / 1e3)
    # e2e: the headline arm (FRAMES_PER_CALL frames per call, serial updates)
    vol.set_pipelined(False)
    e2e_ms = timed(step_e2e_frames, args.steps)
    e2e_value = frames_total / (e2e_ms / 1e3)

    # -- e2e from depth images: 4 B per pixel uploaded, unprojected on the GPU
    from what_irregularity_costs_b200 import scenes as _scenes
    K = _scenes.ROOM_K
    depth_host = [torch.from_numpy(d).pin_memory() for d, _, _ in _DEPTH]
    dstage = [torch.empty(depth_host[0].shape, dtype=torch.float32, device="cuda") for _ in range(2)]
    dbytes = int(sum(d.nbytes for d, _, _ in _DEPTH))

    def step_e2e_depth():
        vol.reset()
        for k in range(N_FRAMES):
            s_ = k & 1
            with torch.cuda.stream(cstream):
                cstream.wait_event(free[s_])
                dstage[s_].copy_(depth_host[k], non_blocking=True)
                copied[s_].record(cstream)
            vstream.wait_event(copied[s_])
            _, R_, t_ = _DEPTH[k]
            vol.integrate_depth(dstage[s_], K, R_, t_)
            free[s_].record(vstream)
        result[0] = vol.block_count()
        result[1] = vol.drop_count()

    vol.set_pipelined(True)
    e2e_depth_ms = timed(step_e2e_depth, args.steps)
    vol.set_pipelined(False)
    blocks_depth = vol.block_count()

    # -- the same with several depth images per call (integrate_depth_frames)
    depth_all = torch.from_numpy(np.stack([d for d, _, _ in _DEPTH])).pin_memory()
    dfpc = max(1, min(fpc, 16))
    dgroups = []
    for lo in range(0, N_FRAMES, dfpc):
        hi = min(N_FRAMES, lo + dfpc)
        dgroups.append((lo, hi, np.stack([_DEPTH[k][1] for k in range(lo, hi)]),
                        np.stack([_DEPTH[k][2] for k in range(lo, hi)])))
    dfstage = [torch.empty((dfpc,) + tuple(depth_all.shape[1:]), dtype=torch.float32, device="cuda")
               for _ in range(2)]

    def step_e2e_depth_frames():
        vol.reset()
        for g, (lo, hi, Rs_, ts_) in enumerate(dgroups):
            s_ = g & 1
            with torch.cuda.stream(cstream):
                cstream.wait_event(free[s_])
                dfstage[s_][: hi - lo].copy_(depth_all[lo:hi], non_blocking=True)
                copied[s_].record(cstream)
            vstream.wait_event(copied[s_])
            vol.integrate_depth_frames(dfstage[s_][: hi - lo], K, Rs_, ts_)
            free[s_].record(vstream)
        result[0] = vol.block_count()
        result[1] = vol.drop_count()

    e2e_depth_frames_ms = timed(step_e2e_depth_frames, args.steps)
    blocks_depth_frames = vol.block_count()
    clocks.__exit__(None, None, None)

    # -- one instrumented step of the headline arm: per-kernel CUDA-event
    # times (every launch of the volume bracketed on its stream; no
    # synchronisation between calls; serial mode, so kernels do not overlap)
    vol.set_pipelined(False)
    vol.set_timing(True)
    vol.kernel_times()  # flush
    base = vol.kernel_times()
    vol.reset()
    for lo, hi, a, b, begin, gcams in groups:
        vol.integrate_frames(d_all[a:b], begin, gcams)
    # Extraction of the trajectory's volume into a device buffer (the
    # marching-tetrahedra kernel alone is timed).
    ext_cap = 1 << 24
    ext_buf = torch.empty((ext_cap, 6), dtype=torch.float32, device="cuda")
    ext_blocks = vol.block_count()
    ext_verts = vol.extract_mesh_device(ext_buf, None, ext_cap, 0.5, 0.0)
    del ext_buf
    # Allocation alone (allocate_blocks), for the allocate Mrays/s figure.
    vol.reset()
    for k in range(N_FRAMES):
        a, b = int(offsets[k]), int(offsets[k + 1])
        vol.allocate_blocks(d_all[a:b], cams[k])
    times = vol.kernel_times()
    vol.set_timing(False)
    per_kernel = {k: (times[k][0] - base[k][0], times[k][1] - base[k][1]) for k in KERNEL_NAMES}
    # -- stage statistics of every call of the headline arm (read back per
    # call; untimed)
    vol.reset()
    updated, records, touched, crossing = [], [], [], []
    for lo, hi, a, b, begin, gcams in groups:
        vol.integrate_frames(d_all[a:b], begin, gcams)
        st = vol.last_update_stats()
        updated.append(st["updated_voxels"])
        records.append(st["records"])
        touched.append(st["touched_blocks"])
        crossing.append(st["crossing_voxels"])
    # -- allocation's L2 atomics (CAS attempts counted by the measurement
    # mode; each new block adds its pool-counter add and its publishing
    # exchange) and the probe-depth histogram of every resolved block run
    vol.reset()
    cas = 0
    for k in range(N_FRAMES):
        a, b = int(offsets[k]), int(offsets[k + 1])
        before = vol.drop_count()
        vol.allocate_counting_cas(d_all[a:b], cams[k])
        cas += vol.drop_count() - before
    alloc_atomics = int(cas) + 2 * vol.block_count()
    vol.reset()
    hist = np.zeros(32, dtype=np.uint64)
    for k in range(N_FRAMES):
        a, b = int(offsets[k]), int(offsets[k + 1])
        hist += vol.allocate_probe_histogram(d_all[a:b], cams[k], n_bins=32)
    probes_mean = float(np.sum(hist * np.arange(32)) / max(1, int(hist.sum())))
    integrate_kernels = ("band", "finish", "group", "select")
    # Launches of the headline arm: per integrate_frames call the set-up
    # kernel and the four passes; reset's two per step.
    launches_per_step = (1 + sum(1 for k in integrate_kernels if per_kernel[k][1] > 0)) * len(groups) + 2
    dominant = max(integrate_kernels, key=lambda k: per_kernel[k][0])

    peak, peak_kind = measured_peak()
    t_alloc = per_kernel["allocate"][0] / 1e3
    t_update = sum(per_kernel[k][0] for k in integrate_kernels) / 1e3
    n_slots = n_points * SLOTS_PER_POINT
    n_rec, n_touch = int(np.sum(records)), int(np.sum(touched))
    # Bytes each kernel must move, every structure touched once. Band walk:
    # 12 B per point read, a 4-byte record per band slot written, and per
    # counted sample a 4-byte count and an 8-byte fixed-point sum reduced
    # (16 B with the read of the voxel's weight).
    alg_total = {
        "band": 12 * n_points + 4 * n_slots + 16 * n_rec,
        "finish": n_touch * 512 * (16 + 36),   # read cnt,w,t,sum; write t,w,r,g,b,cnt,sum
        "group": 4 * n_slots,   # the record of every band slot
        "select": 0,
    }
    # Update as the reference scopes it: positions + tsdf/weight tiles of the
    # touched blocks, read and written; the stricter figure counts only the
    # voxels that were updated.
    update_alg_bytes = 12 * n_points + n_touch * 512 * 2 * 8
    update_alg_bytes_voxels = 12 * n_points + int(np.sum(updated)) * 2 * 8
    # Extraction: each allocated block's 512 voxels and 217 halo voxels read
    # (tsdf and weight, 8 bytes), 24 bytes written per vertex.
    t_extract = per_kernel["extract"][0] / 1e3
    extract_alg_bytes = ext_blocks * (512 + 217) * 8 + 24 * max(ext_verts, 0)
    dom_ms, dom_n = per_kernel[dominant]
    dom_alg = alg_total.get(dominant, 0) / dom_n if dom_n else 0.0
    achieved = dom_alg / (dom_ms / 1e3 / dom_n) / 1e9 if dom_n else 0.0
    roofline = {
        "bound": "hbm", "kernel": dominant, "achieved": achieved, "peak": peak, "unit": "GB/s",
        "frac": achieved / peak, "peak_source": peak_kind,
        # The headline's walk launches are band_frames_kernel (several frames per call).
        "traffic": profile_traffic("band_frames" if dominant == "band" and fpc > 1 else dominant),
        "alg_bytes_per_launch": dom_alg, "mean_launch_us": 1e3 * dom_ms / dom_n if dom_n else None,
    }
    # The roofs the L2-resident kernels are judged against: the band walk's
    # per-sample reductions (a 4-byte count and an 8-byte sum per counted
    # sample) against the measured L2 reduction rate at that 1:1 mix; finish's
    # tile bytes against the measured L2 streaming rate.
    from what_irregularity_costs_b200 import _lib as _l
    l2 = l2_ceilings(_l.load())
    t_band = per_kernel["band"][0] / 1e3
    t_fin = per_kernel["finish"][0] / 1e3
    r32, r64 = l2.get("red_u32_gops"), l2.get("red_u64_gops")
    red_mix = 2.0 / (1.0 / r32 + 1.0 / r64) if r32 and r64 else None
    band_red = 2.0 * n_rec / t_band / 1e9 if t_band else None
    fin_gbps = alg_total["finish"] / t_fin / 1e9 if t_fin else None
    roofline["l2"] = {
        "ceilings": l2,
        "band": {"achieved_red_gops": band_red, "peak_red_gops": red_mix,
                 "frac": band_red / red_mix if band_red and red_mix else None,
                 "unit": "G reductions/s (count u32 + sum u64 per counted sample)"},
        "finish": {"achieved_gbps": fin_gbps, "peak_gbps": l2.get("load16_gbps"),
                   "frac": fin_gbps / l2["load16_gbps"] if fin_gbps and l2.get("load16_gbps") else None,
                   "unit": "GB/s of tile bytes (read + written) against L2 streaming loads"},
    }

    a3 = None
    if rank == 0 and not args.no_a3:
        try:
            a3 = a3_gpu_rate(d_all, offsets, cams, max(1, min(args.steps, 3)), torch)
        except Exception as e:  # reported beside the line, never required
            a3 = {"impl": "reference CUDA arm (A3)", "value": None, "error": str(e)}

    # -- the batched form against the plain arm on the 32-scene mix: a bounded
    # run (batch_warmup + batch_steps steps) reported beside the headline
    batch32 = None
    if rank == 0 and world == 1 and args.batch_steps > 0:
        try:
            from what_irregularity_costs_b200 import workloads
            specs = workloads.scene_mix(32)
            mix = workloads.mix_frames(specs, args.batch_warmup + args.batch_steps)
            fig = batch32_figures(specs, mix, args.batch_steps, args.batch_warmup, torch)
            errs = [e for e in fig["precision_vs_fp64"]["fp16_u16"] if "max_m" in e]
            batch32 = {
                "metric": "frames/s (32-scene batched integrate)",
                "batched_fp16": fig["value"], "plain_fp32": fig["plain_fp32"]["value"],
                "batched_fp32": fig["batched_fp32"]["value"],
                "ratio_fp16_vs_plain": fig["speedup_vs_plain"],
                "ratio_fp32_vs_plain": fig["batched_fp32"]["value"] / fig["plain_fp32"]["value"],
                "blocks_identical": fig["blocks_identical"],
                "fp16_tsdf_err_max_m": max((e["max_m"] for e in errs), default=None),
                "fp16_tsdf_err_rms_m": max((e["rms_m"] for e in errs), default=None),
                "precision_scenes": len(errs),
                "e2e": fig["e2e"], "steps": args.batch_steps, "warmup": args.batch_warmup,
                "shape": fig["shape"], "status": fig["status"],
                "note": "every scene of the mix advances one frame per step; batched arms are the "
                        "work-queued passes replayed from a CUDA graph; plain = each scene through "
                        "osn_tsdf_cuda_integrate on its own stream",
            }
            del mix
            torch.cuda.synchronize()
        except Exception as e:  # reported beside the line, never required
            batch32 = {"error": str(e)}

    # -- serving: a bounded run of the 64-session configuration (each session's
    # trajectory cut at serve_frames frames), realtime Poisson arrivals
    serve64 = None
    if rank == 0 and world == 1 and args.serve_frames > 0:
        try:
            serve64 = serve64_figures(args.serve_frames, torch)
        except Exception as e:  # reported beside the line, never required
            serve64 = {"error": str(e)}

    parity = None
    if rank == 0 and not args.no_parity:
        try:
            parity = parity_vs_oracle(headline_voxels, pts, cams,
                                      f"osn_tsdf_cuda_integrate_frames, {fpc} frames per call")
        except Exception as e:  # reported, never fatal to the line
            parity = {"ok": False, "error": str(e)}

    cpu = None
    if rank == 0 and not args.no_cpu:
        try:
            import oracle
            if oracle.ref_available():
                nf = min(args.ref_frames, N_FRAMES)
                rate, done, threads, t = cpu_reference_rate(pts, cams, budget_s=args.cpu_budget,
                                                            max_frames=nf)
                cpu = {"value": rate, "unit": "frames/s", "cores": threads, "kind": "reference",
                       "sample": f"the first {nf} frames of the trajectory from an empty volume, "
                                 f"repeated: {done} frames in {t:.1f} s (the sample bench.py "
                                 f"--impl reference times)"}
        except Exception as e:  # the baseline is reported, never required
            cpu = {"value": None, "unit": "frames/s", "cores": None, "kind": "reference",
                   "sample": f"failed: {e}"}

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": "frames/s", "n_gpus": world,
            "value_per_frame": frames_total / (per_frame_ms / 1e3),
            "value_serial": frames_total / (serial_ms / 1e3),
            "value_frames_pipelined": frames_total / (frames_pipe_ms / 1e3),
            "mode": f"osn_tsdf_cuda_integrate_frames, {fpc} frames per call, serial updates; "
                    "value_frames_pipelined: the same with pipelined updates; "
                    "value_per_frame: one osn_tsdf_cuda_integrate per frame, pipelined; "
                    "value_serial: one per frame, serial",
            "frames_per_call": fpc,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic: seeded room trajectory (3 spheres, 2 boxes), depth noise "
                    "0.0015 z^2, 5% invalid pixels, FP64 backprojection",
            "config": config_dict(n_points),
            "roofline": roofline,
            "cpu_baseline": cpu,
            "reference_gpu_arm": a3,
            "e2e": {"value": e2e_value, "unit": "frames/s",
                    "h2d_bytes_per_step": int(all_pts.nbytes), "d2h_bytes_per_step": 16,
                    "path": f"osn_tsdf_cuda_integrate_frames ({fpc} frames per call) from pinned host buffers"},
            "e2e_per_frame": {"value": e2e_per_frame, "unit": "frames/s",
                              "h2d_bytes_per_step": int(all_pts.nbytes), "d2h_bytes_per_step": 16,
                              "path": "osn_tsdf_cuda_integrate per frame from pinned host buffers"},
            "e2e_depth": {"value": frames_total / (e2e_depth_ms / 1e3), "unit": "frames/s",
                          "h2d_bytes_per_step": dbytes, "d2h_bytes_per_step": 16,
                          "path": "osn_tsdf_cuda_integrate_depth (unprojection in the band walk)",
                          "blocks": blocks_depth},
            "e2e_depth_frames": {"value": frames_total / (e2e_depth_frames_ms / 1e3), "unit": "frames/s",
                                 "h2d_bytes_per_step": dbytes, "d2h_bytes_per_step": 16,
                                 "path": f"osn_tsdf_cuda_integrate_depth_frames ({dfpc} images per call)",
                                 "blocks": blocks_depth_frames},
            "gpu_launches": int(launches_per_step * args.steps),
            "clocks": clocks.summary(),
            "alloc_mrays_per_s": n_points / t_alloc / 1e6 if t_alloc else None,
            "alloc_l2_atomics": {
                "ops": alloc_atomics, "gops_per_s": alloc_atomics / t_alloc / 1e9 if t_alloc else None,
                "peak_atom_gops": l2.get("atom_u32_gops"),
                "frac": (alloc_atomics / t_alloc / 1e9 / l2["atom_u32_gops"])
                if t_alloc and l2.get("atom_u32_gops") else None,
                "note": "CAS attempts + pool-counter add + publishing exchange per new block, over "
                        "the allocate-only walk of the trajectory; warp key grouping keeps CAS "
                        "attempts near one per new block"},
            "probe_hist": {"bins": [int(x) for x in hist[:12]], "mean_probes": probes_mean,
                           "unit": "block resolutions by slots probed (bin k = k slots)"},
            "parity": parity,
            "batch32": batch32,
            "serve64": serve64,
            "update_gbps": update_alg_bytes / t_update / 1e9 if t_update else None,
            "update_gbps_updated_voxels": update_alg_bytes_voxels / t_update / 1e9 if t_update else None,
            "extract": {"blocks": ext_blocks, "vertices": ext_verts,
                        "ms": round(1e3 * t_extract, 4) if t_extract else None,
                        "gbps": extract_alg_bytes / t_extract / 1e9 if t_extract else None,
                        "frac": extract_alg_bytes / t_extract / 1e9 / peak if t_extract else None,
                        "alg_bytes": extract_alg_bytes},
            "kernel_ms_per_step": {k: round(v[0], 4) for k, v in per_kernel.items()},
            "kernel_launches_per_step": {k: v[1] for k, v in per_kernel.items()},
            "blocks": blocks, "drops": int(drops), "status": status,
            # Per frame of the headline arm (its calls' counts over the frames).
            "updated_voxels_per_frame": float(np.sum(updated)) / N_FRAMES,
            "touched_blocks_per_frame": float(np.sum(touched)) / N_FRAMES,
            "crossing_voxels_per_frame": float(np.sum(crossing)) / N_FRAMES,
            "records_per_frame": float(np.sum(records)) / N_FRAMES,
        }
        print(json.dumps(line))
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def run_batch32(args):
    """The 32-scene batched mix (what_irregularity_costs_b200.workloads): every
    scene advances one frame per step. Arms, each timed with CUDA events over
    the same steps after the same warm-up frames:
      value        batched, FP16 TSDF + uint16 weight, autotuned shape, steps
                   replayed from a CUDA graph (device-resident frames);
      plain_fp32   each scene integrated alone through osn_tsdf_cuda_integrate
                   (its own stream), FP32 storage -- the plain drop-in arm;
      batched_fp32 the batched arm with FP32 storage;
      e2e          the batched arm with every frame copied from pinned host
                   memory on the batch stream inside the timed region;
      precision    max / RMS TSDF error (m) of the FP16 batch against FP64
                   volumes fed the same frames, first 8 scenes.
    """
    from what_irregularity_costs_b200 import workloads
    specs = workloads.scene_mix(32)
    frames = workloads.mix_frames(specs, args.warmup + args.steps)  # before any CUDA use
    import torch
    rank, local, world, dist = dist_setup(args.gpus)
    torch.cuda.set_device(local)
    fig = batch32_figures(specs, frames, args.steps, args.warmup, torch)
    if rank == 0:
        line = {
            "metric": "frames/s (32-scene batched integrate)", "value": fig["value"],
            "unit": "frames/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f16 tsdf / u16 weight storage, f32 running average",
            "data": "synthetic: 32 seeded room scenes (scene_mix seed 4)",
        }
        line.update(fig)
        print(json.dumps(line))
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def batch32_figures(specs, frames, steps, warmup, torch):
    """The arms of the 32-scene batched mix over the same steps (see
    run_batch32), as a dict: value (batched FP16), plain_fp32, batched_fp32,
    speedup_vs_plain, blocks_identical, precision_vs_fp64, e2e, autotune."""
    from what_irregularity_costs_b200 import (STORAGE_FP16_U16, STORAGE_FP32, STORAGE_FP64, Batch,
                                              device_tensor, precision, workloads)

    class _A:  # the step counts the arms below read
        pass
    args = _A()
    args.steps, args.warmup = steps, warmup
    n_steps = args.warmup + args.steps
    dev = workloads.upload(frames, torch)
    active = [[s.index for s in specs if k < len(frames[s.index])] for k in range(n_steps)]
    timed_frames = sum(len(active[k]) for k in range(args.warmup, n_steps))

    def batched(storage, tune, graph=True, e2e=False, shape=None):
        vols = workloads.make_volumes(specs, storage)
        b = Batch(len(specs))
        for v, sp in zip(vols, specs):
            b.add(v, sp.max_points)
        if shape is not None:
            b.set_shape(shape["tiles_per_item"], 1 if shape["probe"] == "lane" else 0,
                        1 if shape["finish_pair"] else 0)
        bstream = torch.cuda.ExternalStream(b.stream_handle())
        tune_res = None
        if tune:  # live autotuning steps (results do not depend on the shape), then reset
            b.autotune(1)
            for k in range(16):
                kk = k % n_steps
                for si in active[kk]:
                    b.set_frame(si, dev[si][kk], frames[si][kk][1])
                b.step()
            tune_res = b.tune_results()
            b.synchronize()
            for v in vols:
                v.reset()
        b.set_graph(graph)
        stage = host = None
        if e2e:
            stage = [torch.empty((sp.max_points, 3), dtype=torch.float32, device="cuda") for sp in specs]
            host = [[torch.from_numpy(p).pin_memory() for p, _ in fr] for fr in frames]
            view = vols[0].device_view()
            bc_dev = device_tensor(view.block_count, (1,), "<i4")
            bc_host = torch.zeros(1, dtype=torch.int32).pin_memory()
        h2d = [0]

        def step(k):
            for si in active[k]:
                if e2e:
                    n = host[si][k].shape[0]
                    with torch.cuda.stream(bstream):
                        stage[si][:n].copy_(host[si][k], non_blocking=True)
                    b.set_frame(si, stage[si][:n], frames[si][k][1])
                    if k >= args.warmup:
                        h2d[0] += n * 12
                else:
                    b.set_frame(si, dev[si][k], frames[si][k][1])
            b.step()
            if e2e:
                with torch.cuda.stream(bstream):
                    bc_host.copy_(bc_dev, non_blocking=True)

        for k in range(args.warmup):
            step(k)
        b.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(bstream)
        for k in range(args.warmup, n_steps):
            step(k)
        e1.record(bstream)
        b.synchronize()
        ms = e0.elapsed_time(e1)
        status = b.status()
        out = {"value": timed_frames / (ms / 1e3), "unit": "frames/s", "ms_per_step": ms / args.steps,
               "status": status, "shape": b.shape(), "graph": graph}
        if e2e:
            out["h2d_bytes_per_step"] = h2d[0] // args.steps
            out["d2h_bytes_per_step"] = 4
        if tune_res is not None:
            out["tune"] = tune_res
        return out, vols, b

    # -- batched FP16 (the batched form), autotuned and graph-replayed
    res16, vols16, b16 = batched(STORAGE_FP16_U16, tune=True)
    shape = res16["shape"]
    keep = list(range(8))
    snap16 = [precision._aligned(vols16[i]) for i in keep]
    blocks16 = [v.block_count() for v in vols16]
    del b16, vols16
    torch.cuda.synchronize()

    # -- e2e: the same batched arm from pinned host buffers
    res_e2e, v_e2e, b_e2e = batched(STORAGE_FP16_U16, tune=False, e2e=True, shape=shape)
    del b_e2e, v_e2e
    torch.cuda.synchronize()

    # -- batched FP32 (same passes, reference storage)
    res32b, v32b, b32b = batched(STORAGE_FP32, tune=False, shape=shape)
    blocks32b = [v.block_count() for v in v32b]
    del b32b, v32b
    torch.cuda.synchronize()

    # -- plain FP32 arm: every scene alone through the drop-in ABI, own streams
    vols = workloads.make_volumes(specs, STORAGE_FP32)
    streams = [torch.cuda.ExternalStream(v.stream_handle()) for v in vols]
    join = torch.cuda.Stream()

    def plain_step(k):
        for si in active[k]:
            vols[si].integrate(dev[si][k], frames[si][k][1])

    for k in range(args.warmup):
        plain_step(k)
    torch.cuda.synchronize()
    p0, p1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    p0.record(join)
    for st in streams:
        st.wait_event(p0)
    for k in range(args.warmup, n_steps):
        plain_step(k)
    for st in streams:
        ev = torch.cuda.Event()
        ev.record(st)
        join.wait_event(ev)
    p1.record(join)
    torch.cuda.synchronize()
    plain_ms = p0.elapsed_time(p1)
    plain = {"value": timed_frames / (plain_ms / 1e3), "unit": "frames/s",
             "ms_per_step": plain_ms / args.steps}
    blocks_plain = [v.block_count() for v in vols]
    snap32 = [precision._aligned(vols[i]) for i in keep]
    del vols
    torch.cuda.synchronize()

    # -- FP64 oracle for the first 8 scenes (alone), same frames
    errs16, errs32 = [], []
    for i in keep:
        sp = specs[i]
        o = workloads.make_volumes([sp], STORAGE_FP64)[0]
        for k in range(len(frames[i])):
            o.integrate(dev[i][k], frames[i][k][1])
        co, mo, wo = precision._aligned(o)
        for snap, errs in ((snap16[i], errs16), (snap32[i], errs32)):
            c, m, w = snap
            if c.shape != co.shape or not np.array_equal(c, co) or not np.array_equal(w, wo):
                errs.append({"scene": i, "mismatch": True})
                continue
            seen = wo > 0
            e = np.abs(m[seen] - mo[seen]) * sp.trunc
            errs.append({"scene": i, "max_m": float(e.max()) if e.size else 0.0,
                         "rms_m": float(np.sqrt(np.mean(e * e))) if e.size else 0.0})
        del o

    line = {
        "value": res16["value"], "unit": "frames/s", "ms_per_step": res16["ms_per_step"],
        "config": {"workload": "32-scene mix: tables 2^14-2^20 (log-uniform), voxels 1-4 cm "
                               "(log-uniform), 160x120..1280x720, 8-256 frames, cap 64; step = "
                               "every active scene integrates its next frame",
                   "scenes": [s.__dict__ for s in specs], "frames_in_window": timed_frames,
                   "l2": "inputs larger than L2: %.0f MB of points in the timed steps"
                         % (sum(dev[si][k].numel() * 4 for k in range(args.warmup, n_steps)
                                for si in active[k]) / 1e6)},
        "shape": shape, "graph": True, "status": res16["status"],
        "plain_fp32": plain, "batched_fp32": res32b,
        "speedup_vs_plain": res16["value"] / plain["value"],
        "blocks_identical": blocks16 == blocks32b == blocks_plain,
        "precision_vs_fp64": {"fp16_u16": errs16, "fp32": errs32},
        "e2e": {"value": res_e2e["value"], "unit": "frames/s",
                "h2d_bytes_per_step": res_e2e["h2d_bytes_per_step"],
                "d2h_bytes_per_step": res_e2e["d2h_bytes_per_step"]},
        "autotune": res16.get("tune"),
    }
    return line


def run_serve64(args):
    """The serving configuration: 64 concurrent sessions of the scene-mix kind
    (FP16 storage), integrate requests as Poisson streams summing to 2000
    frames/s, an extract request after every 50th frame of a session,
    admission against a 120 GB HBM budget (what_irregularity_costs_b200.serving).
    Each session cycles through 8 distinct frames of its trajectory (the host
    generates 512 frames, not ~8,400). Two runs on the same schedule:
      value      realtime arrivals: frames served per second, with p50/p99
                 integrate and extract latency;
      saturated  every request visible at once: the loop's peak throughput.
    """
    from what_irregularity_costs_b200 import workloads
    specs = workloads.scene_mix(64, seed=5)
    frames = workloads.mix_frames([s for s in specs], 8)  # before any CUDA use
    import torch
    from what_irregularity_costs_b200.serving import Server, poisson_schedule
    rank, local, world, dist = dist_setup(args.gpus)
    torch.cuda.set_device(local)
    rate, every, budget = 2000.0, 50, 120e9
    # The work shape the batch autotuner picks on the 32-scene mix (8 tiles per
    # band item, warp-grouped probing, two blocks per finish item).
    shape = (8, 0, 1)
    out = {}
    for mode in ("realtime", "saturated"):
        reqs = poisson_schedule(specs, rate_fps=rate, extract_every=every, seed=11)
        server = Server(budget_bytes=budget, graph=True, shape=shape)
        try:
            out[mode] = server.run(specs, frames, reqs, realtime=(mode == "realtime"),
                                   open_first=True)
            out[mode]["status"] = server.batch.status()
        finally:
            server.close()
    rt = out["realtime"]
    if rank == 0:
        line = {
            "metric": "frames/s (64-session serving, Poisson 2000 frames/s offered)",
            "value": rt["frames_per_s"], "unit": "frames/s", "n_gpus": world,
            "steps": rt["steps"], "warmup": 0, "ms_per_step": 1e3 * rt["wall_s"] / max(rt["steps"], 1),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f16 tsdf / u16 weight storage, f32 running average",
            "data": "synthetic: 64 seeded room sessions (scene_mix seed 5), 8 distinct frames each, cycled",
            "config": {"workload": "64 sessions, Poisson integrate arrivals summing to 2000 frames/s, "
                                   "extract every 50 frames per session, 120 GB HBM admission budget",
                       "sessions": len(specs), "offered_fps": rate, "extract_every": every,
                       "budget_gb": budget / 1e9, "shape": list(shape),
                       "sessions_open_before_first_frame": True},
            "latency_ms": {"integrate": rt["integrate_latency_ms"],
                           "integrate_steady": rt["integrate_latency_ms_steady"],
                           "extract": rt["extract_latency_ms"]},
            "realtime": rt, "saturated": out["saturated"],
            "e2e": {"value": rt["frames_per_s"], "unit": "frames/s",
                    "h2d_bytes_per_step": int(sum(p.nbytes for fr in frames for p, _ in fr) /
                                              sum(len(fr) for fr in frames) * rt["frames_per_step"]),
                    "d2h_bytes_per_step": 0},
        }
        print(json.dumps(line))
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def serve64_figures(max_frames, torch):
    """The serving configuration (run_serve64) with every session's trajectory
    cut at max_frames frames, realtime arrivals only: frames/s and p50/p99
    integrate and extract latency."""
    import dataclasses
    from what_irregularity_costs_b200 import workloads
    from what_irregularity_costs_b200.serving import Server, poisson_schedule
    specs = [dataclasses.replace(sp, frames=min(sp.frames, max_frames))
             for sp in workloads.scene_mix(64, seed=5)]
    frames = workloads.mix_frames(specs, 8)
    rate, every, budget = 2000.0, 50, 120e9
    reqs = poisson_schedule(specs, rate_fps=rate, extract_every=every, seed=11)
    server = Server(budget_bytes=budget, graph=True, shape=(8, 0, 1))
    try:
        rt = server.run(specs, frames, reqs, realtime=True, open_first=True)
        status = server.batch.status()
    finally:
        server.close()
    torch.cuda.synchronize()
    return {"metric": "frames/s (64-session serving, Poisson 2000 frames/s offered)",
            "frames_per_s": rt["frames_per_s"], "frames": rt.get("frames"),
            "latency_ms": {"integrate": rt["integrate_latency_ms"],
                           "integrate_steady": rt.get("integrate_latency_ms_steady"),
                           "extract": rt["extract_latency_ms"]},
            "frames_per_step": rt.get("frames_per_step"), "status": status,
            "config": f"64 sessions (scene_mix seed 5), each cut at {max_frames} frames, 8 distinct "
                      f"frames cycled; extract every {every} frames; {budget / 1e9:.0f} GB budget; "
                      "FP16/u16 storage"}


def run_sweep(args):
    """Irregularity and precision sweep on the room trajectory (640x480 frames):
    voxel sizes 5 mm, 1, 2, 4 cm (trunc 4 voxels, cap 64) on a 2^18-slot table
    (the smallest of the 2^18-2^22 range, so the most load factors are
    reachable), pool = slots. An FP64 volume integrates frames until the block
    count reaches 0.9 of the table (or the frames run out); FP32 and FP16/u16
    volumes then integrate exactly those frames, so all three hold the same
    blocks. In the FP32/FP16 runs, the frame at which the load factor first
    reaches 0.25 / 0.5 / 0.75 / 0.9 runs as: allocate (timed: Mrays/s), a
    probe-histogram pass over the same points (now lookups: the probe depth of
    finding each block at that load factor), update (timed: GB/s of 12 B per
    point + tsdf and weight of every touched block read and written). Load
    factors the trajectory cannot reach at a voxel size are reported as the
    largest reached. Errors of FP32 and FP16 against FP64: max / RMS mean-TSDF
    error (m) and the Chamfer distance of the extracted meshes."""
    n_frames = min(args.frames, N_FRAMES)
    pts, cams = make_trajectory(n_frames)  # before any CUDA use
    import torch
    from what_irregularity_costs_b200 import (STORAGE_FP16_U16, STORAGE_FP32, STORAGE_FP64, CudaVolume,
                                              precision)
    rank, local, world, dist = dist_setup(args.gpus)
    torch.cuda.set_device(local)
    dev = [torch.from_numpy(p).cuda() for p in pts]
    slots = 1 << 18
    targets = [0.25, 0.5, 0.75, 0.9]
    mesh_cap = 1 << 25
    cells = []
    for voxel in (0.005, 0.01, 0.02, 0.04):
        trunc = 4 * voxel
        o = CudaVolume(voxel, slots, trunc, CAP, slots, storage=STORAGE_FP64)
        n_stop = 0
        for k in range(n_frames):
            if o.block_count() >= 0.9 * slots:
                break
            o.integrate(dev[k], cams[k])
            n_stop = k + 1
        mo = o.extract_mesh(mesh_cap)
        row = {"voxel_m": voxel, "slots": slots, "frames": n_stop, "blocks": o.block_count(),
               "lf_reached": o.block_count() / slots, "fp64_drops": int(o.drop_count())}
        for storage, name in ((STORAGE_FP32, "fp32"), (STORAGE_FP16_U16, "fp16_u16")):
            vol = CudaVolume(voxel, slots, trunc, CAP, slots, storage=storage)
            vs = torch.cuda.ExternalStream(vol.stream_handle())
            # Pass 1 (timed): every frame, one event pair, no polling in between.
            for _ in range(2):  # the first pass warms up (allocations, caches)
                vol.reset()
                torch.cuda.synchronize()
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record(vs)
                for k in range(n_stop):
                    vol.integrate(dev[k], cams[k])
                e1.record(vs)
                torch.cuda.synchronize()
            fps = n_stop / (e0.elapsed_time(e1) / 1e3) if n_stop else None
            # Pass 2: the same frames with the load-factor checkpoints.
            vol.reset()
            marks, ti, t_frames = [], 0, []
            for k in range(n_stop):
                lf = vol.block_count() / slots
                if ti < len(targets) and lf >= targets[ti]:
                    e = [torch.cuda.Event(enable_timing=True) for _ in range(4)]
                    e[0].record(vs)
                    vol.allocate_blocks(dev[k], cams[k])
                    e[1].record(vs)
                    hist = vol.allocate_probe_histogram(dev[k], cams[k], n_bins=32)
                    e[2].record(vs)
                    vol.update_voxels(dev[k], cams[k])
                    e[3].record(vs)
                    torch.cuda.synchronize()
                    st = vol.last_update_stats()
                    t_alloc, t_upd = e[0].elapsed_time(e[1]), e[2].elapsed_time(e[3])
                    tb = 4 if storage == STORAGE_FP32 else 2
                    ub = 12 * pts[k].shape[0] + st["touched_blocks"] * 512 * 2 * 2 * tb
                    nz = np.nonzero(hist)[0]
                    marks.append({"target_lf": targets[ti], "lf": lf, "frame": k,
                                  "alloc_mrays_per_s": pts[k].shape[0] / t_alloc / 1e3,
                                  "update_gbps": ub / t_upd / 1e6, "update_ms": t_upd,
                                  "touched_blocks": st["touched_blocks"],
                                  "probe_hist": hist[: int(nz.max()) + 1].tolist() if nz.size else [],
                                  "mean_probes": float((hist * np.arange(hist.size)).sum() / max(hist.sum(), 1))})
                    while ti < len(targets) and lf >= targets[ti]:
                        ti += 1
                else:
                    vol.integrate(dev[k], cams[k])
            torch.cuda.synchronize()
            try:
                err = precision.tsdf_errors(vol, o, trunc)
            except AssertionError as ex:  # block sets or weights differ: reported, not hidden
                err = {"mismatch": str(ex)}
            mesh = vol.extract_mesh(mesh_cap)
            row[name] = {"frames_per_s": fps, "marks": marks,
                         "drops": int(vol.drop_count()), "status": vol.status(),
                         "tsdf_error_vs_fp64": err, "mesh_vs_fp64": precision.mesh_errors(mesh, mo, stride=4)}
            vol.close()
        o.close()
        cells.append(row)
    if rank == 0:
        print(json.dumps({
            "metric": "irregularity and precision sweep (room trajectory 640x480)",
            "value": None, "unit": None, "n_gpus": world, "steps": n_frames, "warmup": 0,
            "ms_per_step": None, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32 and f16/u16 storage vs f64 oracle", "data": "synthetic room trajectory seed 0",
            "config": {"workload": "voxels 5 mm-4 cm x load factor 0.25-0.9 on 2^18 slots x storage",
                       "frames": n_frames, "slots": slots},
            "cells": cells}))
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline leg")
    ap.add_argument("--no-a3", action="store_true", help="skip timing the reference's CUDA arm")
    ap.add_argument("--batch-steps", type=int, default=5,
                    help="timed steps of the 32-scene batched comparison in the room line (0: skip)")
    ap.add_argument("--batch-warmup", type=int, default=3)
    ap.add_argument("--serve-frames", type=int, default=50,
                    help="frames per session of the bounded serving run in the room line (0: skip)")
    ap.add_argument("--no-parity", action="store_true",
                    help="skip the check of the headline run's volume against the oracle")
    ap.add_argument("--cpu-budget", type=float, default=15.0)
    ap.add_argument("--ref-frames", type=int, default=20,
                    help="frames per step of the reference arm")
    ap.add_argument("--frames", type=int, default=N_FRAMES,
                    help="frames of the trajectory per step (fewer: a small profiling case)")
    ap.add_argument("--pool", type=int, default=POOL, help="pool capacity in blocks")
    ap.add_argument("--frames-per-call", type=int, default=FRAMES_PER_CALL,
                    help="frames per integrate_frames call in the headline arm")
    ap.add_argument("--workload", choices=["room", "batch32", "serve64", "sweep"], default="room",
                    help="room: the single-scene trajectory (default); batch32: the 32-scene "
                         "batched mix; serve64: the 64-session serving loop; sweep: voxel size x "
                         "load factor x storage precision")
    args = ap.parse_args()
    set_workload(args.frames, args.pool)
    if args.workload == "batch32" and args.impl == "ours":
        return run_batch32(args)
    if args.workload == "serve64" and args.impl == "ours":
        return run_serve64(args)
    if args.workload == "sweep" and args.impl == "ours":
        return run_sweep(args)
    if args.impl == "reference":
        return run_reference(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
