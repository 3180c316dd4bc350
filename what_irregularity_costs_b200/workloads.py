"""Seeded multi-scene workloads: the 32-scene batched mix and the 64-session
serving mix.

Scene mix (the batched configuration): 32 independent room scenes (a
6x6x3 m room with 3 spheres and 2 boxes placed from the scene's seed, the
seeded orbit trajectory and depth noise of the single-scene benchmark),
each with
  - a hash table of 2^e slots, e uniform in [14, 20] (log-uniform sizes),
    and the reference's pool sizing (slots / 2 blocks);
  - a voxel size log-uniform in [1, 4] cm, truncation 4 voxels, cap 64;
  - a resolution drawn from 160x120, 320x240, 640x480, 1280x720 with the
    intrinsics scaled from fx = fy = 320 at 640x480;
  - a frame count uniform in [8, 256].
All scenes advance one frame per step; a scene whose frames ran out sits the
remaining steps out. The serving mix draws 64 sessions the same way.
"""
from __future__ import annotations

import math
import multiprocessing as mp
import os
from concurrent.futures import ProcessPoolExecutor
from dataclasses import dataclass

import numpy as np

RESOLUTIONS = [(160, 120), (320, 240), (640, 480), (1280, 720)]
CAP = 64.0


@dataclass(frozen=True)
class SceneSpec:
    index: int
    seed: int
    hash_slots: int
    voxel: float
    width: int
    height: int
    frames: int
    cap: float = CAP

    @property
    def pool(self) -> int:
        return self.hash_slots // 2

    @property
    def trunc(self) -> float:
        return 4.0 * self.voxel

    @property
    def max_points(self) -> int:
        return self.width * self.height


def scene_mix(n_scenes: int = 32, seed: int = 4) -> list[SceneSpec]:
    rng = np.random.default_rng(seed)
    out = []
    for k in range(n_scenes):
        e = int(rng.integers(14, 21))
        voxel = float(math.exp(rng.uniform(math.log(0.01), math.log(0.04))))
        w, h = RESOLUTIONS[int(rng.integers(0, len(RESOLUTIONS)))]
        frames = int(rng.integers(8, 257))
        out.append(SceneSpec(k, 1000 + 17 * k + seed, 1 << e, voxel, w, h, frames))
    return out


def _frame_job(args):
    spec_seed, w, h, k = args
    from . import scenes
    scene = scenes.RoomScene.make(spec_seed)
    K = scenes.ROOM_K.scaled(w, h)
    f = scenes.room_frame(scene, k, K)
    return scenes.frame_points(f), f.cam


def mix_frames(specs, n_steps: int, workers: int | None = None):
    """frames[p][k] = (points (n, 3) float32, cam) of specs[p], k < min(frames, n_steps).
    Generated in spawned workers (call before any CUDA use)."""
    jobs, where = [], []
    for pos, s in enumerate(specs):
        for k in range(min(s.frames, n_steps)):
            jobs.append((s.seed, s.width, s.height, k))
            where.append((pos, k))
    workers = workers or min(32, os.cpu_count() or 1)
    ctx = mp.get_context("spawn")
    with ProcessPoolExecutor(max_workers=workers, mp_context=ctx) as ex:
        res = list(ex.map(_frame_job, jobs, chunksize=2))
    frames = [[None] * min(s.frames, n_steps) for s in specs]
    for (si, k), r in zip(where, res):
        frames[si][k] = r
    return frames


def make_volumes(specs, storage: int):
    from .volume import CudaVolume
    return [CudaVolume(s.voxel, s.pool, s.trunc, s.cap, s.hash_slots, storage=storage) for s in specs]


def upload(frames, torch):
    return [[torch.from_numpy(p).cuda() for p, _ in fr] for fr in frames]


def _main():
    """A small batched run of the scene mix (a profiling case): the first
    --scenes scenes integrate --steps frames each through one batch (FP16
    storage, the autotuner's shape for the mix), then the batch status is
    printed."""
    import argparse
    ap = argparse.ArgumentParser()
    ap.add_argument("--scenes", type=int, default=8)
    ap.add_argument("--steps", type=int, default=6)
    args = ap.parse_args()
    specs = scene_mix(32)[: args.scenes]
    frames = mix_frames(specs, args.steps)
    import torch
    from . import STORAGE_FP16_U16, Batch
    dev = upload(frames, torch)
    vols = make_volumes(specs, STORAGE_FP16_U16)
    b = Batch(len(specs))
    b.set_shape(8, 0, 1)
    for v, sp in zip(vols, specs):
        b.add(v, sp.max_points)
    for k in range(args.steps):
        for i, fr in enumerate(frames):
            if k < len(fr):
                b.set_frame(i, dev[i][k], fr[k][1])
        b.step()
    b.synchronize()
    print(f"batched {args.scenes} scenes x {args.steps} steps: status {b.status()}, "
          f"blocks {[v.block_count() for v in vols]}")


if __name__ == "__main__":
    _main()
