"""Python mirror of the batched integrate API (osn_tsdf_batch_* in
include/osn_tsdf_b200.h).

``Batch`` holds up to 64 ``CudaVolume`` scenes; every ``step()`` integrates
the frame set for each scene since the last step, all scenes in one chain
of work-queued passes on the batch's stream (optionally replayed from a CUDA
graph, with an autotuned work shape). Results equal integrating each scene
alone. While attached, a scene is integrated only through the batch; call
``synchronize()`` before reading a scene's volume.
"""
from __future__ import annotations

import ctypes as C
from typing import Sequence

import numpy as np

from . import _lib
from .volume import CudaVolume, _addr, _count


class Batch:
    def __init__(self, max_scenes: int = 64):
        self.lib = _lib.load()
        self.h = self.lib.osn_tsdf_batch_create(int(max_scenes))
        if not self.h:
            raise ValueError("osn_tsdf_batch_create failed (max_scenes must be in [1, 64])")
        self.scenes: list[CudaVolume | None] = []  # by scene slot
        self._keep = []

    def close(self):
        if getattr(self, "h", None):
            self.lib.osn_tsdf_batch_destroy(self.h)
            self.h = None
            self._keep = []

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def add(self, vol: CudaVolume, max_points: int) -> int:
        idx = self.lib.osn_tsdf_batch_add(self.h, vol.h, int(max_points))
        if idx < 0:
            raise ValueError("osn_tsdf_batch_add rejected the volume (full, already attached, "
                             "storage mode differs, or max_points too large)")
        while len(self.scenes) <= idx:
            self.scenes.append(None)
        self.scenes[idx] = vol
        return idx

    def remove(self, scene: int):
        """Detach a scene after the queued steps ran (its slot is reused)."""
        rc = self.lib.osn_tsdf_batch_remove(self.h, int(scene))
        if rc:
            raise ValueError(f"remove: no scene {scene}" if rc == 1 else "remove: CUDA error")
        vol = self.scenes[scene]
        self.scenes[scene] = None
        return vol

    def set_frame(self, scene: int, positions, cam: Sequence[float], radius_m: float = 0.0, n=None):
        count = _count(positions, n)
        self._keep.append(positions)
        rc = self.lib.osn_tsdf_batch_set_frame(self.h, int(scene), _addr(positions), count,
                                               float(cam[0]), float(cam[1]), float(cam[2]),
                                               float(radius_m))
        if rc:
            raise ValueError(f"set_frame: invalid arguments for scene {scene}")

    def step(self):
        rc = self.lib.osn_tsdf_batch_step(self.h)
        if rc:
            raise RuntimeError(f"osn_tsdf_batch_step failed (code {rc})")

    def synchronize(self):
        self.lib.osn_tsdf_batch_synchronize(self.h)
        self._keep = []

    def set_graph(self, on: bool = True):
        self.lib.osn_tsdf_batch_set_graph(self.h, 1 if on else 0)

    def autotune(self, steps_per_shape: int = 3):
        if self.lib.osn_tsdf_batch_autotune(self.h, int(steps_per_shape)):
            raise ValueError("autotune: steps_per_shape must be positive")

    def set_shape(self, tiles_per_item: int, probe: int, finish_pair: int):
        if self.lib.osn_tsdf_batch_set_shape(self.h, tiles_per_item, probe, finish_pair):
            raise ValueError("set_shape: shape out of range")

    def shape(self) -> dict:
        out = np.zeros(3, dtype=np.int32)
        tuning = self.lib.osn_tsdf_batch_shape(self.h, out.ctypes.data)
        return {"tiles_per_item": int(out[0]), "probe": ["warp", "lane"][int(out[1])],
                "finish_pair": bool(out[2]), "tuning": tuning == 1}

    def tune_results(self) -> list:
        ms = np.zeros(32, dtype=np.float64)
        shapes = np.zeros(96, dtype=np.int32)
        n = self.lib.osn_tsdf_batch_tune_results(self.h, ms.ctypes.data, shapes.ctypes.data, 32)
        return [{"tiles_per_item": int(shapes[3 * k]), "probe": ["warp", "lane"][int(shapes[3 * k + 1])],
                 "finish_pair": bool(shapes[3 * k + 2]), "median_ms": float(ms[k])} for k in range(n)]

    def status(self) -> int:
        return int(self.lib.osn_tsdf_batch_status(self.h))

    def stream_handle(self) -> int:
        return int(self.lib.osn_tsdf_batch_stream(self.h) or 0)

    def __len__(self):
        return int(self.lib.osn_tsdf_batch_size(self.h))
