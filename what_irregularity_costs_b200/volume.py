"""Python mirror of the reference's CUDA volume interface, over the C ABI.

``CudaVolume`` wraps one ``OsnTsdfCudaVolume`` of libosn_tsdf_b200.so. Its
methods keep the reference's names and argument meanings
(cpp/include/osn_tsdf/c_api.h:80-126, cpp/include/osn_tsdf/volume_cuda.hpp:24-86):
positions are device-resident float32 ``(n, 3)`` world points (a CUDA torch
tensor or a raw device address), ``cam`` is the camera origin, ``radius_m``
the far cutoff (<= 0 disables). Bad arguments raise ``ValueError`` where the
C ABI returns 1; a failed launch raises ``RuntimeError`` (return code 3).
"""
from __future__ import annotations

import ctypes as C
import os
from typing import Sequence

import numpy as np

from . import _lib

MAX_FRAMES = 32  # OSN_TSDF_MAX_FRAMES: frames per integrate_frames call
MAX_DEPTH_FRAMES = 16  # OSN_TSDF_MAX_DEPTH_FRAMES: images per integrate_depth_frames call
# Kernel ids of the timing table (id 7 is kept for the numbering and records
# no launches).
KERNEL_NAMES = ["allocate", "band", "finish", "group", "select", "extract", "reset", "unused7"]

# Voxel storage modes (OSN_TSDF_STORAGE_* in include/osn_tsdf_b200.h).
STORAGE_FP32, STORAGE_FP16_U16, STORAGE_FP64 = 0, 1, 2
# Table layouts (OSN_TSDF_LAYOUT_*): the reference's pool order, or the pool
# as the table (a block's index is its slot).
LAYOUT_POOL, LAYOUT_SLOT_INDEX = 0, 1
STORAGE_NAMES = {STORAGE_FP32: "fp32", STORAGE_FP16_U16: "fp16_u16", STORAGE_FP64: "fp64"}


def _addr(x) -> int:
    """Device address of a CUDA tensor (or an int address)."""
    if isinstance(x, int):
        return x
    if hasattr(x, "data_ptr"):
        if not x.is_cuda:
            raise ValueError("positions must be a CUDA tensor (device pointer)")
        return int(x.data_ptr())
    raise TypeError(f"expected a CUDA tensor or a device address, got {type(x)!r}")


def _count(x, n):
    if n is not None:
        return int(n)
    if hasattr(x, "shape"):
        if x.dim() != 2 or x.shape[1] != 3:
            raise ValueError("positions must have shape (n, 3)")
        if not x.is_contiguous():
            raise ValueError("positions must be contiguous")
        import torch
        if x.dtype != torch.float32:
            raise ValueError("positions must be float32")
        return int(x.shape[0])
    raise ValueError("n is required with a raw device address")


class _DeviceArray:
    """Zero-copy view of device memory for torch.as_tensor."""

    def __init__(self, ptr: int, shape, typestr: str):
        self.__cuda_array_interface__ = {
            "shape": tuple(shape), "typestr": typestr, "data": (int(ptr), False), "version": 3,
            "strides": None,
        }


def device_tensor(ptr: int, shape, dtype: str):
    """torch view of `shape` elements at device address `ptr` (dtype: numpy typestr)."""
    import torch
    return torch.as_tensor(_DeviceArray(ptr, shape, dtype), device="cuda")


class CudaVolume:
    """One hash-blocked TSDF volume on the GPU (drop-in for the reference's CudaVolume)."""

    def __init__(self, voxel_size_m: float, pool_capacity_blocks: int, trunc_m: float = -1.0,
                 weight_cap: float = 32.0, hash_slots: int = 0, storage: int = STORAGE_FP32,
                 layout: int = LAYOUT_POOL):
        self.lib = _lib.load()
        self.storage = int(storage)
        self.layout = int(layout)
        self.h = self.lib.osn_tsdf_cuda_create_layout(voxel_size_m, pool_capacity_blocks, trunc_m,
                                                      weight_cap, hash_slots, self.storage, self.layout)
        if not self.h:
            raise ValueError("osn_tsdf_cuda_create rejected the parameters or the device "
                             "allocation failed")
        self._keep = []

    # -- lifetime -----------------------------------------------------------
    def close(self):
        if getattr(self, "h", None):
            self.lib.osn_tsdf_cuda_destroy(self.h)
            self.h = None
            self._keep = []

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def _check(self, rc: int, what: str):
        if rc == 1:
            raise ValueError(f"{what}: invalid arguments")
        if rc != 0:
            raise RuntimeError(f"{what}: CUDA launch failed (code {rc})")

    def _batch(self, fn, positions, cam, radius_m, n, what):
        count = _count(positions, n)
        self._keep.append(positions)
        rc = fn(self.h, _addr(positions), count, float(cam[0]), float(cam[1]), float(cam[2]),
                float(radius_m))
        self._check(rc, what)

    # -- the reference's stages --------------------------------------------
    def allocate_blocks(self, positions, cam: Sequence[float], radius_m: float = 0.0, n=None):
        self._batch(self.lib.osn_tsdf_cuda_allocate_blocks, positions, cam, radius_m, n,
                    "allocate_blocks")

    def update_voxels(self, positions, cam: Sequence[float], radius_m: float = 0.0, n=None):
        self._batch(self.lib.osn_tsdf_cuda_update_voxels, positions, cam, radius_m, n,
                    "update_voxels")

    def update_voxels_noalloc(self, positions, cam: Sequence[float], radius_m: float = 0.0,
                              n=None) -> int:
        """update_voxels with no device allocation (the library's fixed scratch array).

        For callers that cannot let the library allocate during the call: a
        serving loop that admits work against a fixed device-memory budget, a
        latency-critical thread that cannot absorb the synchronisation of a
        cudaMalloc/cudaFree. Returns the C ABI code: 0 queued, 4 when the
        batch exceeds OSN_TSDF_NOALLOC_MAX_RECORDS records (nothing queued).
        """
        count = _count(positions, n)
        self._keep.append(positions)
        rc = self.lib.osn_tsdf_cuda_update_voxels_noalloc(
            self.h, _addr(positions), count, float(cam[0]), float(cam[1]), float(cam[2]),
            float(radius_m))
        if rc not in (0, 4):
            self._check(rc, "update_voxels_noalloc")
        return rc

    def integrate(self, positions, cam: Sequence[float], radius_m: float = 0.0, n=None):
        self._batch(self.lib.osn_tsdf_cuda_integrate, positions, cam, radius_m, n, "integrate")

    def integrate_frames(self, positions, frame_begin, cams, radius_m: float = 0.0):
        """integrate() of several consecutive frames in one call: frame k is
        positions[frame_begin[k]:frame_begin[k + 1]] seen from cams[k]
        (positions: a CUDA (N, 3) float32 tensor of all frames' points back to
        back; frame_begin: n_frames + 1 offsets from 0 to N; cams: (n_frames, 3)).
        Same blocks and weights as one integrate() per frame; each voxel's TSDF
        is rounded once per call instead of once per frame. FP32 and FP16
        storage; at most MAX_FRAMES frames."""
        begin = np.ascontiguousarray(np.asarray(frame_begin, dtype=np.int32).reshape(-1))
        cam = np.ascontiguousarray(np.asarray(cams, dtype=np.float32).reshape(-1, 3))
        if begin.size != cam.shape[0] + 1:
            raise ValueError("integrate_frames: frame_begin needs one entry more than cams")
        if _count(positions, None) < int(begin[-1]):
            raise ValueError("integrate_frames: frame_begin reaches past the points")
        self._keep.append(positions)
        rc = self.lib.osn_tsdf_cuda_integrate_frames(self.h, _addr(positions), begin.ctypes.data,
                                                     cam.ctypes.data, int(cam.shape[0]), float(radius_m))
        if rc == 2:
            raise ValueError("integrate_frames: the FP64 oracle integrates one frame per call")
        self._check(rc, "integrate_frames")

    def integrate_depth_frames(self, depth, K, Rs, ts, max_range_m: float = 0.0):
        """integrate_depth() of several images in one call: depth is a
        contiguous (F, H, W) float32 CUDA tensor, Rs (F, 3, 3) and ts (F, 3)
        the images' camera-to-world poses. Same blocks and weights as one
        integrate_depth() per image; each voxel's TSDF is rounded once per
        call. FP32 and FP16 storage; at most MAX_DEPTH_FRAMES images."""
        if not (hasattr(depth, "is_cuda") and depth.is_cuda and depth.dim() == 3 and depth.is_contiguous()):
            raise ValueError("depth must be a contiguous (F, H, W) CUDA tensor")
        import torch
        if depth.dtype != torch.float32:
            raise ValueError("depth must be float32")
        f = int(depth.shape[0])
        Rh = np.ascontiguousarray(np.asarray(Rs, dtype=np.float64).reshape(-1))
        th = np.ascontiguousarray(np.asarray(ts, dtype=np.float64).reshape(-1))
        if Rh.size != 9 * f or th.size != 3 * f:
            raise ValueError("integrate_depth_frames: one pose per image")
        self._keep.append(depth)
        rc = self.lib.osn_tsdf_cuda_integrate_depth_frames(
            self.h, _addr(depth), int(depth.shape[2]), int(depth.shape[1]), f, float(K.fx), float(K.fy),
            float(K.cx), float(K.cy), Rh.ctypes.data, th.ctypes.data, float(max_range_m))
        if rc == 2:
            raise ValueError("integrate_depth_frames: the FP64 oracle integrates one image per call")
        self._check(rc, "integrate_depth_frames")

    def integrate_depth(self, depth, K, R, t, max_range_m: float = 0.0):
        """integrate() from a device depth image (H, W) float32, unprojected on
        the GPU with intrinsics K (fx, fy, cx, cy attributes) and the
        camera-to-world pose R (3x3), t (3,) in FP64; equals integrating the
        host-backprojected points (scenes.backproject)."""
        if not (hasattr(depth, "is_cuda") and depth.is_cuda and depth.dim() == 2 and depth.is_contiguous()):
            raise ValueError("depth must be a contiguous (H, W) CUDA tensor")
        import torch
        if depth.dtype != torch.float32:
            raise ValueError("depth must be float32")
        Rh = np.ascontiguousarray(np.asarray(R, dtype=np.float64).reshape(9))
        th = np.ascontiguousarray(np.asarray(t, dtype=np.float64).reshape(3))
        self._keep.append(depth)
        rc = self.lib.osn_tsdf_cuda_integrate_depth(
            self.h, _addr(depth), int(depth.shape[1]), int(depth.shape[0]), float(K.fx), float(K.fy),
            float(K.cx), float(K.cy), Rh.ctypes.data, th.ctypes.data, float(max_range_m))
        self._check(rc, "integrate_depth")

    def write_mesh_osn1(self, path: str, vert_cap: int = 1 << 22, min_weight: float = 0.5,
                        iso: float = 0.0) -> int:
        """Extract the mesh and write it as an OSN1 file (meshio); returns the
        vertex count."""
        n = self.lib.osn_tsdf_cuda_write_mesh_osn1(self.h, os.fsencode(path), int(vert_cap),
                                                   float(min_weight), float(iso))
        if n == -1:
            raise ValueError("write_mesh_osn1: bad arguments or vert_cap too small")
        if n < 0:
            raise OSError(f"write_mesh_osn1: cannot write {path}")
        return int(n)

    def snapshot(self) -> np.ndarray:
        """The volume's allocated blocks and voxels as a host byte array."""
        n = self.lib.osn_tsdf_cuda_snapshot_bytes(self.h)
        if n < 0:
            raise RuntimeError("snapshot_bytes failed")
        buf = np.empty(int(n), dtype=np.uint8)
        wrote = self.lib.osn_tsdf_cuda_snapshot(self.h, buf.ctypes.data, int(n))
        if wrote != n:
            raise RuntimeError("snapshot failed")
        return buf

    def restore(self, snap: np.ndarray):
        """Replace the contents with a snapshot (same voxel size, truncation,
        cap and storage; pool and table large enough)."""
        snap = np.ascontiguousarray(snap, dtype=np.uint8)
        rc = self.lib.osn_tsdf_cuda_restore(self.h, snap.ctypes.data, int(snap.nbytes))
        self._check(rc, "restore")

    def allocate_counting_cas(self, positions, cam, radius_m=0.0, n=None):
        self._batch(self.lib.osn_tsdf_cuda_allocate_counting_cas, positions, cam, radius_m, n,
                    "allocate_counting_cas")

    def allocate_no_cas(self, positions, cam, radius_m=0.0, n=None):
        self._batch(self.lib.osn_tsdf_cuda_allocate_no_cas, positions, cam, radius_m, n,
                    "allocate_no_cas")

    def allocate_slot_index(self, positions, cam, radius_m=0.0, n=None):
        self._batch(self.lib.osn_tsdf_cuda_allocate_slot_index, positions, cam, radius_m, n,
                    "allocate_slot_index")

    def allocate_probe_histogram(self, positions, cam, radius_m=0.0, n_bins=32, n=None):
        count = _count(positions, n)
        hist = np.zeros(n_bins, dtype=np.uint64)
        self._keep.append(positions)
        rc = self.lib.osn_tsdf_cuda_allocate_probe_histogram(
            self.h, _addr(positions), count, float(cam[0]), float(cam[1]), float(cam[2]),
            float(radius_m), hist.ctypes.data, n_bins)
        self._check(rc, "allocate_probe_histogram")
        return hist

    def extract_mesh(self, vert_cap: int = 4 << 20, min_weight: float = 0.5, iso: float = 0.0,
                     rgb: bool = False):
        """Triangle soup as host arrays: posnor (n, 6) float32 [, rgb (n, 3) uint8]; None on overflow."""
        posnor = np.empty((vert_cap, 6), dtype=np.float32)
        col = np.empty((vert_cap, 3), dtype=np.uint8) if rgb else None
        n = self.lib.osn_tsdf_cuda_extract_mesh(self.h, posnor.ctypes.data,
                                                col.ctypes.data if rgb else None, vert_cap,
                                                min_weight, iso)
        self._keep = []
        if n < 0:
            return (None, None) if rgb else None
        return (posnor[:n], col[:n]) if rgb else posnor[:n]

    def extract_mesh_device(self, posnor, rgb=None, vert_cap=None, min_weight=0.5, iso=0.0) -> int:
        cap = int(vert_cap if vert_cap is not None else posnor.shape[0])
        return self.lib.osn_tsdf_cuda_extract_mesh_device(
            self.h, _addr(posnor), _addr(rgb) if rgb is not None else None, cap, min_weight, iso)

    def reset(self):
        self._check(self.lib.osn_tsdf_cuda_reset(self.h), "reset")
        self._keep = []

    def block_count(self) -> int:
        return self.lib.osn_tsdf_cuda_block_count(self.h)

    def drop_count(self) -> int:
        return self.lib.osn_tsdf_cuda_drop_count(self.h)

    def synchronize(self):
        self.lib.osn_tsdf_cuda_synchronize(self.h)
        self._keep = []

    def valid(self) -> bool:
        return bool(self.lib.osn_tsdf_cuda_valid(self.h))

    # -- extensions ---------------------------------------------------------
    def status(self) -> int:
        return self.lib.osn_tsdf_cuda_status(self.h)

    def set_pipelined(self, on: bool = True):
        """Overlap each update's tail with the next call's band walk (same
        results; +12 bytes per voxel). Not for FP64 storage."""
        rc = self.lib.osn_tsdf_cuda_set_pipelined(self.h, 1 if on else 0)
        if rc == 2:
            raise ValueError("pipelined updates are not available for FP64 storage")
        if rc:
            raise RuntimeError(f"set_pipelined failed (code {rc})")

    # -- streaming by chunk id ---------------------------------------------
    def set_chunk(self, chunk_id: int):
        """Chunk id that later calls give the blocks they allocate or update."""
        self._check(self.lib.osn_tsdf_cuda_set_chunk(self.h, int(chunk_id)), "set_chunk")

    def evict_chunks(self, lo: int, hi: int) -> np.ndarray:
        """Move every block whose chunk id lies in [lo, hi] to a host pack
        (returned as bytes) and remove it from the volume; the remaining blocks
        are compacted and the table rebuilt."""
        n = self.lib.osn_tsdf_cuda_evict_chunks_bytes(self.h, int(lo), int(hi))
        if n < 0:
            raise RuntimeError("evict_chunks_bytes failed")
        buf = np.empty(int(n), dtype=np.uint8)
        wrote = self.lib.osn_tsdf_cuda_evict_chunks(self.h, int(lo), int(hi), buf.ctypes.data, int(n))
        if wrote != n:
            raise RuntimeError(f"evict_chunks failed ({wrote})")
        return buf

    def unpack_chunks(self, pack: np.ndarray):
        """(coords (n, 3) int32, chunk ids (n,) int32, arrays) of a pack from
        evict_chunks: arrays as (n, 512) per voxel array of the storage mode
        (tsdf, weight[, r, g, b]; FP16: float16 means and uint16 weights)."""
        pack = np.ascontiguousarray(pack, dtype=np.uint8)
        n = int(pack[28:32].view(np.int32)[0])  # header: magic, version, storage, 3 floats, n
        off = 64
        coords = pack[off:off + 12 * n].view(np.int32).reshape(n, 3)
        off += 12 * n
        chunks = pack[off:off + 4 * n].view(np.int32)
        off += 4 * n
        kinds = {STORAGE_FP32: ["<f4"] * 5, STORAGE_FP16_U16: ["<f2", "<u2"], STORAGE_FP64: ["<f8", "<f4"]}
        arrays = []
        for dt in kinds[self.storage]:
            size = np.dtype(dt).itemsize * 512 * n
            arrays.append(pack[off:off + size].view(dt).reshape(n, 512))
            off += size
        return coords, chunks, arrays

    def stream_in(self, pack: np.ndarray) -> int:
        """Insert a pack's blocks again; returns how many were skipped because
        the volume holds them again. Raises when the pool filled."""
        pack = np.ascontiguousarray(pack, dtype=np.uint8)
        skipped = C.c_int32(0)
        rc = self.lib.osn_tsdf_cuda_stream_in(self.h, pack.ctypes.data, int(pack.nbytes),
                                              C.addressof(skipped))
        if rc == 2:
            raise RuntimeError("stream_in: the pool filled before every block was restored")
        self._check(rc, "stream_in")
        return int(skipped.value)

    def set_spin_limit(self, iterations: int):
        """Bound each device-side publication wait of later calls to this many
        iterations of ~100 ns (1 .. 2^20, the default). A wait that runs out
        drops its samples and sets bit 0 of status()."""
        rc = self.lib.osn_tsdf_cuda_set_spin_limit(self.h, int(iterations))
        if rc:
            raise ValueError(f"set_spin_limit({iterations}) failed (code {rc})")

    def join(self):
        """Order the volume's stream after every queued update tail."""
        self.lib.osn_tsdf_cuda_join(self.h)

    def stream_handle(self) -> int:
        return int(self.lib.osn_tsdf_cuda_stream(self.h) or 0)

    def device_view(self) -> _lib.OsnTsdfDeviceView:
        view = _lib.OsnTsdfDeviceView()
        rc = self.lib.osn_tsdf_cuda_device_view(self.h, C.byref(view))
        if rc:
            raise RuntimeError("device_view failed")
        return view

    def last_update_stats(self) -> dict:
        out = np.zeros(4, dtype=np.int64)
        self._check(self.lib.osn_tsdf_cuda_last_update_stats(self.h, out.ctypes.data),
                    "last_update_stats")
        return {"updated_voxels": int(out[0]), "records": int(out[1]),
                "touched_blocks": int(out[2]), "crossing_voxels": int(out[3])}

    def set_timing(self, on: bool = True):
        self.lib.osn_tsdf_cuda_set_timing(self.h, 1 if on else 0)

    def kernel_times(self) -> dict:
        ms = np.zeros(len(KERNEL_NAMES), dtype=np.float64)
        launches = np.zeros(len(KERNEL_NAMES), dtype=np.int64)
        self.lib.osn_tsdf_cuda_kernel_times(self.h, ms.ctypes.data, launches.ctypes.data,
                                            len(KERNEL_NAMES))
        return {k: (float(ms[i]), int(launches[i])) for i, k in enumerate(KERNEL_NAMES)}

    # -- read-back helpers (tests, tools) ------------------------------------
    def _rows(self, ptr, cols, typestr):
        """Rows of a per-block device array for every allocated block, in pool
        order (slot-index layout: the occupied slots, ascending)."""
        view = self.device_view()
        if self.layout == LAYOUT_SLOT_INDEX:
            import torch
            keys, idx = self.table()
            slots = np.nonzero((keys >= 0) & (idx == np.arange(keys.shape[0])))[0]
            if slots.size == 0:
                return np.zeros((0, cols), dtype=np.dtype(typestr))
            full = device_tensor(ptr, (view.pool_capacity, cols), typestr)
            return full[torch.from_numpy(slots).cuda()].cpu().numpy()
        n = min(self.block_count(), view.pool_capacity)
        if n <= 0:
            return np.zeros((0, cols), dtype=np.dtype(typestr))
        return device_tensor(ptr, (n, cols), typestr).cpu().numpy()

    def coords(self) -> np.ndarray:
        """Block coordinates in pool order, (block_count, 3) int32."""
        self.synchronize()
        return self._rows(self.device_view().block_coord, 3, "<i4")

    def coord_set(self) -> set:
        return set(map(tuple, self.coords().tolist()))

    def means(self):
        """(coords, mean TSDF, weight) in any storage mode: (block_count, 512) float64
        arrays; the mean is 0 where the weight is 0."""
        view = self.device_view()
        coords = self.coords()
        if coords.shape[0] == 0:
            z = np.zeros((0, 512), dtype=np.float64)
            return coords, z, z.copy()
        if self.storage == STORAGE_FP16_U16:
            mean = self._rows(view.tsdf, 512, "<f2").astype(np.float64)
            w = self._rows(view.weight, 512, "<u2").astype(np.float64)
        else:
            typ = "<f8" if self.storage == STORAGE_FP64 else "<f4"
            t = self._rows(view.tsdf, 512, typ).astype(np.float64)
            w = self._rows(view.weight, 512, "<f4").astype(np.float64)
            mean = np.divide(t, w, out=np.zeros_like(t), where=w > 0)
        return coords, mean, w

    def voxels(self):
        """(coords, tsdf, weight, r, g, b): the five arrays as (block_count, 512) float32
        (FP32 storage: the reference's weighted sums)."""
        if self.storage != STORAGE_FP32:
            raise ValueError("voxels() reads the FP32 layout; use means() for other storage")
        view = self.device_view()
        out = [self.coords()]
        for ptr in (view.tsdf, view.weight, view.r, view.g, view.b):
            out.append(self._rows(ptr, 512, "<f4"))
        return tuple(out)

    def table(self):
        """(keys int64, block_idx int32) of the live table."""
        self.synchronize()
        view = self.device_view()
        size = view.hash_mask + 1
        raw = device_tensor(view.table, (size, 4), "<i4").cpu().numpy()
        keys = raw[:, :2].copy().view(np.int64).reshape(-1)
        return keys, raw[:, 2].copy()
