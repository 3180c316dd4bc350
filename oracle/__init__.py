"""CPU checkers for the TSDF integrate path -- TEST INFRASTRUCTURE ONLY.

Two ctypes wrappers with the same surface:

* ``OracleVolume``: the single-threaded C restatement in ``tsdf_oracle.c``
  (built into ``oracle/_build/liboracle_tsdf.so``).
* ``RefVolume``: the reference's own CPU arm, compiled from its unmodified
  sources plus ``ref_shim.cpp`` into ``oracle/_ref/libosn_tsdf_ref.so``.

Only tests, ``__graft_entry__.smoke()`` and the CPU-baseline leg of
``bench.py`` import this package, and only to check or time the CPU path.
The CUDA library never loads it.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "_build", "liboracle_tsdf.so")
REF_SO = os.path.join(HERE, "_ref", "libosn_tsdf_ref.so")

_f32p = C.POINTER(C.c_float)
_u8p = C.POINTER(C.c_uint8)
_i32p = C.POINTER(C.c_int32)
_i64p = C.POINTER(C.c_int64)


def build(ref_root: str | None = None, gate: bool = False) -> None:
    """Compile the restatement and, when the reference tree is present, the
    reference's CPU and CUDA arms; with gate=True (the library must be built)
    also the reference's own C++ GPU test linked against this library."""
    env = dict(os.environ)
    cmd = ["make", "-s", "-C", HERE, "all"] + (["gate"] if gate else [])
    if ref_root:
        cmd.append(f"REF_ROOT={ref_root}")
    subprocess.run(cmd, check=True, env=env)


def _ptr(a, ctype):
    if a is None:
        return None
    return a.ctypes.data_as(C.POINTER(ctype))


_oracle_lib = None
_ref_lib = None


def oracle_lib():
    global _oracle_lib
    if _oracle_lib is None:
        if not os.path.exists(ORACLE_SO):
            build()
        lib = C.CDLL(ORACLE_SO)
        lib.oracle_create.restype = C.c_void_p
        lib.oracle_create.argtypes = [C.c_float, C.c_int32, C.c_float, C.c_float, C.c_uint32]
        lib.oracle_destroy.argtypes = [C.c_void_p]
        lib.oracle_allocate_blocks.argtypes = [C.c_void_p, _f32p, C.c_int32] + [C.c_float] * 4
        lib.oracle_update_voxels.argtypes = [C.c_void_p, _f32p, _u8p, _f32p, C.c_int32] + [C.c_float] * 4
        lib.oracle_integrate.argtypes = [C.c_void_p, _f32p, _u8p, _f32p, C.c_int32] + [C.c_float] * 4
        lib.oracle_extract_mesh.argtypes = [C.c_void_p, _f32p, _u8p, C.c_int32, C.c_float, C.c_float]
        lib.oracle_block_count.argtypes = [C.c_void_p]
        lib.oracle_drop_count.argtypes = [C.c_void_p]
        lib.oracle_drop_count.restype = C.c_uint64
        lib.oracle_hash_mask.argtypes = [C.c_void_p]
        lib.oracle_hash_mask.restype = C.c_uint32
        lib.oracle_trunc.argtypes = [C.c_void_p]
        lib.oracle_trunc.restype = C.c_float
        lib.oracle_block_coords.argtypes = [C.c_void_p, _i32p]
        lib.oracle_voxels.argtypes = [C.c_void_p, _f32p, _f32p, _f32p, _f32p, _f32p]
        lib.oracle_table.argtypes = [C.c_void_p, _i64p, _i32p]
        lib.oracle_sphere_points.argtypes = [C.c_float, C.c_int32, C.c_int32, _f32p]
        lib.oracle_plane_points.argtypes = [C.c_float, C.c_float, C.c_int32, _f32p]
        _oracle_lib = lib
    return _oracle_lib


def sphere_points(radius: float, n_theta: int, n_phi: int) -> np.ndarray:
    """The reference's analytic sphere cloud (cpp/tests/analytic_scenes.hpp:19-33)."""
    out = np.empty((n_theta * n_phi, 3), dtype=np.float32)
    oracle_lib().oracle_sphere_points(radius, n_theta, n_phi, _ptr(out, C.c_float))
    return out


def plane_points(z0: float, half_extent: float, n: int) -> np.ndarray:
    """The reference's analytic plane patch (cpp/tests/analytic_scenes.hpp:35-46)."""
    out = np.empty((n * n, 3), dtype=np.float32)
    oracle_lib().oracle_plane_points(z0, half_extent, n, _ptr(out, C.c_float))
    return out


def ref_available() -> bool:
    return os.path.exists(REF_SO)


def ref_lib():
    global _ref_lib
    if _ref_lib is None:
        if not os.path.exists(REF_SO):
            raise FileNotFoundError(f"reference CPU arm not built: {REF_SO}")
        lib = C.CDLL(REF_SO)
        lib.ref_create.restype = C.c_void_p
        lib.ref_create.argtypes = [C.c_float, C.c_int32, C.c_float, C.c_float]
        lib.ref_destroy.argtypes = [C.c_void_p]
        lib.ref_set_threads.argtypes = [C.c_void_p, C.c_int32]
        lib.ref_allocate.argtypes = [C.c_void_p, _f32p, C.c_int32] + [C.c_float] * 4
        lib.ref_update.argtypes = [C.c_void_p, _f32p, _u8p, _f32p, C.c_int32] + [C.c_float] * 4
        lib.ref_integrate.argtypes = [C.c_void_p, _f32p, _u8p, _f32p, C.c_int32] + [C.c_float] * 4
        lib.ref_extract.argtypes = [C.c_void_p, _f32p, _u8p, C.c_int32, C.c_float, C.c_float]
        lib.ref_block_count.argtypes = [C.c_void_p]
        lib.ref_drop_count.argtypes = [C.c_void_p]
        lib.ref_drop_count.restype = C.c_uint64
        lib.ref_hash_mask.argtypes = [C.c_void_p]
        lib.ref_hash_mask.restype = C.c_uint32
        lib.ref_block_coords.argtypes = [C.c_void_p, _i32p]
        lib.ref_voxels.argtypes = [C.c_void_p, _f32p, _f32p, _f32p, _f32p, _f32p]
        lib.ref_table.argtypes = [C.c_void_p, _i64p, _i32p]
        # The reference's public C API, used by the timed CPU baseline.
        lib.osn_tsdf_create.restype = C.c_void_p
        lib.osn_tsdf_create.argtypes = [C.c_float, C.c_int32, C.c_float, C.c_float]
        lib.osn_tsdf_destroy.argtypes = [C.c_void_p]
        lib.osn_tsdf_integrate.argtypes = [C.c_void_p, _f32p, _u8p, _f32p, C.c_int32, C.c_int32] + [C.c_float] * 4
        lib.osn_tsdf_extract_mesh.argtypes = [C.c_void_p, _f32p, _u8p, C.c_int32, C.c_float, C.c_float]
        lib.osn_tsdf_block_count.argtypes = [C.c_void_p]
        lib.osn_tsdf_drop_count.argtypes = [C.c_void_p]
        lib.osn_tsdf_drop_count.restype = C.c_uint64
        lib.osn_tsdf_set_thread_count.argtypes = [C.c_void_p, C.c_int32]
        _ref_lib = lib
    return _ref_lib


class _CpuVolume:
    """Shared numpy-facing surface of the two checkers."""

    def _pts(self, points):
        p = np.ascontiguousarray(points, dtype=np.float32).reshape(-1, 3)
        return p, int(p.shape[0])

    def coords(self) -> np.ndarray:
        n = self.block_count()
        out = np.empty((n, 3), dtype=np.int32)
        if n:
            self._coords(out)
        return out

    def coord_set(self) -> set:
        return set(map(tuple, self.coords().tolist()))

    def voxels(self):
        """(coords[n,3], tsdf[n,512], weight[n,512], r, g, b) in pool order."""
        n = self.block_count()
        arrs = [np.empty((n, 512), dtype=np.float32) for _ in range(5)]
        if n:
            self._voxels(*arrs)
        return (self.coords(), *arrs)

    def extract(self, min_weight=0.5, iso=0.0, cap=4 << 20, rgb=False):
        posnor = np.empty((cap, 6), dtype=np.float32)
        col = np.empty((cap, 3), dtype=np.uint8) if rgb else None
        n = self._extract(posnor, col, cap, min_weight, iso)
        if n < 0:
            return None if not rgb else (None, None)
        if rgb:
            return posnor[:n].copy(), col[:n].copy()
        return posnor[:n].copy()


class OracleVolume(_CpuVolume):
    def __init__(self, voxel, pool, trunc=-1.0, weight_cap=32.0, hash_slots=0):
        self.lib = oracle_lib()
        self.h = self.lib.oracle_create(voxel, pool, trunc, weight_cap, hash_slots)
        if not self.h:
            raise ValueError("oracle_create rejected the parameters")

    def __del__(self):
        if getattr(self, "h", None):
            self.lib.oracle_destroy(self.h)
            self.h = None

    def allocate(self, points, cam, radius=0.0):
        p, n = self._pts(points)
        return self.lib.oracle_allocate_blocks(self.h, _ptr(p, C.c_float), n, *map(float, cam), radius)

    def update(self, points, cam, radius=0.0, colors=None, weights=None):
        p, n = self._pts(points)
        c = None if colors is None else np.ascontiguousarray(colors, dtype=np.uint8)
        w = None if weights is None else np.ascontiguousarray(weights, dtype=np.float32)
        return self.lib.oracle_update_voxels(self.h, _ptr(p, C.c_float), _ptr(c, C.c_uint8),
                                             _ptr(w, C.c_float), n, *map(float, cam), radius)

    def integrate(self, points, cam, radius=0.0, colors=None, weights=None):
        rc = self.allocate(points, cam, radius)
        return rc or self.update(points, cam, radius, colors, weights)

    def block_count(self):
        return self.lib.oracle_block_count(self.h)

    def drop_count(self):
        return self.lib.oracle_drop_count(self.h)

    def hash_mask(self):
        return self.lib.oracle_hash_mask(self.h)

    def table(self):
        size = self.hash_mask() + 1
        keys = np.empty(size, dtype=np.int64)
        idx = np.empty(size, dtype=np.int32)
        self.lib.oracle_table(self.h, _ptr(keys, C.c_int64), _ptr(idx, C.c_int32))
        return keys, idx

    def _coords(self, out):
        self.lib.oracle_block_coords(self.h, _ptr(out, C.c_int32))

    def _voxels(self, t, w, r, g, b):
        self.lib.oracle_voxels(self.h, *(_ptr(a, C.c_float) for a in (t, w, r, g, b)))

    def _extract(self, posnor, col, cap, min_w, iso):
        return self.lib.oracle_extract_mesh(self.h, _ptr(posnor, C.c_float), _ptr(col, C.c_uint8),
                                            cap, min_w, iso)


class RefVolume(_CpuVolume):
    """The reference CPU arm (cpp/src/volume.cpp) behind the same surface."""

    def __init__(self, voxel, pool, trunc=-1.0, weight_cap=32.0, threads=1):
        self.lib = ref_lib()
        self.h = self.lib.ref_create(voxel, pool, trunc, weight_cap)
        if not self.h:
            raise ValueError("reference Volume rejected the parameters")
        self.lib.ref_set_threads(self.h, threads)

    def __del__(self):
        if getattr(self, "h", None):
            self.lib.ref_destroy(self.h)
            self.h = None

    def allocate(self, points, cam, radius=0.0):
        p, n = self._pts(points)
        self.lib.ref_allocate(self.h, _ptr(p, C.c_float), n, *map(float, cam), radius)
        return 0

    def update(self, points, cam, radius=0.0, colors=None, weights=None):
        p, n = self._pts(points)
        c = None if colors is None else np.ascontiguousarray(colors, dtype=np.uint8)
        w = None if weights is None else np.ascontiguousarray(weights, dtype=np.float32)
        self.lib.ref_update(self.h, _ptr(p, C.c_float), _ptr(c, C.c_uint8), _ptr(w, C.c_float), n,
                            *map(float, cam), radius)
        return 0

    def integrate(self, points, cam, radius=0.0, colors=None, weights=None):
        p, n = self._pts(points)
        c = None if colors is None else np.ascontiguousarray(colors, dtype=np.uint8)
        w = None if weights is None else np.ascontiguousarray(weights, dtype=np.float32)
        self.lib.ref_integrate(self.h, _ptr(p, C.c_float), _ptr(c, C.c_uint8), _ptr(w, C.c_float),
                               n, *map(float, cam), radius)
        return 0

    def block_count(self):
        return self.lib.ref_block_count(self.h)

    def drop_count(self):
        return self.lib.ref_drop_count(self.h)

    def hash_mask(self):
        return self.lib.ref_hash_mask(self.h)

    def table(self):
        size = self.hash_mask() + 1
        keys = np.empty(size, dtype=np.int64)
        idx = np.empty(size, dtype=np.int32)
        self.lib.ref_table(self.h, _ptr(keys, C.c_int64), _ptr(idx, C.c_int32))
        return keys, idx

    def _coords(self, out):
        self.lib.ref_block_coords(self.h, _ptr(out, C.c_int32))

    def _voxels(self, t, w, r, g, b):
        self.lib.ref_voxels(self.h, *(_ptr(a, C.c_float) for a in (t, w, r, g, b)))

    def _extract(self, posnor, col, cap, min_w, iso):
        return self.lib.ref_extract(self.h, _ptr(posnor, C.c_float), _ptr(col, C.c_uint8), cap,
                                    min_w, iso)
