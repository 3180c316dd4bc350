"""ctypes binding of libosn_tsdf_b200.so (the C ABI in include/osn_tsdf_b200.h).

The library is loaded from the package directory only. If it is missing the
import fails loudly: there is no CPU fallback for the CUDA path.
"""
from __future__ import annotations

import ctypes as C
import os
import re

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
LIB_PATH = os.path.join(HERE, "libosn_tsdf_b200.so")
HEADER = os.path.join(ROOT, "include", "osn_tsdf_b200.h")


class OsnTsdfDeviceView(C.Structure):
    """Mirror of OsnTsdfDeviceView (104 bytes, cpp/include/osn_tsdf/c_api.h:61-78)."""

    _fields_ = [
        ("table", C.c_void_p),
        ("block_count", C.c_void_p),
        ("drop_count", C.c_void_p),
        ("block_coord", C.c_void_p),
        ("tsdf", C.c_void_p),
        ("weight", C.c_void_p),
        ("r", C.c_void_p),
        ("g", C.c_void_p),
        ("b", C.c_void_p),
        ("hash_mask", C.c_uint32),
        ("scratch_base", C.c_uint32),
        ("pool_capacity", C.c_int32),
        ("block_dim", C.c_int32),
        ("voxel_size_m", C.c_float),
        ("trunc_m", C.c_float),
        ("weight_cap", C.c_float),
    ]


assert C.sizeof(OsnTsdfDeviceView) == 104

_P = C.c_void_p
_F = C.c_float
_I = C.c_int32
_SIG = {
    "osn_tsdf_cuda_create": (_P, [_F, _I, _F, _F]),
    "osn_tsdf_cuda_create_ex": (_P, [_F, _I, _F, _F, C.c_uint32, _I]),
    "osn_tsdf_cuda_destroy": (None, [_P]),
    "osn_tsdf_cuda_valid": (_I, [_P]),
    "osn_tsdf_cuda_device_view": (_I, [_P, C.POINTER(OsnTsdfDeviceView)]),
    "osn_tsdf_cuda_allocate_blocks": (_I, [_P, _P, _I, _F, _F, _F, _F]),
    "osn_tsdf_cuda_update_voxels": (_I, [_P, _P, _I, _F, _F, _F, _F]),
    "osn_tsdf_cuda_integrate": (_I, [_P, _P, _I, _F, _F, _F, _F]),
    "osn_tsdf_cuda_integrate_frames": (_I, [_P, _P, _P, _P, _I, _F]),
    "osn_tsdf_cuda_integrate_depth_frames": (_I, [_P, _P, _I, _I, _I, C.c_double, C.c_double, C.c_double,
                                                  C.c_double, _P, _P, _F]),
    "osn_tsdf_cuda_integrate_depth": (_I, [_P, _P, _I, _I, C.c_double, C.c_double, C.c_double,
                                           C.c_double, _P, _P, _F]),
    "osn_tsdf_cuda_extract_mesh": (_I, [_P, _P, _P, _I, _F, _F]),
    "osn_tsdf_cuda_write_mesh_osn1": (_I, [_P, C.c_char_p, _I, _F, _F]),
    "osn_tsdf_cuda_extract_mesh_device": (_I, [_P, _P, _P, _I, _F, _F]),
    "osn_tsdf_cuda_reset": (_I, [_P]),
    "osn_tsdf_cuda_allocate_counting_cas": (_I, [_P, _P, _I, _F, _F, _F, _F]),
    "osn_tsdf_cuda_allocate_no_cas": (_I, [_P, _P, _I, _F, _F, _F, _F]),
    "osn_tsdf_cuda_allocate_slot_index": (_I, [_P, _P, _I, _F, _F, _F, _F]),
    "osn_tsdf_cuda_allocate_probe_histogram": (_I, [_P, _P, _I, _F, _F, _F, _F, _P, _I]),
    "osn_tsdf_cuda_block_count": (_I, [_P]),
    "osn_tsdf_cuda_drop_count": (C.c_uint64, [_P]),
    "osn_tsdf_cuda_synchronize": (None, [_P]),
    "osn_tsdf_cuda_status": (C.c_uint32, [_P]),
    "osn_tsdf_cuda_stream": (_P, [_P]),
    "osn_tsdf_cuda_set_pipelined": (_I, [_P, _I]),
    "osn_tsdf_cuda_set_spin_limit": (_I, [_P, _I]),
    "osn_tsdf_cuda_set_chunk": (_I, [_P, _I]),
    "osn_tsdf_cuda_create_layout": (_P, [_F, _I, _F, _F, C.c_uint32, _I, _I]),
    "osn_tsdf_cuda_layout": (_I, [_P]),
    "osn_tsdf_cuda_evict_chunks_bytes": (C.c_int64, [_P, _I, _I]),
    "osn_tsdf_cuda_evict_chunks": (C.c_int64, [_P, _I, _I, _P, C.c_int64]),
    "osn_tsdf_cuda_stream_in": (_I, [_P, _P, C.c_int64, _P]),
    "osn_tsdf_cuda_l2_probe": (_I, [_I, C.c_int64, _I, _P]),
    "osn_tsdf_cuda_join": (_I, [_P]),
    "osn_tsdf_cuda_storage": (_I, [_P]),
    "osn_tsdf_cuda_snapshot_bytes": (C.c_int64, [_P]),
    "osn_tsdf_cuda_snapshot": (C.c_int64, [_P, _P, C.c_int64]),
    "osn_tsdf_cuda_restore": (_I, [_P, _P, C.c_int64]),
    "osn_tsdf_cuda_last_update_stats": (_I, [_P, _P]),
    "osn_tsdf_cuda_set_timing": (_I, [_P, _I]),
    "osn_tsdf_cuda_kernel_times": (_I, [_P, _P, _P, _I]),
    "osn_tsdf_cuda_update_voxels_noalloc": (_I, [_P, _P, _I, _F, _F, _F, _F]),
    "osn_tsdf_batch_create": (_P, [_I]),
    "osn_tsdf_batch_destroy": (None, [_P]),
    "osn_tsdf_batch_add": (_I, [_P, _P, _I]),
    "osn_tsdf_batch_remove": (_I, [_P, _I]),
    "osn_tsdf_batch_set_frame": (_I, [_P, _I, _P, _I, _F, _F, _F, _F]),
    "osn_tsdf_batch_step": (_I, [_P]),
    "osn_tsdf_batch_synchronize": (_I, [_P]),
    "osn_tsdf_batch_set_graph": (_I, [_P, _I]),
    "osn_tsdf_batch_autotune": (_I, [_P, _I]),
    "osn_tsdf_batch_set_shape": (_I, [_P, _I, _I, _I]),
    "osn_tsdf_batch_shape": (_I, [_P, _P]),
    "osn_tsdf_batch_tune_results": (_I, [_P, _P, _P, _I]),
    "osn_tsdf_batch_status": (C.c_uint32, [_P]),
    "osn_tsdf_batch_stream": (_P, [_P]),
    "osn_tsdf_batch_size": (_I, [_P]),
}

_lib = None


def declared_symbols() -> list[str]:
    """Every function the public header declares."""
    with open(HEADER) as f:
        text = f.read()
    return sorted(set(re.findall(r"\b(osn_tsdf_(?:cuda|batch)_\w+)\s*\(", text)))


def load(path: str | None = None):
    """Load the CUDA library (once). Raises if it has not been built.
    OSN_TSDF_B200_LIB names another build of it (a variant compiled with
    different tuning flags) in place of the in-tree one."""
    global _lib
    if _lib is not None:
        return _lib
    path = path or os.environ.get("OSN_TSDF_B200_LIB") or LIB_PATH
    if not os.path.exists(path):
        raise ImportError(
            f"libosn_tsdf_b200.so not found at {path}; build it with "
            "`python -m what_irregularity_costs_b200.build` (there is no CPU fallback)")
    lib = C.CDLL(path)
    for name, (res, args) in _SIG.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib
