"""B200-native hash-blocked TSDF integrate path (allocate / update / extract).

The compute lives in ``libosn_tsdf_b200.so`` (hand-written sm_100a CUDA behind
the reference's CUDA C ABI, declared in ``include/osn_tsdf_b200.h``). This
package is the Python host mirror of that interface plus the synthetic
scene generators used by the tests and the benchmark.
"""
from .volume import (CudaVolume, device_tensor, KERNEL_NAMES, LAYOUT_POOL,  # noqa: F401
                     LAYOUT_SLOT_INDEX, MAX_DEPTH_FRAMES, MAX_FRAMES, STORAGE_FP32, STORAGE_FP16_U16,
                     STORAGE_FP64, STORAGE_NAMES)
from . import scenes  # noqa: F401
from . import precision  # noqa: F401
from .batch import Batch  # noqa: F401

__all__ = ["CudaVolume", "Batch", "device_tensor", "scenes", "precision", "KERNEL_NAMES",
           "LAYOUT_POOL", "LAYOUT_SLOT_INDEX",
           "MAX_DEPTH_FRAMES", "MAX_FRAMES", "STORAGE_FP32", "STORAGE_FP16_U16", "STORAGE_FP64",
           "STORAGE_NAMES"]
