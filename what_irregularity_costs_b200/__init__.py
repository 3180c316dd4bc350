"""B200-native hash-blocked TSDF integrate path (allocate / update / extract).

The compute lives in ``libosn_tsdf_b200.so`` (hand-written sm_100a CUDA behind
the reference's CUDA C ABI, declared in ``include/osn_tsdf_b200.h``). This
package is the Python host mirror of that interface plus the synthetic
scene generators used by the tests and the benchmark.
"""
from .volume import CudaVolume, device_tensor, KERNEL_NAMES  # noqa: F401
from . import scenes  # noqa: F401

__all__ = ["CudaVolume", "device_tensor", "scenes", "KERNEL_NAMES"]
