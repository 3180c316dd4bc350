"""The C-ABI library loads and exports every symbol the public header declares
(no compute calls: these run without a GPU)."""
import ctypes as C
import os
import re

import pytest

from what_irregularity_costs_b200 import _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

# The reference's CUDA section, cpp/include/osn_tsdf/c_api.h:80-126.
REFERENCE_CUDA_ENTRY_POINTS = [
    "osn_tsdf_cuda_create", "osn_tsdf_cuda_destroy", "osn_tsdf_cuda_valid",
    "osn_tsdf_cuda_device_view", "osn_tsdf_cuda_allocate_blocks", "osn_tsdf_cuda_update_voxels",
    "osn_tsdf_cuda_extract_mesh", "osn_tsdf_cuda_reset", "osn_tsdf_cuda_allocate_counting_cas",
    "osn_tsdf_cuda_allocate_no_cas", "osn_tsdf_cuda_allocate_slot_index",
    "osn_tsdf_cuda_block_count", "osn_tsdf_cuda_drop_count", "osn_tsdf_cuda_synchronize",
]


@pytest.fixture(scope="module")
def lib():
    if not os.path.exists(_lib.LIB_PATH):
        from what_irregularity_costs_b200 import build
        build.build()
    return _lib.load()


def test_header_declares_reference_surface():
    declared = _lib.declared_symbols()
    for name in REFERENCE_CUDA_ENTRY_POINTS:
        assert name in declared, name


def test_library_exports_every_declared_symbol(lib):
    for name in _lib.declared_symbols():
        assert hasattr(lib, name), f"{name} declared but not exported"


def test_ctypes_signatures_cover_header():
    assert set(_lib._SIG) == set(_lib.declared_symbols())


def test_device_view_layout():
    assert C.sizeof(_lib.OsnTsdfDeviceView) == 104
    assert _lib.OsnTsdfDeviceView.hash_mask.offset == 72
    assert _lib.OsnTsdfDeviceView.weight_cap.offset == 96


def test_reference_prototypes_match():
    """Each reference CUDA entry point keeps its parameter list."""
    with open(os.path.join(ROOT, "include", "osn_tsdf_b200.h")) as f:
        ours = re.sub(r"\s+", " ", f.read())
    expected = {
        "osn_tsdf_cuda_create": "float voxel_size_m, int32_t pool_capacity_blocks, float trunc_m, float weight_cap",
        "osn_tsdf_cuda_allocate_blocks": "OsnTsdfCudaVolume* v, const float* d_positions, int32_t n_points, float cam_x, float cam_y, float cam_z, float radius_m",
        "osn_tsdf_cuda_update_voxels": "OsnTsdfCudaVolume* v, const float* d_positions, int32_t n_points, float cam_x, float cam_y, float cam_z, float radius_m",
        "osn_tsdf_cuda_extract_mesh": "OsnTsdfCudaVolume* v, float* buffer_posnor, uint8_t* buffer_rgb, int32_t vert_cap, float min_weight, float iso",
        "osn_tsdf_cuda_device_view": "const OsnTsdfCudaVolume* v, OsnTsdfDeviceView* out",
    }
    for name, params in expected.items():
        assert f"{name}({params})" in ours, name


def test_no_cpu_fallback_when_library_missing(tmp_path):
    with pytest.raises(ImportError):
        saved = _lib._lib
        _lib._lib = None
        try:
            _lib.load(str(tmp_path / "missing.so"))
        finally:
            _lib._lib = saved
