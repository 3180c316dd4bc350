// osn_tsdf_b200: the reference's C++ interface of its CUDA arm (A3),
// implemented by this library.
//
// Re-declares cpp/include/osn_tsdf/volume_cuda.hpp:24-86 (class CudaVolume)
// and the parameter types it takes from cpp/include/osn_tsdf/types.hpp
// (VolumeConfig :94-116, PointBatch :122-135, MeshBuffers :138-142) with the
// same names, namespace, member layout and meaning, so C++ code written
// against the reference's CudaVolume -- its own cpp/tests/test_cuda_analytic.cu
// among it -- compiles against either header and links against
// libosn_tsdf_b200.so instead of the reference's CUDA arm. Include this
// header or the reference's, not both.
//
// Differences from the reference class, each deliberate:
//   - a PointBatch with colours or per-point weights is refused (a message on
//     stderr, nothing queued): this library's kernels integrate unit-weight,
//     grey contributions, which is all the reference's C ABI ever passes;
//   - allocate_blocks_probe_depth and device_view (which returns a type of
//     the reference's private CUDA header) are not provided; the C ABI has
//     osn_tsdf_cuda_allocate_probe_histogram and osn_tsdf_cuda_device_view.
#pragma once

#include <cstddef>
#include <cstdint>

namespace osn_tsdf {

/// Construction parameters (types.hpp:94-116).
struct VolumeConfig {
    float voxel_size_m = 0.01f;
    int32_t pool_capacity_blocks = 1 << 16;
    /// TSDF truncation half-width in metres; <= 0 selects 4 * voxel_size.
    float trunc_m = -1.0f;
    /// Cap on accumulated weight; <= 0 disables.
    float weight_cap = 32.0f;

    float trunc() const { return trunc_m > 0.0f ? trunc_m : 4.0f * voxel_size_m; }
    /// Bytes of the five per-voxel float arrays of the block pool.
    std::size_t pool_bytes() const {
        return static_cast<std::size_t>(pool_capacity_blocks) * 512 * 5 * sizeof(float);
    }
};

/// World-space points to integrate (types.hpp:122-135); positions are DEVICE
/// pointers for CudaVolume.
struct PointBatch {
    const float* positions = nullptr;  // 3 * n, interleaved xyz
    const uint8_t* colors = nullptr;   // must be null here (grey)
    const float* weights = nullptr;    // must be null here (unit weights)
    int32_t n = 0;
    int32_t chunk_id = 0;              // tags the blocks a call allocates or updates (streaming)
    float cam[3] = {0.0f, 0.0f, 0.0f};
    float radius_m = 0.0f;             // far cutoff; <= 0 disables
};

/// Output triangle soup, 6 floats per vertex (types.hpp:138-142); HOST buffers.
struct MeshBuffers {
    float* posnor = nullptr;
    uint8_t* rgb = nullptr;
    int32_t capacity_vertices = 0;
};

struct CudaVolumeImpl;

class CudaVolume {
public:
    explicit CudaVolume(const VolumeConfig& cfg);
    ~CudaVolume();

    CudaVolume(const CudaVolume&) = delete;
    CudaVolume& operator=(const CudaVolume&) = delete;
    CudaVolume(CudaVolume&&) = delete;
    CudaVolume& operator=(CudaVolume&&) = delete;

    /// True when construction obtained all device memory.
    bool valid() const;

    /// Asynchronous on the volume's stream.
    void integrate(const PointBatch& batch);
    void allocate_blocks(const PointBatch& batch);
    void update_voxels(const PointBatch& batch);
    /// Measurement modes of the reference (c_api.h:108-122).
    void allocate_blocks_counting_cas(const PointBatch& batch);
    void allocate_blocks_no_cas(const PointBatch& batch);
    void allocate_blocks_slot_index(const PointBatch& batch);

    /// Copies the mesh to the host buffers; vertex count, or -1 on overflow.
    int32_t extract_mesh(const MeshBuffers& out, float min_weight, float iso) const;

    int32_t block_count() const;
    uint64_t drop_count() const;
    const VolumeConfig& config() const;
    void synchronize() const;
    void reset();

private:
    CudaVolumeImpl* impl_ = nullptr;
};

}  // namespace osn_tsdf
