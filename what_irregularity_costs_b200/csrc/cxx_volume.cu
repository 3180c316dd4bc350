// osn_tsdf::CudaVolume, the reference's C++ class of its CUDA arm
// (cpp/include/osn_tsdf/volume_cuda.hpp:24-86, implemented there by
// cpp/src/volume_cuda.cu:343-480), over this library's Volume: same calls,
// same kernels and results as the C ABI.
#include <cstdio>
#include <new>

#include "../../include/osn_tsdf_b200.hpp"
#include "volume.h"

namespace osn_tsdf {

struct CudaVolumeImpl {
    osn_b200::Volume vol;
    VolumeConfig cfg;
    explicit CudaVolumeImpl(const VolumeConfig& c)
        : vol(c.voxel_size_m, c.pool_capacity_blocks, c.trunc_m, c.weight_cap, 0u), cfg(c) {}
};

namespace {

// The batch as this library's kernels take it; false (and a message) for
// inputs they do not integrate.
bool to_args(const PointBatch& b, osn_b200::BatchArgs& a) {
    if (b.colors || b.weights) {
        std::fprintf(stderr,
                     "[osn_tsdf_b200] CudaVolume: batches with colours or per-point weights are "
                     "not supported (unit-weight grey contributions only); batch skipped\n");
        return false;
    }
    if (!b.positions || b.n <= 0) return false;
    a = osn_b200::BatchArgs{};
    a.pos = b.positions;
    a.n = b.n;
    a.cam_x = b.cam[0];
    a.cam_y = b.cam[1];
    a.cam_z = b.cam[2];
    a.radius_sq = b.radius_m > 0.0f ? b.radius_m * b.radius_m : 0.0f;
    return true;
}

}  // namespace

CudaVolume::CudaVolume(const VolumeConfig& cfg) {
    if (!(cfg.voxel_size_m > 0.0f) || cfg.pool_capacity_blocks <= 0) return;
    impl_ = new (std::nothrow) CudaVolumeImpl(cfg);
    if (impl_ && !impl_->vol.ok()) {
        delete impl_;
        impl_ = nullptr;
    }
}

CudaVolume::~CudaVolume() { delete impl_; }

bool CudaVolume::valid() const { return impl_ != nullptr; }

// The batch's chunk id tags the blocks the call allocates or updates.
void CudaVolume::integrate(const PointBatch& batch) {
    osn_b200::BatchArgs a;
    if (!impl_ || !to_args(batch, a)) return;
    impl_->vol.set_chunk(batch.chunk_id);
    impl_->vol.integrate(a);
}

void CudaVolume::allocate_blocks(const PointBatch& batch) {
    osn_b200::BatchArgs a;
    if (!impl_ || !to_args(batch, a)) return;
    impl_->vol.set_chunk(batch.chunk_id);
    impl_->vol.allocate(a, osn_b200::kAllocInsert, nullptr, 0);
}

void CudaVolume::update_voxels(const PointBatch& batch) {
    osn_b200::BatchArgs a;
    if (!impl_ || !to_args(batch, a)) return;
    impl_->vol.set_chunk(batch.chunk_id);
    impl_->vol.update(a);
}

void CudaVolume::allocate_blocks_counting_cas(const PointBatch& batch) {
    osn_b200::BatchArgs a;
    if (impl_ && to_args(batch, a)) impl_->vol.allocate(a, osn_b200::kAllocCountingCas, nullptr, 0);
}

void CudaVolume::allocate_blocks_no_cas(const PointBatch& batch) {
    osn_b200::BatchArgs a;
    if (impl_ && to_args(batch, a)) impl_->vol.allocate(a, osn_b200::kAllocNoCas, nullptr, 0);
}

void CudaVolume::allocate_blocks_slot_index(const PointBatch& batch) {
    osn_b200::BatchArgs a;
    if (impl_ && to_args(batch, a)) impl_->vol.allocate(a, osn_b200::kAllocSlotIndex, nullptr, 0);
}

int32_t CudaVolume::extract_mesh(const MeshBuffers& out, float min_weight, float iso) const {
    if (!impl_ || !out.posnor || out.capacity_vertices < 0) return -1;
    return impl_->vol.extract(out.posnor, out.rgb, out.capacity_vertices, min_weight, iso, true);
}

int32_t CudaVolume::block_count() const { return impl_ ? impl_->vol.block_count() : 0; }

uint64_t CudaVolume::drop_count() const { return impl_ ? impl_->vol.drop_count() : 0; }

const VolumeConfig& CudaVolume::config() const {
    static const VolumeConfig none{};
    return impl_ ? impl_->cfg : none;
}

void CudaVolume::synchronize() const {
    if (impl_) impl_->vol.synchronize();
}

void CudaVolume::reset() {
    if (impl_) impl_->vol.reset();
}

}  // namespace osn_tsdf
