// Accessors into the reference's own CPU arm -- TEST INFRASTRUCTURE.
//
// Compiled by oracle/Makefile together with the reference's unmodified
// sources (cpp/src/volume.cpp, cpp/src/marching_tets.cpp, cpp/src/c_api.cpp)
// into oracle/_ref/libosn_tsdf_ref.so. The reference keeps its block
// coordinates and voxel arrays private (cpp/include/osn_tsdf/volume.hpp:401-447)
// and its C API exposes only counts and meshes, so this shim opens the class
// up for reading. It changes nothing the reference computes: every mutating
// call goes through the reference's own Volume methods.
#include <atomic>
#include <cstdint>
#include <cstring>
#include <functional>
#include <memory>
#include <new>
#include <thread>
#include <vector>

#define private public
#include "osn_tsdf/volume.hpp"
#undef private

using osn_tsdf::BlockCoord;
using osn_tsdf::HashEntry;
using osn_tsdf::kBlockVoxels;
using osn_tsdf::MeshBuffers;
using osn_tsdf::PointBatch;
using osn_tsdf::Volume;
using osn_tsdf::VolumeConfig;

namespace {
PointBatch make_batch(const float* pos, const uint8_t* col, const float* w, int32_t n, float cx,
                      float cy, float cz, float radius) {
    PointBatch b;
    b.positions = pos;
    b.colors = col;
    b.weights = w;
    b.n = n;
    b.cam[0] = cx;
    b.cam[1] = cy;
    b.cam[2] = cz;
    b.radius_m = radius;
    return b;
}
}  // namespace

extern "C" {

void* ref_create(float voxel, int32_t pool, float trunc, float cap) {
    VolumeConfig cfg;
    cfg.voxel_size_m = voxel;
    cfg.pool_capacity_blocks = pool;
    cfg.trunc_m = trunc;
    cfg.weight_cap = cap;
    try {
        return new Volume(cfg);
    } catch (...) {
        return nullptr;
    }
}

void ref_destroy(void* v) { delete static_cast<Volume*>(v); }

void ref_set_threads(void* v, int32_t n) { static_cast<Volume*>(v)->set_thread_count(n); }

void ref_allocate(void* v, const float* pos, int32_t n, float cx, float cy, float cz, float radius) {
    static_cast<Volume*>(v)->allocate_blocks(make_batch(pos, nullptr, nullptr, n, cx, cy, cz, radius));
}

void ref_update(void* v, const float* pos, const uint8_t* col, const float* w, int32_t n, float cx,
                float cy, float cz, float radius) {
    static_cast<Volume*>(v)->update_voxels(make_batch(pos, col, w, n, cx, cy, cz, radius));
}

void ref_integrate(void* v, const float* pos, const uint8_t* col, const float* w, int32_t n,
                   float cx, float cy, float cz, float radius) {
    static_cast<Volume*>(v)->integrate(make_batch(pos, col, w, n, cx, cy, cz, radius));
}

int32_t ref_extract(void* v, float* posnor, uint8_t* rgb, int32_t cap, float min_w, float iso) {
    MeshBuffers out;
    out.posnor = posnor;
    out.rgb = rgb;
    out.capacity_vertices = cap;
    return static_cast<Volume*>(v)->extract_mesh(out, min_w, iso);
}

int32_t ref_block_count(void* v) { return static_cast<Volume*>(v)->block_count(); }
uint64_t ref_drop_count(void* v) { return static_cast<Volume*>(v)->drop_count(); }
uint32_t ref_hash_mask(void* v) { return static_cast<Volume*>(v)->hash_mask_; }

int32_t ref_block_coords(void* v, int32_t* out) {
    auto* vol = static_cast<Volume*>(v);
    const int32_t n = vol->block_count();
    for (int32_t i = 0; i < n; ++i) {
        const BlockCoord& c = vol->block_coord_[static_cast<std::size_t>(i)];
        out[i * 3 + 0] = c.x;
        out[i * 3 + 1] = c.y;
        out[i * 3 + 2] = c.z;
    }
    return n;
}

int32_t ref_voxels(void* v, float* tsdf, float* weight, float* r, float* g, float* b) {
    auto* vol = static_cast<Volume*>(v);
    const std::size_t n = static_cast<std::size_t>(vol->block_count()) * kBlockVoxels;
    if (tsdf) std::memcpy(tsdf, vol->tsdf_.data(), n * sizeof(float));
    if (weight) std::memcpy(weight, vol->weight_.data(), n * sizeof(float));
    if (r) std::memcpy(r, vol->r_.data(), n * sizeof(float));
    if (g) std::memcpy(g, vol->g_.data(), n * sizeof(float));
    if (b) std::memcpy(b, vol->b_.data(), n * sizeof(float));
    return 0;
}

int32_t ref_table(void* v, int64_t* keys, int32_t* idx) {
    auto* vol = static_cast<Volume*>(v);
    for (std::size_t i = 0; i < vol->table_.size(); ++i) {
        if (keys) keys[i] = vol->table_[i].key;
        if (idx) idx[i] = vol->table_[i].block_idx;
    }
    return 0;
}

}  // extern "C"
