// The C ABI: the reference's CUDA section of cpp/include/osn_tsdf/c_api.h
// (implemented there by cpp/src/c_api_cuda.cu) plus this library's
// extensions, declared in include/osn_tsdf_b200.h.
#include <climits>
#include <cstdio>
#include <cstring>
#include <memory>

#include "../../include/osn_tsdf_b200.h"
#include "volume.h"

using osn_b200::BatchArgs;
using osn_b200::Volume;

static_assert(sizeof(OsnTsdfDeviceView) == 104,
              "OsnTsdfDeviceView must keep the reference's 104-byte layout");

struct OsnTsdfCudaVolume {
    Volume vol;
    OsnTsdfCudaVolume(float voxel, int32_t pool, float trunc, float cap, uint32_t slots, int storage,
                      int layout)
        : vol(voxel, pool, trunc, cap, slots, storage, layout) {}
};

namespace {

BatchArgs batch(const float* pos, int32_t n, float cx, float cy, float cz, float radius) {
    BatchArgs a{};
    a.pos = pos;
    a.n = n;
    a.cam_x = cx;
    a.cam_y = cy;
    a.cam_z = cz;
    a.radius_sq = radius > 0.0f ? radius * radius : 0.0f;
    return a;
}

bool usable(const OsnTsdfCudaVolume* v) { return v && v->vol.ok(); }

// A batch's records carry the 32-bit id point * (2*steps+1) + step.
bool batch_fits(const OsnTsdfCudaVolume* v, int32_t n) {
    const int64_t steps = 2 * (int64_t)v->vol.dev().steps + 1;
    return (int64_t)n * steps < (int64_t(1) << 32);
}

int32_t allocate_mode(OsnTsdfCudaVolume* v, const float* d_positions, int32_t n, float cx,
                      float cy, float cz, float radius, int mode) {
    if (!usable(v) || !d_positions || n <= 0) return 1;
    return v->vol.allocate(batch(d_positions, n, cx, cy, cz, radius), mode, nullptr, 0) ==
                   cudaSuccess
               ? 0
               : 3;
}

}  // namespace

osn_b200::Volume* osn_tsdf_b200_volume_of(OsnTsdfCudaVolume* v) {
    return usable(v) ? &v->vol : nullptr;
}

extern "C" {

OsnTsdfCudaVolume* osn_tsdf_cuda_create(float voxel_size_m, int32_t pool_capacity_blocks,
                                        float trunc_m, float weight_cap) {
    return osn_tsdf_cuda_create_ex(voxel_size_m, pool_capacity_blocks, trunc_m, weight_cap, 0u,
                                   OSN_TSDF_STORAGE_FP32);
}

OsnTsdfCudaVolume* osn_tsdf_cuda_create_ex(float voxel_size_m, int32_t pool_capacity_blocks,
                                           float trunc_m, float weight_cap, uint32_t hash_slots,
                                           int32_t storage) {
    return osn_tsdf_cuda_create_layout(voxel_size_m, pool_capacity_blocks, trunc_m, weight_cap, hash_slots,
                                       storage, OSN_TSDF_LAYOUT_POOL);
}

OsnTsdfCudaVolume* osn_tsdf_cuda_create_layout(float voxel_size_m, int32_t pool_capacity_blocks,
                                               float trunc_m, float weight_cap, uint32_t hash_slots,
                                               int32_t storage, int32_t layout) {
    if (storage != OSN_TSDF_STORAGE_FP32 && storage != OSN_TSDF_STORAGE_FP16_U16 &&
        storage != OSN_TSDF_STORAGE_FP64)
        return nullptr;
    if (layout != OSN_TSDF_LAYOUT_POOL && layout != OSN_TSDF_LAYOUT_SLOT_INDEX) return nullptr;
    if (!(voxel_size_m > 0.0f) || pool_capacity_blocks <= 0) return nullptr;
    auto* v = new (std::nothrow) OsnTsdfCudaVolume(voxel_size_m, pool_capacity_blocks, trunc_m,
                                                   weight_cap, hash_slots, storage, layout);
    if (!v) return nullptr;
    if (!v->vol.ok()) {
        delete v;
        return nullptr;
    }
    return v;
}

void osn_tsdf_cuda_destroy(OsnTsdfCudaVolume* v) { delete v; }

int32_t osn_tsdf_cuda_valid(const OsnTsdfCudaVolume* v) { return usable(v) ? 1 : 0; }

int32_t osn_tsdf_cuda_device_view(const OsnTsdfCudaVolume* v, OsnTsdfDeviceView* out) {
    if (!usable(v) || !out) return 1;
    const auto& d = v->vol.dev();
    out->table = d.table;
    out->block_count = d.block_count;
    out->drop_count = d.drop_count;
    out->block_coord = d.block_coord;
    out->tsdf = d.tsdf;
    out->weight = d.weight;
    out->r = d.r;
    out->g = d.g;
    out->b = d.b;
    out->hash_mask = d.hash_mask;
    out->scratch_base = d.hash_mask + 1;
    out->pool_capacity = d.pool_capacity;
    out->block_dim = osn_b200::kBlockDim;
    out->voxel_size_m = d.voxel_size;
    out->trunc_m = d.trunc;
    out->weight_cap = v->vol.weight_cap();
    return 0;
}

int32_t osn_tsdf_cuda_storage(const OsnTsdfCudaVolume* v) {
    return usable(v) ? v->vol.storage() : -1;
}

int32_t osn_tsdf_cuda_layout(const OsnTsdfCudaVolume* v) {
    return usable(v) ? v->vol.layout() : -1;
}

int32_t osn_tsdf_cuda_allocate_blocks(OsnTsdfCudaVolume* v, const float* d_positions,
                                      int32_t n_points, float cam_x, float cam_y, float cam_z,
                                      float radius_m) {
    return allocate_mode(v, d_positions, n_points, cam_x, cam_y, cam_z, radius_m,
                         osn_b200::kAllocInsert);
}

int32_t osn_tsdf_cuda_update_voxels(OsnTsdfCudaVolume* v, const float* d_positions,
                                    int32_t n_points, float cam_x, float cam_y, float cam_z,
                                    float radius_m) {
    if (!usable(v) || !d_positions || n_points <= 0 || !batch_fits(v, n_points)) return 1;
    return v->vol.update(batch(d_positions, n_points, cam_x, cam_y, cam_z, radius_m)) ==
                   cudaSuccess
               ? 0
               : 3;
}

int32_t osn_tsdf_cuda_integrate(OsnTsdfCudaVolume* v, const float* d_positions, int32_t n_points,
                                float cam_x, float cam_y, float cam_z, float radius_m) {
    if (!usable(v) || !d_positions || n_points <= 0 || !batch_fits(v, n_points)) return 1;
    return v->vol.integrate(batch(d_positions, n_points, cam_x, cam_y, cam_z, radius_m)) ==
                   cudaSuccess
               ? 0
               : 3;
}

static_assert(OSN_TSDF_MAX_FRAMES == osn_b200::kMaxFrames, "one frame limit");

int32_t osn_tsdf_cuda_integrate_frames(OsnTsdfCudaVolume* v, const float* d_positions,
                                       const int32_t* frame_begin, const float* cams_xyz,
                                       int32_t n_frames, float radius_m) {
    if (!usable(v) || !d_positions || !frame_begin || !cams_xyz || n_frames < 1 ||
        n_frames > osn_b200::kMaxFrames || frame_begin[0] != 0)
        return 1;
    for (int32_t k = 0; k < n_frames; ++k)
        if (frame_begin[k + 1] < frame_begin[k]) return 1;
    const int32_t n = frame_begin[n_frames];
    if (n <= 0 || !batch_fits(v, n)) return 1;
    if (v->vol.storage() == osn_b200::kStoreF64) return 2;
    osn_b200::FrameTable t{};
    t.n = n_frames;
    for (int32_t k = 0; k <= n_frames; ++k) {
        t.f[k].begin = frame_begin[k];
        if (k < n_frames) {
            t.f[k].x = cams_xyz[3 * k];
            t.f[k].y = cams_xyz[3 * k + 1];
            t.f[k].z = cams_xyz[3 * k + 2];
        }
    }
    // The batch's own camera is not read by the several-frame walk; the
    // update tail of FP32 / FP16 storage reads no camera.
    const BatchArgs a = batch(d_positions, n, cams_xyz[0], cams_xyz[1], cams_xyz[2], radius_m);
    return v->vol.integrate_frames(a, t) == cudaSuccess ? 0 : 3;
}

int32_t osn_tsdf_cuda_integrate_depth(OsnTsdfCudaVolume* v, const float* d_depth, int32_t width,
                                      int32_t height, double fx, double fy, double cx, double cy,
                                      const double* cam_to_world_R, const double* cam_to_world_t,
                                      float max_range_m) {
    if (!usable(v) || !d_depth || width <= 0 || height <= 0 || !cam_to_world_R || !cam_to_world_t ||
        !(fx != 0.0) || !(fy != 0.0))
        return 1;
    const int64_t n = (int64_t)width * height;
    if (n > INT32_MAX || !batch_fits(v, (int32_t)n)) return 1;
    // The camera origin of the walk is the pose translation as float, as a
    // caller passing backprojected points would pass it.
    BatchArgs a = batch(nullptr, (int32_t)n, (float)cam_to_world_t[0], (float)cam_to_world_t[1],
                        (float)cam_to_world_t[2], 0.0f);
    a.depth.depth = d_depth;
    a.depth.width = width;
    a.depth.max_range = max_range_m;
    a.depth.fx = fx;
    a.depth.fy = fy;
    a.depth.cx = cx;
    a.depth.cy = cy;
    for (int k = 0; k < 9; ++k) a.depth.R[k] = cam_to_world_R[k];
    for (int k = 0; k < 3; ++k) a.depth.t[k] = cam_to_world_t[k];
    return v->vol.integrate(a) == cudaSuccess ? 0 : 3;
}

static_assert(OSN_TSDF_MAX_DEPTH_FRAMES == osn_b200::kMaxDepthFrames, "one depth frame limit");

int32_t osn_tsdf_cuda_integrate_depth_frames(OsnTsdfCudaVolume* v, const float* d_depth, int32_t width,
                                             int32_t height, int32_t n_frames, double fx, double fy,
                                             double cx, double cy, const double* cam_to_world_R,
                                             const double* cam_to_world_t, float max_range_m) {
    if (!usable(v) || !d_depth || width <= 0 || height <= 0 || n_frames < 1 ||
        n_frames > osn_b200::kMaxDepthFrames || !cam_to_world_R || !cam_to_world_t || !(fx != 0.0) ||
        !(fy != 0.0))
        return 1;
    const int64_t npix = (int64_t)width * height;
    const int64_t n = npix * n_frames;
    if (n > INT32_MAX || !batch_fits(v, (int32_t)n)) return 1;
    if (v->vol.storage() == osn_b200::kStoreF64) return 2;
    osn_b200::FrameTable t{};
    osn_b200::PoseTable p{};
    t.n = n_frames;
    p.n = n_frames;
    for (int32_t k = 0; k <= n_frames; ++k) {
        t.f[k].begin = (int32_t)(npix * k);
        if (k == n_frames) break;
        // The camera origin of the walk is the pose translation as float, as
        // for a single depth image.
        t.f[k].x = (float)cam_to_world_t[3 * k];
        t.f[k].y = (float)cam_to_world_t[3 * k + 1];
        t.f[k].z = (float)cam_to_world_t[3 * k + 2];
        for (int j = 0; j < 9; ++j) p.p[k].R[j] = cam_to_world_R[9 * k + j];
        for (int j = 0; j < 3; ++j) p.p[k].t[j] = cam_to_world_t[3 * k + j];
    }
    BatchArgs a = batch(nullptr, (int32_t)n, t.f[0].x, t.f[0].y, t.f[0].z, 0.0f);
    a.depth.depth = d_depth;
    a.depth.width = width;
    a.depth.max_range = max_range_m;
    a.depth.fx = fx;
    a.depth.fy = fy;
    a.depth.cx = cx;
    a.depth.cy = cy;
    for (int j = 0; j < 9; ++j) a.depth.R[j] = cam_to_world_R[j];
    for (int j = 0; j < 3; ++j) a.depth.t[j] = cam_to_world_t[j];
    return v->vol.integrate_frames(a, t, &p) == cudaSuccess ? 0 : 3;
}

int32_t osn_tsdf_cuda_extract_mesh(OsnTsdfCudaVolume* v, float* buffer_posnor, uint8_t* buffer_rgb,
                                   int32_t vert_cap, float min_weight, float iso) {
    if (!usable(v) || !buffer_posnor || vert_cap <= 0) return -1;
    return v->vol.extract(buffer_posnor, buffer_rgb, vert_cap, min_weight, iso, true);
}

int32_t osn_tsdf_cuda_write_mesh_osn1(OsnTsdfCudaVolume* v, const char* path, int32_t vert_cap,
                                      float min_weight, float iso) {
    if (!usable(v) || !path || vert_cap <= 0) return -1;
    std::unique_ptr<float[]> posnor(new (std::nothrow) float[(size_t)vert_cap * 6]);
    if (!posnor) return -1;
    const int32_t n = v->vol.extract(posnor.get(), nullptr, vert_cap, min_weight, iso, true);
    if (n < 0) return -1;
    std::FILE* f = std::fopen(path, "wb");
    if (!f) return -2;
    const uint32_t magic = 0x314e534fu;  // the bytes "OSN1" in little-endian order
    const uint32_t nv = (uint32_t)n;
    bool ok = std::fwrite(&magic, 4, 1, f) == 1 && std::fwrite(&nv, 4, 1, f) == 1;
    if (ok && n > 0) ok = std::fwrite(posnor.get(), sizeof(float), (size_t)n * 6, f) == (size_t)n * 6;
    ok = std::fclose(f) == 0 && ok;
    return ok ? n : -2;
}

int32_t osn_tsdf_cuda_extract_mesh_device(OsnTsdfCudaVolume* v, float* d_posnor, uint8_t* d_rgb,
                                          int32_t vert_cap, float min_weight, float iso) {
    if (!usable(v) || !d_posnor || vert_cap <= 0) return -1;
    return v->vol.extract(d_posnor, d_rgb, vert_cap, min_weight, iso, false);
}

int32_t osn_tsdf_cuda_reset(OsnTsdfCudaVolume* v) {
    if (!usable(v)) return 1;
    return v->vol.reset() == cudaSuccess ? 0 : 3;
}

int32_t osn_tsdf_cuda_allocate_counting_cas(OsnTsdfCudaVolume* v, const float* d_positions,
                                            int32_t n_points, float cam_x, float cam_y,
                                            float cam_z, float radius_m) {
    return allocate_mode(v, d_positions, n_points, cam_x, cam_y, cam_z, radius_m,
                         osn_b200::kAllocCountingCas);
}

int32_t osn_tsdf_cuda_allocate_no_cas(OsnTsdfCudaVolume* v, const float* d_positions,
                                      int32_t n_points, float cam_x, float cam_y, float cam_z,
                                      float radius_m) {
    return allocate_mode(v, d_positions, n_points, cam_x, cam_y, cam_z, radius_m,
                         osn_b200::kAllocNoCas);
}

int32_t osn_tsdf_cuda_allocate_slot_index(OsnTsdfCudaVolume* v, const float* d_positions,
                                          int32_t n_points, float cam_x, float cam_y, float cam_z,
                                          float radius_m) {
    return allocate_mode(v, d_positions, n_points, cam_x, cam_y, cam_z, radius_m,
                         osn_b200::kAllocSlotIndex);
}

int32_t osn_tsdf_cuda_allocate_probe_histogram(OsnTsdfCudaVolume* v, const float* d_positions,
                                               int32_t n_points, float cam_x, float cam_y,
                                               float cam_z, float radius_m, uint64_t* hist,
                                               int32_t n_bins) {
    if (!usable(v) || !d_positions || n_points <= 0 || !hist || n_bins <= 0 || n_bins > 64) return 1;
    unsigned long long* d_hist = nullptr;
    cudaStream_t s = v->vol.stream();
    if (cudaMallocAsync(&d_hist, (size_t)n_bins * sizeof(unsigned long long), s) != cudaSuccess)
        return 3;
    cudaMemsetAsync(d_hist, 0, (size_t)n_bins * sizeof(unsigned long long), s);
    const cudaError_t e = v->vol.allocate(batch(d_positions, n_points, cam_x, cam_y, cam_z, radius_m),
                                          osn_b200::kAllocProbeHist, d_hist, n_bins);
    cudaMemcpyAsync(hist, d_hist, (size_t)n_bins * sizeof(unsigned long long),
                    cudaMemcpyDeviceToHost, s);
    cudaFreeAsync(d_hist, s);
    cudaStreamSynchronize(s);
    return e == cudaSuccess ? 0 : 3;
}

int32_t osn_tsdf_cuda_block_count(const OsnTsdfCudaVolume* v) {
    return usable(v) ? const_cast<OsnTsdfCudaVolume*>(v)->vol.block_count() : 0;
}

uint64_t osn_tsdf_cuda_drop_count(const OsnTsdfCudaVolume* v) {
    return usable(v) ? const_cast<OsnTsdfCudaVolume*>(v)->vol.drop_count() : 0;
}

void osn_tsdf_cuda_synchronize(const OsnTsdfCudaVolume* v) {
    if (usable(v)) const_cast<OsnTsdfCudaVolume*>(v)->vol.synchronize();
}

uint32_t osn_tsdf_cuda_status(const OsnTsdfCudaVolume* v) {
    return usable(v) ? const_cast<OsnTsdfCudaVolume*>(v)->vol.status() : 0u;
}

int32_t osn_tsdf_cuda_set_spin_limit(OsnTsdfCudaVolume* v, int32_t iterations) {
    if (!usable(v)) return 1;
    return v->vol.set_spin_limit(iterations) ? 0 : 1;
}

int32_t osn_tsdf_cuda_set_pipelined(OsnTsdfCudaVolume* v, int32_t enabled) {
    if (!usable(v)) return 1;
    if (enabled && v->vol.storage() == osn_b200::kStoreF64) return 2;
    return v->vol.set_pipelined(enabled != 0) ? 0 : 3;
}

int32_t osn_tsdf_cuda_join(OsnTsdfCudaVolume* v) {
    if (!usable(v)) return 1;
    v->vol.join();
    return 0;
}

void* osn_tsdf_cuda_stream(const OsnTsdfCudaVolume* v) {
    return usable(v) ? (void*)v->vol.stream() : nullptr;
}

int32_t osn_tsdf_cuda_last_update_stats(const OsnTsdfCudaVolume* v, int64_t* out4) {
    if (!usable(v) || !out4) return 1;
    return const_cast<OsnTsdfCudaVolume*>(v)->vol.last_update_stats(out4) ? 0 : 3;
}

int32_t osn_tsdf_cuda_set_timing(OsnTsdfCudaVolume* v, int32_t enabled) {
    if (!usable(v)) return 1;
    v->vol.set_timing(enabled != 0);
    return 0;
}

int32_t osn_tsdf_cuda_kernel_times(OsnTsdfCudaVolume* v, double* ms, int64_t* launches,
                                   int32_t n_ids) {
    if (!usable(v) || n_ids <= 0) return 0;
    return v->vol.kernel_times(ms, launches, n_ids);
}

}  // extern "C"
