// Device-side layout and geometry shared by every kernel of the library.
//
// Layout (bit-compatible with the reference, cpp/include/osn_tsdf/types.hpp):
//   - hash slot: 16 bytes {int64 key, int32 block_idx, int32 pad}; key is the
//     packed block coordinate, kEmptyKey (-1) marks a free slot (types.hpp:44-50,
//     :87-91); the 2^20 slots past the live table hold kScratchKey (-2) as in
//     cpp/src/cuda_impl.cuh:84-85;
//   - key = (x+2^20)<<42 | (y+2^20)<<21 | (z+2^20) (types.hpp:64-69);
//   - slot = Teschner multiply-xor hash & mask (types.hpp:150-155);
//   - voxels: five SoA float arrays of weighted sums, 512 per block at
//     block_idx*512, voxel (lx,ly,lz) at (lz*8+ly)*8+lx (volume.cpp:271-276).
//
// The band walk is written with explicit round-to-nearest intrinsics so that
// no multiply-add is contracted: the reference's CPU arm is compiled for
// baseline x86-64 (no FMA) and every sample position, voxel index and signed
// distance here must round exactly as it does there for the allocated block
// set to be bit-identical.
#pragma once

#include <cstdint>
#include <cuda_fp16.h>
#include <cuda_runtime.h>

namespace osn_b200 {

constexpr int kBlockDim = 8;
constexpr int kBlockVoxels = 512;
constexpr long long kEmptyKey = -1;
constexpr long long kScratchKey = -2;
// A slot whose insertion was rolled back because the pool was full. Lookups
// probe past it (unlike an empty slot), so a block inserted further along the
// probe sequence while the rollback was in flight stays reachable.
constexpr long long kReleasedKey = -3;
constexpr long long kNoKey = -4;  // "no request" marker inside warps; never stored
constexpr long long kCoordBias = 1LL << 20;
constexpr int kCoordBits = 21;
constexpr uint32_t kScratchSlots = 1u << 20;
// Default bound on every device-side wait (iterations of ~100 ns): far above
// any legitimate publication delay, far below a watchdog. A volume may lower
// its own bound (osn_tsdf_cuda_set_spin_limit), e.g. so a test can make a
// wait run out quickly.
constexpr int kSpinLimit = 1 << 20;

// Bits of the device status word.
constexpr uint32_t kStatusSpinTimeout = 1u;
constexpr uint32_t kStatusScratchOverflow = 2u;

// Voxel storage modes (OSN_TSDF_STORAGE_* in include/osn_tsdf_b200.h).
//   kStoreF32     the reference's layout: float weighted sums tsdf, weight,
//                 r, g, b (20 bytes per voxel).
//   kStoreF16U16  the mean normalised TSDF as FP16 and the weight as uint16
//                 (4 bytes per voxel); the running average is formed in FP32
//                 from the stored mean and the batch's exact sums. No colour
//                 arrays: through the C ABI every contribution is grey (128),
//                 so a voxel's mean colour is 128 wherever its weight is set.
//   kStoreF64     the FP64 oracle: double TSDF sums computed from SDFs
//                 evaluated in double at the same band samples, float weights
//                 (integers, exact). No colour arrays.
enum Storage : int { kStoreF32 = 0, kStoreF16U16 = 1, kStoreF64 = 2 };

// Table layouts (OSN_TSDF_LAYOUT_* in include/osn_tsdf_b200.h).
enum Layout : int { kLayoutPool = 0, kLayoutSlotIndex = 1 };

// The largest weight a uint16 voxel holds; the effective cap of kStoreF16U16.
constexpr float kU16WeightMax = 65535.0f;

struct HashEntry {
    long long key;
    int32_t block_idx;
    int32_t pad;
};
static_assert(sizeof(HashEntry) == 16, "hash slot must stay 16 bytes");

struct BlockCoord {
    int32_t x, y, z;
};

// Everything a kernel needs to address one volume.
struct DevVolume {
    HashEntry* table;
    uint32_t hash_mask;
    int32_t pool_capacity;
    int32_t* block_count;
    unsigned long long* drop_count;
    BlockCoord* block_coord;
    float* tsdf;
    float* weight;
    float* r;
    float* g;
    float* b;
    float voxel_size;
    float inv_voxel;  // 1.0f / voxel_size, computed on the host (volume.cpp:148)
    float trunc;
    float inv_trunc;  // 1.0f / trunc (volume.cpp:203)
    float weight_cap;  // effective cap: <= 0 disables (FP32/FP64); at most 65535 for uint16 weights
    int32_t steps;    // max(1, ceil(trunc * inv_voxel)) (volume.cpp:171)
    uint32_t* status;
    int32_t storage;     // Storage
    int32_t spin_limit;  // iterations a publication wait may take (kSpinLimit by default)
    int32_t* block_chunk;  // per pool block: chunk id of the last call that allocated or updated it
    int32_t chunk;         // chunk id of the current call
    // Slot-index layout (opt-in): the pool is the table, a block's pool index
    // is its table slot, so a key found in the table needs no wait for its
    // index (cpp/src/volume_cuda.cu:194-244).
    int32_t slot_index;
};

// Bytes per voxel of the tsdf and weight arrays of a storage mode.
__host__ __device__ constexpr int tsdf_bytes(int storage) {
    return storage == kStoreF16U16 ? 2 : storage == kStoreF64 ? 8 : 4;
}
__host__ __device__ constexpr int weight_bytes(int storage) { return storage == kStoreF16U16 ? 2 : 4; }

// Weight of voxel i (read-only path: kernels that run after the volume's
// weights were last written).
template <int S>
__device__ __forceinline__ float weight_at(const DevVolume& v, size_t i) {
    if constexpr (S == kStoreF16U16)
        return (float)__ldg(reinterpret_cast<const unsigned short*>(v.weight) + i);
    else
        return __ldg(v.weight + i);
}

// Mean normalised TSDF of voxel i given its weight w (sum * (1/w) for FP32
// sums, marching_tets.cpp), the stored value loaded whatever the weight so
// that a caller's weight and value loads are in flight together; meaningful
// only for w > 0.
template <int S>
__device__ __forceinline__ float mean_from(const DevVolume& v, size_t i, float w) {
    if constexpr (S == kStoreF16U16) {
        return __half2float(__ldg(reinterpret_cast<const __half*>(v.tsdf) + i));
    } else if constexpr (S == kStoreF64) {
        const double d = __ldg(reinterpret_cast<const double*>(v.tsdf) + i);
        return w > 0.0f ? (float)(d / (double)w) : 0.0f;
    } else {
        const float t = __ldg(v.tsdf + i);
        return w > 0.0f ? __fmul_rn(t, __fdiv_rn(1.0f, w)) : 0.0f;
    }
}

// A depth image as the point source of a batch: pixel i = v * width + u
// with depth z (metres along the optical axis) becomes the world point
// R [ (u - cx) z / fx, (v - cy) z / fy, z ] + t, evaluated in FP64 and
// rounded to float (crates/tartanair/src/lib.rs:307-340); pixels with a
// non-finite, non-positive or out-of-range depth have no point.
struct DepthSource {
    const float* depth;  // [height * width], device
    int32_t width;
    float max_range;     // <= 0: no limit
    double fx, fy, cx, cy;
    double R[9];         // camera-to-world rotation, row-major
    double t[3];         // camera origin in world
};

// One batch: camera origin and squared far cutoff (0 disables). Points come
// from pos (3 floats each) or, when depth.depth is set, from a depth image
// (n = width * height pixels, in raster order).
struct BatchArgs {
    const float* pos;
    int32_t n;
    float cam_x, cam_y, cam_z;
    float radius_sq;
    DepthSource depth;
};

// Pixel p of a depth image (depth value at index i of the batch's depth
// array) unprojected with the camera-to-world pose (R, t) in FP64, rounded to
// float; false for an invalid pixel (non-finite, <= 0 or beyond max_range).
__device__ __forceinline__ bool unproject_pixel(const DepthSource& d, const double* R, const double* t,
                                                int i, int p, float& px, float& py, float& pz) {
    const float z = d.depth[i];
    px = py = pz = 0.0f;
    if (!isfinite(z) || !(z > 0.0f) || (d.max_range > 0.0f && z > d.max_range)) return false;
    const int v = p / d.width, u = p - v * d.width;
    const double zd = (double)z;
    const double x = __ddiv_rn(__dmul_rn(__dsub_rn((double)u, d.cx), zd), d.fx);
    const double y = __ddiv_rn(__dmul_rn(__dsub_rn((double)v, d.cy), zd), d.fy);
    float w[3];
#pragma unroll
    for (int k = 0; k < 3; ++k)
        w[k] = __double2float_rn(__dadd_rn(
            __dadd_rn(__dadd_rn(__dmul_rn(R[3 * k], x), __dmul_rn(R[3 * k + 1], y)), __dmul_rn(R[3 * k + 2], zd)),
            t[k]));
    px = w[0];
    py = w[1];
    pz = w[2];
    return true;
}

// Point i of a batch; false when it has none (an invalid depth pixel).
// SOURCE: 0 = xyz positions, 1 = depth image, -1 = whichever the batch has.
template <int SOURCE = -1>
__device__ __forceinline__ bool load_point(const BatchArgs& a, int i, float& px, float& py, float& pz) {
    if (SOURCE == 0 || (SOURCE < 0 && a.depth.depth == nullptr)) {
        px = a.pos[(size_t)i * 3 + 0];
        py = a.pos[(size_t)i * 3 + 1];
        pz = a.pos[(size_t)i * 3 + 2];
        return true;
    }
    return unproject_pixel(a.depth, a.depth.R, a.depth.t, i, i, px, py, pz);
}

__device__ __forceinline__ long long pack_key(int32_t x, int32_t y, int32_t z) {
    return (((long long)x + kCoordBias) << (2 * kCoordBits)) |
           (((long long)y + kCoordBias) << kCoordBits) | ((long long)z + kCoordBias);
}

__device__ __forceinline__ uint32_t hash_slot(int32_t x, int32_t y, int32_t z, uint32_t mask) {
    return ((uint32_t)x * 73856093u ^ (uint32_t)y * 19349663u ^ (uint32_t)z * 83492791u) & mask;
}

__device__ __forceinline__ int32_t unpack_axis(long long key, int shift) {
    return (int32_t)((key >> shift) & ((1LL << kCoordBits) - 1)) - (int32_t)kCoordBias;
}

// ---- coherent memory helpers (the table is mutated by other SMs) ----------

__device__ __forceinline__ long long ld_relaxed_s64(const long long* p) {
    long long v;
    asm volatile("ld.relaxed.gpu.global.s64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ int ld_acquire_s32(const int* p) {
    int v;
    asm volatile("ld.acquire.gpu.global.s32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ int ld_relaxed_s32(const int* p) {
    int v;
    asm volatile("ld.relaxed.gpu.global.s32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

// ---- the band walk (volume.cpp:153-196 and :208-296) ----------------------

struct Ray {
    float px, py, pz;
    float ux, uy, uz;
    float dist;
    float cx, cy, cz;  // the camera origin of the point's frame
};

// Point set-up for a point already loaded into (px, py, pz), seen from the
// camera at (cx, cy, cz). False when the point is gated out by the far cutoff
// or sits on the camera (volume.cpp:158-166).
__device__ __forceinline__ bool ray_setup_cam(float radius_sq, float cx, float cy, float cz, float px,
                                              float py, float pz, Ray& r) {
    r.px = px;
    r.py = py;
    r.pz = pz;
    r.cx = cx;
    r.cy = cy;
    r.cz = cz;
    const float dx = __fsub_rn(r.px, cx);
    const float dy = __fsub_rn(r.py, cy);
    const float dz = __fsub_rn(r.pz, cz);
    const float d2 = __fadd_rn(__fadd_rn(__fmul_rn(dx, dx), __fmul_rn(dy, dy)), __fmul_rn(dz, dz));
    if (radius_sq > 0.0f && d2 > radius_sq) return false;
    r.dist = __fsqrt_rn(d2);
    if (!(r.dist > 1e-6f)) return false;
    r.ux = __fdiv_rn(dx, r.dist);
    r.uy = __fdiv_rn(dy, r.dist);
    r.uz = __fdiv_rn(dz, r.dist);
    return true;
}

// The same for a batch with one camera.
__device__ __forceinline__ bool ray_setup_at(const BatchArgs& a, float px, float py, float pz, Ray& r) {
    return ray_setup_cam(a.radius_sq, a.cam_x, a.cam_y, a.cam_z, px, py, pz, r);
}

__device__ __forceinline__ bool ray_setup(const BatchArgs& a, int i, Ray& r) {
    float px, py, pz;
    if (!load_point(a, i, px, py, pz)) return false;
    return ray_setup_at(a, px, py, pz, r);
}

// Band sample s in [-steps, steps]: voxel index and signed distance at the
// voxel CENTRE. False when the voxel is fully occluded (sdf < -trunc), the
// gate both passes apply (volume.cpp:185-191, :260-268).
__device__ __forceinline__ bool band_sample_from(const DevVolume& v, const Ray& r, float cx, float cy,
                                                 float cz, int s, int& vx, int& vy, int& vz, float& sdf) {
    const float t = __fmul_rn((float)s, v.voxel_size);
    vx = (int)floorf(__fmul_rn(__fadd_rn(r.px, __fmul_rn(r.ux, t)), v.inv_voxel));
    vy = (int)floorf(__fmul_rn(__fadd_rn(r.py, __fmul_rn(r.uy, t)), v.inv_voxel));
    vz = (int)floorf(__fmul_rn(__fadd_rn(r.pz, __fmul_rn(r.uz, t)), v.inv_voxel));
    const float ex = __fsub_rn(__fmul_rn(__fadd_rn((float)vx, 0.5f), v.voxel_size), cx);
    const float ey = __fsub_rn(__fmul_rn(__fadd_rn((float)vy, 0.5f), v.voxel_size), cy);
    const float ez = __fsub_rn(__fmul_rn(__fadd_rn((float)vz, 0.5f), v.voxel_size), cz);
    const float dv =
        __fsqrt_rn(__fadd_rn(__fadd_rn(__fmul_rn(ex, ex), __fmul_rn(ey, ey)), __fmul_rn(ez, ez)));
    sdf = __fsub_rn(r.dist, dv);
    return !(sdf < -v.trunc);
}

// A batch with one camera (read from the batch's arguments).
__device__ __forceinline__ bool band_sample(const DevVolume& v, const BatchArgs& a, const Ray& r,
                                            int s, int& vx, int& vy, int& vz, float& sdf) {
    return band_sample_from(v, r, a.cam_x, a.cam_y, a.cam_z, s, vx, vy, vz, sdf);
}

// A batch of several frames: the camera of the point's frame, kept in the ray.
__device__ __forceinline__ bool band_sample_ray(const DevVolume& v, const Ray& r, int s, int& vx,
                                                int& vy, int& vz, float& sdf) {
    return band_sample_from(v, r, r.cx, r.cy, r.cz, s, vx, vy, vz, sdf);
}

// The FP64 oracle's signed distance of the same band sample: the point's
// distance and the voxel centre's distance evaluated in double.
__device__ __forceinline__ double sdf_f64(const DevVolume& v, const BatchArgs& a, float px, float py,
                                          float pz, int vx, int vy, int vz) {
    const double dx = (double)px - (double)a.cam_x;
    const double dy = (double)py - (double)a.cam_y;
    const double dz = (double)pz - (double)a.cam_z;
    const double vs = (double)v.voxel_size;
    const double ex = ((double)vx + 0.5) * vs - (double)a.cam_x;
    const double ey = ((double)vy + 0.5) * vs - (double)a.cam_y;
    const double ez = ((double)vz + 0.5) * vs - (double)a.cam_z;
    return sqrt(dx * dx + dy * dy + dz * dz) - sqrt(ex * ex + ey * ey + ez * ez);
}

__device__ __forceinline__ double clamp_sdf_n_f64(double sdf, float trunc) {
    return fmin(fmax(sdf / (double)trunc, -1.0), 1.0);
}

// ---- lookups after allocation has completed --------------------------------

// Block index of a key, or -1 (volume.cpp:71-92). Only valid in kernels that
// run after the allocating kernel finished, so every index is published and
// the non-coherent 128-bit load of a whole slot is safe.
__device__ __forceinline__ int32_t find_block(const DevVolume& v, int32_t bx, int32_t by, int32_t bz,
                                              long long want) {
    const uint32_t size = v.hash_mask + 1;
    const uint32_t start = hash_slot(bx, by, bz, v.hash_mask);
    for (uint32_t p = 0; p < size; ++p) {
        const int4 raw = __ldg(reinterpret_cast<const int4*>(&v.table[(start + p) & v.hash_mask]));
        const long long key = ((long long)(unsigned)raw.y << 32) | (unsigned)raw.x;
        if (key == want) return (raw.z >= 0 && raw.z < v.pool_capacity) ? raw.z : -1;
        if (key == kEmptyKey) return -1;
    }
    return -1;
}

// ---- insertion (volume.cpp:94-145, volume_cuda.cu:59-107) -------------------

// Allocation modes: the production insert and the reference's measurement
// variants (cpp/include/osn_tsdf/c_api.h:108-122), plus a probe histogram.
enum AllocMode : int {
    kAllocInsert = 0,       // production
    kAllocCountingCas = 1,  // measurement: count CAS attempts into drop_count
    kAllocNoCas = 2,        // measurement: probe, never insert
    kAllocProbeHist = 3,    // measurement: insert and histogram probe depths
    kAllocSlotIndex = 4,    // measurement: block index = slot
    kLookupOnly = 5,        // no insertion: find_block (update after allocation)
};

struct InsertResult {
    int32_t idx;      // >= 0 allocated or found, -1 dropped / absent
    uint32_t probes;  // slots visited
};

// Wait, with an iteration bound, until a claimed slot's index is published
// or its claim is rolled back (pool full). A timeout sets a status bit.
__device__ __forceinline__ int32_t wait_published(const DevVolume& v, HashEntry* e, long long want) {
    for (int it = 0; it < v.spin_limit; ++it) {
        const int idx = ld_acquire_s32(&e->block_idx);
        if (idx >= 0) return idx;
        if (ld_relaxed_s64(&e->key) != want) return -1;
        __nanosleep(64);
    }
    atomicOr(v.status, kStatusSpinTimeout);
    return -1;
}

// Find or insert one block: CAS the key into the first empty slot of its
// linear probe sequence, take a pool index from the counter, write the
// coordinate, fence, publish the index (volume_cuda.cu:82-95). When the pool
// is already full no slot is claimed; a claim that overflows the pool is
// rolled back to kReleasedKey.
//
// In the slot-index layout (and the slot-index measurement mode) the block's
// index is its slot: a claim publishes it at once (coordinate, count, fence,
// index) and a thread that finds the key returns the slot without waiting.
template <int MODE>
__device__ __forceinline__ InsertResult find_or_insert(const DevVolume& v, int32_t bx, int32_t by,
                                                       int32_t bz, long long want) {
    InsertResult res{-1, 0};
    const bool by_slot = MODE == kAllocSlotIndex || (MODE == kAllocInsert && v.slot_index);
    // The measurement mode uses the first pool_capacity slots as the table;
    // the layout's pool is the whole table.
    const uint32_t mask = (MODE == kAllocSlotIndex) ? (uint32_t)v.pool_capacity - 1u : v.hash_mask;
    const uint32_t size = mask + 1;
    const uint32_t start = hash_slot(bx, by, bz, mask);
    for (uint32_t p = 0; p < size; ++p) {
        const uint32_t slot = (start + p) & mask;
        HashEntry* e = &v.table[slot];
        ++res.probes;
        const long long key = ld_relaxed_s64(&e->key);
        if (key == want) {
            if (MODE == kAllocNoCas) { res.idx = 0; return res; }
            if (by_slot) { res.idx = (int32_t)slot; return res; }
            res.idx = wait_published(v, e, want);
            return res;
        }
        if (key == kEmptyKey) {
            if (MODE == kAllocNoCas) return res;
            if (!by_slot && ld_acquire_s32(v.block_count) >= v.pool_capacity) {
                // The pool is full, so no claim can succeed any more -- but the
                // claim that filled it may have been this very key, made after
                // we read the slot. Claimers fence between their CAS and their
                // counter increment, so having seen the full count we see
                // their key if it is there.
                const long long again = ld_relaxed_s64(&e->key);
                if (again == want) {
                    res.idx = wait_published(v, e, want);
                    return res;
                }
                if (again == kEmptyKey) return res;  // absent, and cannot be inserted
                continue;                            // another key took the slot: probe on
            }
            if (MODE == kAllocCountingCas) atomicAdd(v.drop_count, 1ULL);
            const long long prev = (long long)atomicCAS((unsigned long long*)&e->key,
                                                        (unsigned long long)kEmptyKey,
                                                        (unsigned long long)want);
            if (prev == kEmptyKey) {
                if (by_slot) {
                    v.block_coord[slot] = BlockCoord{bx, by, bz};
                    if (v.block_chunk) v.block_chunk[slot] = v.chunk;
                    atomicAdd(v.block_count, 1);
                    __threadfence();
                    atomicExch(&e->block_idx, (int)slot);
                    res.idx = (int32_t)slot;
                    return res;
                }
                __threadfence();  // the claim is visible before the count that reflects it
                const int32_t idx = atomicAdd(v.block_count, 1);
                if (idx >= v.pool_capacity) {
                    atomicSub(v.block_count, 1);
                    atomicExch((unsigned long long*)&e->key, (unsigned long long)kReleasedKey);
                    return res;
                }
                v.block_coord[idx] = BlockCoord{bx, by, bz};
                if (v.block_chunk) v.block_chunk[idx] = v.chunk;
                __threadfence();  // coordinate visible before the index
                atomicExch(&e->block_idx, idx);
                res.idx = idx;
                return res;
            }
            if (prev == want) {
                if (by_slot) { res.idx = (int32_t)slot; return res; }
                res.idx = wait_published(v, e, want);
                return res;
            }
        }
        // Another key, a rolled-back slot or a scratch sentinel: probe on.
    }
    return res;  // table full
}

// ---- fixed-point sums ----------------------------------------------------
//
// Per-voxel sums of normalised SDFs are accumulated as 64-bit integers in
// units of 2^-40 (exact for |value| >= 2^-17, |sum| < 2^23) and added to the
// stored float sum with one rounding, so a sum does not depend on the order
// of its terms.
constexpr double kFixScale = 1099511627776.0;      // 2^40
constexpr double kFixInv = 1.0 / 1099511627776.0;  // 2^-40

// x * 2^40 is exact in float (a power-of-two scale of |x| <= 1), so rounding
// it to an integer in float gives the same value as in double.
__device__ __forceinline__ long long to_fix(float x) { return __float2ll_rn(x * 1099511627776.0f); }
__device__ __forceinline__ long long to_fix(double x) { return __double2ll_rn(x * kFixScale); }

__device__ __forceinline__ float add_fix(float t0, long long sum) {
    return __double2float_rn((double)t0 + (double)sum * kFixInv);
}

// Programmatic dependent launch. A kernel launched with programmatic stream
// serialisation may start before its predecessor on the stream has finished;
// it waits here, before reading anything the predecessor wrote, until that
// grid has completed and its writes are visible. Each kernel lets its own
// dependents launch as soon as all of its CTAs are running, so their launch
// overlaps its execution. Both are no-ops for kernels launched without the
// attribute.
__device__ __forceinline__ void grid_dependency_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void launch_dependents() { asm volatile("griddepcontrol.launch_dependents;"); }

__device__ __forceinline__ unsigned lanemask_lt() {
    unsigned m;
    asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
    return m;
}

}  // namespace osn_b200
