// Update, second half: turn the band walk's per-voxel counts and sums into
// the voxels' new tsdf, weight and colour sums.
//
// Reference: cpp/src/volume.cpp:282-295 and cpp/src/volume_cuda.cu:325-335
// (per sample: cap check, then atomic adds of weight, w*sdf and w*colour).
//
// Semantics. The reference's cap check is a plain read before the adds, so
// which contributions a capped voxel accepts depends on thread timing. This
// library implements the one order-independent reading of it: contributions
// are applied as if in (point index, band step) order, and a contribution is
// accepted while the voxel's weight before it is below the cap. That is what
// the reference's CPU arm computes with one thread, the parity oracle.
// Through the reference's CUDA ABI every contribution has weight 1 and grey
// colour 128, so a voxel with weight w0 before the batch and n records
// accepts the first keep = min(n, ceil(cap - w0)) of them, and its colour
// sums stay exactly 128 * weight (every term is an integer times a power of
// two), so they are written, never read.
//
// The band walk (band_kernels.cu) has left, per voxel, the batch count n and
// the fixed-point sum of the records' normalised SDFs, the list of touched
// blocks, and one record per band slot.
//
//   finish     one 128-thread CTA per touched block, 4 voxels per thread,
//              every array read and written as 128-bit vectors: a voxel that
//              accepts all of its records (keep == n, the common case) gets
//              tsdf + sum, w0 + n, 128 * (w0 + n) and its count and sum back
//              to zero. A voxel that crosses the cap inside the batch
//              reserves a group of n deferred records instead and its block
//              is tagged.
//              Crossing voxels go to one of two lists: small groups (at most
//              kLaneRecords records, most of them) and large ones.
//   group      one pass over the records of the batch, eight per thread: a
//              record of a tagged block whose voxel reserved a group takes
//              the next place of the group (a few percent of the records).
//   values     (FP64 oracle only) one thread per grouped record: its
//              canonical id and its normalised SDF recomputed in double from
//              its point. FP32 / FP16 records carry their band slot, from
//              which deferred reads the id and the value the walk kept.
//   deferred   selects the keep records with the smallest ids of every
//              crossing voxel and finishes it: one half-warp per small group
//              (one record per lane, shuffle ranking), one warp per large group
//              (register ranking up to 256 records, a radix select of the
//              keep-th id beyond that).
//
// Sums are 64-bit fixed point added to the stored sum with one rounding, so
// results do not depend on the order in which threads meet the records:
// repeated runs are bit-identical, and a voxel with one contribution per
// batch gets exactly the reference's fl(tsdf + sdf_n).
#include <mutex>

#include "volume.h"

namespace osn_b200 {
namespace {

constexpr int kFinishThreads = 128;  // 4 voxels per thread, one block per CTA pass
constexpr int kGroupThreads = 256;
constexpr int kDeferThreads = 128;
constexpr int kDeferWarps = kDeferThreads / 32;
constexpr int kRankRegs = 8;
static_assert(kFinishThreads >= kMaxBatchScenes && kGroupThreads >= kMaxBatchScenes &&
                  kDeferThreads >= kMaxBatchScenes,
              "one thread per scene builds the item prefix");  // crossing voxels of up to 256 records are ranked in registers

// Contributions a voxel accepts given its weight w0 before the batch and n
// unit-weight records: the j-th record (0-based, canonical order) is accepted
// iff w0 + j < cap (volume.cpp:289); all values are integers, exact in float.
__device__ __forceinline__ int accept_count(float w0, float cap, int n) {
    if (n == 0) return 0;
    if (!(cap > 0.0f)) return n;
    if (w0 >= cap) return 0;
    const double room = ceil((double)cap - (double)w0);
    return room >= (double)n ? n : (int)room;
}

// ---- finish ----------------------------------------------------------------

// Four consecutive voxels of one storage mode, as registers.
template <int S>
struct Quad {
    float w[4];  // weights
    float t[4];  // FP32: tsdf sums; FP16U16: means
    double d[4]; // FP64: tsdf sums
};

template <int S>
__device__ __forceinline__ void load_quad(const DevVolume& v, size_t q4, Quad<S>& x) {
    if constexpr (S == kStoreF32) {
        const float4 w4 = reinterpret_cast<const float4*>(v.weight)[q4];
        const float4 t4 = reinterpret_cast<const float4*>(v.tsdf)[q4];
        x.w[0] = w4.x; x.w[1] = w4.y; x.w[2] = w4.z; x.w[3] = w4.w;
        x.t[0] = t4.x; x.t[1] = t4.y; x.t[2] = t4.z; x.t[3] = t4.w;
    } else if constexpr (S == kStoreF16U16) {
        const ushort4 w4 = reinterpret_cast<const ushort4*>(v.weight)[q4];
        const uint2 h = reinterpret_cast<const uint2*>(v.tsdf)[q4];
        const __half2 h01 = *reinterpret_cast<const __half2*>(&h.x);
        const __half2 h23 = *reinterpret_cast<const __half2*>(&h.y);
        x.w[0] = (float)w4.x; x.w[1] = (float)w4.y; x.w[2] = (float)w4.z; x.w[3] = (float)w4.w;
        x.t[0] = __low2float(h01); x.t[1] = __high2float(h01);
        x.t[2] = __low2float(h23); x.t[3] = __high2float(h23);
    } else {
        const float4 w4 = reinterpret_cast<const float4*>(v.weight)[q4];
        const double2 d01 = reinterpret_cast<const double2*>(v.tsdf)[2 * q4];
        const double2 d23 = reinterpret_cast<const double2*>(v.tsdf)[2 * q4 + 1];
        x.w[0] = w4.x; x.w[1] = w4.y; x.w[2] = w4.z; x.w[3] = w4.w;
        x.d[0] = d01.x; x.d[1] = d01.y; x.d[2] = d23.x; x.d[3] = d23.y;
    }
}

template <int S>
__device__ __forceinline__ void store_quad(const DevVolume& v, size_t q4, const Quad<S>& x) {
    if constexpr (S == kStoreF32) {
        reinterpret_cast<float4*>(v.tsdf)[q4] = make_float4(x.t[0], x.t[1], x.t[2], x.t[3]);
        reinterpret_cast<float4*>(v.weight)[q4] = make_float4(x.w[0], x.w[1], x.w[2], x.w[3]);
        const float4 c = make_float4(__fmul_rn(128.0f, x.w[0]), __fmul_rn(128.0f, x.w[1]),
                                     __fmul_rn(128.0f, x.w[2]), __fmul_rn(128.0f, x.w[3]));
        __stcs(reinterpret_cast<float4*>(v.r) + q4, c);  // write-only: keep them out of L2
        __stcs(reinterpret_cast<float4*>(v.g) + q4, c);
        __stcs(reinterpret_cast<float4*>(v.b) + q4, c);
    } else if constexpr (S == kStoreF16U16) {
        const __half2 h01 = __floats2half2_rn(x.t[0], x.t[1]);
        const __half2 h23 = __floats2half2_rn(x.t[2], x.t[3]);
        uint2 h;
        h.x = *reinterpret_cast<const unsigned*>(&h01);
        h.y = *reinterpret_cast<const unsigned*>(&h23);
        reinterpret_cast<uint2*>(v.tsdf)[q4] = h;
        reinterpret_cast<ushort4*>(v.weight)[q4] =
            make_ushort4((unsigned short)x.w[0], (unsigned short)x.w[1], (unsigned short)x.w[2],
                         (unsigned short)x.w[3]);
    } else {
        reinterpret_cast<double2*>(v.tsdf)[2 * q4] = make_double2(x.d[0], x.d[1]);
        reinterpret_cast<double2*>(v.tsdf)[2 * q4 + 1] = make_double2(x.d[2], x.d[3]);
        reinterpret_cast<float4*>(v.weight)[q4] = make_float4(x.w[0], x.w[1], x.w[2], x.w[3]);
    }
}

// New stored TSDF of a voxel with weight w0 before the batch that accepts
// keep contributions whose normalised SDFs sum to fix * 2^-40.
//   FP32: the sum gets the batch sum added with one rounding;
//   FP16U16: the mean, (mean * w0 + sum) / (w0 + keep) in FP32, rounded to FP16
//            (the caller rounds);
//   FP64: the double sum.
__device__ __forceinline__ float new_mean_f16(float mean0, float w0, int keep, long long fix) {
    const float sum = __fadd_rn(__fmul_rn(mean0, w0), (float)((double)fix * kFixInv));
    return __fdiv_rn(sum, __fadd_rn(w0, (float)keep));
}

template <int S>
__device__ __forceinline__ void apply_voxel(Quad<S>& x, int q, int keep, long long fix) {
    if constexpr (S == kStoreF32) {
        x.t[q] = add_fix(x.t[q], fix);
    } else if constexpr (S == kStoreF16U16) {
        x.t[q] = new_mean_f16(x.t[q], x.w[q], keep, fix);
    } else {
        x.d[q] = x.d[q] + (double)fix * kFixInv;
    }
    x.w[q] = __fadd_rn(x.w[q], (float)keep);
}

// Per-CTA sum of a per-thread statistic, one global atomic per CTA (the
// control counters share a line: per-warp atomics would serialise there).
__device__ __forceinline__ void cta_add(int* smem_acc, int mine, int* global) {
    const int w = __reduce_add_sync(0xffffffffu, mine);
    if ((threadIdx.x & 31) == 0 && w) atomicAdd(smem_acc, w);
    __syncthreads();
    if (threadIdx.x == 0 && *smem_acc) atomicAdd(global, *smem_acc);
}

// One touched block's quad of voxels, its arrays already loaded: finish
// the voxels that accept all their records, reserve groups for those that
// cross the cap. Warp-synchronous (all lanes of the warp call it).
template <int S>
__device__ __forceinline__ void finish_quad(const DevVolume& v, const UpdateScratch& u, int32_t bi,
                                            size_t q4, int t, int lane, const uint4 c4, Quad<S>& x,
                                            const ulonglong2 a01, const ulonglong2 a23, int& updated) {
    const bool any = (c4.x | c4.y | c4.z | c4.w) != 0u;
    if (!__any_sync(0xffffffffu, any)) return;  // warp-uniform skip
    const uint32_t n[4] = {c4.x, c4.y, c4.z, c4.w};
    unsigned long long acc[4] = {a01.x, a01.y, a23.x, a23.y};
    uint32_t cnt[4] = {0u, 0u, 0u, 0u};
    int keepv[4] = {0, 0, 0, 0};
    // Voxels crossing the cap reserve a group of their n records and an
    // entry in the small (n <= kLaneRecords) or large list; the warp's
    // reservations are summed and made with one atomic per counter.
    uint32_t my_records = 0u;
    uint32_t my_small = 0u, my_large = 0u;
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        if (n[q] == 0u) continue;
        keepv[q] = accept_count(x.w[q], v.weight_cap, (int)n[q]);
        if (keepv[q] != 0 && (uint32_t)keepv[q] != n[q]) {
            my_records += n[q];
            if (n[q] <= (uint32_t)kLaneRecords) ++my_small;
            else ++my_large;
        }
    }
    const unsigned crossers = __ballot_sync(0xffffffffu, my_records > 0u);
    uint32_t rec_base = 0u, small_at = 0u, large_at = 0u;
    bool lists_ok = true;
    if (crossers) {
        uint32_t rec_incl = my_records, s_incl = my_small, l_incl = my_large;
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t ry = __shfl_up_sync(0xffffffffu, rec_incl, o);
            const uint32_t sy = __shfl_up_sync(0xffffffffu, s_incl, o);
            const uint32_t ly = __shfl_up_sync(0xffffffffu, l_incl, o);
            if (lane >= o) {
                rec_incl += ry;
                s_incl += sy;
                l_incl += ly;
            }
        }
        uint32_t rb = 0u;
        unsigned long long lb = 0ull;
        if (lane == 31) {
            rb = atomicAdd(&u.ctl->x_used, rec_incl);
            lb = atomicAdd(&u.ctl->def_lists, (unsigned long long)s_incl |
                                                  ((unsigned long long)l_incl << 32));
        }
        rb = __shfl_sync(0xffffffffu, rb, 31);
        lb = __shfl_sync(0xffffffffu, lb, 31);
        const uint32_t s_tot = __shfl_sync(0xffffffffu, s_incl, 31);
        const uint32_t l_tot = __shfl_sync(0xffffffffu, l_incl, 31);
        rec_base = rb + rec_incl - my_records;
        const uint64_t s0 = lb & 0xFFFFFFFFull, l0 = lb >> 32;
        small_at = (uint32_t)s0 + s_incl - my_small;
        large_at = (uint32_t)l0 + l_incl - my_large;
        // The lists grow towards each other: entries written under a
        // reservation that fits never overlap later ones.
        lists_ok = s0 + s_tot + l0 + l_tot <= (uint64_t)u.dvox_cap;
    }
    if (!any) return;  // no warp-synchronous step follows
    bool crossing = false;
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        if (n[q] == 0u) continue;
        if ((uint32_t)keepv[q] == n[q] || keepv[q] == 0) {
            // All accepted (or none: the voxel was full before the batch).
            if (keepv[q]) {
                apply_voxel<S>(x, q, keepv[q], (long long)acc[q]);
                ++updated;
            }
            acc[q] = 0ull;
        } else {
            // Crosses the cap: its group is filled by the group pass and
            // the voxel finished by the deferred kernel.
            const uint32_t vi = (uint32_t)bi * kBlockVoxels + 4u * t + q;
            const bool small = n[q] <= (uint32_t)kLaneRecords;
            const int entry = small ? (int)small_at : u.dvox_cap - 1 - (int)large_at;
            if ((uint64_t)rec_base + n[q] <= (uint64_t)u.record_cap && lists_ok) {
                u.dvox[entry] = make_int4((int)vi, (int)rec_base, (int)n[q], keepv[q]);
                acc[q] = (unsigned long long)(rec_base + 1u) << 32;  // low half: fill ticket
                cnt[q] = n[q];
            } else {
                // Out of scratch (the status word says so): a reserved
                // list entry still gets an empty group, never a stale one.
                if (lists_ok) u.dvox[entry] = make_int4((int)vi, 0, 0, 0);
                atomicOr(v.status, kStatusScratchOverflow);
                acc[q] = 0ull;
            }
            rec_base += n[q];
            if (small) ++small_at;
            else ++large_at;
            crossing = true;
        }
    }
    if (crossing) u.blk_cross[bi] = u.tag;
    store_quad<S>(v, q4, x);
    reinterpret_cast<uint4*>(u.vcnt)[q4] = make_uint4(cnt[0], cnt[1], cnt[2], cnt[3]);
    reinterpret_cast<ulonglong2*>(u.vacc)[2 * q4] = make_ulonglong2(acc[0], acc[1]);
    reinterpret_cast<ulonglong2*>(u.vacc)[2 * q4 + 1] = make_ulonglong2(acc[2], acc[3]);
}

template <int S>
__device__ __forceinline__ void load_item(const DevVolume& v, const UpdateScratch& u, size_t q4,
                                          uint4& c4, Quad<S>& x, ulonglong2& a01, ulonglong2& a23) {
    c4 = reinterpret_cast<const uint4*>(u.vcnt)[q4];
    load_quad<S>(v, q4, x);
    a01 = reinterpret_cast<const ulonglong2*>(u.vacc)[2 * q4];
    a23 = reinterpret_cast<const ulonglong2*>(u.vacc)[2 * q4 + 1];
}

// Two touched blocks per CTA iteration: the indices of both, then every
// array of both, are in flight together (each CTA pass is two dependent
// round trips, whatever the number of blocks it covers).
template <int S>
__global__ void __launch_bounds__(kFinishThreads)
finish_kernel(DevVolume v, UpdateScratch u) {
    __shared__ int s_updated;
    const int t = threadIdx.x, lane = t & 31;
    if (t == 0) s_updated = 0;
    __syncthreads();
    launch_dependents();
    grid_dependency_wait();
    const int n_touched = min(u.ctl->n_touched, v.pool_capacity);
    int updated = 0;
    for (int ia = blockIdx.x; ia < n_touched; ia += 2 * gridDim.x) {
        const int ib = ia + gridDim.x;
        const bool has_b = ib < n_touched;  // uniform across the CTA
        const int32_t ba = u.touched[ia];
        const int32_t bb = has_b ? u.touched[ib] : ba;
        const size_t qa = (size_t)ba * (kBlockVoxels / 4) + t;  // this thread's 4 voxels
        const size_t qb = (size_t)bb * (kBlockVoxels / 4) + t;
        uint4 ca, cb;
        Quad<S> xa, xb;
        ulonglong2 a01, a23, b01, b23;
        load_item<S>(v, u, qa, ca, xa, a01, a23);
        if (has_b) load_item<S>(v, u, qb, cb, xb, b01, b23);
        finish_quad<S>(v, u, ba, qa, t, lane, ca, xa, a01, a23, updated);
        if (has_b) finish_quad<S>(v, u, bb, qb, t, lane, cb, xb, b01, b23, updated);
    }
    cta_add(&s_updated, updated, &u.ctl->n_updated);
}

// ---- group ---------------------------------------------------------------

// Canonical id and normalised SDF (2^-40 fixed point) of the record in band
// slot `slot`: the value the band walk kept for the slot (the FP64 oracle
// recomputes it from the point in double, with the walk's arithmetic).
template <int S>
__device__ __forceinline__ uint32_t slot_record(const DevVolume& v, const BatchArgs& a,
                                                const UpdateScratch& u, uint32_t slot, long long& fix) {
    const uint32_t n_steps = 2u * (uint32_t)v.steps + 1u;
    if (a.n <= 0) {  // no batch: nothing to recompute (never a valid record)
        fix = 0;
        return 0xFFFFFFFFu;
    }
    const uint32_t s = slot / (uint32_t)a.n, i = slot - s * (uint32_t)a.n;
    if constexpr (S != kStoreF64) {
        // The band walk kept the slot's normalised SDF: no point is read again.
        fix = to_fix(u.slot_val[slot]);
        return i * n_steps + s;
    }
    Ray r;
    int vx = 0, vy = 0, vz = 0;
    float sdf = 0.0f;
    const bool ok = ray_setup(a, (int)i, r);
    if (ok) band_sample(v, a, r, (int)s - v.steps, vx, vy, vz, sdf);
    if constexpr (S == kStoreF64) {
        fix = ok ? to_fix(clamp_sdf_n_f64(sdf_f64(v, a, r.px, r.py, r.pz, vx, vy, vz), v.trunc)) : 0ll;
    } else {
        fix = to_fix(fminf(fmaxf(__fmul_rn(sdf, v.inv_trunc), -1.0f), 1.0f));
    }
    return i * n_steps + s;
}

constexpr int kGroupPerThread = 8;  // records per thread (two 128-bit loads)

// Eight band slots from `first` of one batch: records of voxels that
// reserved a group take the next place of the group.
__device__ __forceinline__ void group_slots(const UpdateScratch& u, uint32_t first, uint32_t n_slots) {
    // Eight consecutive band slots per thread (same step, neighbouring points,
    // so mostly the same block): the block-tag gathers of distinct blocks in
    // flight together, then the (rare) records of crossing voxels take the
    // next place of their voxel's group with their band slot.
    if (first >= n_slots) return;
    uint32_t vi[kGroupPerThread];
    if (first + kGroupPerThread <= n_slots) {
        const uint4 r0 = __ldcs(reinterpret_cast<const uint4*>(u.records + first));
        const uint4 r1 = __ldcs(reinterpret_cast<const uint4*>(u.records + first) + 1);
        vi[0] = r0.x; vi[1] = r0.y; vi[2] = r0.z; vi[3] = r0.w;
        vi[4] = r1.x; vi[5] = r1.y; vi[6] = r1.z; vi[7] = r1.w;
    } else {
#pragma unroll
        for (int m = 0; m < kGroupPerThread; ++m)
            vi[m] = first + m < n_slots ? u.records[first + m] : kNoVoxel;
    }
    uint32_t tag[kGroupPerThread];
    bool same[kGroupPerThread];  // same block as the previous slot: reuse its tag
#pragma unroll
    for (int m = 0; m < kGroupPerThread; ++m) {
        const uint32_t blk = vi[m] / kBlockVoxels;
        same[m] = m > 0 && vi[m] != kNoVoxel && vi[m - 1] != kNoVoxel && vi[m - 1] / kBlockVoxels == blk;
        tag[m] = (vi[m] == kNoVoxel || same[m]) ? 0u : u.blk_cross[blk];
    }
#pragma unroll
    for (int m = 1; m < kGroupPerThread; ++m)
        if (same[m]) tag[m] = tag[m - 1];
    uint32_t hi[kGroupPerThread];
#pragma unroll
    for (int m = 0; m < kGroupPerThread; ++m)
        hi[m] = (vi[m] != kNoVoxel && tag[m] == u.tag) ? (uint32_t)(u.vacc[vi[m]] >> 32) : 0u;
#pragma unroll
    for (int m = 0; m < kGroupPerThread; ++m) {
        if (hi[m] == 0u) continue;  // not a voxel that reserved a group
        const uint32_t tk = (uint32_t)atomicAdd(&u.vacc[vi[m]], 1ull);
        if (tk < u.vcnt[vi[m]]) u.deferred[(size_t)(hi[m] - 1u) + tk] = first + m;
        else atomicOr(u.status, kStatusScratchOverflow);  // state left by a failed update
    }
}

__global__ void __launch_bounds__(kGroupThreads)
group_kernel(UpdateScratch u, uint32_t n_slots) {
    launch_dependents();
    grid_dependency_wait();
    if (u.ctl->def_lists == 0ull) return;  // no voxel crossed the cap in this batch
    group_slots(u, (blockIdx.x * kGroupThreads + threadIdx.x) * kGroupPerThread, n_slots);
}

// ---- values --------------------------------------------------------------

// One thread per grouped record: its band slot becomes its canonical id and
// its normalised SDF (recomputed from the point, the walk's arithmetic with
// the same rounding; the FP64 oracle's value in double).
template <int S>
__global__ void __launch_bounds__(kGroupThreads)
values_kernel(DevVolume v, BatchArgs a, UpdateScratch u) {
    launch_dependents();
    grid_dependency_wait();
    if (u.ctl->def_lists == 0ull) return;
    const uint32_t n = (uint32_t)min((long long)u.ctl->x_used, (long long)u.record_cap);
    for (uint32_t k = blockIdx.x * kGroupThreads + threadIdx.x; k < n; k += gridDim.x * kGroupThreads) {
        long long fix;
        const uint32_t id = slot_record<S>(v, a, u, u.deferred[k], fix);
        u.deferred[k] = id;
        u.deferred_fix[k] = fix;
    }
}

// ---- deferred ------------------------------------------------------------

// Finish a cap-crossing voxel: keep contributions accepted, their values
// summing to fix * 2^-40.
template <int S>
__device__ __forceinline__ void finish_voxel(const DevVolume& v, const UpdateScratch& u, uint32_t vi,
                                             int keep, long long fix) {
    if constexpr (S == kStoreF32) {
        const float wn = __fadd_rn(v.weight[vi], (float)keep);
        v.tsdf[vi] = add_fix(v.tsdf[vi], fix);
        v.weight[vi] = wn;
        const float c = __fmul_rn(128.0f, wn);
        v.r[vi] = c;
        v.g[vi] = c;
        v.b[vi] = c;
    } else if constexpr (S == kStoreF16U16) {
        unsigned short* w16 = reinterpret_cast<unsigned short*>(v.weight);
        __half* h = reinterpret_cast<__half*>(v.tsdf);
        const float w0 = (float)w16[vi];
        h[vi] = __float2half_rn(new_mean_f16(__half2float(h[vi]), w0, keep, fix));
        w16[vi] = (unsigned short)__fadd_rn(w0, (float)keep);
    } else {
        double* d = reinterpret_cast<double*>(v.tsdf);
        d[vi] = d[vi] + (double)fix * kFixInv;
        v.weight[vi] = __fadd_rn(v.weight[vi], (float)keep);
    }
    u.vacc[vi] = 0ull;
    u.vcnt[vi] = 0u;
}

// The keep-th smallest id (1-based) of a group, by four 8-bit radix passes
// with a per-warp histogram. Ids are distinct, so exactly keep ids are <= it.
__device__ uint32_t radix_select(const uint32_t* ids, int n, int keep, uint32_t* hist, int lane) {
    uint32_t prefix = 0u, pmask = 0u;
    int need = keep;
    for (int shift = 24; shift >= 0; shift -= 8) {
        for (int b = lane; b < 256; b += 32) hist[b] = 0u;
        __syncwarp();
        for (int k = lane; k < n; k += 32) {
            const uint32_t id = ids[k];
            if ((id & pmask) == prefix) atomicAdd(&hist[(id >> shift) & 255u], 1u);
        }
        __syncwarp();
        uint32_t c[8];
        int mine = 0;
#pragma unroll
        for (int j = 0; j < 8; ++j) {
            c[j] = hist[lane * 8 + j];
            mine += (int)c[j];
        }
        int incl = mine;
        for (int o = 1; o < 32; o <<= 1) {
            const int y = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += y;
        }
        const int excl = incl - mine;
        const unsigned hit = __ballot_sync(0xffffffffu, excl < need && need <= incl);
        const int owner = hit ? __ffs(hit) - 1 : 0;
        int bucket = 0, below = excl;
        if (lane == owner) {
#pragma unroll
            for (int j = 0; j < 8; ++j) {
                if (below + (int)c[j] >= need) {
                    bucket = lane * 8 + j;
                    break;
                }
                below += (int)c[j];
            }
        }
        bucket = __shfl_sync(0xffffffffu, bucket, owner);
        below = __shfl_sync(0xffffffffu, below, owner);
        prefix |= (uint32_t)bucket << shift;
        pmask |= 255u << shift;
        need -= below;
        __syncwarp();
    }
    return prefix;
}

// Id and fixed-point value of the record at group position pos: as the values
// pass left them (the FP64 oracle), or from the record's band slot (FP32 /
// FP16 storage: id from the slot's point and step, value kept by the walk).
template <int S>
__device__ __forceinline__ void group_record(const UpdateScratch& u, uint32_t n_pts, uint32_t n_steps,
                                             uint32_t pos, uint32_t& id, long long& fix) {
    if constexpr (S == kStoreF64) {
        id = u.deferred[pos];
        fix = u.deferred_fix[pos];
    } else {
        const uint32_t slot = u.deferred[pos];
        const uint32_t st = slot / n_pts;
        id = (slot - st * n_pts) * n_steps + st;
        fix = to_fix(u.slot_val[slot]);
    }
}

// A large group's records as (id, value) arrays in place, by the whole warp.
template <int S>
__device__ __forceinline__ void group_to_ids(const UpdateScratch& u, uint32_t n_pts, uint32_t n_steps,
                                             uint32_t base, int n, int lane) {
    if constexpr (S != kStoreF64) {
        for (int k = lane; k < n; k += 32) {
            uint32_t id;
            long long fix;
            group_record<S>(u, n_pts, n_steps, base + (uint32_t)k, id, fix);
            u.deferred[base + k] = id;
            u.deferred_fix[base + k] = fix;
        }
        __syncwarp();
    }
}

// Sum of the accepted values of a group of at most 32 * R records, by one
// warp: record r * 32 + lane in registers (id and value straight from its
// band slot), ranked by id against every other record with shuffles; a record
// is accepted when fewer than keep ids are below its own. Ids are distinct
// and below 0xFFFFFFFF, so the padding entries never rank below a record.
template <int S, int R>
__device__ __forceinline__ long long rank_group(const UpdateScratch& u, uint32_t n_pts, uint32_t n_steps,
                                                uint32_t base, int n, int keep, int lane) {
    uint32_t id[R];
    long long val[R];
    int rank[R];
#pragma unroll
    for (int r = 0; r < R; ++r) {
        const int k = r * 32 + lane;
        id[r] = 0xFFFFFFFFu;
        val[r] = 0ll;
        rank[r] = 0;
        if (k < n) group_record<S>(u, n_pts, n_steps, base + (uint32_t)k, id[r], val[r]);
    }
#pragma unroll
    for (int rr = 0; rr < R; ++rr) {
#pragma unroll 8
        for (int src = 0; src < 32; ++src) {
            const uint32_t other = __shfl_sync(0xffffffffu, id[rr], src);
#pragma unroll
            for (int r = 0; r < R; ++r) rank[r] += other < id[r] ? 1 : 0;
        }
    }
    long long fix = 0ll;
#pragma unroll
    for (int r = 0; r < R; ++r)
        if (r * 32 + lane < n && rank[r] < keep) fix += val[r];
    return fix;
}

// Sum of the accepted values of a voxel of the large list (e = voxel, group
// base, records, accepted), by one warp, on every lane: register ranking
// sized to the group up to 256 records; beyond, the group's records become
// (id, value) arrays in place and a radix select finds the keep-th id.
template <int S>
__device__ long long large_group_sum(const UpdateScratch& u, uint32_t n_pts, uint32_t n_steps, const int4 e,
                                     uint32_t* hist, int lane) {
    const uint32_t base = (uint32_t)e.y;
    const int n = e.z, keep = e.w;
    long long fix;
    if (n <= 32) {
        fix = rank_group<S, 1>(u, n_pts, n_steps, base, n, keep, lane);
    } else if (n <= 64) {
        fix = rank_group<S, 2>(u, n_pts, n_steps, base, n, keep, lane);
    } else if (n <= 128) {
        fix = rank_group<S, 4>(u, n_pts, n_steps, base, n, keep, lane);
    } else if (n <= 32 * kRankRegs) {
        fix = rank_group<S, kRankRegs>(u, n_pts, n_steps, base, n, keep, lane);
    } else {
        group_to_ids<S>(u, n_pts, n_steps, base, n, lane);
        const uint32_t* ids = u.deferred + base;
        const long long* vals = u.deferred_fix + base;
        const uint32_t last = radix_select(ids, n, keep, hist, lane);
        fix = 0ll;
        for (int k = lane; k < n; k += 32)
            if (ids[k] <= last) fix += vals[k];
    }
    for (int o = 16; o > 0; o >>= 1) fix += __shfl_xor_sync(0xffffffffu, fix, o);
    return fix;
}

template <int S>
__global__ void __launch_bounds__(kDeferThreads)
deferred_kernel(DevVolume v, BatchArgs a, UpdateScratch u) {
    __shared__ uint32_t hist[kDeferWarps][256];
    __shared__ int s_updated;
    if (threadIdx.x == 0) s_updated = 0;
    __syncthreads();
    launch_dependents();
    grid_dependency_wait();
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const uint32_t n_steps = 2u * (uint32_t)v.steps + 1u;
    const unsigned long long lists = u.ctl->def_lists;
    int n_small = (int)(lists & 0xFFFFFFFFull), n_large = (int)(lists >> 32);
    if ((long long)n_small + n_large > (long long)u.dvox_cap) n_small = n_large = 0;  // overflowed
    int updated = 0;

    // Large groups: one warp each.
    const int gw = blockIdx.x * kDeferWarps + warp, nw = gridDim.x * kDeferWarps;
    for (int d = gw; d < n_large; d += nw) {
        const int4 e = u.dvox[u.dvox_cap - 1 - d];  // (voxel, group base, records, accepted)
        const long long fix = large_group_sum<S>(u, (uint32_t)a.n, n_steps, e, hist[warp], lane);
        if (lane == 0) {
            finish_voxel<S>(v, u, (uint32_t)e.x, e.w, fix);
            ++updated;
        }
    }

    // Small groups (at most kLaneRecords = 16 records): one half-warp each,
    // one record per lane, ranked by id with shuffles inside the half.
    static_assert(kLaneRecords == 16, "small groups are ranked by half-warps");
    const int half = lane >> 4, hl = lane & 15;
    for (int d0 = 2 * gw; d0 < n_small; d0 += 2 * nw) {  // uniform across the warp
        const int d = d0 + half;
        const bool live = d < n_small;
        const int4 e = live ? u.dvox[d] : make_int4(0, 0, 0, 0);
        const int n = e.z, keep = e.w;
        const bool mine = live && hl < n;
        uint32_t id = 0xFFFFFFFFu;
        long long val = 0ll;
        if (mine) group_record<S>(u, (uint32_t)a.n, n_steps, (uint32_t)e.y + hl, id, val);
        int rank = 0;
#pragma unroll
        for (int src = 0; src < 16; ++src) rank += __shfl_sync(0xffffffffu, id, src, 16) < id ? 1 : 0;
        long long fix = (mine && rank < keep) ? val : 0ll;
#pragma unroll
        for (int o = 8; o > 0; o >>= 1) fix += __shfl_xor_sync(0xffffffffu, fix, o, 16);
        if (live && hl == 0) {
            finish_voxel<S>(v, u, (uint32_t)e.x, keep, fix);
            ++updated;
        }
    }
    cta_add(&s_updated, updated, &u.ctl->n_updated);
}

// ---- batched steps -----------------------------------------------------

template <typename T>
__device__ __forceinline__ void cta_copy(T* dst, const T* src) {
    static_assert(sizeof(T) % 4 == 0, "descriptor copies go by words");
    const uint32_t* a = reinterpret_cast<const uint32_t*>(src);
    uint32_t* d = reinterpret_cast<uint32_t*>(dst);
    for (int k = threadIdx.x; k < (int)(sizeof(T) / 4); k += blockDim.x) d[k] = a[k];
}

// Scene of global work item `item` given the per-scene item prefix `begin`
// (n + 1 entries, begin[0] = 0).
__device__ __forceinline__ int scene_of(const int* begin, int n, int item) {
    int lo = 0, hi = n;  // begin[lo] <= item < begin[hi]
    while (hi - lo > 1) {
        const int mid = (lo + hi) >> 1;
        if (begin[mid] <= item) lo = mid;
        else hi = mid;
    }
    return lo;
}

// Start of a step: every scene's update counters and the step's queues to
// zero (one CTA).
__global__ void batch_prepare_kernel(StepWork w) {
    grid_dependency_wait();
    constexpr int kWords = (int)(sizeof(UpdateControl) / 4);
    for (int k = threadIdx.x; k < w.n_scenes * kWords; k += blockDim.x) {
        const SceneWork& sw = w.scenes[k / kWords];
        if (sw.band_tiles > 0)  // idle scenes keep their last update's counters
            reinterpret_cast<uint32_t*>(sw.u.ctl)[k % kWords] = 0u;
    }
    if (threadIdx.x < kNumBatchQueues) w.queues[threadIdx.x] = 0u;
    __syncthreads();
    launch_dependents();
}

// Work items a pass has in one scene (read by thread 0 after the previous
// pass completed).
enum MultiPass : int { kPassFinishPairs, kPassFinishSingle, kPassGroup, kPassValues, kPassDeferred };

template <int PASS>
__device__ __forceinline__ int scene_items(const SceneWork& sw) {
    // A scene sitting this step out still holds its previous update's
    // counters (and an empty batch): it has no work in any pass.
    if (sw.band_tiles <= 0) return 0;
    const UpdateControl* c = sw.u.ctl;
    if (PASS == kPassFinishPairs || PASS == kPassFinishSingle) {
        const int nt = min(c->n_touched, sw.v.pool_capacity);
        return PASS == kPassFinishPairs ? (nt + 1) / 2 : nt;
    }
    if (c->def_lists == 0ull) return 0;  // no voxel crossed the cap in this scene
    if (PASS == kPassGroup)
        return (int)(((uint32_t)sw.n_slots + kGroupThreads * kGroupPerThread - 1) /
                     (kGroupThreads * kGroupPerThread));
    if (PASS == kPassValues) {
        const long long x = min((long long)c->x_used, (long long)sw.u.record_cap);
        return (int)((x + kGroupThreads - 1) / kGroupThreads);
    }
    // Deferred: one warp item per large group and per pair of small groups.
    const int n_small = (int)(c->def_lists & 0xFFFFFFFFull), n_large = (int)(c->def_lists >> 32);
    if ((long long)n_small + n_large > (long long)sw.u.dvox_cap) return 0;  // overflowed
    return n_large + (n_small + 1) / 2;
}

// Exclusive item prefix of the scenes into begin[0..n]: one thread per scene
// reads its counts (all in flight together), then a scan in shared memory
// (n <= 64 <= blockDim.x).
template <int PASS>
__device__ __forceinline__ void scene_prefix(const StepWork& w, int* begin) {
    const int t = threadIdx.x;
    if (t < w.n_scenes) begin[t + 1] = scene_items<PASS>(w.scenes[t]);
    if (t == 0) begin[0] = 0;
    __syncthreads();
    if (t == 0)
        for (int k = 1; k <= w.n_scenes; ++k) begin[k] += begin[k - 1];
    __syncthreads();
}

// Finish every touched block of every scene: work items of one or two
// blocks from an atomic queue, the item's scene descriptor staged in shared
// memory (reloaded when the CTA moves to another scene).
template <int S, bool PAIR>
__global__ void __launch_bounds__(kFinishThreads)
finish_multi_kernel(StepWork w) {
    __shared__ SceneWork sw;
    __shared__ int s_begin[kMaxBatchScenes + 1];
    __shared__ int s_item, s_updated;
    const int t = threadIdx.x, lane = t & 31;
    launch_dependents();
    grid_dependency_wait();
    if (t == 0) s_updated = 0;
    scene_prefix<PAIR ? kPassFinishPairs : kPassFinishSingle>(w, s_begin);
    const int total = s_begin[w.n_scenes];
    int cur = -1, updated = 0;
    for (;;) {
        if (t == 0) s_item = (int)atomicAdd(&w.queues[kQFinish], 1u);
        __syncthreads();
        const int item = s_item;
        const bool done = item >= total;  // also on a CTA's first pull when items are few
        const int sc = done ? -1 : scene_of(s_begin, w.n_scenes, item);
        if (sc != cur || done) {
            // Statistics of the scene left behind, then the next descriptor.
            const int wsum = __reduce_add_sync(0xffffffffu, updated);
            if (lane == 0 && wsum) atomicAdd(&s_updated, wsum);
            __syncthreads();
            if (t == 0 && cur >= 0 && s_updated) atomicAdd(&sw.u.ctl->n_updated, s_updated);
            __syncthreads();
            if (t == 0) s_updated = 0;
            updated = 0;
            if (done) break;
            cta_copy(&sw, &w.scenes[sc]);
            __syncthreads();
            cur = sc;
        }
        const int n_touched = min(sw.u.ctl->n_touched, sw.v.pool_capacity);
        const int local = item - s_begin[sc];
        const int ia = PAIR ? 2 * local : local;
        const int ib = ia + 1;
        const bool has_b = PAIR && ib < n_touched;  // uniform across the CTA
        const int32_t ba = sw.u.touched[ia];
        const int32_t bb = has_b ? sw.u.touched[ib] : ba;
        const size_t qa = (size_t)ba * (kBlockVoxels / 4) + t;
        const size_t qb = (size_t)bb * (kBlockVoxels / 4) + t;
        uint4 ca, cb;
        Quad<S> xa, xb;
        ulonglong2 a01, a23, b01, b23;
        load_item<S>(sw.v, sw.u, qa, ca, xa, a01, a23);
        if (has_b) load_item<S>(sw.v, sw.u, qb, cb, xb, b01, b23);
        finish_quad<S>(sw.v, sw.u, ba, qa, t, lane, ca, xa, a01, a23, updated);
        if (has_b) finish_quad<S>(sw.v, sw.u, bb, qb, t, lane, cb, xb, b01, b23, updated);
        __syncthreads();  // s_item and the descriptor are rewritten next
    }
}

// Group the records of every scene that has cap-crossing voxels.
__global__ void __launch_bounds__(kGroupThreads)
group_multi_kernel(StepWork w) {
    __shared__ UpdateScratch su;
    __shared__ int s_begin[kMaxBatchScenes + 1];
    __shared__ int s_item;
    __shared__ uint32_t s_slots;
    const int t = threadIdx.x;
    launch_dependents();
    grid_dependency_wait();
    scene_prefix<kPassGroup>(w, s_begin);
    const int total = s_begin[w.n_scenes];
    int cur = -1;
    for (;;) {
        if (t == 0) s_item = (int)atomicAdd(&w.queues[kQGroup], 1u);
        __syncthreads();
        const int item = s_item;
        if (item >= total) break;
        const int sc = scene_of(s_begin, w.n_scenes, item);
        if (sc != cur) {
            cta_copy(&su, &w.scenes[sc].u);
            if (t == 0) s_slots = (uint32_t)w.scenes[sc].n_slots;
            __syncthreads();
            cur = sc;
        }
        const uint32_t first = ((uint32_t)(item - s_begin[sc]) * kGroupThreads + t) * kGroupPerThread;
        group_slots(su, first, s_slots);
        __syncthreads();
    }
}

// Ids and values of every scene's grouped records.
template <int S>
__global__ void __launch_bounds__(kGroupThreads)
values_multi_kernel(StepWork w) {
    __shared__ SceneWork sw;
    __shared__ int s_begin[kMaxBatchScenes + 1];
    __shared__ int s_item;
    const int t = threadIdx.x;
    launch_dependents();
    grid_dependency_wait();
    scene_prefix<kPassValues>(w, s_begin);
    const int total = s_begin[w.n_scenes];
    int cur = -1;
    for (;;) {
        if (t == 0) s_item = (int)atomicAdd(&w.queues[kQValues], 1u);
        __syncthreads();
        const int item = s_item;
        if (item >= total) break;
        const int sc = scene_of(s_begin, w.n_scenes, item);
        if (sc != cur) {
            cta_copy(&sw, &w.scenes[sc]);
            __syncthreads();
            cur = sc;
        }
        const uint32_t n = (uint32_t)min((long long)sw.u.ctl->x_used, (long long)sw.u.record_cap);
        const uint32_t k = (uint32_t)(item - s_begin[sc]) * kGroupThreads + t;
        if (k < n) {
            long long fix;
            const uint32_t id = slot_record<S>(sw.v, sw.a, sw.u, sw.u.deferred[k], fix);
            sw.u.deferred[k] = id;
            sw.u.deferred_fix[k] = fix;
        }
        __syncthreads();
    }
}

// Select and finish every scene's cap-crossing voxels: warp work items, one
// per large group and one per pair of small groups.
template <int S>
__global__ void __launch_bounds__(kDeferThreads)
deferred_multi_kernel(StepWork w) {
    __shared__ uint32_t hist[kDeferWarps][256];
    __shared__ int s_begin[kMaxBatchScenes + 1];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    launch_dependents();
    grid_dependency_wait();
    scene_prefix<kPassDeferred>(w, s_begin);
    const int total = s_begin[w.n_scenes];
    for (;;) {
        int item = 0;
        if (lane == 0) item = (int)atomicAdd(&w.queues[kQDeferred], 1u);
        item = __shfl_sync(0xffffffffu, item, 0);
        if (item >= total) break;
        const int sc = scene_of(s_begin, w.n_scenes, item);
        const SceneWork& sw = w.scenes[sc];
        const DevVolume& v = sw.v;
        const UpdateScratch& u = sw.u;
        const uint32_t n_steps = 2u * (uint32_t)v.steps + 1u;
        const unsigned long long lists = u.ctl->def_lists;
        const int n_small = (int)(lists & 0xFFFFFFFFull), n_large = (int)(lists >> 32);
        const int local = item - s_begin[sc];
        int done = 0;
        if (local < n_large) {
            const int4 e = u.dvox[u.dvox_cap - 1 - local];
            const long long fix = large_group_sum<S>(u, (uint32_t)sw.a.n, n_steps, e, hist[warp], lane);
            if (lane == 0) finish_voxel<S>(v, u, (uint32_t)e.x, e.w, fix);
            done = 1;
        } else {
            const int half = lane >> 4, hl = lane & 15;
            const int d0 = 2 * (local - n_large);
            const int d = d0 + half;
            const bool live = d < n_small;
            const int4 e = live ? u.dvox[d] : make_int4(0, 0, 0, 0);
            const int n = e.z, keep = e.w;
            const bool mine = live && hl < n;
            uint32_t id = 0xFFFFFFFFu;
            long long val = 0ll;
            if (mine) group_record<S>(u, (uint32_t)sw.a.n, n_steps, (uint32_t)e.y + hl, id, val);
            int rank = 0;
#pragma unroll
            for (int src = 0; src < 16; ++src) rank += __shfl_sync(0xffffffffu, id, src, 16) < id ? 1 : 0;
            long long fix = (mine && rank < keep) ? val : 0ll;
#pragma unroll
            for (int o = 8; o > 0; o >>= 1) fix += __shfl_xor_sync(0xffffffffu, fix, o, 16);
            if (live && hl == 0) finish_voxel<S>(v, u, (uint32_t)e.x, keep, fix);
            done = d0 + 1 < n_small ? 2 : 1;
        }
        if (lane == 0) atomicAdd(&u.ctl->n_updated, done);
    }
}

}  // namespace

// CTAs of Kernel resident at once on the device (one wave), queried once
// per kernel.
template <auto Kernel>
int resident_grid(int threads, int sm_count) {
    static int per_sm = 0;
    static std::once_flag once;
    std::call_once(once, [&] {
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, Kernel, threads, 0) != cudaSuccess ||
            per_sm < 1)
            per_sm = 1;
    });
    return per_sm * sm_count;
}

cudaError_t launch_finish(const DevVolume& v, const UpdateScratch& u, int sm_count, cudaStream_t s) {
    switch (v.storage) {
        case kStoreF16U16: {
            return launch_after(finish_kernel<kStoreF16U16>, resident_grid<finish_kernel<kStoreF16U16>>(kFinishThreads, sm_count),
                                kFinishThreads, s, v, u);
        }
        case kStoreF64: {
            return launch_after(finish_kernel<kStoreF64>, resident_grid<finish_kernel<kStoreF64>>(kFinishThreads, sm_count),
                                kFinishThreads, s, v, u);
        }
        default: {
            return launch_after(finish_kernel<kStoreF32>, resident_grid<finish_kernel<kStoreF32>>(kFinishThreads, sm_count),
                                kFinishThreads, s, v, u);
        }
    }
}

cudaError_t launch_group(const DevVolume& v, const BatchArgs& a, const UpdateScratch& u,
                         cudaStream_t s) {
    const uint32_t n_slots = (uint32_t)a.n * (2u * (uint32_t)v.steps + 1u);
    if (n_slots == 0) return cudaSuccess;
    const uint32_t per_cta = kGroupThreads * (uint32_t)kGroupPerThread;
    return launch_after(group_kernel, (n_slots + per_cta - 1u) / per_cta, kGroupThreads, s, u, n_slots);
}

cudaError_t launch_values(const DevVolume& v, const BatchArgs& a, const UpdateScratch& u, int n_ctas,
                          cudaStream_t s) {
    // FP32 / FP16: the deferred pass reads each record's id and value from its
    // band slot itself; only the FP64 oracle recomputes values from points.
    if (v.storage != kStoreF64) return cudaSuccess;
    switch (v.storage) {
        case kStoreF16U16: return launch_after(values_kernel<kStoreF16U16>, n_ctas, kGroupThreads, s, v, a, u);
        case kStoreF64: return launch_after(values_kernel<kStoreF64>, n_ctas, kGroupThreads, s, v, a, u);
        default: return launch_after(values_kernel<kStoreF32>, n_ctas, kGroupThreads, s, v, a, u);
    }
}

cudaError_t launch_deferred(const DevVolume& v, const BatchArgs& a, const UpdateScratch& u, int sm_count,
                            cudaStream_t s) {
    switch (v.storage) {
        case kStoreF16U16: {
            return launch_after(deferred_kernel<kStoreF16U16>, resident_grid<deferred_kernel<kStoreF16U16>>(kDeferThreads, sm_count),
                                kDeferThreads, s, v, a, u);
        }
        case kStoreF64: {
            return launch_after(deferred_kernel<kStoreF64>, resident_grid<deferred_kernel<kStoreF64>>(kDeferThreads, sm_count),
                                kDeferThreads, s, v, a, u);
        }
        default: {
            return launch_after(deferred_kernel<kStoreF32>, resident_grid<deferred_kernel<kStoreF32>>(kDeferThreads, sm_count),
                                kDeferThreads, s, v, a, u);
        }
    }
}

cudaError_t launch_batch_prepare(const StepWork& w, cudaStream_t s) {
    return launch_after(batch_prepare_kernel, 1, 256, s, w);
}

namespace {
template <int S, bool P>
cudaError_t finish_multi_t(const StepWork& w, int sm_count, cudaStream_t s) {
    return launch_after(finish_multi_kernel<S, P>,
                        resident_grid<finish_multi_kernel<S, P>>(kFinishThreads, sm_count),
                        kFinishThreads, s, w);
}
template <int S>
cudaError_t values_multi_t(const StepWork& w, int sm_count, cudaStream_t s) {
    return launch_after(values_multi_kernel<S>, resident_grid<values_multi_kernel<S>>(kGroupThreads, sm_count),
                        kGroupThreads, s, w);
}
template <int S>
cudaError_t deferred_multi_t(const StepWork& w, int sm_count, cudaStream_t s) {
    return launch_after(deferred_multi_kernel<S>,
                        resident_grid<deferred_multi_kernel<S>>(kDeferThreads, sm_count), kDeferThreads, s,
                        w);
}
}  // namespace

cudaError_t launch_finish_multi(const StepWork& w, int storage, int pair, int sm_count, cudaStream_t s) {
    switch (storage) {
        case kStoreF16U16:
            return pair ? finish_multi_t<kStoreF16U16, true>(w, sm_count, s)
                        : finish_multi_t<kStoreF16U16, false>(w, sm_count, s);
        case kStoreF64:
            return pair ? finish_multi_t<kStoreF64, true>(w, sm_count, s)
                        : finish_multi_t<kStoreF64, false>(w, sm_count, s);
        default:
            return pair ? finish_multi_t<kStoreF32, true>(w, sm_count, s)
                        : finish_multi_t<kStoreF32, false>(w, sm_count, s);
    }
}

cudaError_t launch_group_multi(const StepWork& w, int sm_count, cudaStream_t s) {
    return launch_after(group_multi_kernel, resident_grid<group_multi_kernel>(kGroupThreads, sm_count),
                        kGroupThreads, s, w);
}

cudaError_t launch_values_multi(const StepWork& w, int storage, int sm_count, cudaStream_t s) {
    if (storage != kStoreF64) return cudaSuccess;  // deferred_multi reads the band slots itself
    switch (storage) {
        case kStoreF16U16: return values_multi_t<kStoreF16U16>(w, sm_count, s);
        case kStoreF64: return values_multi_t<kStoreF64>(w, sm_count, s);
        default: return values_multi_t<kStoreF32>(w, sm_count, s);
    }
}

cudaError_t launch_deferred_multi(const StepWork& w, int storage, int sm_count, cudaStream_t s) {
    switch (storage) {
        case kStoreF16U16: return deferred_multi_t<kStoreF16U16>(w, sm_count, s);
        case kStoreF64: return deferred_multi_t<kStoreF64>(w, sm_count, s);
        default: return deferred_multi_t<kStoreF32>(w, sm_count, s);
    }
}

}  // namespace osn_b200
