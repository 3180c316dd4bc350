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
// blocks, and per band slot a record (the voxel) and the normalised SDF.
//
//   finish   one 128-thread CTA per touched block (two per CTA pass), 4
//            voxels per thread, every array read and written as 128-bit
//            vectors: a voxel that accepts all of its records (keep == n,
//            the common case) gets tsdf + sum, w0 + n, 128 * (w0 + n) and
//            its count and sum back to zero. A voxel that crosses the cap
//            inside the batch instead reserves a group of n places (one
//            warp-aggregated atomic), keeps the group's base in its sum word
//            and n in its count word, and sets its bit in the block's
//            crossing bitmap (16 words per block, rewritten for every block
//            finish visits).
//   group    one pass over the band slots of the batch, eight per thread
//            (records loaded as 128-bit vectors): a record whose voxel's bit
//            is set takes the next place of the voxel's group (atomic add on
//            the sum word; its normalised SDF loaded in the same round trip)
//            and stores its canonical id and value there, then counts the
//            voxel's pending
//            records down with an acquire-release atomic. The record that
//            brings the count to zero is the last of its group: its warp
//            loads the whole group, keeps the keep records with the smallest
//            ids (shuffle ranking in registers up to 256 records, a radix
//            select beyond) and finishes the voxel. No pass runs between the
//            grouping and the selection.
//
// The FP64 oracle storage keeps no per-slot values: its group entries hold
// the band slot, and the selection recomputes each record's normalised SDF
// in double from its point.
//
// Sums are 64-bit fixed point added to the stored sum with one rounding, so
// results do not depend on the order in which threads meet the records:
// repeated runs are bit-identical, and a voxel with one contribution per
// batch gets exactly the reference's fl(tsdf + sdf_n).
#include <algorithm>
#include <mutex>

#include "volume.h"

namespace osn_b200 {
namespace {

constexpr int kFinishThreads = 128;  // 4 voxels per thread, one block per CTA pass
constexpr int kGroupThreads = 256;
constexpr int kGroupWarps = kGroupThreads / 32;
constexpr int kGroupPerThread = 8;  // band slots per thread (two 128-bit loads)
constexpr int kRankRegs = 8;        // groups of up to 32 * 8 records are ranked in registers
// Where the ordered selection of cap-crossing voxels runs: 1, in its own
// pass over a list of the crossing voxels that finish writes (no memory
// ordering inside a pass: the pass boundary orders everything); 0, inside
// the group pass, by the warp whose record completes a voxel's group (one
// fence per thread that placed records, one per selected group).
#ifndef OSN_SPLIT_SELECT
#define OSN_SPLIT_SELECT 1
#endif
// The group pass as a persistent grid whose threads load their next chunk of
// records before placing the current one (1), or one chunk per thread (0).
#ifndef OSN_GROUP_PERSISTENT
#define OSN_GROUP_PERSISTENT 0
#endif
constexpr int kSelectThreads = 128;
constexpr int kSelectWarps = kSelectThreads / 32;
// Resident 256-thread CTAs per SM the group pass's registers are sized for:
// the scan is latency-bound, so occupancy hides its round trips.
#ifndef OSN_GROUP_MIN_BLOCKS
#define OSN_GROUP_MIN_BLOCKS 6
#endif
static_assert(kFinishThreads >= kMaxBatchScenes && kGroupThreads >= kMaxBatchScenes,
              "one thread per scene builds the item prefix");

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
// the voxels that accept all their records, open groups for those that
// cross the cap. Warp-synchronous (all lanes of the warp call it).
template <int S>
__device__ __forceinline__ void finish_quad(const DevVolume& v, const UpdateScratch& u, int32_t bi,
                                            size_t q4, int t, int lane, const uint4 c4, Quad<S>& x,
                                            const ulonglong2 a01, const ulonglong2 a23, int& updated) {
    const bool any = (c4.x | c4.y | c4.z | c4.w) != 0u;
    // Warp-uniform skip: no record of this update names these 128 voxels, so
    // the group pass never reads their crossing bits either.
    if (!__any_sync(0xffffffffu, any)) return;
    const uint32_t n[4] = {c4.x, c4.y, c4.z, c4.w};
    unsigned long long acc[4] = {a01.x, a01.y, a23.x, a23.y};
    uint32_t cnt[4] = {0u, 0u, 0u, 0u};
    int keepv[4] = {0, 0, 0, 0};
    // Voxels crossing the cap reserve n places each; the warp's reservations
    // are summed and made with one atomic.
    uint32_t my_records = 0u, my_cross = 0u;
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        if (n[q] == 0u) continue;
        keepv[q] = accept_count(x.w[q], v.weight_cap, (int)n[q]);
        if (keepv[q] != 0 && (uint32_t)keepv[q] != n[q]) {
            my_records += n[q];
            ++my_cross;
        }
    }
    uint32_t rec_base = 0u, x_at = 0u;
    if (__ballot_sync(0xffffffffu, my_records > 0u)) {
        uint32_t rec_incl = my_records, x_incl = my_cross;
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t ry = __shfl_up_sync(0xffffffffu, rec_incl, o);
            const uint32_t xy = __shfl_up_sync(0xffffffffu, x_incl, o);
            if (lane >= o) {
                rec_incl += ry;
                x_incl += xy;
            }
        }
        uint32_t rb = 0u, xb = 0u;
        if (lane == 31) {
            rb = atomicAdd(&u.ctl->x_used, rec_incl);
            xb = (uint32_t)atomicAdd(&u.ctl->n_crossing, (unsigned long long)x_incl);
        }
        rb = __shfl_sync(0xffffffffu, rb, 31);
        xb = __shfl_sync(0xffffffffu, xb, 31);
        rec_base = rb + rec_incl - my_records;
        x_at = xb + x_incl - my_cross;  // this lane's first place in the crossing list
    }
    uint32_t xmask = 0u;  // bit q: voxel 4t + q crosses the cap
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
            // Crosses the cap: the group pass places its records and the
            // last of them finishes it. The sum word holds the group's base
            // + 1 (high half) and the next free place (low half); the count
            // word the records still to be placed.
            if ((uint64_t)rec_base + n[q] <= (uint64_t)u.record_cap && x_at < (uint32_t)u.xlist_cap) {
                acc[q] = (unsigned long long)(rec_base + 1u) << 32;
                cnt[q] = n[q];
                xmask |= 1u << q;
                if (OSN_SPLIT_SELECT) u.xlist[x_at] = (uint32_t)bi * kBlockVoxels + 4u * t + q;
            } else {
                // Out of scratch (only after a failed update left stale
                // counters): the voxel's records are dropped, the status
                // word says so.
                atomicOr(v.status, kStatusScratchOverflow);
                acc[q] = 0ull;
            }
            rec_base += n[q];
            ++x_at;
        }
    }
    // The block's crossing bitmap: voxel 32w + j is bit j of word w, and the
    // four voxels of thread t are bits 4(t % 8) .. 4(t % 8) + 3 of word t / 8.
    uint32_t bits = xmask << (4 * (t & 7));
    bits |= __shfl_xor_sync(0xffffffffu, bits, 1);
    bits |= __shfl_xor_sync(0xffffffffu, bits, 2);
    bits |= __shfl_xor_sync(0xffffffffu, bits, 4);
    if ((t & 7) == 0) u.xbits[(size_t)bi * kXWords + (t >> 3)] = bits;
    if (!any) return;
    store_quad<S>(v, q4, x);
    reinterpret_cast<uint4*>(u.vcnt)[q4] = make_uint4(cnt[0], cnt[1], cnt[2], cnt[3]);
    reinterpret_cast<ulonglong2*>(u.vacc)[2 * q4] = make_ulonglong2(acc[0], acc[1]);
    reinterpret_cast<ulonglong2*>(u.vacc)[2 * q4 + 1] = make_ulonglong2(acc[2], acc[3]);
}

// A touched block now belongs to the current call's chunk.
__device__ __forceinline__ void tag_chunk(const DevVolume& v, int32_t ba, int32_t bb, bool has_b) {
    if (!v.block_chunk) return;
    v.block_chunk[ba] = v.chunk;
    if (has_b) v.block_chunk[bb] = v.chunk;
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
        if (t == 0) tag_chunk(v, ba, bb, has_b);
        finish_quad<S>(v, u, ba, qa, t, lane, ca, xa, a01, a23, updated);
        if (has_b) finish_quad<S>(v, u, bb, qb, t, lane, cb, xb, b01, b23, updated);
    }
    cta_add(&s_updated, updated, &u.ctl->n_updated);
}

// ---- group and select ------------------------------------------------------

// Canonical id of band slot `slot` (point i at step s sits at s * n + i):
// i * (2 * steps + 1) + s, the position of the sample in (point, step) order.
__device__ __forceinline__ uint32_t slot_id(uint32_t slot, uint32_t n_pts, uint32_t n_steps) {
    const uint32_t s = slot / n_pts, i = slot - s * n_pts;
    return i * n_steps + s;
}

// The FP64 oracle's canonical id and normalised SDF (2^-40 fixed point) of
// the record in band slot `slot`, recomputed in double from its point with
// the walk's sample (the same voxel, so the same accepted set).
__device__ __forceinline__ uint32_t slot_record_f64(const DevVolume& v, const BatchArgs& a, uint32_t slot,
                                                    long long& fix) {
    const uint32_t n_steps = 2u * (uint32_t)v.steps + 1u;
    if (a.n <= 0) {  // no batch: nothing to recompute (never a valid record)
        fix = 0;
        return 0xFFFFFFFFu;
    }
    const uint32_t s = slot / (uint32_t)a.n, i = slot - s * (uint32_t)a.n;
    Ray r;
    int vx = 0, vy = 0, vz = 0;
    float sdf = 0.0f;
    const bool ok = ray_setup(a, (int)i, r);
    if (ok) band_sample(v, a, r, (int)s - v.steps, vx, vy, vz, sdf);
    fix = ok ? to_fix(clamp_sdf_n_f64(sdf_f64(v, a, r.px, r.py, r.pz, vx, vy, vz), v.trunc)) : 0ll;
    return i * n_steps + s;
}

// Id and value of a group entry: (id | normalised SDF bits << 32) as the
// group pass stored it, or, for the FP64 oracle, its band slot.
template <int S>
__device__ __forceinline__ void entry_record(const DevVolume& v, const BatchArgs& a, unsigned long long e,
                                             uint32_t& id, long long& fix) {
    if constexpr (S == kStoreF64) {
        id = slot_record_f64(v, a, (uint32_t)e, fix);
    } else {
        id = (uint32_t)e;
        fix = to_fix(__uint_as_float((uint32_t)(e >> 32)));
    }
}

template <int S>
__device__ __forceinline__ uint32_t entry_id(const DevVolume& v, const BatchArgs& a, unsigned long long e) {
    if constexpr (S == kStoreF64)
        return slot_id((uint32_t)e, (uint32_t)a.n, 2u * (uint32_t)v.steps + 1u);
    else
        return (uint32_t)e;
}

// What the selection of one cap-crossing voxel touches, as plain values: an
// out-of-line selection takes these, so no kernel parameter is passed by
// address (which would make every thread copy it to local memory).
struct SelectArgs {
    float* tsdf;
    float* weight;
    float* r;
    float* g;
    float* b;
    unsigned long long* vacc;
    uint32_t* vcnt;
    const unsigned long long* grp;
    int64_t record_cap;
    uint32_t* status;
    float cap;  // effective weight cap
};

__device__ __forceinline__ SelectArgs select_args(const DevVolume& v, const UpdateScratch& u) {
    return SelectArgs{v.tsdf, v.weight, v.r, v.g, v.b, u.vacc, u.vcnt, u.grp, u.record_cap, u.status, v.weight_cap};
}

// Finish a cap-crossing voxel: keep contributions accepted, their values
// summing to fix * 2^-40.
template <int S>
__device__ __forceinline__ void finish_voxel(const SelectArgs& v, uint32_t vi, int keep, long long fix) {
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
    v.vacc[vi] = 0ull;
    v.vcnt[vi] = 0u;
}

// The weight of voxel vi before the batch (finish leaves crossing voxels as they were).
template <int S>
__device__ __forceinline__ float weight_before(const SelectArgs& v, uint32_t vi) {
    if constexpr (S == kStoreF16U16)
        return (float)__ldg(reinterpret_cast<const unsigned short*>(v.weight) + vi);
    else
        return __ldg(v.weight + vi);
}

// Sum of the accepted values of a group of at most 32 * R records, by one
// warp: record r * 32 + lane in registers, ranked by id against every other
// record with shuffles; a record is accepted when fewer than keep ids are
// below its own. Ids are distinct and below 0xFFFFFFFF, so the padding
// entries never rank below a record. Entries are read through L2: they were
// stored by other threads of this grid.
template <int S, int R>
__device__ __forceinline__ long long rank_group(const DevVolume& v, const BatchArgs& a,
                                                const unsigned long long* grp, int n, int keep, int lane) {
    uint32_t id[R];
    long long val[R];
    int rank[R];
#pragma unroll
    for (int r = 0; r < R; ++r) {
        const int k = r * 32 + lane;
        id[r] = 0xFFFFFFFFu;
        val[r] = 0ll;
        rank[r] = 0;
        if (k < n) entry_record<S>(v, a, __ldcg(grp + k), id[r], val[r]);
    }
#pragma unroll
    for (int rr = 0; rr < R; ++rr) {
        const int srcs = min(32, n - rr * 32);  // warp-uniform
        for (int src = 0; src < srcs; ++src) {
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

// The keep-th smallest id (1-based) of a group, by four 8-bit radix passes
// with a per-warp histogram. Ids are distinct, so exactly keep ids are <= it.
template <int S>
__device__ uint32_t radix_select(const DevVolume& v, const BatchArgs& a, const unsigned long long* grp,
                                 int n, int keep, uint32_t* hist, int lane) {
    uint32_t prefix = 0u, pmask = 0u;
    int need = keep;
    for (int shift = 24; shift >= 0; shift -= 8) {
        for (int b = lane; b < 256; b += 32) hist[b] = 0u;
        __syncwarp();
        for (int k = lane; k < n; k += 32) {
            const uint32_t id = entry_id<S>(v, a, __ldcg(grp + k));
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

// Sum of the accepted values of a group of more than 32 records, by one
// warp.
template <int S>
__device__ __forceinline__ long long large_group_sum(const DevVolume& v, const BatchArgs& a,
                                                     const unsigned long long* grp, int n, int keep,
                                                     uint32_t* hist, int lane) {
    if (n <= 64) return rank_group<S, 2>(v, a, grp, n, keep, lane);
    if (n <= 128) return rank_group<S, 4>(v, a, grp, n, keep, lane);
    if (n <= 32 * kRankRegs) return rank_group<S, kRankRegs>(v, a, grp, n, keep, lane);
    const uint32_t last = radix_select<S>(v, a, grp, n, keep, hist, lane);
    long long fix = 0ll;
    for (int k = lane; k < n; k += 32) {
        uint32_t id;
        long long val;
        entry_record<S>(v, a, __ldcg(grp + k), id, val);
        if (id <= last) fix += val;
    }
    return fix;
}

// Select and finish the cap-crossing voxel vi whose group is complete, by
// the whole warp (vi is warp-uniform). The sum word now holds the group's
// base + 1 and its size. Returns 1 on lane 0 (the voxel it finished), else 0.
// v and a are read only by the FP64 oracle, whose entries carry band slots.
template <int S>
__device__ __forceinline__ int select_group(const SelectArgs& sa, const DevVolume& v, const BatchArgs& a,
                                            uint32_t vi, uint32_t* hist, int lane) {
    // Fused selection: the group's other records were placed by other
    // threads of this pass, each with a fence between its entry stores and
    // its countdown; this fence orders the reads below after the countdown
    // that saw the group complete.
    if (!OSN_SPLIT_SELECT) __threadfence();
    const unsigned long long h = __ldcg(&sa.vacc[vi]);
    const uint32_t base = (uint32_t)(h >> 32) - 1u;
    const int n = (int)(uint32_t)h;
    const int keep = accept_count(weight_before<S>(sa, vi), sa.cap, n);
    long long fix = 0ll;
    if ((uint64_t)base + (uint64_t)n > (uint64_t)sa.record_cap) {
        // Counters left by a failed update: nothing to rank.
        if (lane == 0) atomicOr(sa.status, kStatusScratchOverflow);
    } else {
        const unsigned long long* grp = sa.grp + base;
        fix = n <= 32 ? rank_group<S, 1>(v, a, grp, n, keep, lane)
                      : large_group_sum<S>(v, a, grp, n, keep, hist, lane);
    }
    for (int o = 16; o > 0; o >>= 1) fix += __shfl_xor_sync(0xffffffffu, fix, o);
    if (lane != 0) return 0;
    finish_voxel<S>(sa, vi, keep, fix);
    return 1;
}

// The same out of line for the storages whose entries carry their values
// (no volume or batch needed): the selection runs about once per warp, so
// the scan of the band slots keeps its few registers and its occupancy.
template <int S>
__device__ __noinline__ int select_group_out(const SelectArgs sa, uint32_t vi, uint32_t* hist, int lane) {
    static_assert(S != kStoreF64, "the FP64 oracle recomputes values from its batch");
    return select_group<S>(sa, DevVolume{}, BatchArgs{}, vi, hist, lane);
}

// Eight band slots from `first` of one batch, by every thread of the warp
// (warp-synchronous): records of voxels whose crossing bit is set take their
// place in the voxel's group; the warp then selects and finishes every group
// one of its records completed.
// The records of eight band slots from `first` (kNoVoxel past the batch).
__device__ __forceinline__ void load_records(const UpdateScratch& u, uint32_t first, uint32_t n_slots,
                                             uint32_t (&vi)[kGroupPerThread]) {
    if (first + kGroupPerThread <= n_slots) {
        // Eight consecutive band slots: one step, neighbouring points.
        const uint4 r0 = __ldcs(reinterpret_cast<const uint4*>(u.records + first));
        const uint4 r1 = __ldcs(reinterpret_cast<const uint4*>(u.records + first) + 1);
        vi[0] = r0.x; vi[1] = r0.y; vi[2] = r0.z; vi[3] = r0.w;
        vi[4] = r1.x; vi[5] = r1.y; vi[6] = r1.z; vi[7] = r1.w;
    } else {
#pragma unroll
        for (int m = 0; m < kGroupPerThread; ++m)
            vi[m] = first + m < n_slots ? u.records[first + m] : kNoVoxel;
    }
}

// Records of voxels whose crossing bit is set take their place in the
// voxel's group; returns bit m set for slot m placed.
template <int S>
__device__ __forceinline__ uint32_t place_records(const BatchArgs& a, const DevVolume& v, const UpdateScratch& u,
                                                  uint32_t first, const uint32_t (&vi)[kGroupPerThread]) {
    // Crossing bits: one gather per distinct bitmap word among the eight.
    uint32_t word[kGroupPerThread];
    bool same[kGroupPerThread];
#pragma unroll
    for (int m = 0; m < kGroupPerThread; ++m) {
        same[m] = m > 0 && vi[m] != kNoVoxel && vi[m - 1] != kNoVoxel && (vi[m - 1] >> 5) == (vi[m] >> 5);
        word[m] = (vi[m] == kNoVoxel || same[m]) ? 0u : __ldg(&u.xbits[vi[m] >> 5]);
    }
#pragma unroll
    for (int m = 1; m < kGroupPerThread; ++m)
        if (same[m]) word[m] = word[m - 1];
    const uint32_t n_steps = 2u * (uint32_t)v.steps + 1u;
    uint32_t placed = 0u;  // bit m: slot m's record took a place in its group
#pragma unroll
    for (int m = 0; m < kGroupPerThread; ++m) {
        if (vi[m] == kNoVoxel || !((word[m] >> (vi[m] & 31u)) & 1u)) continue;
        const uint32_t slot = first + m;
        // The record's value (FP32 / FP16: the walk kept it) is loaded beside
        // its place ticket, in the same round trip.
        float val = 0.0f;
        if constexpr (S != kStoreF64) val = __ldcs(u.slot_val + slot);
        const unsigned long long tk = atomicAdd(&u.vacc[vi[m]], 1ull);
        const uint64_t pos = (uint64_t)((uint32_t)(tk >> 32) - 1u) + (uint32_t)tk;
        unsigned long long e;
        if constexpr (S == kStoreF64)
            e = slot;
        else
            e = (unsigned long long)slot_id(slot, (uint32_t)a.n, n_steps) |
                ((unsigned long long)__float_as_uint(val) << 32);
        if (pos < (uint64_t)u.record_cap) u.grp[pos] = e;
        else atomicOr(u.status, kStatusScratchOverflow);  // state left by a failed update
        placed |= 1u << m;
    }
    return placed;
}

template <int S>
__device__ __forceinline__ void group_slots(const DevVolume& v, const BatchArgs& a, const UpdateScratch& u,
                                            uint32_t first, uint32_t n_slots, uint32_t* hist, int& updated) {
    const int lane = threadIdx.x & 31;
    uint32_t vi[kGroupPerThread];
    load_records(u, first, n_slots, vi);
    const uint32_t placed = place_records<S>(a, v, u, first, vi);
    if (OSN_SPLIT_SELECT) return;  // the select pass ranks the complete groups
    // Fused selection: this thread's entries are visible before its
    // countdowns; the record that brings a count to zero completed its group.
    uint32_t last = 0u;  // bit m: slot m's record completed its voxel's group
    if (placed) {
        __threadfence();
#pragma unroll
        for (int m = 0; m < kGroupPerThread; ++m)
            if (((placed >> m) & 1u) && atomicSub(&u.vcnt[vi[m]], 1u) == 1u) last |= 1u << m;
    }
    // Every group completed here is selected by the whole warp, one at a
    // time, lowest lane first.
    while (__any_sync(0xffffffffu, last != 0u)) {
        const int src = __ffs(__ballot_sync(0xffffffffu, last != 0u)) - 1;
        uint32_t pick = kNoVoxel;
        bool got = false;
#pragma unroll
        for (int m = 0; m < kGroupPerThread; ++m)
            if (!got && ((last >> m) & 1u)) {
                pick = vi[m];
                got = true;
            }
        if (lane == src) last &= last - 1u;  // its lowest pending group
        const uint32_t gv = __shfl_sync(0xffffffffu, pick, src);
        if constexpr (S == kStoreF64)
            updated += select_group<S>(select_args(v, u), v, a, gv, hist, lane);
        else
            updated += select_group_out<S>(select_args(v, u), gv, hist, lane);
    }
}

template <int S>
__global__ void __launch_bounds__(kGroupThreads, OSN_GROUP_MIN_BLOCKS)
group_kernel(DevVolume v, BatchArgs a, UpdateScratch u, uint32_t n_slots) {
    launch_dependents();
    grid_dependency_wait();
    if (u.ctl->n_crossing == 0ull) return;  // no voxel crossed the cap in this batch
    if (OSN_SPLIT_SELECT) {
        // Placing only: no voxel is finished here, so there is nothing to
        // count and no CTA barrier (each warp leaves when its slots are done).
        if (OSN_GROUP_PERSISTENT) {
            // Persistent grid: each thread walks chunks of eight slots a grid
            // apart, the next chunk's records loaded before this one's are placed.
            const uint32_t stride = gridDim.x * kGroupThreads * kGroupPerThread;
            uint32_t first = (blockIdx.x * kGroupThreads + threadIdx.x) * kGroupPerThread;
            uint32_t cur[kGroupPerThread], nxt[kGroupPerThread];
            load_records(u, first, n_slots, cur);
            for (; first < n_slots; first += stride) {
                load_records(u, first + stride, n_slots, nxt);
                place_records<S>(a, v, u, first, cur);
#pragma unroll
                for (int m = 0; m < kGroupPerThread; ++m) cur[m] = nxt[m];
            }
        } else {
            const uint32_t first = (blockIdx.x * kGroupThreads + threadIdx.x) * kGroupPerThread;
            uint32_t vi[kGroupPerThread];
            load_records(u, first, n_slots, vi);
            place_records<S>(a, v, u, first, vi);
        }
        return;
    }
    __shared__ uint32_t hist[kGroupWarps][256];
    __shared__ int s_updated;
    if (threadIdx.x == 0) s_updated = 0;
    __syncthreads();
    int updated = 0;
    group_slots<S>(v, a, u, (blockIdx.x * kGroupThreads + threadIdx.x) * kGroupPerThread, n_slots,
                   hist[threadIdx.x >> 5], updated);
    cta_add(&s_updated, updated, &u.ctl->n_updated);
}

constexpr int kSelectChunk = 32;   // voxels whose headers a warp loads together (one per lane)
constexpr int kSelectAhead = 4;    // groups whose entries are in flight ahead of the ranking

// Entry `lane` of group j of a chunk (groups of at most 32 records; none for
// larger or invalid groups).
__device__ __forceinline__ unsigned long long chunk_entry(const SelectArgs& sa, uint32_t base, int cnt, int j,
                                                          int m, int lane) {
    const int src = j < m ? j : 0;
    const uint32_t bj = __shfl_sync(0xffffffffu, base, src);
    const int cj = __shfl_sync(0xffffffffu, cnt, src);
    return (j < m && lane < cj && cj <= 32) ? __ldcg(sa.grp + bj + lane) : ~0ull;
}

// The ordered selection of listed crossing voxels d0, d0 + step, ... < end
// by one warp (FP32 / FP16 storage). The warp takes up to 32 of them at a
// time, lane k owning the k-th: each lane loads its voxel's list entry,
// then its group header (base, size), weight and stored TSDF, all lanes
// together; the warp then ranks the groups in order, each group's entries
// (at most 32 records: one per lane) loaded four groups ahead of the
// ranking, larger groups by the whole warp on the spot; finally each lane
// finishes its own voxel from the values it already holds. Returns the
// voxels this lane finished.
template <int S>
__device__ __forceinline__ int select_stream(const SelectArgs& sa, const uint32_t* xlist, long long d0,
                                             long long end, long long step, uint32_t* hist, int lane) {
    static_assert(S != kStoreF64, "the FP64 oracle ranks one voxel at a time");
    int done = 0;
    for (long long c0 = d0; c0 < end; c0 += kSelectChunk * step) {
        const long long dk = c0 + (long long)lane * step;
        const bool mine = dk < end;
        const uint32_t vi = mine ? xlist[dk] : 0u;
        unsigned long long h = 0ull;
        float w0 = 0.0f, t0 = 0.0f;
        if (mine) {
            h = __ldcg(&sa.vacc[vi]);
            if constexpr (S == kStoreF16U16) {
                w0 = (float)reinterpret_cast<const unsigned short*>(sa.weight)[vi];
                t0 = __half2float(reinterpret_cast<const __half*>(sa.tsdf)[vi]);
            } else {
                w0 = sa.weight[vi];
                t0 = sa.tsdf[vi];
            }
        }
        const uint32_t base = (uint32_t)(h >> 32) - 1u;
        const bool valid = mine && (uint64_t)base + (uint64_t)(uint32_t)h <= (uint64_t)sa.record_cap;
        if (mine && !valid) atomicOr(sa.status, kStatusScratchOverflow);  // counters left by a failed update
        const int cnt = valid ? (int)(uint32_t)h : 0;
        const int keep = accept_count(w0, sa.cap, cnt);
        const int m = (int)min((long long)kSelectChunk, (end - c0 + step - 1) / step);  // warp-uniform
        unsigned long long e0 = chunk_entry(sa, base, cnt, 0, m, lane);
        unsigned long long e1 = chunk_entry(sa, base, cnt, 1, m, lane);
        unsigned long long e2 = chunk_entry(sa, base, cnt, 2, m, lane);
        unsigned long long e3 = chunk_entry(sa, base, cnt, 3, m, lane);
        long long my_fix = 0ll;
        for (int j = 0; j < m; ++j) {
            const unsigned long long ej = e0;
            e0 = e1;
            e1 = e2;
            e2 = e3;
            e3 = chunk_entry(sa, base, cnt, j + kSelectAhead, m, lane);
            const int cj = __shfl_sync(0xffffffffu, cnt, j);
            const int kj = __shfl_sync(0xffffffffu, keep, j);
            long long fix = 0ll;
            if (cj <= 32) {  // warp-uniform
                // Padding ids (0xFFFFFFFF) never rank below a record, so the
                // ids are read four lanes at a time up to the group's size.
                const uint32_t id = lane < cj ? (uint32_t)ej : 0xFFFFFFFFu;
                int rank = 0;
                for (int q = 0; q < cj; q += 4) {
#pragma unroll
                    for (int r = 0; r < 4; ++r) rank += __shfl_sync(0xffffffffu, id, q + r) < id ? 1 : 0;
                }
                if (lane < cj && rank < kj) fix = to_fix(__uint_as_float((uint32_t)(ej >> 32)));
                // One value per lane, |fix| <= 2^40: the warp sums of the
                // 20-bit low parts and of the high parts fit 26 bits.
                const uint32_t lo = __reduce_add_sync(0xffffffffu, (uint32_t)fix & 0xFFFFFu);
                const int32_t hi = (int32_t)__reduce_add_sync(0xffffffffu, (uint32_t)(int32_t)(fix >> 20));
                fix = ((long long)hi << 20) + (long long)lo;
            } else {
                const uint32_t bj = __shfl_sync(0xffffffffu, base, j);
                fix = large_group_sum<S>(DevVolume{}, BatchArgs{}, sa.grp + bj, cj, kj, hist, lane);
                for (int o = 16; o > 0; o >>= 1) fix += __shfl_xor_sync(0xffffffffu, fix, o);
            }
            if (lane == j) my_fix = fix;
        }
        if (!mine) continue;
        // Finish the lane's voxel (finish_voxel with the values already loaded).
        const int k = valid ? keep : 0;
        const long long f = valid ? my_fix : 0ll;
        if constexpr (S == kStoreF32) {
            const float wn = __fadd_rn(w0, (float)k);
            sa.tsdf[vi] = add_fix(t0, f);
            sa.weight[vi] = wn;
            const float c = __fmul_rn(128.0f, wn);
            sa.r[vi] = c;
            sa.g[vi] = c;
            sa.b[vi] = c;
        } else {
            reinterpret_cast<__half*>(sa.tsdf)[vi] = __float2half_rn(new_mean_f16(t0, w0, k, f));
            reinterpret_cast<unsigned short*>(sa.weight)[vi] = (unsigned short)__fadd_rn(w0, (float)k);
        }
        sa.vacc[vi] = 0ull;
        sa.vcnt[vi] = 0u;
        ++done;
    }
    return done;
}

// The ordered selection of every cap-crossing voxel of the batch, from the
// list finish wrote (OSN_SPLIT_SELECT): warp w takes voxels w, w + warps,
// ... (so large groups spread over the grid); the FP64 oracle storage, one
// voxel at a time.
template <int S>
__global__ void __launch_bounds__(kSelectThreads)
select_kernel(DevVolume v, BatchArgs a, UpdateScratch u) {
    __shared__ uint32_t hist[kSelectWarps][256];
    __shared__ int s_updated;
    if (threadIdx.x == 0) s_updated = 0;
    __syncthreads();
    launch_dependents();
    grid_dependency_wait();
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const long long n = min((long long)u.ctl->n_crossing, (long long)u.xlist_cap);
    const SelectArgs sa = select_args(v, u);
    const long long gw = (long long)blockIdx.x * kSelectWarps + warp, nw = (long long)gridDim.x * kSelectWarps;
    int updated = 0;
    if constexpr (S == kStoreF64) {
        for (long long d = gw; d < n; d += nw) updated += select_group<S>(sa, v, a, u.xlist[d], hist[warp], lane);
    } else {
        updated += select_stream<S>(sa, u.xlist, gw, n, nw, hist[warp], lane);
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
enum MultiPass : int { kPassFinishPairs, kPassFinishSingle, kPassGroup, kPassSelect };

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
    if (c->n_crossing == 0ull) return 0;  // no voxel crossed the cap in this scene
    if (PASS == kPassSelect) {
        const long long x = min((long long)c->n_crossing, (long long)sw.u.xlist_cap);
        return (int)(sw.v.storage == kStoreF64 ? x : (x + kSelectChunk - 1) / kSelectChunk);  // voxels, or chunks
    }
    return (int)(((uint32_t)sw.n_slots + kGroupThreads * kGroupPerThread - 1) /
                 (kGroupThreads * kGroupPerThread));
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
        if (t == 0) tag_chunk(sw.v, ba, bb, has_b);
        finish_quad<S>(sw.v, sw.u, ba, qa, t, lane, ca, xa, a01, a23, updated);
        if (has_b) finish_quad<S>(sw.v, sw.u, bb, qb, t, lane, cb, xb, b01, b23, updated);
        __syncthreads();  // s_item and the descriptor are rewritten next
    }
}

// Group, select and finish the cap-crossing voxels of every scene that has
// any: work items of 2048 band slots of one scene.
template <int S>
__global__ void __launch_bounds__(kGroupThreads, OSN_GROUP_MIN_BLOCKS)
group_multi_kernel(StepWork w) {
    __shared__ SceneWork sw;
    __shared__ uint32_t hist[kGroupWarps][256];
    __shared__ int s_begin[kMaxBatchScenes + 1];
    __shared__ int s_item, s_updated;
    const int t = threadIdx.x, lane = t & 31;
    launch_dependents();
    grid_dependency_wait();
    if (t == 0) s_updated = 0;
    scene_prefix<kPassGroup>(w, s_begin);
    const int total = s_begin[w.n_scenes];
    int cur = -1, updated = 0;
    for (;;) {
        if (t == 0) s_item = (int)atomicAdd(&w.queues[kQGroup], 1u);
        __syncthreads();
        const int item = s_item;
        const bool done = item >= total;
        const int sc = done ? -1 : scene_of(s_begin, w.n_scenes, item);
        if (sc != cur || done) {
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
        const uint32_t first = ((uint32_t)(item - s_begin[sc]) * kGroupThreads + t) * kGroupPerThread;
        group_slots<S>(sw.v, sw.a, sw.u, first, (uint32_t)sw.n_slots, hist[t >> 5], updated);
        __syncthreads();
    }
}

// The ordered selection of every scene's cap-crossing voxels: warp work
// items, one per listed voxel (OSN_SPLIT_SELECT).
template <int S>
__global__ void __launch_bounds__(kSelectThreads)
select_multi_kernel(StepWork w) {
    __shared__ uint32_t hist[kSelectWarps][256];
    __shared__ int s_begin[kMaxBatchScenes + 1];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    launch_dependents();
    grid_dependency_wait();
    scene_prefix<kPassSelect>(w, s_begin);
    const int total = s_begin[w.n_scenes];
    for (;;) {
        int item = 0;
        if (lane == 0) item = (int)atomicAdd(&w.queues[kQSelect], 1u);
        item = __shfl_sync(0xffffffffu, item, 0);
        if (item >= total) break;
        const int sc = scene_of(s_begin, w.n_scenes, item);
        const SceneWork& sw = w.scenes[sc];
        const SelectArgs sa = select_args(sw.v, sw.u);
        int done;
        if constexpr (S == kStoreF64) {
            done = select_group<S>(sa, sw.v, sw.a, sw.u.xlist[item - s_begin[sc]], hist[warp], lane);
        } else {
            const long long n = min((long long)sw.u.ctl->n_crossing, (long long)sw.u.xlist_cap);
            const long long c0 = (long long)kSelectChunk * (item - s_begin[sc]);
            done = select_stream<S>(sa, sw.u.xlist, c0, min(n, c0 + kSelectChunk), 1, hist[warp], lane);
        }
        done = __reduce_add_sync(0xffffffffu, done);
        if (lane == 0 && done) atomicAdd(&sw.u.ctl->n_updated, done);
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

cudaError_t launch_group(const DevVolume& v, const BatchArgs& a, const UpdateScratch& u, int sm_count,
                         cudaStream_t s) {
    const uint32_t n_slots = (uint32_t)a.n * (2u * (uint32_t)v.steps + 1u);
    if (n_slots == 0) return cudaSuccess;
    const uint32_t per_cta = kGroupThreads * (uint32_t)kGroupPerThread;
    uint32_t grid = (n_slots + per_cta - 1u) / per_cta;
    if (OSN_SPLIT_SELECT && OSN_GROUP_PERSISTENT) {  // persistent: at most one resident wave
        const int res = v.storage == kStoreF16U16 ? resident_grid<group_kernel<kStoreF16U16>>(kGroupThreads, sm_count)
                        : v.storage == kStoreF64  ? resident_grid<group_kernel<kStoreF64>>(kGroupThreads, sm_count)
                                                  : resident_grid<group_kernel<kStoreF32>>(kGroupThreads, sm_count);
        grid = std::min<uint32_t>(grid, (uint32_t)res);
    }
    switch (v.storage) {
        case kStoreF16U16: return launch_after(group_kernel<kStoreF16U16>, grid, kGroupThreads, s, v, a, u, n_slots);
        case kStoreF64: return launch_after(group_kernel<kStoreF64>, grid, kGroupThreads, s, v, a, u, n_slots);
        default: return launch_after(group_kernel<kStoreF32>, grid, kGroupThreads, s, v, a, u, n_slots);
    }
}

cudaError_t launch_select(const DevVolume& v, const BatchArgs& a, const UpdateScratch& u, int sm_count,
                          cudaStream_t s) {
    if (!OSN_SPLIT_SELECT) return cudaSuccess;  // the group pass selects
    switch (v.storage) {
        case kStoreF16U16:
            return launch_after(select_kernel<kStoreF16U16>,
                                resident_grid<select_kernel<kStoreF16U16>>(kSelectThreads, sm_count),
                                kSelectThreads, s, v, a, u);
        case kStoreF64:
            return launch_after(select_kernel<kStoreF64>, resident_grid<select_kernel<kStoreF64>>(kSelectThreads, sm_count),
                                kSelectThreads, s, v, a, u);
        default:
            return launch_after(select_kernel<kStoreF32>, resident_grid<select_kernel<kStoreF32>>(kSelectThreads, sm_count),
                                kSelectThreads, s, v, a, u);
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
cudaError_t select_multi_t(const StepWork& w, int sm_count, cudaStream_t s) {
    return launch_after(select_multi_kernel<S>, resident_grid<select_multi_kernel<S>>(kSelectThreads, sm_count),
                        kSelectThreads, s, w);
}
template <int S>
cudaError_t group_multi_t(const StepWork& w, int sm_count, cudaStream_t s) {
    return launch_after(group_multi_kernel<S>, resident_grid<group_multi_kernel<S>>(kGroupThreads, sm_count),
                        kGroupThreads, s, w);
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

cudaError_t launch_group_multi(const StepWork& w, int storage, int sm_count, cudaStream_t s) {
    switch (storage) {
        case kStoreF16U16: return group_multi_t<kStoreF16U16>(w, sm_count, s);
        case kStoreF64: return group_multi_t<kStoreF64>(w, sm_count, s);
        default: return group_multi_t<kStoreF32>(w, sm_count, s);
    }
}

}  // namespace osn_b200

namespace osn_b200 {
cudaError_t launch_select_multi(const StepWork& w, int storage, int sm_count, cudaStream_t s) {
    if (!OSN_SPLIT_SELECT) return cudaSuccess;  // the group pass selects
    switch (storage) {
        case kStoreF16U16: return select_multi_t<kStoreF16U16>(w, sm_count, s);
        case kStoreF64: return select_multi_t<kStoreF64>(w, sm_count, s);
        default: return select_multi_t<kStoreF32>(w, sm_count, s);
    }
}
}  // namespace osn_b200
