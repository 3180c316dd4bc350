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
//   group      one pass over the records of the batch: a record of a tagged
//              block whose voxel reserved a group puts its slot in the next
//              place of the group (a few percent of the records).
//   deferred   one warp per crossing voxel: each lane recomputes the
//              canonical id and normalised SDF of its records from their
//              points (the walk's arithmetic, same rounding), then the warp
//              selects the keep records with the smallest ids (ranking in
//              registers up to 256 records, a radix select of the keep-th id
//              beyond that) and finishes the voxel.
//
// Sums are 64-bit fixed point added to the stored sum with one rounding, so
// results do not depend on the order in which threads meet the records:
// repeated runs are bit-identical, and a voxel with one contribution per
// batch gets exactly the reference's fl(tsdf + sdf_n).
#include "volume.h"

namespace osn_b200 {
namespace {

constexpr int kFinishThreads = 128;  // 4 voxels per thread, one block per CTA pass
constexpr int kGroupThreads = 256;
constexpr int kDeferThreads = 256;
constexpr int kDeferWarps = kDeferThreads / 32;
constexpr int kRankRegs = 8;  // crossing voxels of up to 256 records are ranked in registers

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

// ---- finish --------------------------------------------------------------

__global__ void __launch_bounds__(kFinishThreads)
finish_kernel(DevVolume v, UpdateScratch u) {
    const int t = threadIdx.x;
    const int n_touched = min(u.ctl->n_touched, v.pool_capacity);
    int updated = 0;
    for (int item = blockIdx.x; item < n_touched; item += gridDim.x) {
        const int32_t bi = u.touched[item];
        const size_t q4 = (size_t)bi * (kBlockVoxels / 4) + t;  // this thread's 4 voxels
        const uint4 c4 = reinterpret_cast<const uint4*>(u.vcnt)[q4];
        if ((c4.x | c4.y | c4.z | c4.w) == 0u) continue;
        const float4 w4 = reinterpret_cast<const float4*>(v.weight)[q4];
        const float4 t4 = reinterpret_cast<const float4*>(v.tsdf)[q4];
        const ulonglong2 a01 = reinterpret_cast<const ulonglong2*>(u.vacc)[2 * q4];
        const ulonglong2 a23 = reinterpret_cast<const ulonglong2*>(u.vacc)[2 * q4 + 1];
        const uint32_t n[4] = {c4.x, c4.y, c4.z, c4.w};
        const float w0[4] = {w4.x, w4.y, w4.z, w4.w};
        float tn[4] = {t4.x, t4.y, t4.z, t4.w};
        float wn[4];
        unsigned long long acc[4] = {a01.x, a01.y, a23.x, a23.y};
        uint32_t cnt[4];
        bool crossing = false;
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            wn[q] = w0[q];
            cnt[q] = 0u;
            if (n[q] == 0u) continue;
            const int keep = accept_count(w0[q], v.weight_cap, (int)n[q]);
            if ((uint32_t)keep == n[q]) {
                tn[q] = add_fix(tn[q], (long long)acc[q]);
                wn[q] = __fadd_rn(w0[q], (float)keep);
                acc[q] = 0ull;
                ++updated;
            } else {
                // Crosses the cap: reserve a group for its records; the
                // group pass fills it and the deferred kernel finishes it.
                const uint32_t vi = (uint32_t)bi * kBlockVoxels + 4u * t + q;
                const uint32_t base = atomicAdd(&u.ctl->x_used, n[q]);
                const int d = atomicAdd(&u.ctl->n_deferred, 1);
                if ((uint64_t)base + n[q] <= (uint64_t)u.record_cap && d < u.dvox_cap) {
                    u.dvox[d] = make_int4((int)vi, (int)base, (int)n[q], keep);
                    acc[q] = (unsigned long long)(base + 1u) << 32;  // low half: fill ticket
                    cnt[q] = n[q];
                } else {
                    atomicOr(v.status, kStatusScratchOverflow);
                    acc[q] = 0ull;
                }
                crossing = true;
            }
        }
        if (crossing) u.blk_cross[bi] = u.tag;
        reinterpret_cast<float4*>(v.tsdf)[q4] = make_float4(tn[0], tn[1], tn[2], tn[3]);
        reinterpret_cast<float4*>(v.weight)[q4] = make_float4(wn[0], wn[1], wn[2], wn[3]);
        const float4 c = make_float4(__fmul_rn(128.0f, wn[0]), __fmul_rn(128.0f, wn[1]),
                                     __fmul_rn(128.0f, wn[2]), __fmul_rn(128.0f, wn[3]));
        __stcs(reinterpret_cast<float4*>(v.r) + q4, c);  // write-only: keep them out of L2
        __stcs(reinterpret_cast<float4*>(v.g) + q4, c);
        __stcs(reinterpret_cast<float4*>(v.b) + q4, c);
        reinterpret_cast<uint4*>(u.vcnt)[q4] = make_uint4(cnt[0], cnt[1], cnt[2], cnt[3]);
        reinterpret_cast<ulonglong2*>(u.vacc)[2 * q4] = make_ulonglong2(acc[0], acc[1]);
        reinterpret_cast<ulonglong2*>(u.vacc)[2 * q4 + 1] = make_ulonglong2(acc[2], acc[3]);
    }
    const unsigned total = __reduce_add_sync(0xffffffffu, (unsigned)updated);
    if ((t & 31) == 0 && total) atomicAdd(&u.ctl->n_updated, (int)total);
}

// ---- group ---------------------------------------------------------------

__global__ void __launch_bounds__(kGroupThreads)
group_kernel(UpdateScratch u, uint32_t n_slots) {
    if (u.ctl->n_deferred == 0) return;  // no voxel crossed the cap in this batch
    // Four records per thread, phase by phase: the block-tag gathers of all
    // four in flight together, then the (rare) records of crossing voxels
    // take the next place of their voxel's group.
    const uint32_t q = blockIdx.x * kGroupThreads + threadIdx.x;  // quad of slots
    if (4u * q >= n_slots) return;
    uint32_t vi[4];
    if (4u * q + 3u < n_slots) {
        const uint4 r = __ldcs(reinterpret_cast<const uint4*>(u.records) + q);
        vi[0] = r.x;
        vi[1] = r.y;
        vi[2] = r.z;
        vi[3] = r.w;
    } else {
#pragma unroll
        for (uint32_t m = 0; m < 4u; ++m) vi[m] = 4u * q + m < n_slots ? u.records[4u * q + m] : kNoVoxel;
    }
    bool cand[4];
#pragma unroll
    for (int m = 0; m < 4; ++m)
        cand[m] = vi[m] != kNoVoxel && u.blk_cross[vi[m] / kBlockVoxels] == u.tag;
    uint32_t hi[4];
#pragma unroll
    for (int m = 0; m < 4; ++m) hi[m] = cand[m] ? (uint32_t)(u.vacc[vi[m]] >> 32) : 0u;
#pragma unroll
    for (int m = 0; m < 4; ++m) {
        if (hi[m] == 0u) continue;  // not a voxel that reserved a group
        const uint32_t t = (uint32_t)atomicAdd(&u.vacc[vi[m]], 1ull);
        if (t < u.vcnt[vi[m]]) u.deferred[(size_t)(hi[m] - 1u) + t] = 4u * q + m;
        else atomicOr(u.status, kStatusScratchOverflow);  // state left by a failed update
    }
}

// ---- deferred ------------------------------------------------------------

// The keep-th smallest id (1-based) of a group, by four 8-bit radix passes
// with a per-warp histogram. Ids are distinct, so exactly keep ids are <= it.
__device__ uint32_t slot_id(const DevVolume& v, const BatchArgs& a, uint32_t slot);

__device__ uint32_t radix_select(const DevVolume& v, const BatchArgs& a, const uint32_t* X, int n,
                                 int keep, uint32_t* hist, int lane) {
    uint32_t prefix = 0u, pmask = 0u;
    int need = keep;
    for (int shift = 24; shift >= 0; shift -= 8) {
        for (int b = lane; b < 256; b += 32) hist[b] = 0u;
        __syncwarp();
        for (int k = lane; k < n; k += 32) {
            const uint32_t id = slot_id(v, a, X[k]);
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

// Canonical id and normalised SDF of the record in band slot `slot`: the
// walk's arithmetic again for this one sample (same rounding).
__device__ __forceinline__ uint32_t slot_record(const DevVolume& v, const BatchArgs& a, uint32_t slot,
                                                float& sdf_n) {
    const uint32_t n_steps = 2u * (uint32_t)v.steps + 1u;
    const uint32_t s = slot / (uint32_t)a.n, i = slot - s * (uint32_t)a.n;
    Ray r;
    int vx, vy, vz;
    float sdf = 0.0f;
    if (ray_setup(a, (int)i, r)) band_sample(v, a, r, (int)s - v.steps, vx, vy, vz, sdf);
    sdf_n = fminf(fmaxf(__fmul_rn(sdf, v.inv_trunc), -1.0f), 1.0f);
    return i * n_steps + s;
}

__device__ __forceinline__ uint32_t slot_id(const DevVolume& v, const BatchArgs& a, uint32_t slot) {
    const uint32_t s = slot / (uint32_t)a.n;
    return (slot - s * (uint32_t)a.n) * (2u * (uint32_t)v.steps + 1u) + s;
}

__global__ void __launch_bounds__(kDeferThreads)
deferred_kernel(DevVolume v, BatchArgs a, UpdateScratch u) {
    __shared__ uint32_t hist[kDeferWarps][256];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int nd = min(u.ctl->n_deferred, u.dvox_cap);
    int updated = 0;
    for (int d = blockIdx.x * kDeferWarps + warp; d < nd; d += gridDim.x * kDeferWarps) {
        const int4 e = u.dvox[d];  // (voxel, group base, records, accepted)
        const uint32_t vi = (uint32_t)e.x;
        const int n = e.z, keep = e.w;
        const uint32_t* X = u.deferred + (uint32_t)e.y;
        long long fix = 0;
        if (n <= 32 * kRankRegs) {
            // Up to 8 records per lane, ranked by id against all others.
            uint32_t id[kRankRegs];
            float val[kRankRegs];
            int rank[kRankRegs];
            const int rows = (n + 31) / 32;
#pragma unroll
            for (int r = 0; r < kRankRegs; ++r) {
                const int k = r * 32 + lane;
                id[r] = 0xFFFFFFFFu;
                val[r] = 0.0f;
                rank[r] = 0;
                if (r < rows && k < n) id[r] = slot_record(v, a, X[k], val[r]);
            }
#pragma unroll
            for (int rr = 0; rr < kRankRegs; ++rr) {
                if (rr >= rows) break;
                const int m = min(32, n - rr * 32);
                for (int src = 0; src < m; ++src) {
                    const uint32_t other = __shfl_sync(0xffffffffu, id[rr], src);
#pragma unroll
                    for (int r = 0; r < kRankRegs; ++r)
                        if (r < rows) rank[r] += other < id[r] ? 1 : 0;
                }
            }
#pragma unroll
            for (int r = 0; r < kRankRegs; ++r)
                if (r < rows && r * 32 + lane < n && rank[r] < keep) fix += to_fix(val[r]);
        } else {
            // The keep-th smallest id by radix select over the group's ids,
            // then the accepted records' values.
            const uint32_t last = radix_select(v, a, X, n, keep, hist[warp], lane);
            for (int k = lane; k < n; k += 32) {
                if (slot_id(v, a, X[k]) > last) continue;
                float val;
                slot_record(v, a, X[k], val);
                fix += to_fix(val);
            }
        }
        for (int o = 16; o > 0; o >>= 1) fix += __shfl_xor_sync(0xffffffffu, fix, o);
        if (lane == 0) {
            const float wn = __fadd_rn(v.weight[vi], (float)keep);
            v.tsdf[vi] = add_fix(v.tsdf[vi], fix);
            v.weight[vi] = wn;
            const float c = __fmul_rn(128.0f, wn);
            v.r[vi] = c;
            v.g[vi] = c;
            v.b[vi] = c;
            u.vacc[vi] = 0ull;
            u.vcnt[vi] = 0u;
            ++updated;
        }
    }
    const unsigned total = __reduce_add_sync(0xffffffffu, (unsigned)updated);
    if (lane == 0 && total) atomicAdd(&u.ctl->n_updated, (int)total);
}

}  // namespace

cudaError_t launch_finish(const DevVolume& v, const UpdateScratch& u, int n_ctas, cudaStream_t s) {
    finish_kernel<<<n_ctas, kFinishThreads, 0, s>>>(v, u);
    return cudaGetLastError();
}

cudaError_t launch_group(const DevVolume& v, const BatchArgs& a, const UpdateScratch& u,
                         cudaStream_t s) {
    const uint32_t n_slots = (uint32_t)a.n * (2u * (uint32_t)v.steps + 1u);
    if (n_slots == 0) return cudaSuccess;
    const uint32_t per_cta = kGroupThreads * 4u;
    group_kernel<<<(n_slots + per_cta - 1u) / per_cta, kGroupThreads, 0, s>>>(u, n_slots);
    return cudaGetLastError();
}

cudaError_t launch_deferred(const DevVolume& v, const BatchArgs& a, const UpdateScratch& u,
                            int n_ctas, cudaStream_t s) {
    deferred_kernel<<<n_ctas, kDeferThreads, 0, s>>>(v, a, u);
    return cudaGetLastError();
}

}  // namespace osn_b200
