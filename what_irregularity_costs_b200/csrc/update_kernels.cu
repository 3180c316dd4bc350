// Update, second half: apply the staged contributions to the block tiles.
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
//
// The count-and-stage walk (walk_kernels.cu) has staged every contribution
// that can still be accepted, in segments of consecutive records, one
// segment per (walk CTA, block), and has given each touched block the offset
// and length of its bin. Here:
//
//   bin       one warp per segment copies its records into the block's
//             contiguous bin (L2-resident traffic);
//   apply     one 128-thread CTA per touched block (persistent, work-queued,
//             many per SM), 4 voxels per thread. The block's five 2 KB tiles
//             are staged into shared memory by cp.async.bulk while the CTA
//             makes one pass over the bin: per-voxel record counts and sums,
//             combined per warp with __match_any_sync before the shared
//             atomics. A voxel accepts all of its records when w0 + n - 1 <
//             cap. Voxels that cross the cap inside the batch are resolved in
//             the CTA: their records are grouped per voxel in shared memory
//             and a warp counts each record's rank by id among its voxel's
//             records; the `keep` lowest are accepted. Blocks with more than
//             2048 records, or more crossing records than the CTA holds, go to
//   big       one 1024-thread CTA per SM and block, same algorithm, crossing
//             records gathered in groups of up to 16384.
//
// Sums are accumulated in 64-bit fixed point (2^-40 resolution, exact for
// |value| >= 2^-17) and added to the stored sum with one rounding, so results
// do not depend on the order in which threads meet the records: repeated runs
// are bit-identical, and a voxel with one contribution per batch gets exactly
// the reference's fl(tsdf + sdf_n).
#include "bulk_copy.cuh"
#include "volume.h"

namespace osn_b200 {
namespace {

constexpr int kApplyThreads = 128;  // 4 voxels per thread
constexpr int kBigThreads = 1024;   // big blocks: one CTA per SM
constexpr int kBigRecords = 2048;   // blocks above this go to the big-block apply
constexpr int kCrossCap = 1024;     // crossing records resolved inside apply
constexpr int kBigCrossCap = 16384; // crossing records resolved inside the big-block apply
constexpr double kFixScale = 1099511627776.0;      // 2^40
constexpr double kFixInv = 1.0 / 1099511627776.0;  // 2^-40

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

__device__ __forceinline__ unsigned long long to_fix(float x) {
    return (unsigned long long)__double2ll_rn((double)x * kFixScale);
}

__device__ __forceinline__ float add_fix(float t0, unsigned long long acc) {
    return __double2float_rn((double)t0 + (double)(long long)acc * kFixInv);
}

// ---- bin -----------------------------------------------------------------

__global__ void __launch_bounds__(256)
update_bin_kernel(UpdateScratch u) {
    // One warp per segment over a grid of ~19k warps, so the descriptor load
    // and the cursor atomic of many segments are in flight at once; four
    // 16-byte records per lane in flight during the copy.
    const int n = (int)min((long long)u.ctl->n_segs, (long long)u.seg_cap);
    const int lane = threadIdx.x & 31;
    const int warps = gridDim.x * (blockDim.x >> 5);
    for (int d = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); d < n; d += warps) {
        const int4 sg = u.segs[d];  // (block, staging offset, length, -)
        int at = 0;
        if (lane == 0) at = u.blk_info[sg.x].x + atomicAdd(&u.blk_cur[sg.x], sg.z);
        at = __shfl_sync(0xffffffffu, at, 0);
        const int4* src = reinterpret_cast<const int4*>(u.records + sg.y);
        int4* dst = reinterpret_cast<int4*>(u.bins + at);
        for (int k = lane; k < sg.z; k += 128) {
            int4 r[4];
#pragma unroll
            for (int q = 0; q < 4; ++q)
                if (k + 32 * q < sg.z) r[q] = src[k + 32 * q];
#pragma unroll
            for (int q = 0; q < 4; ++q)
                if (k + 32 * q < sg.z) dst[k + 32 * q] = r[q];
        }
    }
}

// ---- apply ---------------------------------------------------------------

// One pass over a bin: per-voxel record counts and fixed-point sums in
// shared memory. Four records per thread are loaded before any is used, and
// lanes holding the same voxel combine before the shared atomics.
template <int NT>
__device__ __forceinline__ void accumulate_bin(const Record* recs, int nrec, int* cnt,
                                               unsigned long long* sum) {
    constexpr int kU = 4;
    const int t = threadIdx.x, lane = t & 31;
    for (int k0 = 0; k0 < nrec; k0 += NT * kU) {
        Record rec[kU];
#pragma unroll
        for (int q = 0; q < kU; ++q) {
            const int k = k0 + q * NT + t;
            if (k < nrec) rec[q] = recs[k];
        }
#pragma unroll
        for (int q = 0; q < kU; ++q) {
            const bool ok = k0 + q * NT + t < nrec;
            const uint32_t lv = ok ? (rec[q].lv & 511u) : 0u;
            const unsigned long long fx = ok ? to_fix(__fmul_rn(rec[q].sdf_n, rec[q].w_in)) : 0ull;
            const unsigned m = __ballot_sync(0xffffffffu, ok);
            if (ok) {
                const unsigned grp = __match_any_sync(m, lv);
                unsigned long long acc = 0ull;
                for (unsigned g = grp; g; g &= g - 1) acc += __shfl_sync(grp, fx, __ffs(g) - 1);
                if (lane == __ffs(grp) - 1) {
                    atomicAdd(&cnt[lv], __popc(grp));
                    atomicAdd(&sum[lv], acc);
                }
            }
        }
    }
}

// A warp per crossing voxel: rank each of the voxel's records by id among
// them; the `keep` smallest ids are accepted and their values summed.
__device__ __forceinline__ unsigned long long ranked_sum(const uint32_t* cid, const float* cval,
                                                         int beg, int n, int keep, int lane) {
    unsigned long long acc = 0ull;
    for (int e = lane; e < n; e += 32) {
        const uint32_t ide = cid[beg + e];
        int rank = 0;
        for (int f = 0; f < n; ++f) rank += cid[beg + f] < ide ? 1 : 0;
        if (rank < keep) acc += to_fix(cval[beg + e]);
    }
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    return acc;
}

struct __align__(128) ApplySmem {
    float tile[5][kBlockVoxels];  // weight, tsdf, r, g, b (bulk-copy destination)
    uint64_t bar;
    int cnt[kBlockVoxels];
    unsigned long long sum[kBlockVoxels];
    short ci[kBlockVoxels];  // crossing index of a voxel, or -1
    short cl[kBlockVoxels];  // voxel of a crossing index
    int cstart[kBlockVoxels];
    int ccur[kBlockVoxels];
    uint32_t cid[kCrossCap];
    float cval[kCrossCap];
    int item, flags, ncv, warp_tot[kApplyThreads / 32];
};

__global__ void __launch_bounds__(kApplyThreads)
update_apply_kernel(DevVolume v, UpdateScratch u) {
    extern __shared__ __align__(128) unsigned char apply_smem[];
    ApplySmem& S = *reinterpret_cast<ApplySmem*>(apply_smem);
    const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
    const int n_touched = u.ctl->n_touched;
    if (t == 0) {
        mbar_init(&S.bar, 1);
        mbar_fence_init();
        S.flags = 0;
        S.ncv = 0;
    }
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        S.cnt[4 * t + q] = 0;
        S.sum[4 * t + q] = 0ull;
    }
    __syncthreads();

    float* const arrays[5] = {v.weight, v.tsdf, v.r, v.g, v.b};
    uint32_t round = 0;  // copies issued so far: the barrier phase to wait for
    for (;;) {
        if (t == 0) S.item = atomicAdd(&u.ctl->work, 1);
        __syncthreads();
        const int item = S.item;
        if (item >= n_touched) break;
        const int32_t bi = u.touched[item];
        const int4 info = u.blk_info[bi];  // (bin offset, records, -, -)
        if (info.y > kBigRecords) {
            if (t == 0) u.big_list[atomicAdd(&u.ctl->n_big, 1)] = bi;
            __syncthreads();  // everyone has read S.item before it is reused
            continue;         // no copy was issued for this block
        }
        if (t == 0) {
            // The previous block's tiles were last read before the barrier
            // above; order those reads before the copies overwrite them.
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            mbar_arrive_expect_tx(&S.bar, 5u * kBlockVoxels * 4u);
            for (int k = 0; k < 5; ++k)
                bulk_load(S.tile[k], arrays[k] + (size_t)bi * kBlockVoxels, kBlockVoxels * 4, &S.bar);
        }
        const Record* recs = u.bins + info.x;
        const int nrec = info.y;

        accumulate_bin<kApplyThreads>(recs, nrec, S.cnt, S.sum);
        const bool landed = mbar_wait(&S.bar, round & 1u, kSpinLimit);
        if (__syncthreads_or(!landed)) {
            if (t == 0) atomicOr(v.status, kStatusSpinTimeout);
            mbar_wait(&S.bar, round & 1u, kSpinLimit);  // the copies must land before exit
            return;
        }
        ++round;

        const float4 w0 = reinterpret_cast<const float4*>(S.tile[0])[t];
        const float4 t0 = reinterpret_cast<const float4*>(S.tile[1])[t];
        const float w0a[4] = {w0.x, w0.y, w0.z, w0.w};
        int keep[4];
        int flags = 0;
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const int n = S.cnt[4 * t + q];
            keep[q] = accept_count(w0a[q], v.weight_cap, n);
            if (keep[q] > 0) flags |= 1;
            if (keep[q] > 0 && keep[q] < n) flags |= 2;
        }
        if (flags) atomicOr(&S.flags, flags);
        __syncthreads();
        const int block_flags = S.flags;
        bool deferred = false;

        if (block_flags & 2) {
            // Ordered selection for the voxels crossing the cap.
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                const int lv = 4 * t + q;
                short ci = -1;
                if (keep[q] > 0 && keep[q] < S.cnt[lv]) {
                    ci = (short)atomicAdd(&S.ncv, 1);
                    S.cl[ci] = (short)lv;
                }
                S.ci[lv] = ci;
            }
            __syncthreads();
            const int ncv = S.ncv;
            int local[4], mine = 0;
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                const int ci = 4 * t + q;
                local[q] = ci < ncv ? S.cnt[S.cl[ci]] : 0;
                mine += local[q];
            }
            int incl = mine;
            for (int o = 1; o < 32; o <<= 1) {
                const int y = __shfl_up_sync(0xffffffffu, incl, o);
                if (lane >= o) incl += y;
            }
            if (lane == 31) S.warp_tot[warp] = incl;
            __syncthreads();
            int before = 0, total = 0;
#pragma unroll
            for (int w = 0; w < kApplyThreads / 32; ++w) {
                if (w < warp) before += S.warp_tot[w];
                total += S.warp_tot[w];
            }
            if (total > kCrossCap) {
                // More crossing records than this CTA holds: the big-block
                // CTA (room for kBigCrossCap) takes the whole block.
                deferred = true;
                if (t == 0) u.big_list[atomicAdd(&u.ctl->n_big, 1)] = bi;
            } else {
                if (t == 0) atomicAdd(&u.ctl->n_crossing, 1);
                int run = before + incl - mine;
#pragma unroll
                for (int q = 0; q < 4; ++q) {
                    const int ci = 4 * t + q;
                    if (ci < ncv) {
                        S.cstart[ci] = run;
                        S.ccur[ci] = 0;
                    }
                    run += local[q];
                }
                __syncthreads();
                for (int k = t; k < nrec; k += kApplyThreads) {
                    const Record rec = recs[k];
                    const int ci = S.ci[rec.lv & 511u];
                    if (ci < 0) continue;
                    const int pos = S.cstart[ci] + atomicAdd(&S.ccur[ci], 1);
                    S.cid[pos] = rec.id;
                    S.cval[pos] = __fmul_rn(rec.sdf_n, rec.w_in);
                }
                __syncthreads();
                for (int ci = warp; ci < ncv; ci += kApplyThreads / 32) {
                    const int lv = S.cl[ci];
                    const int n = S.cnt[lv];
                    const int k = accept_count(S.tile[0][lv], v.weight_cap, n);
                    const unsigned long long acc = ranked_sum(S.cid, S.cval, S.cstart[ci], n, k, lane);
                    if (lane == 0) S.sum[lv] = acc;
                }
            }
            __syncthreads();
        }

        if (!deferred && (block_flags & 1)) {
            const float t0a[4] = {t0.x, t0.y, t0.z, t0.w};
            float tn[4], wn[4], dc[4];
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                tn[q] = keep[q] > 0 ? add_fix(t0a[q], S.sum[4 * t + q]) : t0a[q];
                wn[q] = __fadd_rn(w0a[q], (float)keep[q]);
                dc[q] = __fmul_rn(128.0f, (float)keep[q]);
            }
            const size_t v4 = (size_t)bi * (kBlockVoxels / 4) + t;
            reinterpret_cast<float4*>(v.tsdf)[v4] = make_float4(tn[0], tn[1], tn[2], tn[3]);
            reinterpret_cast<float4*>(v.weight)[v4] = make_float4(wn[0], wn[1], wn[2], wn[3]);
#pragma unroll
            for (int ch = 0; ch < 3; ++ch) {
                float4 x = reinterpret_cast<const float4*>(S.tile[2 + ch])[t];
                x.x = __fadd_rn(x.x, dc[0]);
                x.y = __fadd_rn(x.y, dc[1]);
                x.z = __fadd_rn(x.z, dc[2]);
                x.w = __fadd_rn(x.w, dc[3]);
                reinterpret_cast<float4*>(arrays[2 + ch])[v4] = x;
            }
            if (t == 0) atomicAdd(&u.ctl->n_accepted, 1);
        }
        if (t == 0 && !deferred) u.blk_cur[bi] = 0;  // done with its bin
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            S.cnt[4 * t + q] = 0;
            S.sum[4 * t + q] = 0ull;
        }
        __syncthreads();
        if (t == 0) {
            S.flags = 0;
            S.ncv = 0;
        }
    }
}

// ---- apply, big blocks ----------------------------------------------------
//
// Blocks with more than kBigRecords records, and blocks whose cap-crossing
// records overflow the regular CTA: one 1024-thread CTA per SM (persistent
// over the big list), so a 20k-record block is one pass of ~20 records per
// thread. Threads 0-511 own one voxel each. Crossing voxels are resolved in
// the CTA as in the regular apply, in groups of up to kBigCrossCap records.
struct BigSmem {
    int cnt[kBlockVoxels];
    unsigned long long sum[kBlockVoxels];
    short ci[kBlockVoxels];
    short cl[kBlockVoxels];
    int cstart[kBlockVoxels];
    int ccur[kBlockVoxels];
    uint32_t cid[kBigCrossCap];
    float cval[kBigCrossCap];
    int item, flags, ncv, group_hi, warp_tot[kBigThreads / 32];
};

__global__ void __launch_bounds__(kBigThreads, 1)
update_apply_big_kernel(DevVolume v, UpdateScratch u) {
    extern __shared__ __align__(16) unsigned char big_smem[];
    BigSmem& S = *reinterpret_cast<BigSmem*>(big_smem);
    const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
    const int n_items = u.ctl->n_big;
    if (n_items == 0) return;
    for (int k = t; k < kBlockVoxels; k += kBigThreads) {
        S.cnt[k] = 0;
        S.sum[k] = 0ull;
    }
    if (t == 0) {
        S.flags = 0;
        S.ncv = 0;
    }
    for (;;) {
        if (t == 0) S.item = atomicAdd(&u.ctl->work_big, 1);
        __syncthreads();
        const int item = S.item;
        if (item >= n_items) break;
        const int32_t bi = u.big_list[item];
        const int4 info = u.blk_info[bi];
        const Record* recs = u.bins + info.x;
        const int nrec = info.y;
        const bool owner = t < kBlockVoxels;
        const size_t vox = (size_t)bi * kBlockVoxels + t;
        const float w0 = owner ? v.weight[vox] : 0.0f;

        accumulate_bin<kBigThreads>(recs, nrec, S.cnt, S.sum);
        __syncthreads();

        const int n = owner ? S.cnt[t] : 0;
        const int keep = owner ? accept_count(w0, v.weight_cap, n) : 0;
        const bool crossing = keep > 0 && keep < n;
        if (keep > 0) atomicOr(&S.flags, crossing ? 3 : 1);
        __syncthreads();
        const int block_flags = S.flags;

        if (block_flags & 2) {
            if (owner) {
                short ci = -1;
                if (crossing) {
                    ci = (short)atomicAdd(&S.ncv, 1);
                    S.cl[ci] = (short)t;
                }
                S.ci[t] = ci;
            }
            __syncthreads();
            const int ncv = S.ncv;
            const int mine = t < ncv ? S.cnt[S.cl[t]] : 0;
            int incl = mine;
            for (int o = 1; o < 32; o <<= 1) {
                const int y = __shfl_up_sync(0xffffffffu, incl, o);
                if (lane >= o) incl += y;
            }
            if (lane == 31) S.warp_tot[warp] = incl;
            __syncthreads();
            if (warp == 0) {
                int w = S.warp_tot[lane];
                for (int o = 1; o < 32; o <<= 1) {
                    const int y = __shfl_up_sync(0xffffffffu, w, o);
                    if (lane >= o) w += y;
                }
                S.warp_tot[lane] = w;  // inclusive per warp
            }
            __syncthreads();
            if (t == 0) atomicAdd(&u.ctl->n_crossing, 1);
            if (t < ncv) S.cstart[t] = (warp ? S.warp_tot[warp - 1] : 0) + incl - mine;
            __syncthreads();
            // Crossing voxels in groups whose records fit the buffer: one
            // pass over the bin gathers a group, warps rank its voxels.
            for (int lo = 0; lo < ncv;) {
                if (t == 0) {
                    int hi = lo + 1;
                    while (hi < ncv && S.cstart[hi] + S.cnt[S.cl[hi]] - S.cstart[lo] <= kBigCrossCap) ++hi;
                    S.group_hi = hi;
                }
                __syncthreads();
                const int hi = S.group_hi;
                const int base = S.cstart[lo];
                if (S.cnt[S.cl[lo]] <= kBigCrossCap) {
                    if (t >= lo && t < hi) S.ccur[t] = 0;
                    __syncthreads();
                    for (int k = t; k < nrec; k += kBigThreads) {
                        const Record rec = recs[k];
                        const int ci = S.ci[rec.lv & 511u];
                        if (ci < lo || ci >= hi) continue;
                        const int pos = S.cstart[ci] - base + atomicAdd(&S.ccur[ci], 1);
                        S.cid[pos] = rec.id;
                        S.cval[pos] = __fmul_rn(rec.sdf_n, rec.w_in);
                    }
                    __syncthreads();
                    for (int ci = lo + warp; ci < hi; ci += kBigThreads / 32) {
                        const int lv = S.cl[ci];
                        const int nv = S.cnt[lv];
                        const int kv = accept_count(v.weight[(size_t)bi * kBlockVoxels + lv], v.weight_cap, nv);
                        const unsigned long long acc =
                            ranked_sum(S.cid, S.cval, S.cstart[ci] - base, nv, kv, lane);
                        if (lane == 0) S.sum[lv] = acc;
                    }
                } else {
                    // One voxel with more records than the buffer holds (only
                    // an adversarial batch gets here): rank its records
                    // against the bin in global memory.
                    const int lv = S.cl[lo];
                    const int kv = accept_count(v.weight[(size_t)bi * kBlockVoxels + lv], v.weight_cap,
                                                S.cnt[lv]);
                    if (t == 0) S.sum[lv] = 0ull;
                    __syncthreads();
                    for (int k = t; k < nrec; k += kBigThreads) {
                        const Record rec = recs[k];
                        if ((int)(rec.lv & 511u) != lv) continue;
                        int rank = 0;
                        for (int f = 0; f < nrec; ++f) {
                            const Record o = recs[f];
                            rank += ((int)(o.lv & 511u) == lv && o.id < rec.id) ? 1 : 0;
                        }
                        if (rank < kv) atomicAdd(&S.sum[lv], to_fix(__fmul_rn(rec.sdf_n, rec.w_in)));
                    }
                }
                __syncthreads();
                lo = hi;
            }
        }

        if (keep > 0) {
            v.tsdf[vox] = add_fix(v.tsdf[vox], S.sum[t]);
            v.weight[vox] = __fadd_rn(w0, (float)keep);
            const float dc = __fmul_rn(128.0f, (float)keep);
            v.r[vox] = __fadd_rn(v.r[vox], dc);
            v.g[vox] = __fadd_rn(v.g[vox], dc);
            v.b[vox] = __fadd_rn(v.b[vox], dc);
        }
        if (t == 0) {
            if (block_flags & 1) atomicAdd(&u.ctl->n_accepted, 1);
            u.blk_cur[bi] = 0;  // done with its bin
        }
        if (owner) {
            S.cnt[t] = 0;
            S.sum[t] = 0ull;
        }
        __syncthreads();
        if (t == 0) {
            S.flags = 0;
            S.ncv = 0;
        }
    }
}

}  // namespace

cudaError_t launch_update_bin(const UpdateScratch& u, int n_ctas, cudaStream_t s) {
    update_bin_kernel<<<n_ctas, 256, 0, s>>>(u);
    return cudaGetLastError();
}

cudaError_t launch_update_apply(const DevVolume& v, const UpdateScratch& u, int n_ctas,
                                cudaStream_t s) {
    update_apply_kernel<<<n_ctas, kApplyThreads, sizeof(ApplySmem), s>>>(v, u);
    return cudaGetLastError();
}

cudaError_t launch_update_apply_big(const DevVolume& v, const UpdateScratch& u, int n_ctas,
                                    cudaStream_t s) {
    update_apply_big_kernel<<<n_ctas, kBigThreads, sizeof(BigSmem), s>>>(v, u);
    return cudaGetLastError();
}

cudaError_t prepare_update_kernels() {
    cudaError_t e = cudaFuncSetAttribute(update_apply_big_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)sizeof(BigSmem));
    if (e != cudaSuccess) return e;
    return cudaFuncSetAttribute(update_apply_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)sizeof(ApplySmem));
}

size_t apply_smem_bytes() { return sizeof(ApplySmem); }

}  // namespace osn_b200
