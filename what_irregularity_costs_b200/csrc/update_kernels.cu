// Update, second half: apply the binned contributions to the block tiles.
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
// segment per (walk CTA, block), and given each touched block its range of
// segment slots. Here:
//
//   place     files each segment descriptor under its block (one thread per
//             segment);
//   apply     one 128-thread CTA per touched block (persistent, work-queued),
//             4 voxels per thread, 128-bit tile loads and stores. One pass
//             over the block's segments counts each voxel's records and sums
//             their values; a voxel accepts all of them when w0 + n - 1 < cap.
//             A block in which some voxel would cross the cap inside this
//             batch is deferred, untouched, to
//   crossing  one 256-thread CTA per deferred block: an exact radix select
//             (4-bit digits over the record ids) finds the id of each
//             crossing voxel's last accepted record, then the block is
//             applied with that threshold.
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

constexpr int kCrossThreads = 256;   // two voxels per thread
constexpr int kDigitBits = 4;
constexpr int kDigits = 1 << kDigitBits;
constexpr double kFixScale = 1099511627776.0;        // 2^40
constexpr double kFixInv = 1.0 / 1099511627776.0;    // 2^-40

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

__device__ __forceinline__ unsigned long long to_fix(float sdf_n, float w_in) {
    return (unsigned long long)__double2ll_rn((double)__fmul_rn(sdf_n, w_in) * kFixScale);
}

__device__ __forceinline__ float add_fix(float t0, unsigned long long acc) {
    return __double2float_rn((double)t0 + (double)(long long)acc * kFixInv);
}

// Visit every record of a block, warp w taking segments w, w + W, ...
template <int NTHREADS, class F>
__device__ __forceinline__ void for_block_records(const UpdateScratch& u, const int4& info, F&& f) {
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    for (int g = warp; g < info.y; g += NTHREADS / 32) {
        const int2 sg = u.seg_list[info.x + g];
        for (int k = lane; k < sg.y; k += 32) f(u.records[sg.x + k]);
    }
}

__global__ void __launch_bounds__(256)
update_place_kernel(UpdateScratch u) {
    const int n = (int)min((long long)u.ctl->n_segs, (long long)u.seg_cap);
    for (int d = blockIdx.x * blockDim.x + threadIdx.x; d < n; d += gridDim.x * blockDim.x) {
        const int4 sg = u.segs[d];
        const int4 info = u.blk_info[sg.x];
        const int k = atomicAdd(&u.blk_cur[sg.x], 1);
        if (k < info.y) u.seg_list[info.x + k] = make_int2(sg.y, sg.z);
    }
}

// ---- apply: warp-specialised, bulk-copy staged --------------------------
//
// Warp 0 is the producer: it takes the next touched block from the work
// cursor, loads the block's segment descriptors, and issues cp.async.bulk
// copies of the block's five 2 KB tiles (weight, tsdf, r, g, b) and of every
// record segment into one of kStages shared-memory stages, completing on the
// stage's "full" mbarrier. Warps 1-4 are consumers (4 voxels per thread):
// they wait for a full stage, apply it, and release it on its "empty"
// mbarrier, so the copies of the next blocks overlap the current one.
// Blocks with more records or segments than a stage holds are applied from
// global memory by the same consumers.
//
// Voxels that cross the cap inside the batch are resolved in the CTA: their
// records are grouped per voxel in shared memory and each record's rank by
// id among its voxel's records is counted by a warp; the `keep` lowest-ranked
// are accepted. Blocks whose crossing records exceed kCrossCap are deferred
// to update_crossing_kernel.
constexpr int kConsumerWarps = 4;
constexpr int kConsumers = 32 * kConsumerWarps;
constexpr int kApplyCta = kConsumers + 32;
constexpr int kStages = 3;
constexpr int kStageRecords = 1024;
constexpr int kStageSegs = 256;  // 8 descriptors per producer lane
constexpr int kCrossCap = 2048;
constexpr int kModeDone = 0, kModeShared = 1, kModeGlobal = 2;
constexpr int kConsumerBar = 1;

struct __align__(128) ApplyStage {
    float tile[5][kBlockVoxels];  // weight, tsdf, r, g, b
    Record rec[kStageRecords];
    int4 info;                    // (first segment slot, segments, records, block)
    int mode;
};

struct ApplySmem {
    ApplyStage st[kStages];
    uint64_t full[kStages];
    uint64_t empty[kStages];
    int cnt[kBlockVoxels];
    unsigned long long sum[kBlockVoxels];
    short ci[kBlockVoxels];  // crossing index of a voxel, or -1
    short cl[kBlockVoxels];  // voxel of a crossing index
    int cstart[kBlockVoxels];
    int ccur[kBlockVoxels];
    uint32_t cid[kCrossCap];
    float cval[kCrossCap];
    int flags, ncv, ncrec, warp_tot[kConsumerWarps];
};

// Records of a block for the consumers: from the stage, or from global
// memory through the block's segments (consumer warps take segments in turn).
template <class F>
__device__ __forceinline__ void consumer_records(const UpdateScratch& u, const ApplyStage& st,
                                                 int c, F&& f) {
    if (st.mode == kModeShared) {
        for (int k = c; k < st.info.z; k += kConsumers) f(st.rec[k]);
    } else {
        const int warp = c >> 5, lane = c & 31;
        for (int g = warp; g < st.info.y; g += kConsumerWarps) {
            const int2 sg = u.seg_list[st.info.x + g];
            for (int k = lane; k < sg.y; k += 32) f(u.records[sg.x + k]);
        }
    }
}

__global__ void __launch_bounds__(kApplyCta)
update_apply_kernel(DevVolume v, UpdateScratch u) {
    extern __shared__ __align__(128) unsigned char apply_smem[];
    ApplySmem& S = *reinterpret_cast<ApplySmem*>(apply_smem);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int n_touched = u.ctl->n_touched;

    if (threadIdx.x == 0) {
        for (int k = 0; k < kStages; ++k) {
            mbar_init(&S.full[k], 1);
            mbar_init(&S.empty[k], kConsumerWarps);
        }
        mbar_fence_init();
        S.flags = 0;
        S.ncv = 0;
    }
    for (int k = threadIdx.x; k < kBlockVoxels; k += kApplyCta) {
        S.cnt[k] = 0;
        S.sum[k] = 0ull;
    }
    __syncthreads();

    if (warp == 0) {
        // ---- producer ----
        float* const arrays[5] = {v.weight, v.tsdf, v.r, v.g, v.b};
        int issued[kStages];  // last use of each stage this warp filled, -1 none
#pragma unroll
        for (int k = 0; k < kStages; ++k) issued[k] = -1;
        for (int it = 0;; ++it) {
            const int s = it % kStages;
            const uint32_t use = (uint32_t)(it / kStages);
            if (use > 0 && !mbar_wait(&S.empty[s], (use - 1) & 1u, kSpinLimit)) {
                if (lane == 0) atomicOr(v.status, kStatusSpinTimeout);
                break;
            }
            int item = 0;
            if (lane == 0) item = atomicAdd(&u.ctl->work, 1);
            item = __shfl_sync(0xffffffffu, item, 0);
            ApplyStage& st = S.st[s];
            issued[s] = (int)use;
            if (item >= n_touched) {
                if (lane == 0) {
                    st.mode = kModeDone;
                    mbar_arrive(&S.full[s]);
                }
                break;
            }
            int bi = 0;
            int4 info = make_int4(0, 0, 0, 0);
            if (lane == 0) {
                bi = u.touched[item];
                info = u.blk_info[bi];
            }
            bi = __shfl_sync(0xffffffffu, bi, 0);
            info.x = __shfl_sync(0xffffffffu, info.x, 0);
            info.y = __shfl_sync(0xffffffffu, info.y, 0);
            info.z = __shfl_sync(0xffffffffu, info.z, 0);
            info.w = bi;
            if (info.z > kStageRecords || info.y > kStageSegs) {
                if (lane == 0) {
                    st.info = info;
                    st.mode = kModeGlobal;
                    mbar_arrive(&S.full[s]);
                }
                continue;
            }
            int2 sg[kStageSegs / 32];
            int mine = 0;
#pragma unroll
            for (int q = 0; q < kStageSegs / 32; ++q) {
                const int d = lane + 32 * q;
                sg[q] = d < info.y ? u.seg_list[info.x + d] : make_int2(0, 0);
                mine += sg[q].y;
            }
            int incl = mine;
            for (int o = 1; o < 32; o <<= 1) {
                const int y = __shfl_up_sync(0xffffffffu, incl, o);
                if (lane >= o) incl += y;
            }
            if (lane == 0) {
                st.info = info;
                st.mode = kModeShared;
                mbar_arrive_expect_tx(&S.full[s], 5u * kBlockVoxels * 4u + (uint32_t)info.z * 16u);
            }
            __syncwarp();
            if (lane < 5)
                bulk_load(st.tile[lane], arrays[lane] + (size_t)bi * kBlockVoxels, kBlockVoxels * 4,
                          &S.full[s]);
            int off = incl - mine;
#pragma unroll
            for (int q = 0; q < kStageSegs / 32; ++q) {
                if (sg[q].y > 0) {
                    bulk_load(&st.rec[off], u.records + sg[q].x, (uint32_t)sg[q].y * 16u, &S.full[s]);
                    off += sg[q].y;
                }
            }
        }
        // Never leave with copies in flight: wait (bounded) until the last
        // fill of every stage has landed. Stages the consumers already used
        // return at once.
#pragma unroll
        for (int k = 0; k < kStages; ++k)
            if (issued[k] >= 0 && !mbar_wait(&S.full[k], (uint32_t)issued[k] & 1u, kSpinLimit) &&
                lane == 0)
                atomicOr(v.status, kStatusSpinTimeout);
        return;
    }

    // ---- consumers ----
    const int c = threadIdx.x - 32;
    const int cw = c >> 5;
    for (int it = 0;; ++it) {
        const int s = it % kStages;
        const uint32_t use = (uint32_t)(it / kStages);
        if (!mbar_wait(&S.full[s], use & 1u, kSpinLimit)) {
            if (c == 0) atomicOr(v.status, kStatusSpinTimeout);
            break;
        }
        const ApplyStage& st = S.st[s];
        const int mode = st.mode;
        if (mode == kModeDone) break;
        const int4 info = st.info;
        const int32_t bi = info.w;
        const size_t v4 = (size_t)bi * (kBlockVoxels / 4) + c;
        float4 w0, t0;
        if (mode == kModeShared) {
            w0 = reinterpret_cast<const float4*>(st.tile[0])[c];
            t0 = reinterpret_cast<const float4*>(st.tile[1])[c];
        } else {
            w0 = reinterpret_cast<const float4*>(v.weight)[v4];
            t0 = reinterpret_cast<const float4*>(v.tsdf)[v4];
        }

        consumer_records(u, st, c, [&](const Record& rec) {
            const uint32_t lv = rec.lv & 511u;
            atomicAdd(&S.cnt[lv], 1);
            atomicAdd(&S.sum[lv], to_fix(rec.sdf_n, rec.w_in));
        });
        named_sync(kConsumerBar, kConsumers);

        const float w0a[4] = {w0.x, w0.y, w0.z, w0.w};
        int keep[4];
        int flags = 0;
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const int n = S.cnt[4 * c + q];
            keep[q] = accept_count(w0a[q], v.weight_cap, n);
            if (keep[q] > 0) flags |= 1;
            if (keep[q] > 0 && keep[q] < n) flags |= 2;
        }
        if (flags) atomicOr(&S.flags, flags);
        named_sync(kConsumerBar, kConsumers);
        const int block_flags = S.flags;
        bool deferred = false;

        if (block_flags & 2) {
            // Ordered selection for the voxels crossing the cap.
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                const int lv = 4 * c + q;
                short ci = -1;
                if (keep[q] > 0 && keep[q] < S.cnt[lv]) {
                    ci = (short)atomicAdd(&S.ncv, 1);
                    S.cl[ci] = (short)lv;
                }
                S.ci[lv] = ci;
            }
            named_sync(kConsumerBar, kConsumers);
            const int ncv = S.ncv;
            int local[4], mine = 0;
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                const int ci = 4 * c + q;
                local[q] = ci < ncv ? S.cnt[S.cl[ci]] : 0;
                mine += local[q];
            }
            int incl = mine;
            for (int o = 1; o < 32; o <<= 1) {
                const int y = __shfl_up_sync(0xffffffffu, incl, o);
                if ((c & 31) >= o) incl += y;
            }
            if ((c & 31) == 31) S.warp_tot[cw] = incl;
            named_sync(kConsumerBar, kConsumers);
            int before = 0, total = 0;
#pragma unroll
            for (int w = 0; w < kConsumerWarps; ++w) {
                if (w < cw) before += S.warp_tot[w];
                total += S.warp_tot[w];
            }
            int run = before + incl - mine;
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                const int ci = 4 * c + q;
                if (ci < ncv) {
                    S.cstart[ci] = run;
                    S.ccur[ci] = 0;
                }
                run += local[q];
            }
            if (c == 0) atomicAdd(&u.ctl->n_crossing, 1);
            if (total > kCrossCap) {
                deferred = true;
                if (c == 0) u.cross_list[atomicAdd(&u.ctl->n_deferred, 1)] = bi;
            } else {
                named_sync(kConsumerBar, kConsumers);
                consumer_records(u, st, c, [&](const Record& rec) {
                    const int ci = S.ci[rec.lv & 511u];
                    if (ci < 0) return;
                    const int pos = S.cstart[ci] + atomicAdd(&S.ccur[ci], 1);
                    S.cid[pos] = rec.id;
                    S.cval[pos] = __fmul_rn(rec.sdf_n, rec.w_in);
                });
                named_sync(kConsumerBar, kConsumers);
                const int lane_c = c & 31;
                for (int ci = cw; ci < ncv; ci += kConsumerWarps) {
                    const int lv = S.cl[ci];
                    const int n = S.cnt[lv];
                    const int beg = S.cstart[ci];
                    const float wv = mode == kModeShared ? st.tile[0][lv]
                                                         : v.weight[(size_t)bi * kBlockVoxels + lv];
                    const int k = accept_count(wv, v.weight_cap, n);
                    unsigned long long acc = 0ull;
                    for (int e = lane_c; e < n; e += 32) {
                        const uint32_t ide = S.cid[beg + e];
                        int rank = 0;
                        for (int f = 0; f < n; ++f) rank += S.cid[beg + f] < ide ? 1 : 0;
                        if (rank < k)
                            acc += (unsigned long long)__double2ll_rn((double)S.cval[beg + e] * kFixScale);
                    }
                    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
                    if (lane_c == 0) S.sum[lv] = acc;
                }
            }
            named_sync(kConsumerBar, kConsumers);
        }

        if (!deferred && (block_flags & 1)) {
            const float t0a[4] = {t0.x, t0.y, t0.z, t0.w};
            float tn[4], wn[4], dc[4];
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                tn[q] = keep[q] > 0 ? add_fix(t0a[q], S.sum[4 * c + q]) : t0a[q];
                wn[q] = __fadd_rn(w0a[q], (float)keep[q]);
                dc[q] = __fmul_rn(128.0f, (float)keep[q]);
            }
            reinterpret_cast<float4*>(v.tsdf)[v4] = make_float4(tn[0], tn[1], tn[2], tn[3]);
            reinterpret_cast<float4*>(v.weight)[v4] = make_float4(wn[0], wn[1], wn[2], wn[3]);
            float* rgb[3] = {v.r, v.g, v.b};
#pragma unroll
            for (int ch = 0; ch < 3; ++ch) {
                float4 x = mode == kModeShared ? reinterpret_cast<const float4*>(st.tile[2 + ch])[c]
                                               : reinterpret_cast<const float4*>(rgb[ch])[v4];
                x.x = __fadd_rn(x.x, dc[0]);
                x.y = __fadd_rn(x.y, dc[1]);
                x.z = __fadd_rn(x.z, dc[2]);
                x.w = __fadd_rn(x.w, dc[3]);
                reinterpret_cast<float4*>(rgb[ch])[v4] = x;
            }
            if (c == 0) atomicAdd(&u.ctl->n_accepted, 1);
        }
        if (c == 0 && !deferred) u.blk_cur[bi] = 0;  // done with its segments
        named_sync(kConsumerBar, kConsumers);
        if ((c & 31) == 0) mbar_arrive(&S.empty[s]);
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            S.cnt[4 * c + q] = 0;
            S.sum[4 * c + q] = 0ull;
        }
        if (c == 0) {
            S.flags = 0;
            S.ncv = 0;
        }
        named_sync(kConsumerBar, kConsumers);
    }
}

// Blocks with voxels that cross the cap inside this batch. The records of
// the crossing voxels are compacted into shared memory once (when they fit),
// and the radix select runs only over the id bits that differ within the
// block: a 640x480 frame's block spans ids of a few hundred rows, ~20 bits,
// i.e. 5 four-bit passes. Histograms are kept for crossing voxels only.
constexpr int kCrossList = 4096;

struct CrossSmem {
    int cnt[kBlockVoxels];
    unsigned long long sum[kBlockVoxels];
    int keep[kBlockVoxels];
    short ci[kBlockVoxels];      // crossing index of a voxel, or -1
    short lv[kBlockVoxels];      // voxel of a crossing index
    uint32_t prefix[kBlockVoxels];
    int rank[kBlockVoxels];
    uint32_t hist[kBlockVoxels * kDigits];
    uint32_t id[kCrossList];
    float val[kCrossList];
    unsigned short lci[kCrossList];
    int item, ncv, nlist;
    unsigned int minid, maxid;
};

__global__ void __launch_bounds__(kCrossThreads, 2)
update_crossing_kernel(DevVolume v, UpdateScratch u) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    CrossSmem& S = *reinterpret_cast<CrossSmem*>(smem_raw);
    int* s_cnt = S.cnt;
    unsigned long long* s_sum = S.sum;
    int* s_keep = S.keep;
    short* s_ci = S.ci;
    short* s_lv = S.lv;
    uint32_t* s_prefix = S.prefix;
    int* s_rank = S.rank;
    uint32_t* s_hist = S.hist;
    uint32_t* s_id = S.id;
    float* s_val = S.val;
    unsigned short* s_lci = S.lci;
    int& s_item = S.item;
    int& s_ncv = S.ncv;
    int& s_nlist = S.nlist;
    unsigned int& s_minid = S.minid;
    unsigned int& s_maxid = S.maxid;

    const int t = threadIdx.x;
    const int n_items = u.ctl->n_deferred;
    for (;;) {
        if (t == 0) {
            s_item = atomicAdd(&u.ctl->work2, 1);
            s_ncv = 0;
            s_nlist = 0;
            s_minid = 0xffffffffu;
            s_maxid = 0u;
        }
        for (int k = t; k < kBlockVoxels; k += kCrossThreads) {
            s_cnt[k] = 0;
            s_sum[k] = 0ull;
        }
        __syncthreads();
        const int item = s_item;
        if (item >= n_items) break;
        const int32_t bi = u.cross_list[item];
        const int4 info = u.blk_info[bi];

        for_block_records<kCrossThreads>(u, info, [&](const Record& rec) {
            const uint32_t lv = rec.lv & 511u;
            atomicAdd(&s_cnt[lv], 1);
            atomicAdd(&s_sum[lv], to_fix(rec.sdf_n, rec.w_in));
        });
        __syncthreads();

        for (int k = t; k < kBlockVoxels; k += kCrossThreads) {
            const float w0 = v.weight[(size_t)bi * kBlockVoxels + k];
            const int n = s_cnt[k];
            const int keep = accept_count(w0, v.weight_cap, n);
            s_keep[k] = keep;
            short ci = -1;
            if (keep > 0 && keep < n) {
                ci = (short)atomicAdd(&s_ncv, 1);
                s_lv[ci] = (short)k;
                s_rank[ci] = keep;
                s_sum[k] = 0ull;  // re-summed over the accepted records below
            }
            s_ci[k] = ci;
        }
        __syncthreads();

        // Compact the crossing voxels' records.
        for_block_records<kCrossThreads>(u, info, [&](const Record& rec) {
            const int ci = s_ci[rec.lv & 511u];
            if (ci < 0) return;
            atomicMin(&s_minid, rec.id);
            atomicMax(&s_maxid, rec.id);
            const int slot = atomicAdd(&s_nlist, 1);
            if (slot < kCrossList) {
                s_id[slot] = rec.id;
                s_val[slot] = __fmul_rn(rec.sdf_n, rec.w_in);
                s_lci[slot] = (unsigned short)ci;
            }
        });
        __syncthreads();
        const int ncv = s_ncv;
        const bool spill = s_nlist > kCrossList;  // too many: read them from the segments
        const int n_list = s_nlist;
        const uint32_t diff = s_minid ^ s_maxid;
        const int hi_bit = diff ? 31 - __clz(diff) : 0;
        const int top = (hi_bit / kDigitBits) * kDigitBits;
        const uint32_t common = top + kDigitBits >= 32 ? 0u : (s_minid >> (top + kDigitBits)) << (top + kDigitBits);
        for (int c = t; c < ncv; c += kCrossThreads) s_prefix[c] = common;

        // Radix select over the differing bits, most significant digit first:
        // afterwards s_prefix[c] is the id of crossing voxel c's keep-th
        // smallest record, i.e. its last accepted one.
        for (int shift = top; shift >= 0; shift -= kDigitBits) {
            for (int k = t; k < ncv * kDigits; k += kCrossThreads) s_hist[k] = 0u;
            __syncthreads();
            auto count_digit = [&](uint32_t id, int ci) {
                if (((uint64_t)id >> (shift + kDigitBits)) !=
                    ((uint64_t)s_prefix[ci] >> (shift + kDigitBits)))
                    return;
                atomicAdd(&s_hist[ci * kDigits + ((id >> shift) & (kDigits - 1))], 1u);
            };
            if (spill) {
                for_block_records<kCrossThreads>(u, info, [&](const Record& rec) {
                    const int ci = s_ci[rec.lv & 511u];
                    if (ci >= 0) count_digit(rec.id, ci);
                });
            } else {
                for (int k = t; k < n_list; k += kCrossThreads) count_digit(s_id[k], s_lci[k]);
            }
            __syncthreads();
            for (int c = t; c < ncv; c += kCrossThreads) {
                int acc = 0, d = 0;
                const int rank = s_rank[c];
                for (; d < kDigits - 1; ++d) {
                    const int h = (int)s_hist[c * kDigits + d];
                    if (acc + h >= rank) break;
                    acc += h;
                }
                s_rank[c] = rank - acc;
                s_prefix[c] |= (uint32_t)d << shift;
            }
            __syncthreads();
        }

        // Sum the accepted records of the crossing voxels.
        auto add_accepted = [&](uint32_t id, int ci, float val) {
            if (id <= s_prefix[ci])
                atomicAdd(&s_sum[s_lv[ci]], (unsigned long long)__double2ll_rn((double)val * kFixScale));
        };
        if (spill) {
            for_block_records<kCrossThreads>(u, info, [&](const Record& rec) {
                const int ci = s_ci[rec.lv & 511u];
                if (ci >= 0) add_accepted(rec.id, ci, __fmul_rn(rec.sdf_n, rec.w_in));
            });
        } else {
            for (int k = t; k < n_list; k += kCrossThreads) add_accepted(s_id[k], s_lci[k], s_val[k]);
        }
        __syncthreads();

        int any = 0;
        for (int k = t; k < kBlockVoxels; k += kCrossThreads) {
            const int keep = s_keep[k];
            if (keep <= 0) continue;
            any = 1;
            const size_t vox = (size_t)bi * kBlockVoxels + k;
            v.tsdf[vox] = add_fix(v.tsdf[vox], s_sum[k]);
            v.weight[vox] = __fadd_rn(v.weight[vox], (float)keep);
            const float dc = __fmul_rn(128.0f, (float)keep);
            v.r[vox] = __fadd_rn(v.r[vox], dc);
            v.g[vox] = __fadd_rn(v.g[vox], dc);
            v.b[vox] = __fadd_rn(v.b[vox], dc);
        }
        const int any_keep = __syncthreads_or(any);
        if (t == 0) {
            if (any_keep) atomicAdd(&u.ctl->n_accepted, 1);
            u.blk_cur[bi] = 0;  // done with its segments
        }
    }
}

}  // namespace

cudaError_t launch_update_apply(const DevVolume& v, const UpdateScratch& u, int n_ctas,
                                cudaStream_t s) {
    update_apply_kernel<<<n_ctas, kApplyCta, sizeof(ApplySmem), s>>>(v, u);
    return cudaGetLastError();
}

cudaError_t launch_update_place(const UpdateScratch& u, int n_ctas, cudaStream_t s) {
    update_place_kernel<<<n_ctas, 256, 0, s>>>(u);
    return cudaGetLastError();
}

cudaError_t prepare_update_kernels() {
    cudaError_t e = cudaFuncSetAttribute(update_crossing_kernel,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)sizeof(CrossSmem));
    if (e != cudaSuccess) return e;
    return cudaFuncSetAttribute(update_apply_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)sizeof(ApplySmem));
}

size_t apply_smem_bytes() { return sizeof(ApplySmem); }

cudaError_t launch_update_crossing(const DevVolume& v, const UpdateScratch& u, int n_ctas,
                                   cudaStream_t s) {
    update_crossing_kernel<<<n_ctas, kCrossThreads, sizeof(CrossSmem), s>>>(v, u);
    return cudaGetLastError();
}

}  // namespace osn_b200
