// Update: accumulate a batch's truncation bands into the allocated blocks.
//
// Reference: cpp/src/volume.cpp:200-299 (CPU arm: band walk, find_block, cap
// check, five atomic adds per sample) and cpp/src/volume_cuda.cu:302-337
// (CUDA arm: the same, one thread per point, red.add.f32 scatter).
//
// Semantics. The reference's cap check is a plain read before the adds
// (volume.cpp:283-291), so which contributions a capped voxel accepts depends
// on thread timing. This library implements the one order-independent
// reading of it: contributions are applied as if in (point index, band step)
// order, and a contribution is accepted while the voxel's weight before it is
// below the cap. That is exactly what the reference's CPU arm computes with
// one thread, which is the parity oracle.
//
// B200 design: a scatter of 5 float atomics per sample is bound by L2 atomic
// throughput, not by HBM, and cannot honour an ordered cap. Instead the
// contributions are binned by block and each touched block is updated by one
// CTA in one read-modify-write of its tiles:
//   count   walk + lookup, per-block record counts (warp-aggregated atomics),
//           list of touched blocks
//   scan    exclusive scan of the counts -> each block's bin
//   scatter walk + lookup again, write 16-byte records into the bins
//   apply   one CTA per touched block (persistent, work-queued): per-voxel
//           record counts, the number of contributions each voxel accepts
//           (closed form for unit weights), an exact radix select of the
//           accepted ids for the few voxels that cross the cap inside this
//           batch, then one coalesced read and write of the block's tiles.
//
// The accepted sdf values of a voxel are summed in 64-bit fixed point
// (2^-40 resolution, exact for |value| >= 2^-17) and added to the stored sum
// with one rounding, so the result does not depend on the order in which
// the CTA's threads meet the records: repeated runs are bit-identical, and a
// voxel with one contribution per batch gets exactly the reference's
// fl(tsdf + sdf_n).
#include "volume.h"

namespace osn_b200 {
namespace {

constexpr int kWalkThreads = 256;
constexpr int kScanThreads = 1024;
constexpr int kApplyThreads = 512;  // one thread per voxel of a block
constexpr int kDigitBits = 4;
constexpr int kDigits = 1 << kDigitBits;
constexpr double kFixScale = 1099511627776.0;        // 2^40
constexpr double kFixInv = 1.0 / 1099511627776.0;    // 2^-40

// Per-thread cache of the last looked-up block, and the warp-cooperative
// lookup for samples whose block differs from it: one leader per distinct key.
struct BlockCache {
    long long key = kNoKey;
    int32_t bi = -1;
};

__device__ __forceinline__ int32_t lookup_coop(const DevVolume& v, BlockCache& c, bool have,
                                               long long key, int bx, int by, int bz, int lane) {
    const bool need = have && key != c.key;
    const unsigned need_mask = __ballot_sync(0xffffffffu, need);
    if (need) {
        const unsigned grp = __match_any_sync(need_mask, key);
        const int leader = __ffs(grp) - 1;
        int32_t bi = -1;
        if (lane == leader) bi = find_block(v, bx, by, bz, key);
        bi = __shfl_sync(grp, bi, leader);
        c.key = key;
        c.bi = bi;
    }
    return have ? c.bi : -1;
}

// ---- count ---------------------------------------------------------------

__device__ __forceinline__ void flush_run(const UpdateScratch& u, int32_t bi, int32_t len,
                                          bool pending, int lane) {
    const unsigned m = __ballot_sync(0xffffffffu, pending);
    if (pending) {
        const unsigned grp = __match_any_sync(m, bi);
        const int leader = __ffs(grp) - 1;
        const int total = __reduce_add_sync(grp, len);
        if (lane == leader) {
            const int old = atomicAdd(&u.blk_cnt[bi], total);
            if (old == 0) {
                const int slot = atomicAdd(&u.ctl->n_touched, 1);
                u.touched[slot] = bi;
            }
        }
    }
}

__global__ void __launch_bounds__(kWalkThreads, 4)
update_count_kernel(DevVolume v, BatchArgs a, UpdateScratch u) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int lane = threadIdx.x & 31;
    Ray r;
    const bool live = i < a.n && ray_setup(a, i, r);
    if (!__any_sync(0xffffffffu, live)) return;

    BlockCache cache;
    int32_t run_bi = -1, run_len = 0;
    for (int s = -v.steps; s <= v.steps; ++s) {
        int vx = 0, vy = 0, vz = 0;
        float sdf = 0.0f;
        const bool have = live && band_sample(v, a, r, s, vx, vy, vz, sdf);
        const int bx = vx >> 3, by = vy >> 3, bz = vz >> 3;
        const long long key = have ? pack_key(bx, by, bz) : kNoKey;
        const int32_t bi = lookup_coop(v, cache, have, key, bx, by, bz, lane);
        // Run-length per ray: consecutive samples usually share a block.
        const bool ends = run_len > 0 && bi != run_bi && bi >= 0;
        flush_run(u, run_bi, run_len, ends, lane);
        if (ends) run_len = 0;
        if (bi >= 0) {
            run_bi = bi;
            ++run_len;
        }
    }
    flush_run(u, run_bi, run_len, run_len > 0, lane);
}

// ---- scan ----------------------------------------------------------------

// Single CTA: exclusive scan of the touched blocks' counts into bins.
__global__ void __launch_bounds__(kScanThreads)
update_scan_kernel(UpdateScratch u) {
    __shared__ int warp_sums[kScanThreads / 32];
    __shared__ int carry;
    const int n = u.ctl->n_touched;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (threadIdx.x == 0) carry = 0;
    __syncthreads();
    for (int base = 0; base < n; base += kScanThreads) {
        const int k = base + threadIdx.x;
        const int bi = k < n ? u.touched[k] : -1;
        const int c = bi >= 0 ? u.blk_cnt[bi] : 0;
        int x = c;
        for (int o = 1; o < 32; o <<= 1) {
            const int y = __shfl_up_sync(0xffffffffu, x, o);
            if (lane >= o) x += y;
        }
        if (lane == 31) warp_sums[warp] = x;
        __syncthreads();
        if (warp == 0) {
            int w = warp_sums[lane];
            for (int o = 1; o < 32; o <<= 1) {
                const int y = __shfl_up_sync(0xffffffffu, w, o);
                if (lane >= o) w += y;
            }
            warp_sums[lane] = w;
        }
        __syncthreads();
        const int excl = carry + (warp ? warp_sums[warp - 1] : 0) + x - c;
        if (bi >= 0) u.blk_bin[bi] = make_int2(excl, c);
        __syncthreads();
        if (threadIdx.x == kScanThreads - 1) carry = excl + c;
        __syncthreads();
    }
    if (threadIdx.x == 0) u.ctl->n_records = carry;
}

// ---- scatter -------------------------------------------------------------

__global__ void __launch_bounds__(kWalkThreads, 4)
update_scatter_kernel(DevVolume v, BatchArgs a, UpdateScratch u) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int lane = threadIdx.x & 31;
    Ray r;
    const bool live = i < a.n && ray_setup(a, i, r);
    if (!__any_sync(0xffffffffu, live)) return;

    const uint32_t n_steps = 2u * (uint32_t)v.steps + 1u;
    BlockCache cache;
    for (int s = -v.steps; s <= v.steps; ++s) {
        int vx = 0, vy = 0, vz = 0;
        float sdf = 0.0f;
        const bool have = live && band_sample(v, a, r, s, vx, vy, vz, sdf);
        const int bx = vx >> 3, by = vy >> 3, bz = vz >> 3;
        const long long key = have ? pack_key(bx, by, bz) : kNoKey;
        const int32_t bi = lookup_coop(v, cache, have, key, bx, by, bz, lane);
        const bool emit = bi >= 0;
        const unsigned m = __ballot_sync(0xffffffffu, emit);
        if (emit) {
            const unsigned grp = __match_any_sync(m, bi);
            const int leader = __ffs(grp) - 1;
            const int cnt = __popc(grp);
            int base = 0;
            if (lane == leader) {
                const int old = atomicSub(&u.blk_cnt[bi], cnt);
                base = u.blk_bin[bi].x + old - cnt;
            }
            base = __shfl_sync(grp, base, leader);
            const long long pos = (long long)base + __popc(grp & lanemask_lt());
            if (pos >= 0 && pos < u.record_cap) {
                float sdf_n = __fmul_rn(sdf, v.inv_trunc);
                sdf_n = fminf(fmaxf(sdf_n, -1.0f), 1.0f);
                Record rec;
                rec.id = (uint32_t)i * n_steps + (uint32_t)(s + v.steps);
                rec.lv = (uint32_t)(((vz & 7) * kBlockDim + (vy & 7)) * kBlockDim + (vx & 7));
                rec.sdf_n = sdf_n;
                rec.w_in = 1.0f;
                *reinterpret_cast<int4*>(&u.records[pos]) = *reinterpret_cast<const int4*>(&rec);
            } else {
                atomicOr(v.status, kStatusScratchOverflow);
            }
        }
    }
}

// ---- apply ---------------------------------------------------------------

// Contributions voxel `v` accepts, given its weight w0 before the batch and
// n unit-weight records: j-th record (0-based, canonical order) is accepted
// iff w0 + j < cap (volume.cpp:289), all integer-valued so exact in float.
__device__ __forceinline__ int accept_count(float w0, float cap, int n) {
    if (n == 0) return 0;
    if (!(cap > 0.0f)) return n;
    if (w0 >= cap) return 0;
    const double room = ceil((double)cap - (double)w0);
    return room >= (double)n ? n : (int)room;
}

__global__ void __launch_bounds__(kApplyThreads, 2)
update_apply_kernel(DevVolume v, UpdateScratch u) {
    __shared__ int s_cnt[kBlockVoxels];
    __shared__ int s_keep[kBlockVoxels];
    __shared__ unsigned long long s_acc[kBlockVoxels];
    __shared__ uint32_t s_thr[kBlockVoxels];
    __shared__ uint32_t s_hist[kBlockVoxels * kDigits];
    __shared__ int s_item;

    const int t = threadIdx.x;
    const int n_touched = u.ctl->n_touched;
    for (;;) {
        if (t == 0) s_item = atomicAdd(&u.ctl->work, 1);
        __syncthreads();
        const int item = s_item;
        if (item >= n_touched) break;
        const int32_t bi = u.touched[item];
        const int2 bin = u.blk_bin[bi];
        const Record* recs = u.records + bin.x;
        const int nrec = bin.y;
        const size_t vox = (size_t)bi * kBlockVoxels + t;

        const float w0 = v.weight[vox];
        const float t0 = v.tsdf[vox];
        s_cnt[t] = 0;
        s_acc[t] = 0ull;
        __syncthreads();

        // Pass A: records per voxel.
        for (int k = t; k < nrec; k += kApplyThreads) atomicAdd(&s_cnt[recs[k].lv & 511u], 1);
        __syncthreads();

        const int n_v = s_cnt[t];
        const int keep = accept_count(w0, v.weight_cap, n_v);
        s_keep[t] = keep;
        const bool crossing = keep > 0 && keep < n_v;
        const int any_crossing = __syncthreads_or(crossing);

        if (any_crossing) {
            // Exact selection of the `keep` smallest ids of each crossing
            // voxel: radix select over the 32-bit id, 4 bits per pass.
            uint32_t prefix = 0;
            int rank = keep;  // 1-based rank of the last accepted id
            for (int shift = 32 - kDigitBits; shift >= 0; shift -= kDigitBits) {
                for (int k = t; k < kBlockVoxels * kDigits; k += kApplyThreads) s_hist[k] = 0u;
                s_thr[t] = prefix;
                __syncthreads();
                for (int k = t; k < nrec; k += kApplyThreads) {
                    const Record rec = recs[k];
                    const uint32_t lv = rec.lv & 511u;
                    const int kl = s_keep[lv];
                    if (kl <= 0 || kl >= s_cnt[lv]) continue;
                    const uint64_t hi = (uint64_t)rec.id >> (shift + kDigitBits);
                    if (hi != ((uint64_t)s_thr[lv] >> (shift + kDigitBits))) continue;
                    atomicAdd(&s_hist[lv * kDigits + ((rec.id >> shift) & (kDigits - 1))], 1u);
                }
                __syncthreads();
                if (crossing) {
                    int acc = 0;
                    int d = 0;
                    for (; d < kDigits; ++d) {
                        const int h = (int)s_hist[t * kDigits + d];
                        if (acc + h >= rank) break;
                        acc += h;
                    }
                    rank -= acc;
                    prefix |= (uint32_t)d << shift;
                }
                __syncthreads();
            }
            s_thr[t] = prefix;
            __syncthreads();
        }

        // Pass B: accumulate accepted contributions.
        for (int k = t; k < nrec; k += kApplyThreads) {
            const Record rec = recs[k];
            const uint32_t lv = rec.lv & 511u;
            const int kl = s_keep[lv];
            if (kl <= 0) continue;
            if (kl < s_cnt[lv] && rec.id > s_thr[lv]) continue;
            const double x = (double)__fmul_rn(rec.sdf_n, rec.w_in);
            atomicAdd(&s_acc[lv], (unsigned long long)__double2ll_rn(x * kFixScale));
        }
        __syncthreads();

        if (keep > 0) {
            const double sum = (double)(long long)s_acc[t] * kFixInv;
            v.tsdf[vox] = __double2float_rn((double)t0 + sum);
            v.weight[vox] = __fadd_rn(w0, (float)keep);
            const float dc = __fmul_rn(128.0f, (float)keep);
            v.r[vox] = __fadd_rn(v.r[vox], dc);
            v.g[vox] = __fadd_rn(v.g[vox], dc);
            v.b[vox] = __fadd_rn(v.b[vox], dc);
        }
        const int any_keep = __syncthreads_or(keep > 0);
        if (t == 0) {
            if (any_keep) atomicAdd(&u.ctl->n_accepted, 1);
            if (any_crossing) atomicAdd(&u.ctl->n_crossing, 1);
        }
    }
}

}  // namespace

cudaError_t launch_update_count(const DevVolume& v, const BatchArgs& a, const UpdateScratch& u,
                                cudaStream_t s) {
    const int grid = (a.n + kWalkThreads - 1) / kWalkThreads;
    update_count_kernel<<<grid, kWalkThreads, 0, s>>>(v, a, u);
    return cudaGetLastError();
}

cudaError_t launch_update_scan(const DevVolume&, const UpdateScratch& u, cudaStream_t s) {
    update_scan_kernel<<<1, kScanThreads, 0, s>>>(u);
    return cudaGetLastError();
}

cudaError_t launch_update_scatter(const DevVolume& v, const BatchArgs& a, const UpdateScratch& u,
                                  cudaStream_t s) {
    const int grid = (a.n + kWalkThreads - 1) / kWalkThreads;
    update_scatter_kernel<<<grid, kWalkThreads, 0, s>>>(v, a, u);
    return cudaGetLastError();
}

cudaError_t launch_update_apply(const DevVolume& v, const UpdateScratch& u, int n_ctas,
                                cudaStream_t s) {
    update_apply_kernel<<<n_ctas, kApplyThreads, 0, s>>>(v, u);
    return cudaGetLastError();
}

}  // namespace osn_b200
