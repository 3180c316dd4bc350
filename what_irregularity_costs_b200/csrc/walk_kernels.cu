// The band walk with CTA-cooperative block resolution: allocate, and
// count-and-stage (the first half of update, fused with allocation in
// integrate).
//
// Reference: cpp/src/volume.cpp:147-198 and :200-299 (one sample at a time:
// find_or_insert / find_block per sample) and cpp/src/volume_cuda.cu:160-192,
// :259-269, :302-337 (one thread per point, one hash probe sequence per
// sample).
//
// B200 design. A CTA walks 256 rays (consecutive points, i.e. neighbouring
// pixels of a depth frame). Every band sample is first binned into a small
// open-addressed table of the CTA's distinct blocks in shared memory; only
// then does one thread per DISTINCT block probe the global table (lookup, or
// the insertion protocol), in parallel. A CTA of a 640x480 frame touches ~10-30
// blocks for ~2300 samples, so the global table sees two orders of magnitude
// fewer probes than one per sample.
//
// The band is walked once per batch: the count-and-stage tail writes the
// CTA's records grouped by block into one contiguous staging range (one
// global atomic per CTA reserves it) and publishes one segment descriptor
// (block, offset, length) per (CTA, block); the last CTA to finish turns the
// per-block counts into per-block bins, and a small kernel then copies each
// segment into its block's bin (update_kernels.cu).
//
// Samples whose voxel already holds the cap's weight are dropped before they
// are staged: under "accept while weight before < cap" they cannot be
// accepted in any order, so dropping them changes no result and saves the
// records and the apply work for the saturated surface.
//
// The band is processed in chunks of kChunk samples per ray held in
// registers (9 = the whole band at the default truncation of 4 voxels).
#include "volume.h"

namespace osn_b200 {
namespace {

constexpr int kWalkThreads = 256;
constexpr int kChunk = 9;
constexpr int kCtaSlots = 512;
constexpr int kScanPer = 16;  // touched blocks per thread per scan pass
constexpr long long kCtaEmpty = -1;

enum Tail : int {
    kTailDrops = 0,  // allocate only: count dropped samples
    kTailStage = 1,  // count, stage records, publish segments; the last CTA scans
};

// Per-sample state packed in one register: slot (9 bits), voxel in block
// (9 bits), rank within the slot for this chunk (12 bits), valid, overflow.
constexpr uint32_t kSlotMask = 0x1FFu;
constexpr int kLvShift = 9;
constexpr int kRankShift = 18;
constexpr uint32_t kRankMask = 0xFFFu;
constexpr uint32_t kValid = 1u << 30;
constexpr uint32_t kOverflow = 1u << 31;

struct CtaTable {
    long long key[kCtaSlots];
    int32_t bi[kCtaSlots];
    int32_t cnt[kCtaSlots];
    int32_t base[kCtaSlots];
    int32_t list[kCtaSlots];
    int32_t n_list;
    int32_t n_resolved;
    uint32_t drops;
    int32_t last;
    int32_t cta_base;
    int32_t warp_sums[kWalkThreads / 32];
    unsigned int hist[64];
};

// Slot of `key` in the CTA table (inserting it), or -1 when the table is full.
__device__ __forceinline__ int cta_slot(CtaTable& T, long long key, int bx, int by, int bz) {
    const uint32_t h = hash_slot(bx, by, bz, kCtaSlots - 1);
    for (int p = 0; p < kCtaSlots; ++p) {
        const int s = (int)((h + p) & (kCtaSlots - 1));
        const long long k = *(volatile long long*)&T.key[s];
        if (k == key) return s;
        if (k == kCtaEmpty) {
            const long long prev = (long long)atomicCAS((unsigned long long*)&T.key[s],
                                                        (unsigned long long)kCtaEmpty,
                                                        (unsigned long long)key);
            if (prev == kCtaEmpty) {
                T.list[atomicAdd(&T.n_list, 1)] = s;
                return s;
            }
            if (prev == key) return s;
        }
    }
    return -1;
}

template <int MODE>
__device__ __forceinline__ int32_t resolve(const DevVolume& v, int bx, int by, int bz, long long key,
                                           unsigned int* hist, int n_bins) {
    if (MODE == kLookupOnly) return find_block(v, bx, by, bz, key);
    const InsertResult r = find_or_insert<MODE>(v, bx, by, bz, key);
    if (MODE == kAllocProbeHist) atomicAdd(&hist[min(r.probes, (uint32_t)(n_bins - 1))], 1u);
    return r.idx;
}

// Rare path: a sample whose block did not fit the CTA table is resolved on
// its own. Kept out of line so the unrolled sample loop stays in registers.
template <int MODE>
__device__ __noinline__ int32_t resolve_sample(const DevVolume& v, const BatchArgs& a, const Ray& r,
                                               int s, unsigned int* hist, int n_bins) {
    int vx, vy, vz;
    float sdf;
    band_sample(v, a, r, s, vx, vy, vz, sdf);
    const int bx = vx >> 3, by = vy >> 3, bz = vz >> 3;
    return resolve<MODE>(v, bx, by, bz, pack_key(bx, by, bz), hist, n_bins);
}

// CTA-wide exclusive scan of one int per thread; returns the exclusive
// prefix and writes the total to *total.
__device__ __forceinline__ int cta_exclusive_scan(CtaTable& T, int x, int* total) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    int incl = x;
    for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += y;
    }
    if (lane == 31) T.warp_sums[warp] = incl;
    __syncthreads();
    if (warp == 0) {
        int w = lane < kWalkThreads / 32 ? T.warp_sums[lane] : 0;
        for (int o = 1; o < 32; o <<= 1) {
            const int y = __shfl_up_sync(0xffffffffu, w, o);
            if (lane >= o) w += y;
        }
        if (lane < kWalkThreads / 32) T.warp_sums[lane] = w;
    }
    __syncthreads();
    const int excl = (warp ? T.warp_sums[warp - 1] : 0) + incl - x;
    *total = T.warp_sums[kWalkThreads / 32 - 1];
    __syncthreads();
    return excl;
}

// Exclusive scan of the touched blocks' record counts into per-block bins,
// run by the last CTA once every CTA's segments are out: blk_info[bi] =
// (bin offset, record count). The per-block counters go back to zero for the
// next batch.
__device__ void scan_blocks(CtaTable& T, const UpdateScratch& u) {
    const int n = ld_relaxed_s32(&u.ctl->n_touched);
    int carry = 0;
    for (int base = 0; base < n; base += kWalkThreads * kScanPer) {
        int b[kScanPer], c[kScanPer];
        int local = 0;
        const int first = base + threadIdx.x * kScanPer;
#pragma unroll
        for (int q = 0; q < kScanPer; ++q)
            b[q] = first + q < n ? ld_relaxed_s32(&u.touched[first + q]) : -1;
#pragma unroll
        for (int q = 0; q < kScanPer; ++q) {
            c[q] = b[q] >= 0 ? ld_relaxed_s32(&u.blk_cnt[b[q]]) : 0;
            local += c[q];
        }
        int total = 0;
        int run = carry + cta_exclusive_scan(T, local, &total);
#pragma unroll
        for (int q = 0; q < kScanPer; ++q) {
            if (b[q] >= 0) {
                u.blk_info[b[q]] = make_int4(run, c[q], 0, 0);
                u.blk_cnt[b[q]] = 0;
            }
            run += c[q];
        }
        carry += total;
    }
    if (threadIdx.x == 0) u.ctl->cta_done = 0;
}

template <int MODE, int TAIL>
__global__ void __launch_bounds__(kWalkThreads, 4)
walk_kernel(DevVolume v, BatchArgs a, UpdateScratch u, unsigned long long* hist, int n_bins) {
    __shared__ CtaTable T;
    const int tid = threadIdx.x;
    for (int s = tid; s < kCtaSlots; s += kWalkThreads) {
        T.key[s] = kCtaEmpty;
        T.cnt[s] = 0;
    }
    if (MODE == kAllocProbeHist)
        for (int s = tid; s < 64; s += kWalkThreads) T.hist[s] = 0u;
    if (tid == 0) {
        T.n_list = 0;
        T.n_resolved = 0;
        T.drops = 0u;
    }
    __syncthreads();

    const int i = blockIdx.x * kWalkThreads + tid;
    Ray r;
    const bool live = i < a.n && ray_setup(a, i, r);
    const bool sat_check = TAIL != kTailDrops && v.weight_cap > 0.0f;
    const bool counts_drops = MODE != kLookupOnly &&
                              MODE != kAllocNoCas && MODE != kAllocCountingCas;
    const uint32_t n_steps = 2u * (uint32_t)v.steps + 1u;
    uint32_t drops = 0;

    for (int c0 = -v.steps; c0 <= v.steps; c0 += kChunk) {
        uint32_t st[kChunk];
        float sd[kChunk];

        // Phase 1: walk; bin every sample into the CTA's block table (a
        // thread looks its block up only when it changes along the ray).
        long long last_key = kNoKey;
        int last_slot = -1;
#pragma unroll
        for (int j = 0; j < kChunk; ++j) {
            st[j] = 0u;
            sd[j] = 0.0f;
            const int s = c0 + j;
            int vx, vy, vz;
            float sdf;
            if (live && s <= v.steps && band_sample(v, a, r, s, vx, vy, vz, sdf)) {
                const int bx = vx >> 3, by = vy >> 3, bz = vz >> 3;  // floor_div(v, 8)
                const long long key = pack_key(bx, by, bz);
                if (key != last_key) {
                    last_key = key;
                    last_slot = cta_slot(T, key, bx, by, bz);
                }
                const uint32_t lv = (uint32_t)(((vz & 7) * kBlockDim + (vy & 7)) * kBlockDim + (vx & 7));
                st[j] = kValid | (lv << kLvShift) |
                        (last_slot >= 0 ? (uint32_t)last_slot : kOverflow);
                sd[j] = sdf;
            }
        }
        __syncthreads();

        // Phase 2: one thread per new distinct block resolves it globally.
        const int n_list = T.n_list;
        for (int k = T.n_resolved + tid; k < n_list; k += kWalkThreads) {
            const int s = T.list[k];
            const long long key = T.key[s];
            const int bx = unpack_axis(key, 2 * kCoordBits);
            const int by = unpack_axis(key, kCoordBits);
            const int bz = unpack_axis(key, 0);
            T.bi[s] = resolve<MODE>(v, bx, by, bz, key, T.hist, min(n_bins, 64));
        }
        __syncthreads();
        if (tid == 0) T.n_resolved = n_list;

        // Phase 3: drops and the saturation gate (loads of all samples in
        // flight together), then ranks within the CTA, one shared-memory
        // atomic per (warp, block).
#pragma unroll
        for (int j = 0; j < kChunk; ++j) {
            if (!(st[j] & kValid)) continue;
            const uint32_t lv = (st[j] >> kLvShift) & 511u;
            int32_t bi;
            if (st[j] & kOverflow) {
                // CTA table full: resolve this sample on its own (rare).
                bi = resolve_sample<MODE>(v, a, r, c0 + j, T.hist, min(n_bins, 64));
            } else {
                bi = T.bi[st[j] & kSlotMask];
            }
            if (bi < 0) {
                if (counts_drops) ++drops;
                st[j] = 0u;
                continue;
            }
            if (TAIL == kTailDrops) continue;
            if (sat_check && __ldg(&v.weight[(size_t)bi * kBlockVoxels + lv]) >= v.weight_cap) {
                st[j] = 0u;
                continue;
            }
            if (st[j] & kOverflow) {
                // Its own one-record segment, straight to global memory.
                const int pos = atomicAdd(&u.ctl->n_records, 1);
                const int d = atomicAdd(&u.ctl->n_segs, 1);
                if (pos < u.record_cap && d < u.seg_cap) {
                    Record rec;
                    rec.id = (uint32_t)i * n_steps + (uint32_t)(c0 + j + v.steps);
                    rec.lv = lv;
                    rec.sdf_n = fminf(fmaxf(__fmul_rn(sd[j], v.inv_trunc), -1.0f), 1.0f);
                    rec.w_in = 1.0f;
                    *reinterpret_cast<int4*>(&u.records[pos]) = *reinterpret_cast<const int4*>(&rec);
                    u.segs[d] = make_int4(bi, pos, 1, 0);
                    if (atomicAdd(&u.blk_cnt[bi], 1) == 0)
                        u.touched[atomicAdd(&u.ctl->n_touched, 1)] = bi;
                } else {
                    atomicOr(v.status, kStatusScratchOverflow);
                }
                st[j] = 0u;
            }
        }
        if (TAIL != kTailDrops) {
#pragma unroll
            for (int j = 0; j < kChunk; ++j) {
                const bool rankable = (st[j] & kValid) != 0u;
                const unsigned m = __ballot_sync(0xffffffffu, rankable);
                if (rankable) {
                    const uint32_t slot = st[j] & kSlotMask;
                    const unsigned grp = __match_any_sync(m, slot);
                    const int leader = __ffs(grp) - 1;
                    int base = 0;
                    if ((tid & 31) == leader) base = atomicAdd(&T.cnt[slot], __popc(grp));
                    base = __shfl_sync(grp, base, leader);
                    const uint32_t rank = (uint32_t)base + __popc(grp & lanemask_lt());
                    st[j] |= (rank & kRankMask) << kRankShift;
                }
            }
        }
        if (TAIL == kTailDrops) continue;
        __syncthreads();

        // Phase 4: the CTA's staging range (one global atomic), segment
        // offsets by a CTA scan over its blocks, one descriptor per block.
        int my_cnt = 0, my_off = 0, total = 0;
        const int k4 = tid;  // n_list <= kCtaSlots = 2 * kWalkThreads
        int c_a = 0, c_b = 0;
        if (k4 < n_list) c_a = T.cnt[T.list[k4]];
        if (k4 + kWalkThreads < n_list) c_b = T.cnt[T.list[k4 + kWalkThreads]];
        my_cnt = c_a + c_b;
        my_off = cta_exclusive_scan(T, my_cnt, &total);
        if (tid == 0) T.cta_base = total ? atomicAdd(&u.ctl->n_records, total) : 0;
        __syncthreads();
        const int cta_base = T.cta_base;
        if (cta_base + total > u.record_cap) {
            if (tid == 0) atomicOr(v.status, kStatusScratchOverflow);
        } else {
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                const int k = k4 + h * kWalkThreads;
                const int c = h ? c_b : c_a;
                if (k >= n_list || c == 0) continue;
                const int s = T.list[k];
                const int32_t bi = T.bi[s];
                const int off = cta_base + my_off + (h ? c_a : 0);
                T.base[s] = off;
                const int d = atomicAdd(&u.ctl->n_segs, 1);
                if (d < u.seg_cap) {
                    u.segs[d] = make_int4(bi, off, c, 0);
                    if (atomicAdd(&u.blk_cnt[bi], c) == 0)
                        u.touched[atomicAdd(&u.ctl->n_touched, 1)] = bi;
                } else {
                    atomicOr(v.status, kStatusScratchOverflow);
                    T.base[s] = -1;
                }
            }
        }
        __syncthreads();

        // Phase 5: the records, grouped by block inside the CTA's range.
        if (cta_base + total <= u.record_cap) {
#pragma unroll
            for (int j = 0; j < kChunk; ++j) {
                if (!(st[j] & kValid)) continue;
                const int base = T.base[st[j] & kSlotMask];
                if (base < 0) continue;
                const long long pos = (long long)base + ((st[j] >> kRankShift) & kRankMask);
                Record rec;
                rec.id = (uint32_t)i * n_steps + (uint32_t)(c0 + j + v.steps);
                rec.lv = (st[j] >> kLvShift) & 511u;
                rec.sdf_n = fminf(fmaxf(__fmul_rn(sd[j], v.inv_trunc), -1.0f), 1.0f);
                rec.w_in = 1.0f;
                *reinterpret_cast<int4*>(&u.records[pos]) = *reinterpret_cast<const int4*>(&rec);
            }
        }
        for (int k = tid; k < n_list; k += kWalkThreads) T.cnt[T.list[k]] = 0;
        __syncthreads();
    }

    if (counts_drops) {
        const unsigned total = __reduce_add_sync(0xffffffffu, drops);
        if ((tid & 31) == 0 && total) atomicAdd(&T.drops, total);
    }
    __syncthreads();
    if (tid == 0 && T.drops) atomicAdd(v.drop_count, (unsigned long long)T.drops);
    if (MODE == kAllocProbeHist) {
        for (int k = tid; k < min(n_bins, 64); k += kWalkThreads)
            if (T.hist[k]) atomicAdd(&hist[k], (unsigned long long)T.hist[k]);
    }

    if (TAIL == kTailStage) {
        // The last CTA to finish turns the per-block counts into bins.
        __syncthreads();
        if (tid == 0) {
            __threadfence();
            T.last = atomicAdd(&u.ctl->cta_done, 1) == (int)gridDim.x - 1;
        }
        __syncthreads();
        if (T.last) {
            __threadfence();
            scan_blocks(T, u);
        }
    }
}

template <int MODE, int TAIL>
cudaError_t launch_walk(const DevVolume& v, const BatchArgs& a, const UpdateScratch& u,
                        unsigned long long* hist, int n_bins, cudaStream_t s) {
    const int grid = (a.n + kWalkThreads - 1) / kWalkThreads;
    walk_kernel<MODE, TAIL><<<grid, kWalkThreads, 0, s>>>(v, a, u, hist, n_bins);
    return cudaGetLastError();
}

}  // namespace

cudaError_t launch_allocate(const DevVolume& v, const BatchArgs& a, int mode,
                            unsigned long long* hist, int n_bins, cudaStream_t s) {
    if (a.n <= 0) return cudaSuccess;
    const UpdateScratch none{};
    switch (mode) {
        case kAllocInsert: return launch_walk<kAllocInsert, kTailDrops>(v, a, none, hist, n_bins, s);
        case kAllocCountingCas: return launch_walk<kAllocCountingCas, kTailDrops>(v, a, none, hist, n_bins, s);
        case kAllocNoCas: return launch_walk<kAllocNoCas, kTailDrops>(v, a, none, hist, n_bins, s);
        case kAllocProbeHist: return launch_walk<kAllocProbeHist, kTailDrops>(v, a, none, hist, n_bins, s);
        case kAllocSlotIndex: return launch_walk<kAllocSlotIndex, kTailDrops>(v, a, none, hist, n_bins, s);
        default: return cudaErrorInvalidValue;
    }
}

cudaError_t launch_update_stage(const DevVolume& v, const BatchArgs& a, const UpdateScratch& u,
                                bool insert, cudaStream_t s) {
    if (a.n <= 0) return cudaSuccess;
    return insert ? launch_walk<kAllocInsert, kTailStage>(v, a, u, nullptr, 1, s)
                  : launch_walk<kLookupOnly, kTailStage>(v, a, u, nullptr, 1, s);
}

}  // namespace osn_b200
