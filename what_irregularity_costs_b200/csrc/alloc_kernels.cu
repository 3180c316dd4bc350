// Allocate: insert every block the batch's truncation bands touch.
//
// Reference: cpp/src/volume.cpp:147-198 (CPU arm) and cpp/src/volume_cuda.cu:59-107,
// :259-269 (CUDA arm, one thread per point, one compare-exchange per sample).
//
// B200 design. One thread walks one point's band (2*steps+1 samples), but a
// sample only becomes a table request when its block differs from the
// previous sample of the same ray, and requests are deduplicated across the
// warp with __match_any_sync on the 64-bit key before any thread touches the
// table: only one leader per distinct key probes and compare-exchanges. The
// 32 rays of a warp come from neighbouring pixels and share most blocks, so
// the probe traffic and CAS contention drop by an order of magnitude against
// one probe per sample. The table (16 B slots, 2^16-2^22 of them) stays
// resident in the 126 MB L2; probes and CASes are L2 transactions.
//
// Insertion protocol (the reference's, volume_cuda.cu:82-95): CAS the key into
// an empty slot, take a pool index from the counter, write the coordinate,
// fence, publish the index. A request that finds its key already claimed
// waits, with an iteration bound, for the index to be published or the claim
// rolled back; a timeout sets a status bit instead of hanging.
#include "volume.h"

namespace osn_b200 {
namespace {

constexpr int kAllocThreads = 256;

// Result of one leader's request.
struct InsertResult {
    int32_t idx;      // >= 0 allocated or found, -1 dropped
    uint32_t probes;  // slots visited
};

__device__ int32_t wait_published(const DevVolume& v, HashEntry* e, long long want) {
    for (int it = 0; it < kSpinLimit; ++it) {
        const int idx = ld_acquire_s32(&e->block_idx);
        if (idx >= 0) return idx;
        // The claim was rolled back (pool full): the block does not exist.
        if (ld_relaxed_s64(&e->key) != want) return -1;
        __nanosleep(64);
    }
    atomicOr(v.status, kStatusSpinTimeout);
    return -1;
}

template <int MODE>
__device__ InsertResult find_or_insert(const DevVolume& v, int32_t bx, int32_t by, int32_t bz,
                                       long long want) {
    InsertResult res{-1, 0};
    const uint32_t mask = (MODE == kAllocSlotIndex) ? (uint32_t)v.pool_capacity - 1u : v.hash_mask;
    const uint32_t size = mask + 1;
    const uint32_t start = hash_slot(bx, by, bz, mask);
    for (uint32_t p = 0; p < size; ++p) {
        const uint32_t slot = (start + p) & mask;
        HashEntry* e = &v.table[slot];
        ++res.probes;
        long long key = ld_relaxed_s64(&e->key);
        if (key == want) {
            if (MODE == kAllocNoCas) { res.idx = 0; return res; }
            if (MODE == kAllocSlotIndex) { res.idx = (int32_t)slot; return res; }
            res.idx = wait_published(v, e, want);
            return res;
        }
        if (key == kEmptyKey) {
            if (MODE == kAllocNoCas) return res;
            if (MODE != kAllocSlotIndex &&
                ld_relaxed_s32(v.block_count) >= v.pool_capacity) {
                // Pool already full: the insert could only be rolled back.
                return res;
            }
            if (MODE == kAllocCountingCas) atomicAdd(v.drop_count, 1ULL);
            const long long prev = (long long)atomicCAS((unsigned long long*)&e->key,
                                                        (unsigned long long)kEmptyKey,
                                                        (unsigned long long)want);
            if (prev == kEmptyKey) {
                if (MODE == kAllocSlotIndex) {
                    v.block_coord[slot] = BlockCoord{bx, by, bz};
                    atomicAdd(v.block_count, 1);
                    __threadfence();
                    atomicExch(&e->block_idx, (int)slot);
                    res.idx = (int32_t)slot;
                    return res;
                }
                const int32_t idx = atomicAdd(v.block_count, 1);
                if (idx >= v.pool_capacity) {
                    atomicSub(v.block_count, 1);
                    atomicExch((unsigned long long*)&e->key, (unsigned long long)kReleasedKey);
                    return res;
                }
                v.block_coord[idx] = BlockCoord{bx, by, bz};
                __threadfence();  // coordinate visible before the index
                atomicExch(&e->block_idx, idx);
                res.idx = idx;
                return res;
            }
            key = prev;
            if (prev == want) {
                if (MODE == kAllocSlotIndex) { res.idx = (int32_t)slot; return res; }
                res.idx = wait_published(v, e, want);
                return res;
            }
        }
        // Another key, a rolled-back slot or a scratch sentinel: probe on.
    }
    return res;  // table full
}

template <int MODE>
__global__ void __launch_bounds__(kAllocThreads, 4)
alloc_kernel(DevVolume v, BatchArgs a, unsigned long long* hist, int n_bins) {
    __shared__ unsigned int s_hist[64];
    if (MODE == kAllocProbeHist) {
        for (int k = threadIdx.x; k < 64; k += blockDim.x) s_hist[k] = 0u;
        __syncthreads();
    }
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int lane = threadIdx.x & 31;
    Ray r;
    const bool live = i < a.n && ray_setup(a, i, r);

    unsigned drops = 0;
    if (__any_sync(0xffffffffu, live)) {
        long long last_key = kNoKey;
        bool last_ok = true;
        for (int s = -v.steps; s <= v.steps; ++s) {
            long long key = kNoKey;
            int bx = 0, by = 0, bz = 0;
            bool fresh = false;
            if (live) {
                int vx, vy, vz;
                float sdf;
                if (band_sample(v, a, r, s, vx, vy, vz, sdf)) {
                    bx = vx >> 3;  // floor_div(v, 8) for int32 (types.hpp:162-165)
                    by = vy >> 3;
                    bz = vz >> 3;
                    key = pack_key(bx, by, bz);
                    if (key == last_key) {
                        if (!last_ok) ++drops;  // same block, already known to be dropped
                    } else {
                        fresh = true;
                    }
                }
            }
            const unsigned want_mask = __ballot_sync(0xffffffffu, fresh);
            if (fresh) {
                const unsigned grp = __match_any_sync(want_mask, key);
                const int leader = __ffs(grp) - 1;
                int ok = 0;
                if (lane == leader) {
                    const InsertResult res = find_or_insert<MODE>(v, bx, by, bz, key);
                    ok = res.idx >= 0;
                    if (MODE == kAllocProbeHist) {
                        atomicAdd(&s_hist[min(res.probes, (uint32_t)min(n_bins, 64) - 1u)], 1u);
                    }
                }
                ok = __shfl_sync(grp, ok, leader);
                last_key = key;
                last_ok = ok != 0;
                if (!ok && MODE != kAllocNoCas) ++drops;
            }
        }
    }
    if (MODE != kAllocNoCas && MODE != kAllocCountingCas) {
        const unsigned total = __reduce_add_sync(0xffffffffu, drops);
        if (lane == 0 && total) atomicAdd(v.drop_count, (unsigned long long)total);
    }
    if (MODE == kAllocProbeHist) {
        __syncthreads();
        for (int k = threadIdx.x; k < min(n_bins, 64); k += blockDim.x)
            if (s_hist[k]) atomicAdd(&hist[k], (unsigned long long)s_hist[k]);
    }
}

}  // namespace

cudaError_t launch_allocate(const DevVolume& v, const BatchArgs& a, int mode,
                            unsigned long long* hist, int n_bins, cudaStream_t s) {
    if (a.n <= 0) return cudaSuccess;
    const int grid = (a.n + kAllocThreads - 1) / kAllocThreads;
    switch (mode) {
        case kAllocInsert: alloc_kernel<kAllocInsert><<<grid, kAllocThreads, 0, s>>>(v, a, hist, n_bins); break;
        case kAllocCountingCas: alloc_kernel<kAllocCountingCas><<<grid, kAllocThreads, 0, s>>>(v, a, hist, n_bins); break;
        case kAllocNoCas: alloc_kernel<kAllocNoCas><<<grid, kAllocThreads, 0, s>>>(v, a, hist, n_bins); break;
        case kAllocProbeHist: alloc_kernel<kAllocProbeHist><<<grid, kAllocThreads, 0, s>>>(v, a, hist, n_bins); break;
        case kAllocSlotIndex: alloc_kernel<kAllocSlotIndex><<<grid, kAllocThreads, 0, s>>>(v, a, hist, n_bins); break;
        default: return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

}  // namespace osn_b200
