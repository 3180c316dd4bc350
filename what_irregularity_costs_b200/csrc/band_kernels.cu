// The band walk: allocate, and count-and-sum (the first half of update,
// fused with allocation in integrate).
//
// Reference: cpp/src/volume.cpp:147-198 and :200-299 (one sample at a time:
// find_or_insert / find_block per sample) and cpp/src/volume_cuda.cu:160-192,
// :259-269, :302-337 (one thread per point, one hash probe sequence per
// sample).
//
// One thread walks one point's band (2*steps+1 samples, kChunk at a time in
// registers); a persistent grid of CTAs strides over tiles of 128
// consecutive points (neighbouring pixels of a frame). Along a ray the block
// changes rarely, so a thread keeps the runs of equal blocks of its chunk
// (their keys in a per-thread column of shared memory) and resolves each
// once. The resolution is warp-cooperative: for each run index the warp's
// lanes group equal block keys with __match_any_sync and only the lowest lane
// of a group probes the global table (and inserts), then broadcasts the pool
// index with a shuffle -- neighbouring pixels share blocks, so the table sees
// a fraction of the per-sample probes and far fewer contending CAS attempts
// on a new block.
//
// Update tail. The group leader also tags the block as touched by this update
// (one atomic exchange; the first tagger appends it to the touched list).
// Every band sample whose voxel can still accept a contribution adds one to
// the voxel's batch count and its normalised SDF, in 2^-40 fixed point, to
// the voxel's 64-bit sum: two fire-and-forget L2 reductions, whose order does
// not matter. Every band slot (point i, step s) also gets a 4-byte record at
// records[(s + steps) * n + i] -- step-major, so each store of a warp is one
// contiguous 128-byte line -- holding the voxel's global index or kNoVoxel;
// only voxels that cross the cap read them again (their canonical order is
// the record position).
//
// Samples whose voxel already holds the cap's weight are left out: under
// "accept while weight before < cap" they cannot be accepted in any order,
// so leaving them out changes no result.
#include <algorithm>
#include <mutex>

#include "volume.h"

namespace osn_b200 {
namespace {

constexpr int kBandThreads = 128;
constexpr int kChunk = 9;  // samples per ray held in registers (the whole band at 4 voxels)

// Per-sample state: voxel within block (9 bits), run index (4 bits), valid.
constexpr uint32_t kLvMask = 0x1FFu;
constexpr int kRunShift = 9;
constexpr uint32_t kValid = 1u << 30;

template <int MODE>
__device__ __forceinline__ int32_t resolve(const DevVolume& v, int bx, int by, int bz, long long key,
                                           unsigned long long* hist, int n_bins) {
    if (MODE == kLookupOnly) return find_block(v, bx, by, bz, key);
    const InsertResult r = find_or_insert<MODE>(v, bx, by, bz, key);
    if (MODE == kAllocProbeHist && n_bins > 0)
        atomicAdd(&hist[min(r.probes, (uint32_t)(n_bins - 1))], 1ull);
    return r.idx;
}

template <int MODE, bool RECORDS>
__global__ void __launch_bounds__(kBandThreads)
band_kernel(DevVolume v, BatchArgs a, UpdateScratch u, unsigned long long* hist, int n_bins) {
    // Per-thread columns: run q of thread t at [q][t] (no bank conflicts).
    __shared__ long long run_key[kChunk][kBandThreads];
    __shared__ int32_t run_bi[kChunk][kBandThreads];
    const int t = threadIdx.x;
    const int lane = t & 31;
    const bool counts_drops = MODE != kLookupOnly && MODE != kAllocNoCas && MODE != kAllocCountingCas;
    const bool sat_check = RECORDS && v.weight_cap > 0.0f;
    const int n_tiles = (a.n + kBandThreads - 1) / kBandThreads;
    uint32_t drops = 0, counted = 0;

    for (int tile = blockIdx.x; tile < n_tiles; tile += gridDim.x) {
        const int i = tile * kBandThreads + t;
        Ray r;
        const bool live = i < a.n && ray_setup(a, i, r);
        uint32_t* rec = RECORDS ? u.records + i : nullptr;  // slot (s = -steps, i)

        for (int c0 = -v.steps; c0 <= v.steps; c0 += kChunk) {
            uint32_t st[kChunk];
            float sd[kChunk];
            int n_run = 0;
            long long last = kNoKey;

            // Phase 1: the chunk's samples; distinct blocks in walk order.
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
                    // A straight ray leaves a block (a convex box) for good, so
                    // equal consecutive keys are the only repeats.
                    if (key != last) {
                        last = key;
                        run_key[n_run][t] = key;
                        ++n_run;
                    }
                    const uint32_t lv =
                        (uint32_t)(((vz & 7) * kBlockDim + (vy & 7)) * kBlockDim + (vx & 7));
                    st[j] = kValid | lv | (uint32_t)(n_run - 1) << kRunShift;
                    sd[j] = sdf;
                }
            }

            // Phase 2: warp rounds, one per run index; one probe per distinct key.
            for (int q = 0; q < kChunk; ++q) {
                if (!__any_sync(0xffffffffu, q < n_run)) break;
                const long long key = q < n_run ? run_key[q][t] : kNoKey;
                const unsigned grp = __match_any_sync(0xffffffffu, key);
                const int leader = __ffs(grp) - 1;
                int32_t bi = -1;
                if (key != kNoKey && lane == leader) {
                    const int bx = unpack_axis(key, 2 * kCoordBits);
                    const int by = unpack_axis(key, kCoordBits);
                    const int bz = unpack_axis(key, 0);
                    bi = resolve<MODE>(v, bx, by, bz, key, hist, n_bins);
                    if (RECORDS && bi >= 0 && atomicExch(&u.blk_touch[bi], u.tag) != u.tag)
                        u.touched[atomicAdd(&u.ctl->n_touched, 1)] = bi;
                }
                run_bi[q][t] = __shfl_sync(0xffffffffu, bi, leader);
            }

            // Phase 3: drops; then every sample's weight gather in flight
            // together; then the saturation gate, counts, sums and records.
            uint32_t vox[kChunk];
#pragma unroll
            for (int j = 0; j < kChunk; ++j) {
                vox[j] = kNoVoxel;
                if (st[j] & kValid) {
                    const int32_t bi = run_bi[(st[j] >> kRunShift) & 15u][t];
                    if (bi < 0) {
                        if (counts_drops) ++drops;
                    } else {
                        vox[j] = (uint32_t)bi * kBlockVoxels + (st[j] & kLvMask);
                    }
                }
            }
            if (RECORDS) {
                float w0[kChunk];
#pragma unroll
                for (int j = 0; j < kChunk; ++j)
                    w0[j] = (sat_check && vox[j] != kNoVoxel) ? __ldg(&v.weight[vox[j]]) : 0.0f;
#pragma unroll
                for (int j = 0; j < kChunk; ++j) {
                    if (c0 + j > v.steps) break;
                    uint32_t out = kNoVoxel;
                    if (vox[j] != kNoVoxel && !(sat_check && w0[j] >= v.weight_cap)) {
                        out = vox[j];
                        const float sdf_n = fminf(fmaxf(__fmul_rn(sd[j], v.inv_trunc), -1.0f), 1.0f);
                        atomicAdd(&u.vcnt[out], 1u);
                        atomicAdd(&u.vacc[out], (unsigned long long)to_fix(sdf_n));
                        ++counted;
                    }
                    if (i < a.n) *rec = out;
                    rec += a.n;
                }
            }
        }
    }

    if (counts_drops) {
        const unsigned total = __reduce_add_sync(0xffffffffu, drops);
        if (lane == 0 && total) atomicAdd(v.drop_count, (unsigned long long)total);
    }
    if (RECORDS) {
        const unsigned total = __reduce_add_sync(0xffffffffu, counted);
        if (lane == 0 && total) atomicAdd(&u.ctl->n_records, (int)total);
    }
}

template <int MODE, bool RECORDS>
cudaError_t launch(const DevVolume& v, const BatchArgs& a, const UpdateScratch& u,
                   unsigned long long* hist, int n_bins, int sm_count, cudaStream_t s) {
    if (a.n <= 0) return cudaSuccess;
    // Persistent grid: as many CTAs as are resident at once (queried once
    // per instantiation), striding over the point tiles.
    static int per_sm = 0;
    static std::once_flag once;
    std::call_once(once, [] {
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, band_kernel<MODE, RECORDS>,
                                                          kBandThreads, 0) != cudaSuccess ||
            per_sm < 1)
            per_sm = 1;
    });
    const int tiles = (a.n + kBandThreads - 1) / kBandThreads;
    const int grid = std::min(tiles, per_sm * sm_count);
    band_kernel<MODE, RECORDS><<<grid, kBandThreads, 0, s>>>(v, a, u, hist, n_bins);
    return cudaGetLastError();
}

}  // namespace

cudaError_t launch_allocate(const DevVolume& v, const BatchArgs& a, int mode,
                            unsigned long long* hist, int n_bins, int sm_count, cudaStream_t s) {
    const UpdateScratch none{};
    switch (mode) {
        case kAllocInsert: return launch<kAllocInsert, false>(v, a, none, nullptr, 0, sm_count, s);
        case kAllocCountingCas:
            return launch<kAllocCountingCas, false>(v, a, none, nullptr, 0, sm_count, s);
        case kAllocNoCas: return launch<kAllocNoCas, false>(v, a, none, nullptr, 0, sm_count, s);
        case kAllocProbeHist:
            return launch<kAllocProbeHist, false>(v, a, none, hist, n_bins, sm_count, s);
        case kAllocSlotIndex: return launch<kAllocSlotIndex, false>(v, a, none, nullptr, 0, sm_count, s);
        default: return cudaErrorInvalidValue;
    }
}

cudaError_t launch_band_records(const DevVolume& v, const BatchArgs& a, const UpdateScratch& u,
                                bool insert, int sm_count, cudaStream_t s) {
    return insert ? launch<kAllocInsert, true>(v, a, u, nullptr, 0, sm_count, s)
                  : launch<kLookupOnly, true>(v, a, u, nullptr, 0, sm_count, s);
}

}  // namespace osn_b200
