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
// of a group probes the global table (and inserts), leaving the pool index in
// shared memory for the group -- neighbouring pixels share blocks, so the
// table sees a fraction of the per-sample probes and far fewer contending CAS
// attempts on a new block. The groups of all run indices are formed first and
// each leader then resolves its runs with their home-slot probes in flight
// together, so a chunk waits for about one table access, not one per run.
//
// Update tail. The group leader also tags the block as touched by this update
// (one atomic exchange unless a cached read already shows the tag; the first
// tagger appends it to the touched list).
// Every band sample whose voxel can still accept a contribution adds one to
// the voxel's batch count and its normalised SDF, in 2^-40 fixed point, to
// the voxel's 64-bit sum: fire-and-forget L2 reductions, whose order does not
// matter, issued once per run of consecutive lanes that share the voxel. Every band slot (point i, step s) also gets a 4-byte record at
// records[(s + steps) * n + i] -- step-major, so each store of a warp is one
// contiguous 128-byte line -- holding the voxel's global index or kNoVoxel;
// only voxels that cross the cap read them again (their canonical order is
// the record position).
//
// Samples whose voxel already holds the cap's weight are left out: under
// "accept while weight before < cap" they cannot be accepted in any order,
// so leaving them out changes no result.
//
// Several frames per call (band_frames_kernel, band_depth_frames_kernel): the
// same walk, each point seen from the camera of its frame (a per-call table
// the set-up kernel stores; depth images also carry their poses). The points
// of frame k precede those of frame k+1, so the canonical (point, step) order
// is (frame, point, step) order and the cap keeps what per-frame calls keep.
#include <algorithm>
#include <climits>
#include <mutex>

#include "volume.h"

namespace osn_b200 {
namespace {

constexpr int kBandThreads = kBatchTilePoints;
static_assert(kBandThreads >= kMaxBatchScenes, "one thread per scene builds the item prefix");
#ifndef OSN_BAND_CHUNK
#define OSN_BAND_CHUNK 9
#endif
constexpr int kChunk = OSN_BAND_CHUNK;  // samples per ray held in registers (9: the whole band at 4 voxels)
// Resident CTAs per SM the register budget is sized for. The several-frame
// and batched walks: 7 (72 registers), measured 1.4 % faster on the room
// trajectory than 8 (64 registers) and 6; the one-frame walk: 8 (at 7 it
// measured 6 % slower, its batches are a third of the size).
#ifndef OSN_BAND_MIN_BLOCKS
#define OSN_BAND_MIN_BLOCKS 8
#endif
#ifndef OSN_BAND_FRAMES_MIN_BLOCKS
#define OSN_BAND_FRAMES_MIN_BLOCKS 7
#endif
constexpr int kBandMinBlocks = OSN_BAND_MIN_BLOCKS;
constexpr int kBandFramesMinBlocks = OSN_BAND_FRAMES_MIN_BLOCKS;

// Band records and slot values are read once more, by the group pass of the
// same update: stored with the streaming hint (1, evict-first) or as
// ordinary write-back stores that may stay in L2 (0).
// 1: a several-frame walk is launched with programmatic stream serialisation
// behind its one-CTA set-up kernel, so its CTAs are resident when the set-up
// ends (they wait for it on the device; measured 0.8 % faster on the room
// trajectory); 0: an ordinary launch.
#ifndef OSN_BAND_PDL
#define OSN_BAND_PDL 1
#endif

#ifndef OSN_BAND_STREAM_RECORDS
#define OSN_BAND_STREAM_RECORDS 1
#endif

template <typename T>
__device__ __forceinline__ void store_slot(T* p, T x) {
    if (OSN_BAND_STREAM_RECORDS) __stcs(p, x);
    else *p = x;
}

// Per-sample state: voxel within block (9 bits), run index (4 bits), valid.
constexpr uint32_t kLvMask = 0x1FFu;
constexpr int kRunShift = 9;
constexpr uint32_t kValid = 1u << 30;

template <int MODE>
__device__ __forceinline__ int32_t resolve(const DevVolume& v, long long key,
                                           unsigned long long* hist, int n_bins) {
    const int bx = unpack_axis(key, 2 * kCoordBits);
    const int by = unpack_axis(key, kCoordBits);
    const int bz = unpack_axis(key, 0);
    if (MODE == kLookupOnly) return find_block(v, bx, by, bz, key);
    const InsertResult r = find_or_insert<MODE>(v, bx, by, bz, key);
    if (MODE == kAllocProbeHist && n_bins > 0)
        atomicAdd(&hist[min(r.probes, (uint32_t)(n_bins - 1))], 1ull);
    return r.idx;
}

// Modes whose first probe may be answered from the block's home slot alone.
template <int MODE>
__device__ __forceinline__ constexpr bool has_fast_probe() {
    return MODE == kAllocInsert || MODE == kLookupOnly;
}

// The block's home-slot entry, through L1. A slot goes empty -> claimed
// (key, -1) -> published (key, index) and never changes again within an
// update, so an entry that shows this key with a valid index is final, and
// with no concurrent insertion (lookup) an empty home slot means absent.
template <int MODE>
__device__ __forceinline__ int4 home_entry(const DevVolume& v, long long key) {
    if (!has_fast_probe<MODE>()) return make_int4(0, 0, -1, 0);
    const uint32_t h = hash_slot(unpack_axis(key, 2 * kCoordBits), unpack_axis(key, kCoordBits),
                                 unpack_axis(key, 0), v.hash_mask);
    const int4* e = reinterpret_cast<const int4*>(&v.table[h]);
    return MODE == kLookupOnly ? __ldg(e) : __ldca(e);
}

// The pool index the home entry settles, or -2 when the full probe is needed.
template <int MODE>
__device__ __forceinline__ int32_t settle_home(const DevVolume& v, int4 raw, long long key) {
    if (!has_fast_probe<MODE>()) return -2;
    const long long k0 = ((long long)(unsigned)raw.y << 32) | (unsigned)raw.x;
    if (k0 == key && raw.z >= 0 && raw.z < v.pool_capacity) return raw.z;
    if (MODE == kLookupOnly && k0 == kEmptyKey) return -1;
    return -2;
}

// The full probe (and insertion) protocol, out of line: it is the rare path
// of the fast-probe modes and keeps their walk loop in registers.
template <int MODE>
__device__ __noinline__ int32_t resolve_slow(HashEntry* table, uint32_t hash_mask, int32_t pool,
                                             int32_t* block_count, unsigned long long* drop_count,
                                             BlockCoord* block_coord, uint32_t* status,
                                             int32_t spin_limit, int32_t* block_chunk, int32_t chunk,
                                             int32_t slot_index, long long key) {
    DevVolume v{};
    v.table = table;
    v.hash_mask = hash_mask;
    v.pool_capacity = pool;
    v.block_count = block_count;
    v.drop_count = drop_count;
    v.block_coord = block_coord;
    v.status = status;
    v.spin_limit = spin_limit;
    v.block_chunk = block_chunk;
    v.chunk = chunk;
    v.slot_index = slot_index;
    return resolve<MODE>(v, key, nullptr, 0);
}

template <int MODE>
__device__ __forceinline__ int32_t resolve_from(const DevVolume& v, int4 raw, long long key,
                                                unsigned long long* hist, int n_bins) {
    if (!has_fast_probe<MODE>()) return resolve<MODE>(v, key, hist, n_bins);
    const int32_t bi = settle_home<MODE>(v, raw, key);
    if (bi != -2) return bi;
    return resolve_slow<MODE>(v.table, v.hash_mask, v.pool_capacity, v.block_count, v.drop_count,
                              v.block_coord, v.status, v.spin_limit, v.block_chunk, v.chunk, v.slot_index,
                              key);
}

// Tag a block as touched by this update; the first tagger appends it to the
// touched list. A cached read that already shows the tag saves the exchange
// (a stale read can only show an older tag). The appends of the lanes that
// arrive together take their places with one atomic on the list's counter.
__device__ __forceinline__ void tag_touched(const UpdateScratch& u, int32_t bi, uint32_t seen) {
    const bool add = bi >= 0 && seen != u.tag && atomicExch(&u.blk_touch[bi], u.tag) != u.tag;
    const unsigned act = __activemask();
    const unsigned want = __ballot_sync(act, add);
    if (!want) return;
    const int ldr = __ffs(want) - 1;
    int base = 0;
    if ((int)(threadIdx.x & 31) == ldr) base = atomicAdd(&u.ctl->n_touched, __popc(want));
    base = __shfl_sync(act, base, ldr);
    if (add) u.touched[base + __popc(want & lanemask_lt())] = bi;
}

// Fire-and-forget L2 reductions (no value comes back, nothing waits).
__device__ __forceinline__ void red_add(uint32_t* p, uint32_t x) {
    asm volatile("red.global.add.u32 [%0], %1;" ::"l"(p), "r"(x));
}
__device__ __forceinline__ void red_add(unsigned long long* p, unsigned long long x) {
    asm volatile("red.global.add.u64 [%0], %1;" ::"l"(p), "l"(x));
}

// Shared memory of one band CTA: per-thread run columns, run q of thread t
// at [q][t] (no bank conflicts).
struct BandSmem {
    long long run_key[kChunk][kBandThreads];
    int32_t run_bi[kChunk][kBandThreads];   // written by the run's group leader
    uint8_t run_src[kChunk][kBandThreads];  // leader lane of the run's group
};

// Walk point i (already loaded into px, py, pz; i >= a.n for lanes without a
// point) through its band: runs, warp-cooperative block resolution, then
// the update tail. Called by every thread of the CTA, warp-synchronously.
// Block resolution schemes of the band walk.
constexpr int kProbeWarp = 0;  // equal keys grouped across the warp, one leader probes
constexpr int kProbeLane = 1;  // every lane probes its own runs (L1 shares the loads)

// FRAMES: the batch holds several frames; (cx, cy, cz) is the camera of
// point i's frame (otherwise the batch's one camera is used).
template <int MODE, bool RECORDS, int S, int PROBE = kProbeWarp, bool FRAMES = false>
__device__ __forceinline__ void band_point(const DevVolume& v, const BatchArgs& a, const UpdateScratch& u,
                                           int i, bool has, float px, float py, float pz, BandSmem& sm,
                                           uint32_t& drops, uint32_t& counted,
                                           unsigned long long* hist, int n_bins, float cx = 0.0f,
                                           float cy = 0.0f, float cz = 0.0f) {
    static_assert(!(FRAMES && S == kStoreF64), "the FP64 oracle integrates one frame per batch");
    const int t = threadIdx.x;
    const int lane = t & 31, wbase = t & ~31;
    const bool counts_drops = MODE != kLookupOnly && MODE != kAllocNoCas && MODE != kAllocCountingCas;
    const bool sat_check = RECORDS && v.weight_cap > 0.0f;
    auto& run_key = sm.run_key;
    auto& run_bi = sm.run_bi;
    auto& run_src = sm.run_src;
    Ray r;
    const bool live = i < a.n && has &&
                      (FRAMES ? ray_setup_cam(a.radius_sq, cx, cy, cz, px, py, pz, r)
                              : ray_setup_at(a, px, py, pz, r));
    uint32_t* rec = RECORDS ? u.records + i : nullptr;  // slot (s = -steps, i)

    for (int c0 = -v.steps; c0 <= v.steps; c0 += kChunk) {
        uint32_t st[kChunk];
        float sd[kChunk];
        int n_run = 0;
        long long last = kNoKey;

        // Phase 1: the chunk's samples; runs of equal blocks in walk order.
#pragma unroll
        for (int j = 0; j < kChunk; ++j) {
            st[j] = 0u;
            sd[j] = 0.0f;
            const int s = c0 + j;
            int vx, vy, vz;
            float sdf;
            if (live && s <= v.steps &&
                (FRAMES ? band_sample_ray(v, r, s, vx, vy, vz, sdf) : band_sample(v, a, r, s, vx, vy, vz, sdf))) {
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

        // Phase 2a: group equal keys across the warp, one round per run
        // index; the lowest lane of a group leads it. (Per-lane probing: every
        // lane leads its own runs.)
        uint32_t lead = 0u;
        if constexpr (PROBE == kProbeWarp) {
            for (int q = 0; q < kChunk; ++q) {
                if (!__any_sync(0xffffffffu, q < n_run)) break;
                const long long key = q < n_run ? run_key[q][t] : kNoKey;
                const unsigned grp = __match_any_sync(0xffffffffu, key);
                const int leader = __ffs(grp) - 1;
                if (q < n_run) run_src[q][t] = (uint8_t)leader;
                if (key != kNoKey && lane == leader) lead |= 1u << q;
            }
        } else {
            for (int q = 0; q < n_run; ++q) run_src[q][t] = (uint8_t)lane;
            lead = n_run ? (1u << n_run) - 1u : 0u;
        }
        // Phase 2b: each leader resolves its runs two at a time, both
        // home-slot probes (and then both tag reads) in flight together.
        while (lead) {
            const int qa = __ffs(lead) - 1;
            lead &= lead - 1u;
            const int qb = lead ? __ffs(lead) - 1 : -1;
            if (qb >= 0) lead &= lead - 1u;
            const long long ka = run_key[qa][t];
            const long long kb = qb >= 0 ? run_key[qb][t] : kNoKey;
            const int4 ra = home_entry<MODE>(v, ka);
            const int4 rb = qb >= 0 ? home_entry<MODE>(v, kb) : make_int4(0, 0, -1, 0);
            const int32_t ba = resolve_from<MODE>(v, ra, ka, hist, n_bins);
            const int32_t bb = qb >= 0 ? resolve_from<MODE>(v, rb, kb, hist, n_bins) : -1;
            run_bi[qa][t] = ba;
            if (qb >= 0) run_bi[qb][t] = bb;
            if (RECORDS) {
                const uint32_t sa = ba >= 0 ? __ldca(&u.blk_touch[ba]) : u.tag;
                const uint32_t sb = bb >= 0 ? __ldca(&u.blk_touch[bb]) : u.tag;
                tag_touched(u, ba, sa);
                tag_touched(u, bb, sb);
            }
        }
        __syncwarp();

        // Phase 3: drops; then every sample's weight gather in flight
        // together; then the saturation gate, counts, sums and records.
        uint32_t vox[kChunk];
#pragma unroll
        for (int j = 0; j < kChunk; ++j) {
            vox[j] = kNoVoxel;
            if (st[j] & kValid) {
                const uint32_t q = (st[j] >> kRunShift) & 15u;
                const int32_t bi = run_bi[q][wbase + run_src[q][t]];
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
                w0[j] = (sat_check && vox[j] != kNoVoxel) ? weight_at<S>(v, vox[j]) : 0.0f;
#pragma unroll
            for (int j = 0; j < kChunk; ++j) {
                if (c0 + j > v.steps) break;
                uint32_t out = kNoVoxel;
                if (vox[j] != kNoVoxel && !(sat_check && w0[j] >= v.weight_cap)) {
                    out = vox[j];
                    long long fix;
                    if constexpr (S == kStoreF64) {
                        // The oracle's value of the same sample, in double.
                        const long long key = run_key[(st[j] >> kRunShift) & 15u][t];
                        const uint32_t lv = st[j] & kLvMask;
                        const int vx = unpack_axis(key, 2 * kCoordBits) * kBlockDim + (int)(lv & 7u);
                        const int vy = unpack_axis(key, kCoordBits) * kBlockDim + (int)((lv >> 3) & 7u);
                        const int vz = unpack_axis(key, 0) * kBlockDim + (int)(lv >> 6);
                        fix = to_fix(clamp_sdf_n_f64(sdf_f64(v, a, r.px, r.py, r.pz, vx, vy, vz), v.trunc));
                    } else {
                        const float sdf_n = fminf(fmaxf(__fmul_rn(sd[j], v.inv_trunc), -1.0f), 1.0f);
                        fix = to_fix(sdf_n);
                        // Kept for the records of voxels that cross the cap, so the
                        // update tail never reads the batch's points again.
                        store_slot(u.slot_val + (rec - u.records), sdf_n);
                    }
                    red_add(&u.vcnt[out], 1u);
                    red_add(&u.vacc[out], (unsigned long long)fix);
                    ++counted;
                }
                if (i < a.n) store_slot(rec, out);  // read again by the group pass
                rec += a.n;
            }
        }
        __syncwarp();  // run columns are rewritten by the next chunk
    }
}

// The camera of every point of a batch with one camera: nothing to track.
struct OneCamera {
    float cx = 0.0f, cy = 0.0f, cz = 0.0f;
    __device__ __forceinline__ void at(int) {}
};

// The camera of each point of a batch of several frames. A thread's points
// only move forward (tile += grid size), so its frame does too: one
// comparison per tile, and a table read only where the frame changes.
struct FrameCursor {
    const FrameCam* frames;
    int32_t n, f, next;
    float cx, cy, cz;
    __device__ __forceinline__ FrameCursor(const FrameCam* fr, int32_t nf) : frames(fr), n(nf), f(0) {
        load();
    }
    __device__ __forceinline__ void load() {
        cx = __ldg(&frames[f].x);
        cy = __ldg(&frames[f].y);
        cz = __ldg(&frames[f].z);
        next = f + 1 < n ? __ldg(&frames[f + 1].begin) : INT_MAX;
    }
    __device__ __forceinline__ void at(int i) {
        while (i >= next) {  // the last frame's bound is INT_MAX
            ++f;
            load();
        }
    }
};

// Where a batch's points come from: xyz positions or one depth image.
template <int SOURCE>
struct BatchPoints {
    const BatchArgs& a;
    __device__ __forceinline__ bool load(int i, float& px, float& py, float& pz) const {
        return load_point<SOURCE>(a, i, px, py, pz);
    }
};

// Several depth images of npix pixels back to back: pixel i belongs to image
// i / npix, unprojected with that image's pose (staged in shared memory).
struct DepthFramesPoints {
    const BatchArgs& a;
    const FramePose* pose;
    int32_t npix;
    __device__ __forceinline__ bool load(int i, float& px, float& py, float& pz) const {
        const int f = i / npix;
        return unproject_pixel(a.depth, pose[f].R, pose[f].t, i, i - f * npix, px, py, pz);
    }
};

// A persistent CTA's share of a batch: tiles of 128 points, strided by the
// grid, then the CTA's drop and record counts.
template <int MODE, bool RECORDS, int S, bool FRAMES, typename Points, typename Camera>
__device__ __forceinline__ void band_tiles(const DevVolume& v, const BatchArgs& a, const UpdateScratch& u,
                                           unsigned long long* hist, int n_bins, const Points pts,
                                           Camera cam) {
    __shared__ BandSmem sm;
    const int t = threadIdx.x;
    const int lane = t & 31;
    const bool counts_drops = MODE != kLookupOnly && MODE != kAllocNoCas && MODE != kAllocCountingCas;
    const int n_tiles = (a.n + kBandThreads - 1) / kBandThreads;
    uint32_t drops = 0, counted = 0;
    __shared__ unsigned s_drops, s_counted;
    if (t == 0) {
        s_drops = 0u;
        s_counted = 0u;
    }
    __syncthreads();
    launch_dependents();  // the finish pass may be scheduled as CTAs retire

    // The point of the next tile is loaded one tile ahead.
    float nx = 0.0f, ny = 0.0f, nz = 0.0f;
    bool nhas = false;
    {
        const int i0 = blockIdx.x * kBandThreads + t;
        if (blockIdx.x < n_tiles && i0 < a.n) nhas = pts.load(i0, nx, ny, nz);
    }
    for (int tile = blockIdx.x; tile < n_tiles; tile += gridDim.x) {
        const int i = tile * kBandThreads + t;
        const float px = nx, py = ny, pz = nz;
        const bool has = nhas;
        const int inext = i + gridDim.x * kBandThreads;
        nhas = false;
        if (inext < a.n) nhas = pts.load(inext, nx, ny, nz);
        cam.at(i);
        band_point<MODE, RECORDS, S, kProbeWarp, FRAMES>(v, a, u, i, has, px, py, pz, sm, drops, counted,
                                                         hist, n_bins, cam.cx, cam.cy, cam.cz);
    }

    // Counters: one global atomic per CTA (per-warp atomics on one line serialise).
    const unsigned wd = counts_drops ? __reduce_add_sync(0xffffffffu, drops) : 0u;
    const unsigned wc = RECORDS ? __reduce_add_sync(0xffffffffu, counted) : 0u;
    if (lane == 0 && wd) atomicAdd(&s_drops, wd);
    if (lane == 0 && wc) atomicAdd(&s_counted, wc);
    __syncthreads();
    if (t == 0 && s_drops) atomicAdd(v.drop_count, (unsigned long long)s_drops);
    if (t == 0 && s_counted) atomicAdd(&u.ctl->n_records, (int)s_counted);
}

template <int MODE, bool RECORDS, int S, bool DEPTH = false>
__global__ void __launch_bounds__(kBandThreads, kBandMinBlocks)
band_kernel(DevVolume v, BatchArgs a, UpdateScratch u, unsigned long long* hist, int n_bins) {
    band_tiles<MODE, RECORDS, S, false>(v, a, u, hist, n_bins, BatchPoints<DEPTH ? 1 : 0>{a}, OneCamera{});
}

// Integrate (allocate + count-and-sum) of a batch of several frames: the
// single-frame walk with each point's camera taken from the frame table.
template <int S>
__global__ void __launch_bounds__(kBandThreads, kBandFramesMinBlocks)
band_frames_kernel(DevVolume v, BatchArgs a, UpdateScratch u, const FrameCam* frames, int32_t n_frames) {
    if (OSN_BAND_PDL) grid_dependency_wait();  // the set-up kernel's frame table and zeroed counters
    band_tiles<kAllocInsert, true, S, true>(v, a, u, nullptr, 0, BatchPoints<0>{a}, FrameCursor(frames, n_frames));
}

// The same for several depth images of equal size: each CTA stages the
// images' poses in shared memory first.
template <int S>
__global__ void __launch_bounds__(kBandThreads, kBandFramesMinBlocks)
band_depth_frames_kernel(DevVolume v, BatchArgs a, UpdateScratch u, const FrameCam* frames,
                         const FramePose* poses, int32_t n_frames) {
    __shared__ FramePose s_pose[kMaxDepthFrames];
    if (OSN_BAND_PDL) grid_dependency_wait();  // the set-up kernel's tables and zeroed counters
    constexpr int kWords = (int)(sizeof(FramePose) / sizeof(double));
    for (int k = threadIdx.x; k < n_frames * kWords; k += blockDim.x)
        reinterpret_cast<double*>(s_pose)[k] = __ldg(reinterpret_cast<const double*>(poses) + k);
    __syncthreads();
    band_tiles<kAllocInsert, true, S, true>(v, a, u, nullptr, 0, DepthFramesPoints{a, s_pose, a.n / n_frames},
                                            FrameCursor(frames, n_frames));
}

// Set-up of a several-frame integrate, in place of the control block's
// memset: zero the control block and store the frame table where the band
// walk reads it (one CTA; static indices only, so the table stays in the
// parameter space).
__global__ void frames_setup_kernel(UpdateControl* ctl, FrameCam* dst, const FrameTable t) {
    if (OSN_BAND_PDL) launch_dependents();  // the walk's CTAs may take their places now
    const int k = threadIdx.x;
    if (k < (int)(sizeof(UpdateControl) / sizeof(uint32_t))) reinterpret_cast<uint32_t*>(ctl)[k] = 0u;
#pragma unroll
    for (int j = 0; j <= kMaxFrames; ++j)
        if (j == k && j <= t.n) dst[j] = t.f[j];
}

// The same for several depth images, with their poses.
__global__ void frames_setup_depth_kernel(UpdateControl* ctl, FrameCam* dst, const FrameTable t,
                                          FramePose* pdst, const PoseTable p) {
    if (OSN_BAND_PDL) launch_dependents();
    const int k = threadIdx.x;
    if (k < (int)(sizeof(UpdateControl) / sizeof(uint32_t))) reinterpret_cast<uint32_t*>(ctl)[k] = 0u;
#pragma unroll
    for (int j = 0; j <= kMaxFrames; ++j)
        if (j == k && j <= t.n) dst[j] = t.f[j];
#pragma unroll
    for (int j = 0; j < kMaxDepthFrames; ++j)
        if (j == k && j < p.n) pdst[j] = p.p[j];
}

// ---- batched steps -----------------------------------------------------

// Copy a POD descriptor into shared memory with the whole CTA.
template <typename T>
__device__ __forceinline__ void cta_copy(T* dst, const T* src) {
    static_assert(sizeof(T) % 4 == 0, "descriptor copies go by words");
    const uint32_t* s = reinterpret_cast<const uint32_t*>(src);
    uint32_t* d = reinterpret_cast<uint32_t*>(dst);
    for (int k = threadIdx.x; k < (int)(sizeof(T) / 4); k += blockDim.x) d[k] = s[k];
}

// Scene of global work item `item` given the per-scene item prefix `begin`
// (n + 1 entries, begin[0] = 0): the last scene whose range starts at or
// before it.
__device__ __forceinline__ int scene_of(const int* begin, int n, int item) {
    int lo = 0, hi = n;  // begin[lo] <= item < begin[hi]
    while (hi - lo > 1) {
        const int mid = (lo + hi) >> 1;
        if (begin[mid] <= item) lo = mid;
        else hi = mid;
    }
    return lo;
}

// Allocate + count-and-sum walk of every scene of a step. Work items are
// runs of tiles_per_item consecutive 128-point tiles of one scene, handed
// out by an atomic queue to a persistent grid; the CTA keeps the current
// item's scene descriptor in shared memory and flushes its per-scene
// counters whenever it moves to another scene.
template <int S, int PROBE>
__global__ void __launch_bounds__(kBandThreads, kBandFramesMinBlocks)
band_multi_kernel(StepWork w) {
    __shared__ BandSmem sm;
    __shared__ SceneWork sw;
    __shared__ int s_begin[kMaxBatchScenes + 1];
    __shared__ int s_item;
    __shared__ unsigned s_drops, s_counted;
    const int t = threadIdx.x, lane = t & 31;
    launch_dependents();
    grid_dependency_wait();
    // Item prefix: one thread per scene, then a scan (n <= 64 <= blockDim.x).
    if (t < w.n_scenes)
        s_begin[t + 1] = (w.scenes[t].band_tiles + w.band_tiles_per_item - 1) / w.band_tiles_per_item;
    if (t == 0) {
        s_begin[0] = 0;
        s_drops = 0u;
        s_counted = 0u;
    }
    __syncthreads();
    if (t == 0)
        for (int k = 1; k <= w.n_scenes; ++k) s_begin[k] += s_begin[k - 1];
    __syncthreads();
    const int total = s_begin[w.n_scenes];
    int cur = -1;
    uint32_t drops = 0u, counted = 0u;
    for (;;) {
        if (t == 0) s_item = (int)atomicAdd(&w.queues[kQBand], 1u);
        __syncthreads();
        const int item = s_item;
        const bool done = item >= total;  // also on a CTA's first pull when items are few
        const int sc = done ? -1 : scene_of(s_begin, w.n_scenes, item);
        if (sc != cur || done) {
            // Flush the counters of the scene left behind, then load the next one.
            const unsigned wd = __reduce_add_sync(0xffffffffu, drops);
            const unsigned wc = __reduce_add_sync(0xffffffffu, counted);
            if (lane == 0 && wd) atomicAdd(&s_drops, wd);
            if (lane == 0 && wc) atomicAdd(&s_counted, wc);
            __syncthreads();
            if (t == 0 && cur >= 0) {
                if (s_drops) atomicAdd(sw.v.drop_count, (unsigned long long)s_drops);
                if (s_counted) atomicAdd(&sw.u.ctl->n_records, (int)s_counted);
            }
            __syncthreads();
            if (t == 0) {
                s_drops = 0u;
                s_counted = 0u;
            }
            drops = counted = 0u;
            if (done) break;
            cta_copy(&sw, &w.scenes[sc]);
            __syncthreads();
            cur = sc;
        }
        const int first = (item - s_begin[sc]) * w.band_tiles_per_item;
        const int last = min(first + w.band_tiles_per_item, sw.band_tiles);
        for (int tile = first; tile < last; ++tile) {
            const int i = tile * kBandThreads + t;
            float px = 0.0f, py = 0.0f, pz = 0.0f;
            const bool has = i < sw.a.n && load_point(sw.a, i, px, py, pz);
            band_point<kAllocInsert, true, S, PROBE>(sw.v, sw.a, sw.u, i, has, px, py, pz, sm, drops,
                                                    counted, nullptr, 0);
        }
        __syncthreads();  // s_item and the descriptor are rewritten next
    }
}

template <int MODE, bool RECORDS, int S = kStoreF32, bool DEPTH = false>
cudaError_t launch(const DevVolume& v, const BatchArgs& a, const UpdateScratch& u,
                   unsigned long long* hist, int n_bins, int sm_count, cudaStream_t s) {
    if (a.n <= 0) return cudaSuccess;
    // Persistent grid: as many CTAs as are resident at once (queried once
    // per instantiation), striding over the point tiles.
    static int per_sm = 0;
    static std::once_flag once;
    std::call_once(once, [] {
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, band_kernel<MODE, RECORDS, S, DEPTH>,
                                                          kBandThreads, 0) != cudaSuccess ||
            per_sm < 1)
            per_sm = 1;
    });
    const int tiles = (a.n + kBandThreads - 1) / kBandThreads;
    const int grid = std::min(tiles, per_sm * sm_count);
    band_kernel<MODE, RECORDS, S, DEPTH><<<grid, kBandThreads, 0, s>>>(v, a, u, hist, n_bins);
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
    if (a.depth.depth != nullptr) {  // integrate from a depth image (allocates)
        if (!insert) return cudaErrorInvalidValue;
        switch (v.storage) {
            case kStoreF16U16:
                return launch<kAllocInsert, true, kStoreF16U16, true>(v, a, u, nullptr, 0, sm_count, s);
            case kStoreF64:
                return launch<kAllocInsert, true, kStoreF64, true>(v, a, u, nullptr, 0, sm_count, s);
            default:
                return launch<kAllocInsert, true, kStoreF32, true>(v, a, u, nullptr, 0, sm_count, s);
        }
    }
    switch (v.storage) {
        case kStoreF16U16:
            return insert ? launch<kAllocInsert, true, kStoreF16U16>(v, a, u, nullptr, 0, sm_count, s)
                          : launch<kLookupOnly, true, kStoreF16U16>(v, a, u, nullptr, 0, sm_count, s);
        case kStoreF64:
            return insert ? launch<kAllocInsert, true, kStoreF64>(v, a, u, nullptr, 0, sm_count, s)
                          : launch<kLookupOnly, true, kStoreF64>(v, a, u, nullptr, 0, sm_count, s);
        default:
            return insert ? launch<kAllocInsert, true>(v, a, u, nullptr, 0, sm_count, s)
                          : launch<kLookupOnly, true>(v, a, u, nullptr, 0, sm_count, s);
    }
}

namespace {
template <int S>
cudaError_t launch_band_frames_t(const DevVolume& v, const BatchArgs& a, const UpdateScratch& u,
                                 const FrameCam* frames, int32_t n_frames, int sm_count, cudaStream_t s) {
    static int per_sm = 0;
    static std::once_flag once;
    std::call_once(once, [] {
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, band_frames_kernel<S>, kBandThreads, 0) !=
                cudaSuccess ||
            per_sm < 1)
            per_sm = 1;
    });
    const int tiles = (a.n + kBandThreads - 1) / kBandThreads;
    const int grid = std::min(tiles, per_sm * sm_count);
    if (OSN_BAND_PDL) return launch_after(band_frames_kernel<S>, grid, kBandThreads, s, v, a, u, frames, n_frames);
    band_frames_kernel<S><<<grid, kBandThreads, 0, s>>>(v, a, u, frames, n_frames);
    return cudaGetLastError();
}
template <int S>
cudaError_t launch_band_depth_frames_t(const DevVolume& v, const BatchArgs& a, const UpdateScratch& u,
                                       const FrameCam* frames, const FramePose* poses, int32_t n_frames,
                                       int sm_count, cudaStream_t s) {
    static int per_sm = 0;
    static std::once_flag once;
    std::call_once(once, [] {
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, band_depth_frames_kernel<S>, kBandThreads,
                                                          0) != cudaSuccess ||
            per_sm < 1)
            per_sm = 1;
    });
    const int tiles = (a.n + kBandThreads - 1) / kBandThreads;
    const int grid = std::min(tiles, per_sm * sm_count);
    if (OSN_BAND_PDL)
        return launch_after(band_depth_frames_kernel<S>, grid, kBandThreads, s, v, a, u, frames, poses, n_frames);
    band_depth_frames_kernel<S><<<grid, kBandThreads, 0, s>>>(v, a, u, frames, poses, n_frames);
    return cudaGetLastError();
}
}  // namespace

cudaError_t launch_frames_setup(UpdateControl* ctl, FrameCam* d_frames, const FrameTable& t, cudaStream_t s) {
    frames_setup_kernel<<<1, 64, 0, s>>>(ctl, d_frames, t);
    return cudaGetLastError();
}

cudaError_t launch_frames_setup_depth(UpdateControl* ctl, FrameCam* d_frames, const FrameTable& t,
                                      FramePose* d_poses, const PoseTable& p, cudaStream_t s) {
    frames_setup_depth_kernel<<<1, 64, 0, s>>>(ctl, d_frames, t, d_poses, p);
    return cudaGetLastError();
}

cudaError_t launch_band_depth_frames(const DevVolume& v, const BatchArgs& a, const UpdateScratch& u,
                                     const FrameCam* d_frames, const FramePose* d_poses, int32_t n_frames,
                                     int sm_count, cudaStream_t s) {
    if (a.n <= 0 || n_frames < 1 || n_frames > kMaxDepthFrames || a.n % n_frames != 0)
        return cudaErrorInvalidValue;
    switch (v.storage) {
        case kStoreF32: return launch_band_depth_frames_t<kStoreF32>(v, a, u, d_frames, d_poses, n_frames, sm_count, s);
        case kStoreF16U16:
            return launch_band_depth_frames_t<kStoreF16U16>(v, a, u, d_frames, d_poses, n_frames, sm_count, s);
        default: return cudaErrorInvalidValue;
    }
}

cudaError_t launch_band_frames(const DevVolume& v, const BatchArgs& a, const UpdateScratch& u,
                               const FrameCam* d_frames, int32_t n_frames, int sm_count, cudaStream_t s) {
    if (a.n <= 0) return cudaSuccess;
    switch (v.storage) {
        case kStoreF32: return launch_band_frames_t<kStoreF32>(v, a, u, d_frames, n_frames, sm_count, s);
        case kStoreF16U16: return launch_band_frames_t<kStoreF16U16>(v, a, u, d_frames, n_frames, sm_count, s);
        default: return cudaErrorInvalidValue;  // the FP64 oracle integrates one frame per batch
    }
}

namespace {
template <int S, int PROBE>
cudaError_t launch_band_multi_t(const StepWork& w, int sm_count, cudaStream_t s) {
    static int per_sm = 0;
    static std::once_flag once;
    std::call_once(once, [] {
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, band_multi_kernel<S, PROBE>,
                                                          kBandThreads, 0) != cudaSuccess ||
            per_sm < 1)
            per_sm = 1;
    });
    return launch_after(band_multi_kernel<S, PROBE>, per_sm * sm_count, kBandThreads, s, w);
}
}  // namespace

cudaError_t launch_band_multi(const StepWork& w, int storage, int probe, int sm_count, cudaStream_t s) {
    const bool lane = probe == kProbeLane;
    switch (storage) {
        case kStoreF16U16:
            return lane ? launch_band_multi_t<kStoreF16U16, kProbeLane>(w, sm_count, s)
                        : launch_band_multi_t<kStoreF16U16, kProbeWarp>(w, sm_count, s);
        case kStoreF64:
            return lane ? launch_band_multi_t<kStoreF64, kProbeLane>(w, sm_count, s)
                        : launch_band_multi_t<kStoreF64, kProbeWarp>(w, sm_count, s);
        default:
            return lane ? launch_band_multi_t<kStoreF32, kProbeLane>(w, sm_count, s)
                        : launch_band_multi_t<kStoreF32, kProbeWarp>(w, sm_count, s);
    }
}

}  // namespace osn_b200
