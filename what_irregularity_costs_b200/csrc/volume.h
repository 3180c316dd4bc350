// Host-side state of one volume, shared by the kernel translation units.
#pragma once

#include <cstdint>
#include <utility>
#include <vector>

#include <cuda_runtime.h>

#include "tsdf_device.cuh"

namespace osn_b200 {

struct SceneWork;  // one volume's part of a batched step (below)

// Kernel ids for the timing table (documented in include/osn_tsdf_b200.h).
enum KernelId : int {
    kKAllocate = 0,      // allocate-only band walk
    kKBand = 1,          // count-and-sum band walk (fused with allocation in integrate)
    kKFinish = 2,        // per touched block: finish every voxel that accepts all its records
    kKGroup = 3,         // records of voxels that cross the cap: grouped per voxel, ordered
                         // cap selection, voxel finished
    kKSelect = 4,        // ordered cap selection of the crossing voxels (its own pass)
    kKExtract = 5,
    kKReset = 6,
    kKUnused7 = 7,       // no longer launched
    kNumKernelIds = 8,
};

// Counters an update pass keeps on the device (one small struct, cleared by
// one memset at the start of every update).
struct UpdateControl {
    int32_t n_records;   // band records counted (contributions that can be accepted)
    int32_t n_touched;   // blocks that received a band sample
    int32_t n_updated;   // voxels whose sums were rewritten
    int32_t pad0;
    uint32_t x_used;     // group places reserved by voxels that cross the cap
    int32_t pad1;
    unsigned long long n_crossing;  // voxels that cross the cap inside the batch
    int32_t pad[8];
};
static_assert(sizeof(UpdateControl) == 64, "control block is read back as 64 bytes");

// One band slot (point i, step s) at records[s * n + i]: the voxel's global
// index (block index * 512 + (lz*8+ly)*8+lx), or kNoVoxel for a culled,
// dropped or saturated sample.
constexpr uint32_t kNoVoxel = 0xFFFFFFFFu;

// Words of a block's crossing bitmap (one bit per voxel).
constexpr int kXWords = kBlockVoxels / 32;

// Global voxel indices are 32-bit with one value reserved, which bounds the
// pool at 2^23 - 1 blocks (4 G voxels).
constexpr int32_t kMaxPoolBlocks = (1 << 23) - 1;

// Several consecutive frames integrated as one batch: frame k's points are
// [f[k].begin, f[k + 1].begin) of the batch, seen from the camera at
// (f[k].x, f[k].y, f[k].z); f[n].begin is the batch's point count.
constexpr int kMaxFrames = 32;
struct FrameCam {
    int32_t begin;
    float x, y, z;
};
struct FrameTable {
    int32_t n;
    FrameCam f[kMaxFrames + 1];
};
// Several depth images as one batch: image k's camera-to-world pose (the
// unprojection of its pixels; the walk's camera is (float)t).
constexpr int kMaxDepthFrames = 16;
struct FramePose {
    double R[9];  // row-major
    double t[3];
};
struct PoseTable {
    int32_t n;
    FramePose p[kMaxDepthFrames];
};

struct UpdateScratch {
    UpdateControl* ctl = nullptr;
    uint32_t* records = nullptr;  // [record_cap] one per band slot
    float* slot_val = nullptr;    // [record_cap] normalised SDF of each counted slot (FP32 / FP16
                                  // storage; null for the FP64 oracle, which recomputes it)
    // [record_cap] records of the voxels that cross the cap, grouped per
    // voxel: canonical id | normalised SDF bits << 32 (the band slot for the
    // FP64 oracle, which recomputes both).
    unsigned long long* grp = nullptr;
    int64_t record_cap = 0;
    // [xlist_cap] the voxels that cross the cap in this update (written by
    // finish for the select pass); a crossing voxel has at least two records.
    uint32_t* xlist = nullptr;
    int64_t xlist_cap = 0;
    // Owned by the volume. Per voxel: zero between updates.
    uint32_t* vcnt = nullptr;            // records of the voxel in this batch (of a crossing voxel:
                                         // records still to be placed in its group)
    unsigned long long* vacc = nullptr;  // fixed-point sum of their sdf_n (of a crossing voxel: group
                                         // base + 1 << 32 | next place)
    // Per block, tagged with the update number instead of being cleared.
    uint32_t* blk_touch = nullptr;  // update that last touched the block
    // [pool * kXWords] per block: bit lv set when voxel lv crosses the cap in
    // this update; rewritten by finish for every block whose voxels it reads.
    uint32_t* xbits = nullptr;
    int32_t* touched = nullptr;     // [pool] blocks touched by this update
    uint32_t* status = nullptr;     // the volume's status word
    uint32_t tag = 0;               // this update's number (never 0)
};

class Volume {
public:
    // layout: kLayoutPool (the reference's: pool indices from a counter) or
    // kLayoutSlotIndex (the pool is the table; a block's index is its slot).
    Volume(float voxel, int32_t pool, float trunc_m, float weight_cap, uint32_t hash_slots,
           int storage = kStoreF32, int layout = kLayoutPool);
    ~Volume();
    Volume(const Volume&) = delete;
    Volume& operator=(const Volume&) = delete;

    bool ok() const { return ok_; }
    const DevVolume& dev() const { return dv_; }
    int device() const { return device_; }  // the CUDA device the volume was created on
    cudaStream_t stream() const { return stream_; }
    float voxel_size() const { return dv_.voxel_size; }
    float trunc() const { return dv_.trunc; }
    float weight_cap() const { return weight_cap_; }  // as given at creation
    int storage() const { return dv_.storage; }
    int layout() const { return dv_.slot_index ? kLayoutSlotIndex : kLayoutPool; }
    int32_t pool() const { return dv_.pool_capacity; }
    uint32_t hash_mask() const { return dv_.hash_mask; }

    // Stages (all asynchronous on stream()). Return a cudaError_t of the launch.
    cudaError_t allocate(const BatchArgs& a, int mode, unsigned long long* hist, int n_bins);
    cudaError_t update(const BatchArgs& a);
    // allocate + update in one pass over the points (same results).
    cudaError_t integrate(const BatchArgs& a);
    // integrate() of several consecutive frames as one batch (a.n = all
    // their points; t gives each frame's first point and camera). FP32 and
    // FP16 storage.
    cudaError_t integrate_frames(const BatchArgs& a, const FrameTable& t, const PoseTable* poses = nullptr);
    // update() with its control counters and records in caller-provided
    // device memory instead of the volume's own (grown) buffer; the counters
    // are copied to the volume's own control block afterwards.
    cudaError_t update_static_scratch(const BatchArgs& a, void* scratch);
    int32_t extract(float* posnor, uint8_t* rgb, int32_t cap, float min_w, float iso, bool host_out);
    cudaError_t reset();

    int32_t block_count();
    uint64_t drop_count();
    uint32_t status();
    void synchronize() {
        join();
        cudaStreamSynchronize(stream_);
    }
    bool last_update_stats(int64_t out[4]);

    // Pipelined updates. When on, an update's band walk runs on stream() and
    // its tail (finish, group) on an internal stream, so the
    // next update's walk overlaps this one's tail; the per-update scratch
    // alternates between two sets. Every reader of results joins first.
    // Not available for the FP64 oracle storage (its tail reads the points).
    bool set_pipelined(bool on);
    // Chunk id that later calls give the blocks they allocate or update
    // (streaming: evict_chunks moves a range of chunks to host memory).
    void set_chunk(int32_t chunk) { dv_.chunk = chunk; }
    int32_t chunk() const { return dv_.chunk; }
    // Blocks whose chunk id lies in [lo, hi]: bytes of their pack, and the
    // eviction itself (pack written to host, blocks removed, the others
    // compacted to the front of the pool, table rebuilt); stream_in puts a
    // pack's blocks back (blocks already present are left and counted in
    // *skipped). chunks.cu.
    int64_t evict_bytes(int32_t lo, int32_t hi);
    int64_t evict_chunks(int32_t lo, int32_t hi, void* host, int64_t cap);
    int32_t stream_in(const void* host, int64_t size, int32_t* skipped);
    // Bound of every publication wait of this volume's later calls, in
    // iterations of ~100 ns (1 .. kSpinLimit).
    bool set_spin_limit(int32_t iterations) {
        if (iterations < 1 || iterations > kSpinLimit) return false;
        dv_.spin_limit = iterations;
        return true;
    }
    bool pipelined() const { return pipelined_; }
    // Make stream() wait for every queued update tail.
    void join();

    // Snapshot of the allocated blocks through host memory (snapshot.cu):
    // bytes needed, write (returns bytes or -1), restore into this volume
    // (same voxel size, truncation, cap and storage; 0 ok, 1 bad snapshot,
    // 3 CUDA error). All wait for the stream.
    int64_t snapshot_bytes();
    int64_t snapshot(void* host, int64_t cap);
    int32_t restore(const void* host, int64_t size);

    // Batched steps: make room for batches of up to max_points points (call
    // before any stream capture), then describe one batch for a batched
    // step on stream s (takes the next update number).
    bool reserve_batch(int32_t max_points);
    SceneWork batch_work(const BatchArgs& a, cudaStream_t s);

    // Timing.
    void set_timing(bool on) { timing_ = on; }
    int kernel_times(double* ms, int64_t* launches, int n_ids);
    void mark_start(int id, cudaStream_t s = nullptr);
    void mark_end(int id, cudaStream_t s = nullptr);

private:
    bool alloc_device(uint32_t hash_slots);
    cudaError_t run_update(const BatchArgs& a, const UpdateScratch& u, bool insert,
                           const FrameTable* frames = nullptr, const PoseTable* poses = nullptr);
    bool ensure_records(int64_t n_records);
    // The allocated blocks' pool indices: 0..n-1 in the pool layout (returns
    // nullptr), the occupied slots listed on the device in the slot-index
    // layout (returns the list; n = block count).
    const int32_t* block_list(int32_t n);
    int32_t* block_list_ = nullptr;  // slot-index layout: [pool] occupied slots
    int32_t* list_count_ = nullptr;
    bool ensure_mesh(int32_t cap, bool rgb);

    bool ok_ = false;
    int device_ = -1;
    DevVolume dv_{};
    float weight_cap_ = 0.0f;
    cudaStream_t stream_ = nullptr;
    UpdateScratch us_{};
    uint32_t update_tag_ = 0;  // number of the last update (block tags)

    // Pipelining: the second scratch set (its ctl, records, slot_val, vcnt,
    // vacc and touched), the tail stream and the hand-over events.
    bool pipelined_ = false;
    cudaStream_t tail_ = nullptr;
    UpdateScratch us2_{};
    cudaEvent_t band_done_[2] = {nullptr, nullptr};
    cudaEvent_t tail_done_[2] = {nullptr, nullptr};
    uint64_t n_updates_ = 0;
    UpdateControl* last_ctl_ = nullptr;  // counters of the last update
    bool alloc_second_set();
    void free_second_set();
    int sm_count_ = 148;

    // Extraction scratch (device output for the host-copy path, counters).
    float* mesh_posnor_ = nullptr;
    uint8_t* mesh_rgb_ = nullptr;
    int32_t mesh_cap_ = 0;
    int32_t* mesh_ctl_ = nullptr;  // [0] vertex count, [1] overflow flag
    FrameCam* d_frames_ = nullptr;  // frame table of the last several-frame integrate
    FramePose* d_poses_ = nullptr;  // poses of the last several-image depth integrate

    // Pinned host staging for small reads.
    int64_t* host_small_ = nullptr;

    // Timing.
    struct Pending {
        int id;
        cudaEvent_t start, end;
    };
    bool timing_ = false;
    std::vector<Pending> pending_;
    std::vector<cudaEvent_t> event_pool_;
    cudaEvent_t open_start_ = nullptr;
    double acc_ms_[kNumKernelIds] = {};
    int64_t acc_launches_[kNumKernelIds] = {};
};

// Launch `kernel` with programmatic stream serialisation: it may begin while
// the previous kernel on the stream is still running, and waits for it in
// grid_dependency_wait().
template <typename... KArgs, typename... Args>
cudaError_t launch_after(void (*kernel)(KArgs...), dim3 grid, dim3 block, cudaStream_t s,
                         Args&&... args) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = 0;
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, kernel, std::forward<Args>(args)...);
}

// Launchers (one per translation unit).
cudaError_t launch_allocate(const DevVolume& v, const BatchArgs& a, int mode,
                            unsigned long long* hist, int n_bins, int sm_count, cudaStream_t s);
cudaError_t launch_reset_table(HashEntry* first, uint32_t count, long long key, cudaStream_t s);
// Re-insert the keys of pool blocks 0..n-1 (coordinates from block_coord)
// into an empty table, block i at pool index i (snapshot.cu).
cudaError_t launch_rebuild_table(const DevVolume& v, int32_t n_blocks, cudaStream_t s);
// The voxel arrays of a storage mode (tsdf, weight[, r, g, b]) and their
// bytes per voxel; returns how many (snapshot.cu).
size_t voxel_arrays(int storage, const DevVolume& d, void* out[5], size_t bytes[5]);
// Zero the voxels of n blocks: pool indices 0..n-1, or those of a list.
cudaError_t launch_reset_voxels(const DevVolume& v, int32_t n_blocks, const int32_t* list, cudaStream_t s);
// List the occupied slots of the table (slot-index layout) into out.
cudaError_t launch_list_blocks(const DevVolume& v, int32_t* out, int32_t* count, cudaStream_t s);
// Extraction over n blocks: pool indices 0..n-1, or those of a list.
cudaError_t launch_extract(const DevVolume& v, int32_t n_blocks, const int32_t* list, float min_w, float iso,
                           float* posnor, uint8_t* rgb, int32_t cap, int32_t* ctl, cudaStream_t s);

// The update pipeline: band walk (counts, sums, records) -> finish -> group
// (grouping, ordered selection and finishing of the voxels that cross the cap).
cudaError_t launch_band_records(const DevVolume& v, const BatchArgs& a, const UpdateScratch& u,
                                bool insert, int sm_count, cudaStream_t s);
// Several-frame integrate: the set-up kernel (control block zeroed, frame
// table stored) and the band walk with per-frame cameras (FP32 / FP16 storage).
cudaError_t launch_frames_setup(UpdateControl* ctl, FrameCam* d_frames, const FrameTable& t, cudaStream_t s);
cudaError_t launch_band_frames(const DevVolume& v, const BatchArgs& a, const UpdateScratch& u,
                               const FrameCam* d_frames, int32_t n_frames, int sm_count, cudaStream_t s);
// The same for depth images (a.depth set): poses stored by the set-up, the
// walk unprojecting image i / (width * height) with its pose.
cudaError_t launch_frames_setup_depth(UpdateControl* ctl, FrameCam* d_frames, const FrameTable& t,
                                      FramePose* d_poses, const PoseTable& p, cudaStream_t s);
cudaError_t launch_band_depth_frames(const DevVolume& v, const BatchArgs& a, const UpdateScratch& u,
                                     const FrameCam* d_frames, const FramePose* d_poses, int32_t n_frames,
                                     int sm_count, cudaStream_t s);
cudaError_t launch_finish(const DevVolume& v, const UpdateScratch& u, int sm_count, cudaStream_t s);
cudaError_t launch_group(const DevVolume& v, const BatchArgs& a, const UpdateScratch& u, int sm_count,
                         cudaStream_t s);
cudaError_t launch_select(const DevVolume& v, const BatchArgs& a, const UpdateScratch& u, int sm_count,
                          cudaStream_t s);

}  // namespace osn_b200

// The Volume behind a C-ABI handle, or nullptr when the handle is NULL or invalid.
struct OsnTsdfCudaVolume;
osn_b200::Volume* osn_tsdf_b200_volume_of(OsnTsdfCudaVolume* v);

namespace osn_b200 {

// ---- batched steps: many volumes integrate one frame each per step -------

constexpr int kMaxBatchScenes = 64;
constexpr int kBatchTilePoints = 128;  // points per band tile (the band CTA size)
constexpr int kBandTilesPerItemMax = 8;

// One scene of a batched step (device memory, rewritten every step).
struct SceneWork {
    DevVolume v;
    BatchArgs a;
    UpdateScratch u;
    int32_t band_tiles;  // ceil(a.n / kBandThreads); 0 when the scene is idle this step
    int32_t n_slots;     // band slots a.n * (2 * steps + 1)
};

// Work queues of one step, one counter per pass (zeroed by the prepare pass).
enum BatchQueue : int { kQBand = 0, kQFinish, kQGroup, kQSelect, kNumBatchQueues };

// Tunable shape of a batched step (chosen by the batch autotuner).
struct BatchShape {
    int band_tiles_per_item = 4;  // band work item: this many 128-point tiles of one scene
    int probe = 0;                // 0: warp-deduplicated block resolution, 1: per-lane
    int finish_pair = 1;          // finish work item: 1 = two touched blocks, 0 = one
};

// Everything a batched pass reads: the scene table and the queues.
struct StepWork {
    SceneWork* scenes;     // [n_scenes]
    int32_t n_scenes;
    int32_t band_tiles_per_item;
    uint32_t* queues;      // [kNumBatchQueues]
    uint32_t* status;      // batch status word (bounded waits, overflows)
};

cudaError_t launch_batch_prepare(const StepWork& w, cudaStream_t s);
cudaError_t launch_band_multi(const StepWork& w, int storage, int probe, int sm_count, cudaStream_t s);
cudaError_t launch_finish_multi(const StepWork& w, int storage, int pair, int sm_count, cudaStream_t s);
cudaError_t launch_group_multi(const StepWork& w, int storage, int sm_count, cudaStream_t s);
cudaError_t launch_select_multi(const StepWork& w, int storage, int sm_count, cudaStream_t s);

}  // namespace osn_b200
