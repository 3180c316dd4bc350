// Host-side state of one volume, shared by the kernel translation units.
#pragma once

#include <cstdint>
#include <vector>

#include <cuda_runtime.h>

#include "tsdf_device.cuh"

namespace osn_b200 {

// Kernel ids for the timing table (documented in include/osn_tsdf_b200.h).
enum KernelId : int {
    kKAllocate = 0,        // allocate-only walk
    kKUpdateStage = 1,     // count-and-stage walk (fused with allocation in integrate)
    kKUpdateApplyBig = 2,  // tile read-modify-write of blocks above 2048 records
    kKUpdateBin = 3,       // copy staged segments into contiguous per-block bins
    kKUpdateApply = 4,     // tile read-modify-write (blocks up to 2048 records)
    kKExtract = 5,
    kKReset = 6,
    kNumKernelIds = 7,
};

// Counters an update pass keeps on the device (one small struct, cleared by
// one memset at the start of every update).
struct UpdateControl {
    int32_t n_touched;   // blocks that received at least one record
    int32_t n_records;   // records staged
    int32_t work;        // apply-kernel work cursor
    int32_t n_accepted;  // blocks that accepted at least one contribution
    int32_t n_crossing;  // blocks that needed ordered cap selection
    int32_t cta_done;    // stage-kernel CTAs finished (the last one scans)
    int32_t n_segs;      // segment descriptors published
    int32_t n_big;       // blocks handed to the big-block apply
    int32_t work_big;    // big-block apply work cursor
    int32_t pad[7];
};

// One binned contribution: 16 bytes, written and read as one vector.
struct __align__(16) Record {
    uint32_t id;   // point * (2*steps+1) + (s + steps): the canonical order
    uint32_t lv;   // voxel within the block, (lz*8+ly)*8+lx
    float sdf_n;   // clamp(sdf / trunc, -1, 1)
    float w_in;    // contribution weight (1 through the reference ABI)
};
static_assert(sizeof(Record) == 16, "record must stay one 128-bit vector");

struct UpdateScratch {
    int32_t* blk_cnt = nullptr;     // [pool] records per block; back to 0 after every update
    int32_t* blk_cur = nullptr;     // [pool] bin filling cursor; back to 0 after every update
    int4* blk_info = nullptr;       // [pool] (bin offset, records, -, -)
    int32_t* touched = nullptr;     // [pool] touched block indices
    int32_t* big_list = nullptr;    // [pool] blocks with more records than a small CTA takes
    UpdateControl* ctl = nullptr;
    Record* records = nullptr;      // staged records, grouped per (walk CTA, block)
    Record* bins = nullptr;         // the same records, contiguous per block
    int64_t record_cap = 0;
    int4* segs = nullptr;           // segment descriptors (block, staging offset, length, -)
    int64_t seg_cap = 0;
};

class Volume {
public:
    Volume(float voxel, int32_t pool, float trunc_m, float weight_cap, uint32_t hash_slots);
    ~Volume();
    Volume(const Volume&) = delete;
    Volume& operator=(const Volume&) = delete;

    bool ok() const { return ok_; }
    const DevVolume& dev() const { return dv_; }
    cudaStream_t stream() const { return stream_; }
    float voxel_size() const { return dv_.voxel_size; }
    float trunc() const { return dv_.trunc; }
    float weight_cap() const { return dv_.weight_cap; }
    int32_t pool() const { return dv_.pool_capacity; }
    uint32_t hash_mask() const { return dv_.hash_mask; }

    // Stages (all asynchronous on stream()). Return a cudaError_t of the launch.
    cudaError_t allocate(const BatchArgs& a, int mode, unsigned long long* hist, int n_bins);
    cudaError_t update(const BatchArgs& a);
    // allocate + update in one pass over the points (same results).
    cudaError_t integrate(const BatchArgs& a);
    // update() with its control counters and records in caller-provided
    // device memory instead of the volume's own (grown) buffer.
    cudaError_t update_static_scratch(const BatchArgs& a, void* scratch);
    int32_t extract(float* posnor, uint8_t* rgb, int32_t cap, float min_w, float iso, bool host_out);
    cudaError_t reset();

    int32_t block_count();
    uint64_t drop_count();
    uint32_t status();
    void synchronize() { cudaStreamSynchronize(stream_); }
    bool last_update_stats(int64_t out[4]);

    // Timing.
    void set_timing(bool on) { timing_ = on; }
    int kernel_times(double* ms, int64_t* launches, int n_ids);
    void mark_start(int id);
    void mark_end(int id);

private:
    bool alloc_device(uint32_t hash_slots);
    cudaError_t run_update(const BatchArgs& a, const UpdateScratch& u, bool insert);
    bool ensure_records(int64_t n_records, int64_t n_segs);
    bool ensure_mesh(int32_t cap, bool rgb);

    bool ok_ = false;
    DevVolume dv_{};
    cudaStream_t stream_ = nullptr;
    UpdateScratch us_{};
    int sm_count_ = 148;
    int apply_ctas_per_sm_ = 2;

    // Extraction scratch (device output for the host-copy path, counters).
    float* mesh_posnor_ = nullptr;
    uint8_t* mesh_rgb_ = nullptr;
    int32_t mesh_cap_ = 0;
    int32_t* mesh_ctl_ = nullptr;  // [0] vertex count, [1] overflow flag

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

// Launchers (one per translation unit).
cudaError_t launch_allocate(const DevVolume& v, const BatchArgs& a, int mode,
                            unsigned long long* hist, int n_bins, cudaStream_t s);
cudaError_t launch_reset_table(HashEntry* first, uint32_t count, long long key, cudaStream_t s);
cudaError_t launch_reset_voxels(const DevVolume& v, int32_t n_blocks, cudaStream_t s);
cudaError_t launch_extract(const DevVolume& v, int32_t n_blocks, float min_w, float iso,
                           float* posnor, uint8_t* rgb, int32_t cap, int32_t* ctl, cudaStream_t s);

// The update pipeline: stage (+ per-block bins) -> bin -> apply -> big-block apply.
cudaError_t launch_update_stage(const DevVolume& v, const BatchArgs& a, const UpdateScratch& u,
                                bool insert, cudaStream_t s);
cudaError_t launch_update_bin(const UpdateScratch& u, int n_ctas, cudaStream_t s);
cudaError_t launch_update_apply(const DevVolume& v, const UpdateScratch& u, int n_ctas,
                                cudaStream_t s);
cudaError_t launch_update_apply_big(const DevVolume& v, const UpdateScratch& u, int n_ctas,
                                    cudaStream_t s);
// One-time kernel attributes (dynamic shared memory of apply and crossing).
cudaError_t prepare_update_kernels();
size_t apply_smem_bytes();

}  // namespace osn_b200

// The Volume behind a C-ABI handle, or nullptr when the handle is NULL or invalid.
struct OsnTsdfCudaVolume;
osn_b200::Volume* osn_tsdf_b200_volume_of(OsnTsdfCudaVolume* v);
