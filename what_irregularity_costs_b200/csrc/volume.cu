// Host side of one volume: device memory, the volume's stream, stage
// sequencing, counters and kernel timing.
//
// Reference: cpp/src/cuda_impl.cuh:44-112 (device allocation, table fill,
// scratch slots) and cpp/src/volume_cuda.cu:343-480 (stream-ordered stages,
// reset, counters).
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>

#include "volume.h"

namespace osn_b200 {

namespace {
uint32_t next_pow2(uint32_t v) {  // cpp/src/volume.cpp:14-19
    if (v < 2) return 2;
    --v;
    v |= v >> 1; v |= v >> 2; v |= v >> 4; v |= v >> 8; v |= v >> 16;
    return v + 1;
}

#define OSN_TRY(expr)                                                                       \
    do {                                                                                    \
        const cudaError_t err_ = (expr);                                                    \
        if (err_ != cudaSuccess) {                                                          \
            std::fprintf(stderr, "[osn_tsdf_b200] %s:%d: %s -> %s\n", __FILE__, __LINE__,   \
                         #expr, cudaGetErrorString(err_));                                  \
            return false;                                                                   \
        }                                                                                   \
    } while (0)
}  // namespace

Volume::Volume(float voxel, int32_t pool, float trunc_m, float weight_cap, uint32_t hash_slots,
               int storage, int layout) {
    if (!(voxel > 0.0f) || pool <= 0) return;
    if (storage != kStoreF32 && storage != kStoreF16U16 && storage != kStoreF64) return;
    if (layout != kLayoutPool && layout != kLayoutSlotIndex) return;
    if (hash_slots != 0 && (hash_slots < 2 || (hash_slots & (hash_slots - 1)) != 0)) return;
    if (layout == kLayoutSlotIndex) {
        // The pool is the table: one block of voxels per slot.
        const uint64_t size = hash_slots ? hash_slots : next_pow2((uint32_t)pool * 2u);
        if (size > (uint64_t)kMaxPoolBlocks) return;
        pool = (int32_t)size;
        hash_slots = (uint32_t)size;
        dv_.slot_index = 1;
    }
    if (pool > kMaxPoolBlocks) {
        std::fprintf(stderr, "[osn_tsdf_b200] pool of %d blocks exceeds the supported %d\n", pool,
                     kMaxPoolBlocks);
        return;
    }
    dv_.voxel_size = voxel;
    dv_.inv_voxel = 1.0f / voxel;
    dv_.trunc = trunc_m > 0.0f ? trunc_m : 4.0f * voxel;  // types.hpp:104-106
    dv_.inv_trunc = 1.0f / dv_.trunc;
    // uint16 weights saturate at 65535: that is the cap when none (or a larger
    // one) is given.
    dv_.storage = storage;
    dv_.weight_cap = storage == kStoreF16U16
                         ? (weight_cap > 0.0f ? std::min(weight_cap, kU16WeightMax) : kU16WeightMax)
                         : weight_cap;
    weight_cap_ = weight_cap;
    dv_.pool_capacity = pool;
    dv_.steps = std::max(1, (int32_t)std::ceil(dv_.trunc * dv_.inv_voxel));
    dv_.spin_limit = kSpinLimit;
    ok_ = alloc_device(hash_slots);
}

bool Volume::alloc_device(uint32_t hash_slots) {
    const uint32_t size = hash_slots ? hash_slots : next_pow2((uint32_t)dv_.pool_capacity * 2u);
    dv_.hash_mask = size - 1;
    const size_t n_vox = (size_t)dv_.pool_capacity * kBlockVoxels;
    int dev = 0;
    OSN_TRY(cudaGetDevice(&dev));
    device_ = dev;
    OSN_TRY(cudaDeviceGetAttribute(&sm_count_, cudaDevAttrMultiProcessorCount, dev));
    OSN_TRY(cudaStreamCreate(&stream_));
    OSN_TRY(cudaMalloc(&dv_.table, ((size_t)size + kScratchSlots) * sizeof(HashEntry)));
    OSN_TRY(cudaMalloc(&dv_.block_count, sizeof(int32_t)));
    OSN_TRY(cudaMalloc(&dv_.drop_count, sizeof(unsigned long long)));
    OSN_TRY(cudaMalloc(&dv_.status, sizeof(uint32_t)));
    OSN_TRY(cudaMalloc(&dv_.block_coord, (size_t)dv_.pool_capacity * sizeof(BlockCoord)));
    OSN_TRY(cudaMalloc(&dv_.block_chunk, (size_t)dv_.pool_capacity * sizeof(int32_t)));
    const size_t t_bytes = n_vox * (size_t)tsdf_bytes(dv_.storage);
    const size_t w_bytes = n_vox * (size_t)weight_bytes(dv_.storage);
    const bool rgb = dv_.storage == kStoreF32;
    OSN_TRY(cudaMalloc(&dv_.tsdf, t_bytes));
    OSN_TRY(cudaMalloc(&dv_.weight, w_bytes));
    if (rgb) {
        OSN_TRY(cudaMalloc(&dv_.r, n_vox * sizeof(float)));
        OSN_TRY(cudaMalloc(&dv_.g, n_vox * sizeof(float)));
        OSN_TRY(cudaMalloc(&dv_.b, n_vox * sizeof(float)));
    }
    OSN_TRY(cudaMalloc(&us_.vcnt, n_vox * sizeof(uint32_t)));
    OSN_TRY(cudaMalloc(&us_.vacc, n_vox * sizeof(unsigned long long)));
    OSN_TRY(cudaMalloc(&us_.blk_touch, (size_t)dv_.pool_capacity * sizeof(uint32_t)));
    OSN_TRY(cudaMalloc(&us_.xbits, (size_t)dv_.pool_capacity * kXWords * sizeof(uint32_t)));
    OSN_TRY(cudaMalloc(&us_.touched, (size_t)dv_.pool_capacity * sizeof(int32_t)));
    OSN_TRY(cudaMalloc(&us_.ctl, sizeof(UpdateControl)));
    us_.status = dv_.status;
    OSN_TRY(cudaMalloc(&mesh_ctl_, 2 * sizeof(int32_t)));
    if (dv_.slot_index) {
        OSN_TRY(cudaMalloc(&block_list_, (size_t)dv_.pool_capacity * sizeof(int32_t)));
        OSN_TRY(cudaMalloc(&list_count_, sizeof(int32_t)));
    }
    OSN_TRY(cudaMallocHost(&host_small_, 8 * sizeof(int64_t)));

    // The table must hold kEmptyKey, not zero: zero is a valid packed key.
    // The scratch slots past it hold kScratchKey and are never rewritten.
    OSN_TRY(launch_reset_table(dv_.table, size, kEmptyKey, stream_));
    OSN_TRY(launch_reset_table(dv_.table + size, kScratchSlots, kScratchKey, stream_));
    OSN_TRY(cudaMemsetAsync(dv_.block_count, 0, sizeof(int32_t), stream_));
    OSN_TRY(cudaMemsetAsync(dv_.drop_count, 0, sizeof(unsigned long long), stream_));
    OSN_TRY(cudaMemsetAsync(dv_.status, 0, sizeof(uint32_t), stream_));
    OSN_TRY(cudaMemsetAsync(dv_.block_chunk, 0, (size_t)dv_.pool_capacity * sizeof(int32_t), stream_));
    OSN_TRY(cudaMemsetAsync(dv_.tsdf, 0, t_bytes, stream_));
    OSN_TRY(cudaMemsetAsync(dv_.weight, 0, w_bytes, stream_));
    if (rgb) {
        OSN_TRY(cudaMemsetAsync(dv_.r, 0, n_vox * sizeof(float), stream_));
        OSN_TRY(cudaMemsetAsync(dv_.g, 0, n_vox * sizeof(float), stream_));
        OSN_TRY(cudaMemsetAsync(dv_.b, 0, n_vox * sizeof(float), stream_));
    }
    OSN_TRY(cudaMemsetAsync(us_.vcnt, 0, n_vox * sizeof(uint32_t), stream_));
    OSN_TRY(cudaMemsetAsync(us_.vacc, 0, n_vox * sizeof(unsigned long long), stream_));
    OSN_TRY(cudaMemsetAsync(us_.blk_touch, 0, (size_t)dv_.pool_capacity * sizeof(uint32_t), stream_));
    OSN_TRY(cudaMemsetAsync(us_.xbits, 0, (size_t)dv_.pool_capacity * kXWords * sizeof(uint32_t), stream_));
    OSN_TRY(cudaMemsetAsync(us_.ctl, 0, sizeof(UpdateControl), stream_));
    OSN_TRY(cudaStreamSynchronize(stream_));
    return true;
}

Volume::~Volume() {
    if (pipelined_) set_pipelined(false);
    if (stream_) cudaStreamSynchronize(stream_);
    cudaFree(dv_.table);
    cudaFree(dv_.block_count);
    cudaFree(dv_.drop_count);
    cudaFree(dv_.status);
    cudaFree(dv_.block_coord);
    cudaFree(dv_.block_chunk);
    cudaFree(dv_.tsdf);
    cudaFree(dv_.weight);
    cudaFree(dv_.r);
    cudaFree(dv_.g);
    cudaFree(dv_.b);
    cudaFree(us_.vcnt);
    cudaFree(us_.vacc);
    cudaFree(us_.blk_touch);
    cudaFree(us_.xbits);
    cudaFree(us_.touched);
    cudaFree(us_.ctl);
    cudaFree(us_.records);
    cudaFree(us_.slot_val);
    cudaFree(us_.grp);
    cudaFree(us_.xlist);
    cudaFree(mesh_posnor_);
    cudaFree(mesh_rgb_);
    cudaFree(mesh_ctl_);
    cudaFree(block_list_);
    cudaFree(list_count_);
    cudaFree(d_frames_);
    cudaFree(d_poses_);
    if (host_small_) cudaFreeHost(host_small_);
    for (auto& p : pending_) {
        cudaEventDestroy(p.start);
        cudaEventDestroy(p.end);
    }
    for (auto e : event_pool_) cudaEventDestroy(e);
    if (stream_) cudaStreamDestroy(stream_);
}

// ---- timing ------------------------------------------------------------

void Volume::mark_start(int, cudaStream_t s) {
    if (!timing_) return;
    cudaEvent_t e;
    if (!event_pool_.empty()) {
        e = event_pool_.back();
        event_pool_.pop_back();
    } else {
        cudaEventCreate(&e);
    }
    cudaEventRecord(e, s ? s : stream_);
    open_start_ = e;
}

void Volume::mark_end(int id, cudaStream_t s) {
    if (!timing_ || !open_start_) return;
    cudaEvent_t e;
    if (!event_pool_.empty()) {
        e = event_pool_.back();
        event_pool_.pop_back();
    } else {
        cudaEventCreate(&e);
    }
    cudaEventRecord(e, s ? s : stream_);
    pending_.push_back(Pending{id, open_start_, e});
    open_start_ = nullptr;
}

int Volume::kernel_times(double* ms, int64_t* launches, int n_ids) {
    synchronize();
    for (auto& p : pending_) {
        float t = 0.0f;
        if (cudaEventElapsedTime(&t, p.start, p.end) == cudaSuccess) {
            acc_ms_[p.id] += t;
            acc_launches_[p.id] += 1;
        }
        event_pool_.push_back(p.start);
        event_pool_.push_back(p.end);
    }
    pending_.clear();
    const int n = std::min(n_ids, (int)kNumKernelIds);
    for (int k = 0; k < n; ++k) {
        if (ms) ms[k] = acc_ms_[k];
        if (launches) launches[k] = acc_launches_[k];
    }
    return n;
}

// ---- stages ------------------------------------------------------------

cudaError_t Volume::allocate(const BatchArgs& a, int mode, unsigned long long* hist, int n_bins) {
    mark_start(kKAllocate);
    const cudaError_t e = launch_allocate(dv_, a, mode, hist, n_bins, sm_count_, stream_);
    mark_end(kKAllocate);
    return e;
}

bool Volume::ensure_records(int64_t n_records) {
    if (n_records <= us_.record_cap) return true;
    // Grows only; waits for in-flight work that may still read the old buffers.
    synchronize();
    cudaFree(us_.records);
    cudaFree(us_.slot_val);
    cudaFree(us_.grp);
    cudaFree(us_.xlist);
    us_.records = nullptr;
    us_.slot_val = nullptr;
    us_.grp = nullptr;
    us_.xlist = nullptr;
    us_.record_cap = 0;
    us_.xlist_cap = 0;
    if (cudaMalloc(&us_.records, (size_t)n_records * sizeof(uint32_t)) != cudaSuccess) return false;
    if (dv_.storage != kStoreF64 &&
        cudaMalloc(&us_.slot_val, (size_t)n_records * sizeof(float)) != cudaSuccess)
        return false;
    // Groups partition the records of crossing voxels: at most one place per record.
    if (cudaMalloc(&us_.grp, (size_t)n_records * sizeof(unsigned long long)) != cudaSuccess) return false;
    const int64_t n_cross = n_records / 2 + 1;  // a crossing voxel holds at least two records
    if (cudaMalloc(&us_.xlist, (size_t)n_cross * sizeof(uint32_t)) != cudaSuccess) return false;
    us_.record_cap = n_records;
    us_.xlist_cap = n_cross;
    if (pipelined_) {  // the second set's records and slot values grow with the first
        cudaFree(us2_.records);
        cudaFree(us2_.slot_val);
        us2_.records = nullptr;
        us2_.slot_val = nullptr;
        if (cudaMalloc(&us2_.records, (size_t)n_records * sizeof(uint32_t)) != cudaSuccess) return false;
        if (cudaMalloc(&us2_.slot_val, (size_t)n_records * sizeof(float)) != cudaSuccess) return false;
    }
    return true;
}

// ---- pipelining --------------------------------------------------------

bool Volume::alloc_second_set() {
    const size_t n_vox = (size_t)dv_.pool_capacity * kBlockVoxels;
    us2_ = UpdateScratch{};
    if (cudaMalloc(&us2_.ctl, sizeof(UpdateControl)) != cudaSuccess) return false;
    if (cudaMalloc(&us2_.vcnt, n_vox * sizeof(uint32_t)) != cudaSuccess) return false;
    if (cudaMalloc(&us2_.vacc, n_vox * sizeof(unsigned long long)) != cudaSuccess) return false;
    if (cudaMalloc(&us2_.touched, (size_t)dv_.pool_capacity * sizeof(int32_t)) != cudaSuccess) return false;
    if (us_.record_cap > 0) {
        if (cudaMalloc(&us2_.records, (size_t)us_.record_cap * sizeof(uint32_t)) != cudaSuccess) return false;
        if (cudaMalloc(&us2_.slot_val, (size_t)us_.record_cap * sizeof(float)) != cudaSuccess) return false;
    }
    if (cudaMemsetAsync(us2_.ctl, 0, sizeof(UpdateControl), stream_) != cudaSuccess) return false;
    if (cudaMemsetAsync(us2_.vcnt, 0, n_vox * sizeof(uint32_t), stream_) != cudaSuccess) return false;
    if (cudaMemsetAsync(us2_.vacc, 0, n_vox * sizeof(unsigned long long), stream_) != cudaSuccess)
        return false;
    return cudaStreamSynchronize(stream_) == cudaSuccess;
}

void Volume::free_second_set() {
    cudaFree(us2_.ctl);
    cudaFree(us2_.vcnt);
    cudaFree(us2_.vacc);
    cudaFree(us2_.touched);
    cudaFree(us2_.records);
    cudaFree(us2_.slot_val);
    us2_ = UpdateScratch{};
}

bool Volume::set_pipelined(bool on) {
    if (on == pipelined_) return true;
    synchronize();
    if (!on) {
        pipelined_ = false;
        free_second_set();
        for (int k = 0; k < 2; ++k) {
            if (band_done_[k]) cudaEventDestroy(band_done_[k]);
            if (tail_done_[k]) cudaEventDestroy(tail_done_[k]);
            band_done_[k] = tail_done_[k] = nullptr;
        }
        if (tail_) cudaStreamDestroy(tail_);
        tail_ = nullptr;
        if (last_ctl_ != us_.ctl && last_ctl_ != nullptr) last_ctl_ = nullptr;  // its set is gone
        return true;
    }
    if (dv_.storage == kStoreF64) return false;  // the oracle's tail reads the points
    if (cudaStreamCreate(&tail_) != cudaSuccess) return false;
    for (int k = 0; k < 2; ++k) {
        if (cudaEventCreateWithFlags(&band_done_[k], cudaEventDisableTiming) != cudaSuccess ||
            cudaEventCreateWithFlags(&tail_done_[k], cudaEventDisableTiming) != cudaSuccess ||
            cudaEventRecord(tail_done_[k], stream_) != cudaSuccess)
            return false;
    }
    if (!alloc_second_set()) {
        free_second_set();
        return false;
    }
    n_updates_ = 0;
    pipelined_ = true;
    return true;
}

void Volume::join() {
    if (pipelined_ && n_updates_ > 0) cudaStreamWaitEvent(stream_, tail_done_[(n_updates_ - 1) & 1], 0);
}

cudaError_t Volume::run_update(const BatchArgs& a, const UpdateScratch& scratch, bool insert,
                               const FrameTable* frames, const PoseTable* poses) {
    // Pipelined: this update's scratch set alternates; its walk waits only for
    // the tail two updates back (the last user of that set), its tail for its
    // walk. The walk's saturation filter may read weights the previous tail is
    // still writing: weights only grow, and finish decides acceptance from the
    // final weights, so a stale read only lets through a sample finish rejects.
    const bool pipe = pipelined_ && scratch.ctl == us_.ctl;  // not the fixed no-alloc scratch
    if (pipelined_ && !pipe) join();
    // Block tags are update numbers; at the (theoretical) wrap, clear them.
    if (++update_tag_ == 0u) {
        join();
        cudaMemsetAsync(us_.blk_touch, 0, (size_t)dv_.pool_capacity * sizeof(uint32_t), stream_);
        update_tag_ = 1u;
    }
    UpdateScratch u = scratch;
    const int p = (int)(n_updates_ & 1);
    if (pipe && p == 1) {
        u.ctl = us2_.ctl;
        u.records = us2_.records;
        u.slot_val = us2_.slot_val;
        u.vcnt = us2_.vcnt;
        u.vacc = us2_.vacc;
        u.touched = us2_.touched;
    }
    u.tag = update_tag_;
    cudaStream_t tail = pipe ? tail_ : stream_;
    cudaError_t e = cudaSuccess;
    if (pipe) e = cudaStreamWaitEvent(stream_, tail_done_[p], 0);
    if (e == cudaSuccess)
        e = poses    ? launch_frames_setup_depth(u.ctl, d_frames_, *frames, d_poses_, *poses, stream_)
            : frames ? launch_frames_setup(u.ctl, d_frames_, *frames, stream_)
                     : cudaMemsetAsync(u.ctl, 0, sizeof(UpdateControl), stream_);
    if (e != cudaSuccess) return e;
    mark_start(kKBand);
    e = poses    ? launch_band_depth_frames(dv_, a, u, d_frames_, d_poses_, frames->n, sm_count_, stream_)
        : frames ? launch_band_frames(dv_, a, u, d_frames_, frames->n, sm_count_, stream_)
                 : launch_band_records(dv_, a, u, insert, sm_count_, stream_);
    mark_end(kKBand);
    if (e != cudaSuccess) return e;
    if (pipe) {
        if ((e = cudaEventRecord(band_done_[p], stream_)) != cudaSuccess) return e;
        if ((e = cudaStreamWaitEvent(tail_, band_done_[p], 0)) != cudaSuccess) return e;
    }
    last_ctl_ = u.ctl;
    mark_start(kKFinish, tail);
    e = launch_finish(dv_, u, sm_count_, tail);
    mark_end(kKFinish, tail);
    if (e != cudaSuccess) return e;
    mark_start(kKGroup, tail);
    e = launch_group(dv_, a, u, sm_count_, tail);
    mark_end(kKGroup, tail);
    if (e != cudaSuccess) return e;
    mark_start(kKSelect, tail);
    e = launch_select(dv_, a, u, sm_count_, tail);
    mark_end(kKSelect, tail);
    if (e != cudaSuccess) return e;
    if (pipe) {
        if ((e = cudaEventRecord(tail_done_[p], tail_)) != cudaSuccess) return e;
        ++n_updates_;
    }
    return cudaSuccess;
}

// Records a batch of n points needs: one per band slot.
static int64_t batch_records(int32_t n, int32_t steps) { return (int64_t)n * (2 * steps + 1); }

cudaError_t Volume::update(const BatchArgs& a) {
    if (!ensure_records(batch_records(a.n, dv_.steps))) return cudaErrorMemoryAllocation;
    return run_update(a, us_, false);
}

cudaError_t Volume::integrate(const BatchArgs& a) {
    if (!ensure_records(batch_records(a.n, dv_.steps))) return cudaErrorMemoryAllocation;
    return run_update(a, us_, true);
}

cudaError_t Volume::integrate_frames(const BatchArgs& a, const FrameTable& t, const PoseTable* poses) {
    if (dv_.storage == kStoreF64) return cudaErrorInvalidValue;  // one frame per oracle batch
    if ((poses != nullptr) != (a.depth.depth != nullptr)) return cudaErrorInvalidValue;
    if (!d_frames_ && cudaMalloc(&d_frames_, sizeof(FrameCam) * (kMaxFrames + 1)) != cudaSuccess) {
        d_frames_ = nullptr;
        return cudaErrorMemoryAllocation;
    }
    if (poses && !d_poses_ && cudaMalloc(&d_poses_, sizeof(FramePose) * kMaxDepthFrames) != cudaSuccess) {
        d_poses_ = nullptr;
        return cudaErrorMemoryAllocation;
    }
    if (!ensure_records(batch_records(a.n, dv_.steps))) return cudaErrorMemoryAllocation;
    return run_update(a, us_, true, &t, poses);
}

bool Volume::ensure_mesh(int32_t cap, bool rgb) {
    if (cap > mesh_cap_ || (rgb && !mesh_rgb_)) {
        cudaStreamSynchronize(stream_);
        cudaFree(mesh_posnor_);
        cudaFree(mesh_rgb_);
        mesh_posnor_ = nullptr;
        mesh_rgb_ = nullptr;
        mesh_cap_ = 0;
        const int32_t c = std::max(cap, mesh_cap_);
        if (cudaMalloc(&mesh_posnor_, (size_t)c * 6 * sizeof(float)) != cudaSuccess) return false;
        if (rgb && cudaMalloc(&mesh_rgb_, (size_t)c * 3) != cudaSuccess) return false;
        mesh_cap_ = c;
    }
    return true;
}

int32_t Volume::extract(float* posnor, uint8_t* rgb, int32_t cap, float min_w, float iso,
                        bool host_out) {
    join();
    const int32_t n_blocks = block_count();  // waits for the stream
    if (n_blocks <= 0) return 0;
    float* d_pos = posnor;
    uint8_t* d_rgb = rgb;
    if (host_out) {
        if (!ensure_mesh(cap, rgb != nullptr)) return -1;
        d_pos = mesh_posnor_;
        d_rgb = rgb ? mesh_rgb_ : nullptr;
    }
    if (cudaMemsetAsync(mesh_ctl_, 0, 2 * sizeof(int32_t), stream_) != cudaSuccess) return -1;
    const int32_t nb = std::min(n_blocks, dv_.pool_capacity);
    const int32_t* list = block_list(nb);
    if (dv_.slot_index && !list) return -1;
    mark_start(kKExtract);
    const cudaError_t e = launch_extract(dv_, nb, list, min_w, iso, d_pos, d_rgb, cap, mesh_ctl_, stream_);
    mark_end(kKExtract);
    if (e != cudaSuccess) return -1;
    int32_t* hs = reinterpret_cast<int32_t*>(host_small_);
    if (cudaMemcpyAsync(hs, mesh_ctl_, 2 * sizeof(int32_t), cudaMemcpyDeviceToHost, stream_) !=
            cudaSuccess ||
        cudaStreamSynchronize(stream_) != cudaSuccess)
        return -1;
    const int32_t n = hs[0], ovf = hs[1];
    if (ovf) return -1;
    if (host_out && n > 0) {
        if (cudaMemcpyAsync(posnor, mesh_posnor_, (size_t)n * 6 * sizeof(float),
                            cudaMemcpyDeviceToHost, stream_) != cudaSuccess)
            return -1;
        if (rgb && cudaMemcpyAsync(rgb, mesh_rgb_, (size_t)n * 3, cudaMemcpyDeviceToHost,
                                   stream_) != cudaSuccess)
            return -1;
        if (cudaStreamSynchronize(stream_) != cudaSuccess) return -1;
    }
    return n;
}

const int32_t* Volume::block_list(int32_t n) {
    if (!dv_.slot_index || n <= 0) return nullptr;
    if (cudaMemsetAsync(list_count_, 0, sizeof(int32_t), stream_) != cudaSuccess ||
        launch_list_blocks(dv_, block_list_, list_count_, stream_) != cudaSuccess)
        return nullptr;
    return block_list_;
}

bool Volume::reserve_batch(int32_t max_points) {
    // A batch drives the volume's updates with its own scratch use: serial.
    if (pipelined_) set_pipelined(false);
    return max_points > 0 && ensure_records(batch_records(max_points, dv_.steps));
}

SceneWork Volume::batch_work(const BatchArgs& a, cudaStream_t s) {
    // Block tags are update numbers; at the (theoretical) wrap, clear them.
    if (++update_tag_ == 0u) {
        cudaMemsetAsync(us_.blk_touch, 0, (size_t)dv_.pool_capacity * sizeof(uint32_t), s);
        update_tag_ = 1u;
    }
    SceneWork w{};
    w.v = dv_;
    w.a = a;
    w.u = us_;
    w.u.tag = update_tag_;
    w.band_tiles = (a.n + kBatchTilePoints - 1) / kBatchTilePoints;
    w.n_slots = (int32_t)batch_records(a.n, dv_.steps);
    return w;
}

cudaError_t Volume::reset() {
    join();
    const int32_t n_blocks = std::min(block_count(), dv_.pool_capacity);
    const int32_t* list = block_list(n_blocks);  // before the table is cleared
    if (dv_.slot_index && n_blocks > 0 && !list) return cudaErrorUnknown;
    mark_start(kKReset);
    cudaError_t e = launch_reset_voxels(dv_, n_blocks, list, stream_);
    if (e == cudaSuccess) e = launch_reset_table(dv_.table, dv_.hash_mask + 1, kEmptyKey, stream_);
    mark_end(kKReset);
    if (e == cudaSuccess) e = cudaMemsetAsync(dv_.block_count, 0, sizeof(int32_t), stream_);
    if (e == cudaSuccess) e = cudaMemsetAsync(dv_.drop_count, 0, sizeof(unsigned long long), stream_);
    if (e == cudaSuccess) e = cudaMemsetAsync(dv_.status, 0, sizeof(uint32_t), stream_);
    // The per-voxel batch state is back to zero after every completed update;
    // an update that stopped on an error may have left some behind.
    const size_t n_vox = (size_t)dv_.pool_capacity * kBlockVoxels;
    if (e == cudaSuccess) e = cudaMemsetAsync(us_.vcnt, 0, n_vox * sizeof(uint32_t), stream_);
    if (e == cudaSuccess)
        e = cudaMemsetAsync(us_.vacc, 0, n_vox * sizeof(unsigned long long), stream_);
    if (pipelined_ && e == cudaSuccess) e = cudaMemsetAsync(us2_.vcnt, 0, n_vox * sizeof(uint32_t), stream_);
    if (pipelined_ && e == cudaSuccess)
        e = cudaMemsetAsync(us2_.vacc, 0, n_vox * sizeof(unsigned long long), stream_);
    if (e == cudaSuccess) e = cudaStreamSynchronize(stream_);
    return e;
}

int32_t Volume::block_count() {
    join();
    int32_t* hs = reinterpret_cast<int32_t*>(host_small_);
    cudaMemcpyAsync(hs, dv_.block_count, sizeof(int32_t), cudaMemcpyDeviceToHost, stream_);
    cudaStreamSynchronize(stream_);
    return hs[0];
}

uint64_t Volume::drop_count() {
    join();
    uint64_t* hs = reinterpret_cast<uint64_t*>(host_small_);
    cudaMemcpyAsync(hs, dv_.drop_count, sizeof(uint64_t), cudaMemcpyDeviceToHost, stream_);
    cudaStreamSynchronize(stream_);
    return hs[0];
}

uint32_t Volume::status() {
    join();
    uint32_t* hs = reinterpret_cast<uint32_t*>(host_small_);
    cudaMemcpyAsync(hs, dv_.status, sizeof(uint32_t), cudaMemcpyDeviceToHost, stream_);
    cudaStreamSynchronize(stream_);
    return hs[0];
}

bool Volume::last_update_stats(int64_t out[4]) {
    join();
    UpdateControl c{};
    if (cudaMemcpyAsync(host_small_, last_ctl_ ? last_ctl_ : us_.ctl, sizeof(UpdateControl),
                        cudaMemcpyDeviceToHost,
                        stream_) != cudaSuccess ||
        cudaStreamSynchronize(stream_) != cudaSuccess)
        return false;
    std::memcpy(&c, host_small_, sizeof(UpdateControl));
    out[0] = c.n_updated;
    out[1] = c.n_records;
    out[2] = c.n_touched;
    out[3] = (int64_t)c.n_crossing;
    return true;
}

}  // namespace osn_b200
