// Batched integrate: many independent volumes (scenes) integrate one frame
// each per step, in one chain of work-queued passes.
//
// No counterpart in the reference, whose arms integrate one volume per call
// (cpp/src/volume_cuda.cu:384-455). Each step runs, on the batch's stream:
//
//   table upload  one SceneWork per scene (volume, batch, scratch, update
//                 number), from a pinned double buffer;
//   prepare       zero the active scenes' update counters and the queues;
//   band_multi    allocate + count-and-sum walk of every scene: work items
//                 of a few 128-point tiles of one scene from an atomic queue;
//   finish_multi, group_multi, select_multi
//                 the single-volume passes over every scene's touched
//                 blocks, band records and cap-crossing voxels, work-queued
//                 the same way (per-scene item counts prefix-summed on device).
//
// The passes after the upload are launched with programmatic stream
// serialisation and can be captured once into a CUDA graph and replayed
// every step (their arguments only point at the table). An autotuner runs
// the next steps with each candidate shape (tiles per band item, block
// resolution scheme, blocks per finish item) and keeps the fastest; every
// shape computes bit-identical results, so tuning uses live steps.
#include <algorithm>
#include <cstdio>
#include <cstring>
#include <vector>

#include "../../include/osn_tsdf_b200.h"
#include "volume.h"

namespace osn_b200 {

class Batch {
public:
    explicit Batch(int max_scenes) : max_scenes_(max_scenes) {
        if (max_scenes <= 0 || max_scenes > kMaxBatchScenes) return;
        int dev = 0;
        if (cudaGetDevice(&dev) != cudaSuccess) return;
        if (cudaDeviceGetAttribute(&sm_count_, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) return;
        if (cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking) != cudaSuccess) return;
        if (cudaMalloc(&d_scenes_, (size_t)max_scenes * sizeof(SceneWork)) != cudaSuccess) return;
        if (cudaMalloc(&d_queues_, kNumBatchQueues * sizeof(uint32_t)) != cudaSuccess) return;
        if (cudaMalloc(&d_status_, sizeof(uint32_t)) != cudaSuccess) return;
        if (cudaMemset(d_status_, 0, sizeof(uint32_t)) != cudaSuccess) return;
        for (int k = 0; k < 2; ++k) {
            if (cudaMallocHost(&h_table_[k], (size_t)max_scenes * sizeof(SceneWork)) != cudaSuccess) return;
            if (cudaEventCreateWithFlags(&table_free_[k], cudaEventDisableTiming) != cudaSuccess) return;
            if (cudaEventRecord(table_free_[k], stream_) != cudaSuccess) return;
        }
        if (cudaMallocHost(&h_status_, sizeof(uint32_t)) != cudaSuccess) return;
        ok_ = true;
    }

    ~Batch() {
        if (stream_) cudaStreamSynchronize(stream_);
        drop_graph();
        for (auto& t : tune_log_) {
            cudaEventDestroy(t.start);
            cudaEventDestroy(t.end);
        }
        for (int k = 0; k < 2; ++k) {
            if (h_table_[k]) cudaFreeHost(h_table_[k]);
            if (table_free_[k]) cudaEventDestroy(table_free_[k]);
        }
        if (h_status_) cudaFreeHost(h_status_);
        cudaFree(d_scenes_);
        cudaFree(d_queues_);
        cudaFree(d_status_);
        if (stream_) cudaStreamDestroy(stream_);
    }

    bool ok() const { return ok_; }
    cudaStream_t stream() const { return stream_; }
    int size() const { return live_; }

    // Attach a volume (into the first free scene slot); every scene of a
    // batch shares one storage mode.
    int add(Volume* v, int32_t max_points) {
        if (!v || max_points <= 0) return -1;
        if (storage_ >= 0 && live_ > 0 && v->storage() != storage_) return -1;
        if ((int64_t)max_points * (2 * (int64_t)v->dev().steps + 1) >= (int64_t(1) << 32)) return -1;
        for (Volume* o : vols_)
            if (o == v) return -1;
        int slot = -1;
        for (int k = 0; k < (int)vols_.size(); ++k)
            if (!vols_[k]) {
                slot = k;
                break;
            }
        if (slot < 0 && (int)vols_.size() >= max_scenes_) return -1;
        // Room for the largest frame now (no allocation during a step), and
        // the volume's own queued work done before the batch stream uses it.
        if (!v->reserve_batch(max_points)) return -1;
        v->synchronize();
        storage_ = v->storage();
        if (slot < 0) {
            slot = (int)vols_.size();
            vols_.push_back(nullptr);
            max_points_.push_back(0);
            pending_.push_back(BatchArgs{});
            drop_graph();  // the table grew
        }
        vols_[slot] = v;
        max_points_[slot] = max_points;
        pending_[slot] = BatchArgs{};
        ++live_;
        return slot;
    }

    // Detach a scene after the steps queued so far have run; its slot is
    // reused by the next add.
    int remove(int scene) {
        if (scene < 0 || scene >= (int)vols_.size() || !vols_[scene]) return 1;
        if (cudaStreamSynchronize(stream_) != cudaSuccess) return 3;
        vols_[scene] = nullptr;
        pending_[scene] = BatchArgs{};
        --live_;
        return 0;
    }

    Volume* volume(int scene) const {
        return scene >= 0 && scene < (int)vols_.size() ? vols_[scene] : nullptr;
    }

    int set_frame(int scene, const BatchArgs& a) {
        if (scene < 0 || scene >= (int)vols_.size() || !vols_[scene] || !a.pos || a.n <= 0 ||
            a.n > max_points_[scene])
            return 1;
        pending_[scene] = a;
        return 0;
    }

    // One step over every scene with a frame set since the last step.
    cudaError_t step() {
        const int n = (int)vols_.size();
        if (n == 0) return cudaSuccess;
        const int k = cur_;
        cur_ ^= 1;
        cudaError_t e = cudaEventSynchronize(table_free_[k]);  // its previous upload has run
        if (e != cudaSuccess) return e;
        SceneWork* table = h_table_[k];
        for (int s = 0; s < n; ++s) {
            if (!vols_[s]) {  // free slot: no work, nothing to point at
                table[s] = SceneWork{};
                continue;
            }
            if (pending_[s].n > 0) {
                table[s] = vols_[s]->batch_work(pending_[s], stream_);
            } else {
                // Idle this step: no items, counters left as they are.
                SceneWork idle = vols_[s]->batch_work(BatchArgs{}, stream_);
                idle.band_tiles = 0;
                idle.n_slots = 0;
                table[s] = idle;
            }
            pending_[s] = BatchArgs{};
        }
        e = cudaMemcpyAsync(d_scenes_, table, (size_t)n * sizeof(SceneWork), cudaMemcpyHostToDevice, stream_);
        if (e != cudaSuccess) return e;
        if ((e = cudaEventRecord(table_free_[k], stream_)) != cudaSuccess) return e;

        const BatchShape shape = next_shape();
        cudaEvent_t t0 = nullptr, t1 = nullptr;
        if (tuning_) {
            cudaEventCreate(&t0);
            cudaEventCreate(&t1);
            cudaEventRecord(t0, stream_);
        }
        const StepWork w = work(n, shape);
        const bool have = exec_ && graph_n_ == n && same(graph_shape_, shape);
        if (graph_on_ && !tuning_ && (have || (ran_n_ == n && same(ran_shape_, shape)))) {
            // Captured after one uncaptured run of the same passes (so every
            // one-time host query has happened), then replayed.
            if (!have) {
                drop_graph();
                if ((e = capture(w, shape)) != cudaSuccess) return e;
            }
            e = cudaGraphLaunch(exec_, stream_);
        } else {
            e = passes(w, shape);
            ran_n_ = n;
            ran_shape_ = shape;
        }
        if (tuning_) {
            cudaEventRecord(t1, stream_);
            tune_log_.push_back(TuneStep{tune_index_, t0, t1});
            advance_tuning();
        }
        return e;
    }

    cudaError_t synchronize() { return cudaStreamSynchronize(stream_); }

    uint32_t status() {
        uint32_t st = 0;
        if (cudaMemcpyAsync(h_status_, d_status_, sizeof(uint32_t), cudaMemcpyDeviceToHost, stream_) ==
                cudaSuccess &&
            cudaStreamSynchronize(stream_) == cudaSuccess)
            st = *h_status_;
        for (Volume* v : vols_)
            if (v) st |= v->status();
        return st;
    }

    void set_graph(bool on) {
        graph_on_ = on;
        if (!on) drop_graph();
    }

    void set_shape(const BatchShape& s) {
        shape_ = s;
        tuning_ = false;
    }
    BatchShape shape() const { return shape_; }
    bool tuning() const { return tuning_; }

    // Try every candidate shape for steps_per_shape of the next steps, then
    // keep the one with the smallest median step time.
    void autotune(int steps_per_shape) {
        candidates_.clear();
        for (int tiles : {1, 2, 4, 8})
            for (int probe : {0, 1})
                for (int pair : {1, 0}) {
                    BatchShape s;
                    s.band_tiles_per_item = tiles;
                    s.probe = probe;
                    s.finish_pair = pair;
                    candidates_.push_back(s);
                }
        steps_per_shape_ = std::max(1, steps_per_shape);
        tune_index_ = 0;
        tune_step_ = 0;
        tuning_ = true;
    }

    // Median step time of each candidate so far (ms), in candidate order.
    std::vector<double> tune_results() {
        cudaStreamSynchronize(stream_);
        std::vector<std::vector<double>> per(candidates_.size());
        for (auto& t : tune_log_) {
            float ms = 0.0f;
            if (cudaEventElapsedTime(&ms, t.start, t.end) == cudaSuccess) per[t.shape].push_back(ms);
        }
        std::vector<double> med(candidates_.size(), -1.0);
        for (size_t c = 0; c < per.size(); ++c) {
            auto& v = per[c];
            if (v.empty()) continue;
            std::sort(v.begin(), v.end());
            med[c] = v[v.size() / 2];
        }
        return med;
    }

private:
    struct TuneStep {
        int shape;
        cudaEvent_t start, end;
    };

    static bool same(const BatchShape& a, const BatchShape& b) {
        return a.band_tiles_per_item == b.band_tiles_per_item && a.probe == b.probe &&
               a.finish_pair == b.finish_pair;
    }

    StepWork work(int n, const BatchShape& shape) const {
        StepWork w{};
        w.scenes = d_scenes_;
        w.n_scenes = n;
        w.band_tiles_per_item = std::max(1, std::min(shape.band_tiles_per_item, kBandTilesPerItemMax));
        w.queues = d_queues_;
        w.status = d_status_;
        return w;
    }

    cudaError_t passes(const StepWork& w, const BatchShape& shape) {
        cudaError_t e = launch_batch_prepare(w, stream_);
        if (e == cudaSuccess) e = launch_band_multi(w, storage_, shape.probe, sm_count_, stream_);
        if (e == cudaSuccess) e = launch_finish_multi(w, storage_, shape.finish_pair, sm_count_, stream_);
        if (e == cudaSuccess) e = launch_group_multi(w, storage_, sm_count_, stream_);
        if (e == cudaSuccess) e = launch_select_multi(w, storage_, sm_count_, stream_);
        return e;
    }

    cudaError_t capture(const StepWork& w, const BatchShape& shape) {
        cudaError_t e = cudaStreamBeginCapture(stream_, cudaStreamCaptureModeThreadLocal);
        if (e != cudaSuccess) return e;
        const cudaError_t le = passes(w, shape);
        cudaGraph_t g = nullptr;
        e = cudaStreamEndCapture(stream_, &g);
        if (le != cudaSuccess) e = le;
        if (e == cudaSuccess) e = cudaGraphInstantiate(&exec_, g, 0);
        if (g) cudaGraphDestroy(g);
        if (e != cudaSuccess) {
            exec_ = nullptr;
            return e;
        }
        graph_n_ = w.n_scenes;
        graph_shape_ = shape;
        return cudaSuccess;
    }

    void drop_graph() {
        if (exec_) cudaGraphExecDestroy(exec_);
        exec_ = nullptr;
        graph_n_ = -1;
    }

    BatchShape next_shape() const { return tuning_ ? candidates_[tune_index_] : shape_; }

    void advance_tuning() {
        if (++tune_step_ < steps_per_shape_) return;
        tune_step_ = 0;
        if (++tune_index_ < (int)candidates_.size()) return;
        // Done: keep the fastest median.
        const std::vector<double> med = tune_results();
        int best = -1;
        for (size_t c = 0; c < med.size(); ++c)
            if (med[c] >= 0.0 && (best < 0 || med[c] < med[best])) best = (int)c;
        if (best >= 0) shape_ = candidates_[best];
        tuning_ = false;
        tune_index_ = 0;
    }

    bool ok_ = false;
    int max_scenes_;
    int sm_count_ = 148;
    int storage_ = -1;
    int live_ = 0;  // attached scenes
    cudaStream_t stream_ = nullptr;
    std::vector<Volume*> vols_;
    std::vector<int32_t> max_points_;
    std::vector<BatchArgs> pending_;
    SceneWork* d_scenes_ = nullptr;
    uint32_t* d_queues_ = nullptr;
    uint32_t* d_status_ = nullptr;
    uint32_t* h_status_ = nullptr;
    SceneWork* h_table_[2] = {nullptr, nullptr};
    cudaEvent_t table_free_[2] = {nullptr, nullptr};
    int cur_ = 0;

    BatchShape shape_{};
    bool graph_on_ = false;
    int ran_n_ = -1;           // scenes and shape of the last uncaptured step
    BatchShape ran_shape_{};
    cudaGraphExec_t exec_ = nullptr;
    int graph_n_ = -1;
    BatchShape graph_shape_{};

    bool tuning_ = false;
    std::vector<BatchShape> candidates_;
    int steps_per_shape_ = 1, tune_index_ = 0, tune_step_ = 0;
    std::vector<TuneStep> tune_log_;

public:
    const std::vector<BatchShape>& candidates() const { return candidates_; }
};

}  // namespace osn_b200

struct OsnTsdfBatch {
    osn_b200::Batch b;
    explicit OsnTsdfBatch(int n) : b(n) {}
};

namespace {
osn_b200::Batch* batch_of(OsnTsdfBatch* b) { return b && b->b.ok() ? &b->b : nullptr; }
}  // namespace

extern "C" {

OsnTsdfBatch* osn_tsdf_batch_create(int32_t max_scenes) {
    auto* b = new (std::nothrow) OsnTsdfBatch(max_scenes);
    if (b && !b->b.ok()) {
        delete b;
        return nullptr;
    }
    return b;
}

void osn_tsdf_batch_destroy(OsnTsdfBatch* b) { delete b; }

int32_t osn_tsdf_batch_add(OsnTsdfBatch* b, OsnTsdfCudaVolume* v, int32_t max_points) {
    osn_b200::Batch* x = batch_of(b);
    osn_b200::Volume* vol = osn_tsdf_b200_volume_of(v);
    if (!x || !vol) return -1;
    return x->add(vol, max_points);
}

int32_t osn_tsdf_batch_remove(OsnTsdfBatch* b, int32_t scene) {
    osn_b200::Batch* x = batch_of(b);
    if (!x) return 1;
    return x->remove(scene);
}

int32_t osn_tsdf_batch_set_frame(OsnTsdfBatch* b, int32_t scene, const float* d_positions,
                                 int32_t n_points, float cam_x, float cam_y, float cam_z,
                                 float radius_m) {
    osn_b200::Batch* x = batch_of(b);
    if (!x) return 1;
    osn_b200::BatchArgs a{};
    a.pos = d_positions;
    a.n = n_points;
    a.cam_x = cam_x;
    a.cam_y = cam_y;
    a.cam_z = cam_z;
    a.radius_sq = radius_m > 0.0f ? radius_m * radius_m : 0.0f;
    return x->set_frame(scene, a);
}

int32_t osn_tsdf_batch_step(OsnTsdfBatch* b) {
    osn_b200::Batch* x = batch_of(b);
    if (!x) return 1;
    return x->step() == cudaSuccess ? 0 : 3;
}

int32_t osn_tsdf_batch_synchronize(OsnTsdfBatch* b) {
    osn_b200::Batch* x = batch_of(b);
    if (!x) return 1;
    return x->synchronize() == cudaSuccess ? 0 : 3;
}

int32_t osn_tsdf_batch_set_graph(OsnTsdfBatch* b, int32_t enabled) {
    osn_b200::Batch* x = batch_of(b);
    if (!x) return 1;
    x->set_graph(enabled != 0);
    return 0;
}

int32_t osn_tsdf_batch_autotune(OsnTsdfBatch* b, int32_t steps_per_shape) {
    osn_b200::Batch* x = batch_of(b);
    if (!x || steps_per_shape <= 0) return 1;
    x->autotune(steps_per_shape);
    return 0;
}

int32_t osn_tsdf_batch_set_shape(OsnTsdfBatch* b, int32_t tiles_per_item, int32_t probe,
                                 int32_t finish_pair) {
    osn_b200::Batch* x = batch_of(b);
    if (!x || tiles_per_item < 1 || tiles_per_item > osn_b200::kBandTilesPerItemMax || probe < 0 ||
        probe > 1 || finish_pair < 0 || finish_pair > 1)
        return 1;
    osn_b200::BatchShape s;
    s.band_tiles_per_item = tiles_per_item;
    s.probe = probe;
    s.finish_pair = finish_pair;
    x->set_shape(s);
    return 0;
}

int32_t osn_tsdf_batch_shape(OsnTsdfBatch* b, int32_t* out3) {
    osn_b200::Batch* x = batch_of(b);
    if (!x || !out3) return -1;
    const osn_b200::BatchShape s = x->shape();
    out3[0] = s.band_tiles_per_item;
    out3[1] = s.probe;
    out3[2] = s.finish_pair;
    return x->tuning() ? 1 : 0;
}

int32_t osn_tsdf_batch_tune_results(OsnTsdfBatch* b, double* ms, int32_t* shapes, int32_t n_max) {
    osn_b200::Batch* x = batch_of(b);
    if (!x || n_max <= 0) return 0;
    const std::vector<double> med = x->tune_results();
    const auto& cand = x->candidates();
    const int n = std::min<int>((int)med.size(), n_max);
    for (int k = 0; k < n; ++k) {
        if (ms) ms[k] = med[k];
        if (shapes) {
            shapes[3 * k + 0] = cand[k].band_tiles_per_item;
            shapes[3 * k + 1] = cand[k].probe;
            shapes[3 * k + 2] = cand[k].finish_pair;
        }
    }
    return n;
}

uint32_t osn_tsdf_batch_status(OsnTsdfBatch* b) {
    osn_b200::Batch* x = batch_of(b);
    return x ? x->status() : 0u;
}

void* osn_tsdf_batch_stream(OsnTsdfBatch* b) {
    osn_b200::Batch* x = batch_of(b);
    return x ? (void*)x->stream() : nullptr;
}

int32_t osn_tsdf_batch_size(OsnTsdfBatch* b) {
    osn_b200::Batch* x = batch_of(b);
    return x ? x->size() : 0;
}

}  // extern "C"
