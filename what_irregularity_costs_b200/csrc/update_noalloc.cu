// update_voxels without any device allocation.
//
// The regular update_voxels keeps its per-call scratch (the binned
// contribution records) in a buffer the volume grows with cudaMalloc the
// first time a batch needs more room, which also waits for the volume's
// stream and frees the old buffer. Some callers cannot allow that: code
// that records the integrate into a CUDA graph (allocation is not permitted
// while a stream is being captured), serving loops that admit work against a
// fixed device-memory budget and must not see memory appear behind their
// back, and latency-critical threads that cannot absorb the synchronisation
// cudaMalloc/cudaFree imply. This entry point gives them the same update
// with its scratch in one fixed array compiled into the library.
//
// The array is a file-scope __device__ variable of kNoAllocScratchBytes
// (72 MiB + 256 bytes): the control counters, the staging area and the bins
// for kNoAllocMaxRecords 16-byte records each, and kNoAllocMaxSegments
// 16-byte segment descriptors, i.e. batches with
// n_points * (2 * steps + 1) <= 2,097,152 (a 480x360 frame at 9 band steps
// per point fits; a 640x480 frame must be split in two). Every GPU on which
// the library's code is loaded holds the array until the process exits.
// Every call shares it and it keeps the last call's contents; the counters
// that must start at zero are cleared at the start of each call. Two calls
// whose work overlaps on the GPU (two volumes on different streams, say)
// race on the array and corrupt each other's results: serialise them.
#include <algorithm>
#include <cstdio>
#include <mutex>

#include "../../include/osn_tsdf_b200.h"
#include "volume.h"

namespace osn_b200 {

namespace {

constexpr size_t kNoAllocHeaderBytes = 256;  // UpdateControl, padded
constexpr int64_t kNoAllocMaxRecords = OSN_TSDF_NOALLOC_MAX_RECORDS;
constexpr int64_t kNoAllocMaxSegments = (int64_t)1 << 19;
constexpr size_t kNoAllocRecordBytes = (size_t)kNoAllocMaxRecords * sizeof(Record);
constexpr size_t kNoAllocScratchBytes =
    kNoAllocHeaderBytes + 2 * kNoAllocRecordBytes + (size_t)kNoAllocMaxSegments * sizeof(int4);
static_assert(sizeof(UpdateControl) <= kNoAllocHeaderBytes, "control block must fit the header");

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

constexpr int kMaxDevices = 64;
std::mutex g_setup_mutex;
void* g_scratch_addr[kMaxDevices] = {};

// Device address of the array on the current device. In host code the
// array's name is only a stand-in for the symbol, not a device address, so
// it is resolved once per device with cudaGetSymbolAddress (with that device
// current) and cached. Resolving it may load this file's module on the
// device, which is not allowed during stream capture: make the first call on
// each device before capturing.
void* scratch_address(int device) {
    if (device < 0 || device >= kMaxDevices) return nullptr;
    std::lock_guard<std::mutex> lock(g_setup_mutex);
    if (!g_scratch_addr[device]) {
        void* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess) {
            std::fprintf(stderr, "[osn_tsdf_b200] cudaGetSymbolAddress(no-alloc scratch) failed on "
                                 "device %d: %s\n", device, cudaGetErrorString(e));
            return nullptr;
        }
        g_scratch_addr[device] = p;
    }
    return g_scratch_addr[device];
}

}  // namespace

cudaError_t Volume::update_static_scratch(const BatchArgs& a, void* scratch) {
    unsigned char* base = static_cast<unsigned char*>(scratch);
    UpdateScratch u = us_;
    u.ctl = reinterpret_cast<UpdateControl*>(base);
    u.records = reinterpret_cast<Record*>(base + kNoAllocHeaderBytes);
    u.bins = reinterpret_cast<Record*>(base + kNoAllocHeaderBytes + kNoAllocRecordBytes);
    u.record_cap = kNoAllocMaxRecords;
    u.segs = reinterpret_cast<int4*>(base + kNoAllocHeaderBytes + 2 * kNoAllocRecordBytes);
    u.seg_cap = kNoAllocMaxSegments;
    // Only the control counters must start at zero (run_update clears them);
    // the records of the previous call are overwritten before they are read.
    return run_update(a, u, false);
}

}  // namespace osn_b200

extern "C" int32_t osn_tsdf_cuda_update_voxels_noalloc(OsnTsdfCudaVolume* v,
                                                       const float* d_positions, int32_t n_points,
                                                       float cam_x, float cam_y, float cam_z,
                                                       float radius_m) {
    osn_b200::Volume* vol = osn_tsdf_b200_volume_of(v);
    if (!vol || !d_positions || n_points <= 0) return 1;
    const int64_t records = (int64_t)n_points * (2 * (int64_t)vol->dev().steps + 1);
    const int64_t segments = std::min<int64_t>(records, (int64_t)((n_points + 255) / 256) * 512);
    if (records > osn_b200::kNoAllocMaxRecords || segments > osn_b200::kNoAllocMaxSegments) {
        std::fprintf(stderr,
                     "[osn_tsdf_b200] update_voxels_noalloc: batch of %d points needs %lld records, "
                     "above the fixed maximum of %lld (n_points * (2*steps+1)); split the batch\n",
                     n_points, (long long)records, (long long)osn_b200::kNoAllocMaxRecords);
        return 4;
    }
    int device = 0;
    if (cudaGetDevice(&device) != cudaSuccess) return 3;
    void* scratch = osn_b200::scratch_address(device);
    if (!scratch) return 3;
    osn_b200::BatchArgs a;
    a.pos = d_positions;
    a.n = n_points;
    a.cam_x = cam_x;
    a.cam_y = cam_y;
    a.cam_z = cam_z;
    a.radius_sq = radius_m > 0.0f ? radius_m * radius_m : 0.0f;
    return vol->update_static_scratch(a, scratch) == cudaSuccess ? 0 : 3;
}
