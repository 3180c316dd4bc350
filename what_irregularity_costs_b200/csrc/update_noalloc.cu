// update_voxels without any device allocation.
//
// The regular update_voxels keeps its per-call scratch (one record per band
// slot, the grouped records of voxels that cross the cap, and their list) in
// buffers the volume grows with cudaMalloc the first time a batch needs more
// room, which also waits for the volume's stream and frees the old buffers. Some callers cannot allow that: code
// that records the integrate into a CUDA graph (allocation is not permitted
// while a stream is being captured), serving loops that admit work against a
// fixed device-memory budget and must not see memory appear behind their
// back, and latency-critical threads that cannot absorb the synchronisation
// cudaMalloc/cudaFree imply. This entry point gives them the same update
// with its scratch in one fixed array compiled into the library.
//
// The array is a file-scope __device__ variable of kNoAllocScratchBytes
// (56 MiB + 256 bytes): the control counters, kNoAllocMaxRecords 4-byte band
// records and 4-byte slot values, as many 4-byte ids and 8-byte values of
// crossing voxels' records, and half as many 16-byte crossing-voxel entries,
// i.e. batches with
// n_points * (2 * steps + 1) <= 2,097,152 (a 480x360 frame at 9 band steps
// per point fits; a 640x480 frame must be split in two). The per-voxel and
// per-block state the update also uses belongs to the volume and was
// allocated with it. Every GPU on which
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
constexpr int64_t kNoAllocMaxDeferred = kNoAllocMaxRecords / 2;
constexpr size_t kNoAllocRecordBytes = (size_t)kNoAllocMaxRecords * sizeof(uint32_t);
constexpr size_t kNoAllocDeferredBytes = (size_t)kNoAllocMaxRecords * sizeof(uint32_t);
constexpr size_t kNoAllocFixBytes = (size_t)kNoAllocMaxRecords * sizeof(long long);
constexpr size_t kNoAllocSlotValBytes = (size_t)kNoAllocMaxRecords * sizeof(float);
constexpr size_t kNoAllocScratchBytes = kNoAllocHeaderBytes + kNoAllocRecordBytes +
                                        kNoAllocDeferredBytes + kNoAllocFixBytes +
                                        (size_t)kNoAllocMaxDeferred * sizeof(int4) + kNoAllocSlotValBytes;
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
    u.records = reinterpret_cast<uint32_t*>(base + kNoAllocHeaderBytes);
    u.deferred = reinterpret_cast<uint32_t*>(base + kNoAllocHeaderBytes + kNoAllocRecordBytes);
    u.deferred_fix = reinterpret_cast<long long*>(base + kNoAllocHeaderBytes + kNoAllocRecordBytes +
                                                  kNoAllocDeferredBytes);
    u.dvox = reinterpret_cast<int4*>(base + kNoAllocHeaderBytes + kNoAllocRecordBytes +
                                     kNoAllocDeferredBytes + kNoAllocFixBytes);
    u.slot_val = dv_.storage == kStoreF64
                     ? nullptr
                     : reinterpret_cast<float*>(base + kNoAllocScratchBytes - kNoAllocSlotValBytes);
    u.record_cap = kNoAllocMaxRecords;
    u.dvox_cap = (int32_t)kNoAllocMaxDeferred;
    // Only the control counters must start at zero (run_update clears them);
    // every record slot is rewritten before it is read, and deferred records
    // and entries are read only where this call placed them.
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
    if (records > osn_b200::kNoAllocMaxRecords) {
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
    osn_b200::BatchArgs a{};
    a.pos = d_positions;
    a.n = n_points;
    a.cam_x = cam_x;
    a.cam_y = cam_y;
    a.cam_z = cam_z;
    a.radius_sq = radius_m > 0.0f ? radius_m * radius_m : 0.0f;
    return vol->update_static_scratch(a, scratch) == cudaSuccess ? 0 : 3;
}
