// update_voxels without any device allocation.
//
// The regular update_voxels keeps its per-call scratch (one record and one
// normalised SDF per band slot, and the grouped records of voxels that
// cross the cap) in buffers the volume grows with cudaMalloc the first time
// a batch needs more room, which also waits for the volume's stream and
// frees the old buffers. Some callers cannot allow that: serving loops that
// admit work against a fixed device-memory budget (memory appearing behind
// their back breaks the budget, and a failed cudaMalloc in the middle of a
// request has no good recovery), and latency-critical threads that cannot
// absorb the device-wide synchronisation cudaMalloc and cudaFree imply. This
// entry point gives them the same update with its scratch in one fixed
// array compiled into the library.
//
// The array is a file-scope __device__ variable of kNoAllocScratchBytes
// (36 MiB + 256 bytes): the control counters, then kNoAllocMaxRecords 4-byte
// band records, as many 4-byte normalised SDFs and as many 8-byte group
// entries, and half as many 4-byte crossing-voxel entries, i.e. batches with
// n_points * (2 * steps + 1) <= 2,097,152 (a
// 480x360 frame at 9 band steps per point fits; a 640x480 frame must be
// split in two). The per-voxel and per-block state the update also uses
// belongs to the volume and was allocated with it. Every GPU on which the
// library's code is loaded holds the array until the process exits.
// Every call shares it and it keeps the last call's contents; the counters
// that must start at zero are cleared at the start of each call. Two calls
// whose work overlaps on the GPU (two volumes on different streams, say)
// race on the array and corrupt each other's results: serialise them. The
// calling thread's current device must be the volume's.
#include <algorithm>
#include <cstdio>
#include <mutex>

#include "../../include/osn_tsdf_b200.h"
#include "volume.h"

namespace osn_b200 {

namespace {

constexpr size_t kNoAllocHeaderBytes = 256;  // UpdateControl, padded
constexpr int64_t kNoAllocMaxRecords = OSN_TSDF_NOALLOC_MAX_RECORDS;
constexpr size_t kNoAllocRecordBytes = (size_t)kNoAllocMaxRecords * sizeof(uint32_t);
constexpr size_t kNoAllocSlotValBytes = (size_t)kNoAllocMaxRecords * sizeof(float);
constexpr size_t kNoAllocGroupBytes = (size_t)kNoAllocMaxRecords * sizeof(unsigned long long);
constexpr int64_t kNoAllocMaxCrossing = kNoAllocMaxRecords / 2;  // at least two records each
constexpr size_t kNoAllocCrossBytes = (size_t)kNoAllocMaxCrossing * sizeof(uint32_t);
constexpr size_t kNoAllocScratchBytes = kNoAllocHeaderBytes + kNoAllocRecordBytes + kNoAllocSlotValBytes +
                                        kNoAllocGroupBytes + kNoAllocCrossBytes;
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
    u.slot_val = dv_.storage == kStoreF64
                     ? nullptr
                     : reinterpret_cast<float*>(base + kNoAllocHeaderBytes + kNoAllocRecordBytes);
    u.grp = reinterpret_cast<unsigned long long*>(base + kNoAllocHeaderBytes + kNoAllocRecordBytes +
                                                  kNoAllocSlotValBytes);
    u.xlist = reinterpret_cast<uint32_t*>(base + kNoAllocHeaderBytes + kNoAllocRecordBytes +
                                          kNoAllocSlotValBytes + kNoAllocGroupBytes);
    u.record_cap = kNoAllocMaxRecords;
    u.xlist_cap = kNoAllocMaxCrossing;
    // Only the control counters must start at zero (run_update clears them);
    // every record slot is rewritten before it is read, and group entries are
    // read only where this call placed them.
    cudaError_t e = run_update(a, u, false);
    if (e != cudaSuccess) return e;
    // The call's counters into the volume's own control block (stream order),
    // so last_update_stats keeps describing this volume whatever later calls
    // on other volumes leave in the shared array.
    e = cudaMemcpyAsync(us_.ctl, u.ctl, sizeof(UpdateControl), cudaMemcpyDeviceToDevice, stream_);
    if (e == cudaSuccess) last_ctl_ = us_.ctl;
    return e;
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
    if (device != vol->device()) {
        // The array's address is per device: another device's copy would be
        // a wrong (or unreachable) address for this volume's kernels.
        std::fprintf(stderr,
                     "[osn_tsdf_b200] update_voxels_noalloc: current device %d is not the volume's "
                     "device %d; make the volume's device current first\n",
                     device, vol->device());
        return 1;
    }
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
