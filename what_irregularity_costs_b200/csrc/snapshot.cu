// Snapshot and restore of a volume's contents through host memory.
//
// No counterpart in the reference (cpp/src/volume_cuda.cu has reset only,
// :362-382). A volume's state is its allocated blocks: the coordinates of
// pool slots 0..block_count-1 and the first block_count * 512 voxels of each
// voxel array (blocks take pool indices in order, so each array's used part
// is one contiguous prefix), plus the drop counter. The hash table is not
// saved: restore re-inserts every block's key (same pool index) with a
// kernel, so a restored volume continues exactly as the original would
// (slot positions may differ; lookups, updates and extraction do not depend
// on them). Used to checkpoint a volume or to move an idle session out of HBM
// and back.
//
// Layout: SnapshotHeader, int32[3] coordinates per block, then the prefixes
// of tsdf, weight (and r, g, b for FP32 storage), in that order.
#include <cstring>

#include "../../include/osn_tsdf_b200.h"
#include "volume.h"

namespace osn_b200 {
namespace {

struct SnapshotHeader {
    char magic[8];
    int32_t version;
    int32_t storage;
    float voxel_size, trunc, weight_cap;
    int32_t block_count;
    unsigned long long drop_count;
    int32_t reserved[6];
};
static_assert(sizeof(SnapshotHeader) == 64, "snapshot header is 64 bytes");
constexpr char kMagic[8] = {'O', 'S', 'N', 'B', '2', '0', '0', '\0'};

// Re-insert block i's key into an empty table (one thread per block; the
// keys are distinct, so a claim only ever meets other keys).
__global__ void rebuild_table_kernel(DevVolume v, int32_t n_blocks) {
    const int32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n_blocks) return;
    const BlockCoord c = v.block_coord[i];
    const long long key = pack_key(c.x, c.y, c.z);
    const uint32_t size = v.hash_mask + 1;
    const uint32_t start = hash_slot(c.x, c.y, c.z, v.hash_mask);
    for (uint32_t p = 0; p < size; ++p) {
        HashEntry* e = &v.table[(start + p) & v.hash_mask];
        const long long prev = (long long)atomicCAS((unsigned long long*)&e->key,
                                                    (unsigned long long)kEmptyKey, (unsigned long long)key);
        if (prev == kEmptyKey) {
            e->block_idx = i;
            return;
        }
    }
    atomicOr(v.status, kStatusScratchOverflow);  // table full: cannot happen with block_count <= slots
}

}  // namespace

size_t voxel_arrays(int storage, const DevVolume& d, void* out[5], size_t bytes[5]) {
    const int n = storage == kStoreF32 ? 5 : 2;
    out[0] = d.tsdf;
    bytes[0] = (size_t)tsdf_bytes(storage);
    out[1] = d.weight;
    bytes[1] = (size_t)weight_bytes(storage);
    if (n == 5) {
        out[2] = d.r;
        out[3] = d.g;
        out[4] = d.b;
        bytes[2] = bytes[3] = bytes[4] = 4;
    }
    return (size_t)n;
}

cudaError_t launch_rebuild_table(const DevVolume& v, int32_t n_blocks, cudaStream_t s) {
    if (n_blocks <= 0) return cudaSuccess;
    rebuild_table_kernel<<<(n_blocks + 255) / 256, 256, 0, s>>>(v, n_blocks);
    return cudaGetLastError();
}

int64_t Volume::snapshot_bytes() {
    if (dv_.slot_index) return -1;  // the pool-order layout only
    const int64_t b = std::min(block_count(), dv_.pool_capacity);
    void* arr[5];
    size_t per[5];
    const size_t n = voxel_arrays(dv_.storage, dv_, arr, per);
    int64_t total = (int64_t)sizeof(SnapshotHeader) + b * (int64_t)sizeof(BlockCoord);
    for (size_t k = 0; k < n; ++k) total += b * kBlockVoxels * (int64_t)per[k];
    return total;
}

int64_t Volume::snapshot(void* host, int64_t cap) {
    const int64_t need = snapshot_bytes();  // waits for the stream
    if (need < 0 || !host || cap < need) return -1;
    const int32_t b = std::min(block_count(), dv_.pool_capacity);
    SnapshotHeader h{};
    std::memcpy(h.magic, kMagic, sizeof(kMagic));
    h.version = 1;
    h.storage = dv_.storage;
    h.voxel_size = dv_.voxel_size;
    h.trunc = dv_.trunc;
    h.weight_cap = weight_cap_;
    h.block_count = b;
    h.drop_count = drop_count();
    unsigned char* p = static_cast<unsigned char*>(host);
    std::memcpy(p, &h, sizeof(h));
    p += sizeof(h);
    if (cudaMemcpyAsync(p, dv_.block_coord, (size_t)b * sizeof(BlockCoord), cudaMemcpyDeviceToHost,
                        stream_) != cudaSuccess)
        return -1;
    p += (size_t)b * sizeof(BlockCoord);
    void* arr[5];
    size_t per[5];
    const size_t n = voxel_arrays(dv_.storage, dv_, arr, per);
    for (size_t k = 0; k < n; ++k) {
        const size_t bytes = (size_t)b * kBlockVoxels * per[k];
        if (cudaMemcpyAsync(p, arr[k], bytes, cudaMemcpyDeviceToHost, stream_) != cudaSuccess) return -1;
        p += bytes;
    }
    if (cudaStreamSynchronize(stream_) != cudaSuccess) return -1;
    return need;
}

int32_t Volume::restore(const void* host, int64_t size) {
    if (dv_.slot_index || !host || size < (int64_t)sizeof(SnapshotHeader)) return 1;
    SnapshotHeader h;
    std::memcpy(&h, host, sizeof(h));
    if (std::memcmp(h.magic, kMagic, sizeof(kMagic)) != 0 || h.version != 1) return 1;
    if (h.storage != dv_.storage || h.voxel_size != dv_.voxel_size || h.trunc != dv_.trunc ||
        h.weight_cap != weight_cap_ || h.block_count < 0 || h.block_count > dv_.pool_capacity ||
        (int64_t)h.block_count > (int64_t)dv_.hash_mask + 1)
        return 1;
    const int32_t b = h.block_count;
    void* arr[5];
    size_t per[5];
    const size_t n = voxel_arrays(dv_.storage, dv_, arr, per);
    int64_t need = (int64_t)sizeof(h) + (int64_t)b * (int64_t)sizeof(BlockCoord);
    for (size_t k = 0; k < n; ++k) need += (int64_t)b * kBlockVoxels * (int64_t)per[k];
    if (size < need) return 1;
    if (reset() != cudaSuccess) return 3;  // empty table, zeroed blocks, counters cleared
    const unsigned char* p = static_cast<const unsigned char*>(host) + sizeof(h);
    if (cudaMemcpyAsync(dv_.block_coord, p, (size_t)b * sizeof(BlockCoord), cudaMemcpyHostToDevice,
                        stream_) != cudaSuccess)
        return 3;
    p += (size_t)b * sizeof(BlockCoord);
    for (size_t k = 0; k < n; ++k) {
        const size_t bytes = (size_t)b * kBlockVoxels * per[k];
        if (cudaMemcpyAsync(arr[k], p, bytes, cudaMemcpyHostToDevice, stream_) != cudaSuccess) return 3;
        p += bytes;
    }
    if (launch_rebuild_table(dv_, b, stream_) != cudaSuccess) return 3;
    if (cudaMemcpyAsync(dv_.block_count, &b, sizeof(int32_t), cudaMemcpyHostToDevice, stream_) !=
            cudaSuccess ||
        cudaMemcpyAsync(dv_.drop_count, &h.drop_count, sizeof(unsigned long long),
                        cudaMemcpyHostToDevice, stream_) != cudaSuccess ||
        cudaStreamSynchronize(stream_) != cudaSuccess)
        return 3;
    return 0;
}

}  // namespace osn_b200

extern "C" {

int64_t osn_tsdf_cuda_snapshot_bytes(OsnTsdfCudaVolume* v) {
    osn_b200::Volume* vol = osn_tsdf_b200_volume_of(v);
    return vol ? vol->snapshot_bytes() : -1;
}

int64_t osn_tsdf_cuda_snapshot(OsnTsdfCudaVolume* v, void* host_buffer, int64_t capacity) {
    osn_b200::Volume* vol = osn_tsdf_b200_volume_of(v);
    return vol ? vol->snapshot(host_buffer, capacity) : -1;
}

int32_t osn_tsdf_cuda_restore(OsnTsdfCudaVolume* v, const void* host_buffer, int64_t size) {
    osn_b200::Volume* vol = osn_tsdf_b200_volume_of(v);
    return vol ? vol->restore(host_buffer, size) : 1;
}

}  // extern "C"
