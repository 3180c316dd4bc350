// Streaming: blocks evicted to host memory and streamed back in, keyed by
// chunk id.
//
// The reference declares a chunk id on every point batch
// (cpp/include/osn_tsdf/types.hpp:127, PointBatch::chunk_id) and its FFI
// carries it (crates/tsdf-ffi/src/lib.rs:150), but no arm reads it. Here a
// volume has a current chunk id (osn_tsdf_cuda_set_chunk; the C++ class
// takes PointBatch::chunk_id), and every block carries the chunk id of the
// last call that allocated or updated it. A caller whose scene outgrows the
// pool -- a long trajectory through a large space, a session over its memory
// budget -- moves the blocks of chunks it has left behind to host memory:
//
//   evict    the blocks whose chunk id lies in [lo, hi] are gathered (with
//            their coordinates, chunk ids and voxel arrays) into a host pack,
//            the remaining blocks are moved to the front of the pool in their
//            old order, the vacated pool tail is zeroed and the table is
//            rebuilt from the remaining blocks. Their pool indices change,
//            their contents do not; freed pool entries take new blocks.
//   stream   a pack's blocks are inserted again (the production insert,
//   in       fresh pool indices) with their voxels and chunk ids; a block
//            that is present again (re-observed after its eviction) is left
//            as it is and counted as skipped.
//
// Pack layout: ChunkPackHeader, int32[3] coordinates per block, int32 chunk
// ids, then the blocks' tsdf and weight (and r, g, b for FP32 storage)
// arrays, 512 voxels per block, each array contiguous.
#include <algorithm>
#include <cstring>
#include <vector>

#include "../../include/osn_tsdf_b200.h"
#include "volume.h"

namespace osn_b200 {
namespace {

struct ChunkPackHeader {
    char magic[8];
    int32_t version;
    int32_t storage;
    float voxel_size, trunc, weight_cap;
    int32_t n_blocks;
    int32_t lo, hi;  // the evicted chunk range
    int32_t reserved[6];
};
static_assert(sizeof(ChunkPackHeader) == 64, "pack header is 64 bytes");
constexpr char kPackMagic[8] = {'O', 'S', 'N', 'C', 'H', 'N', 'K', '\0'};
constexpr int kCopyThreads = 128;

// Blocks of a pack or of a gather on the device: coordinates, chunk ids and
// up to five voxel arrays of n blocks each.
struct BlockSet {
    BlockCoord* coord;
    int32_t* chunk;
    unsigned char* arr[5];
    int32_t elem[5];  // bytes per voxel of each array
    int32_t n_arr;
};

// One block's span of every voxel array, by a whole CTA in 16-byte pieces
// (a span is 512 voxels of 2, 4 or 8 bytes: a multiple of 16 bytes).
__device__ __forceinline__ void copy_block(const BlockSet& dst, int32_t di, const BlockSet& src, int32_t si) {
    for (int k = 0; k < src.n_arr; ++k) {
        const size_t span = (size_t)kBlockVoxels * (size_t)src.elem[k];
        const uint4* s = reinterpret_cast<const uint4*>(src.arr[k] + (size_t)si * span);
        uint4* d = reinterpret_cast<uint4*>(dst.arr[k] + (size_t)di * span);
        for (int j = threadIdx.x; j < (int)(span / 16); j += blockDim.x) d[j] = s[j];
    }
}

// staging[p] = pool[order[p]] for p < n (one CTA per block).
__global__ void gather_blocks_kernel(BlockSet pool, BlockSet staging, const int32_t* order, int32_t n) {
    const int32_t p = blockIdx.x;
    if (p >= n) return;
    const int32_t src = order[p];
    if (threadIdx.x == 0) {
        staging.coord[p] = pool.coord[src];
        staging.chunk[p] = pool.chunk[src];
    }
    copy_block(staging, p, pool, src);
}

// Insert pack block p (one CTA per block): absent keys take a pool index
// from the production insert and get the pack's voxels and chunk id; keys
// already present are left alone and counted; a full pool is counted too.
__global__ void stream_in_kernel(DevVolume v, BlockSet pool, BlockSet pack, int32_t n, int32_t* counts) {
    const int32_t p = blockIdx.x;
    if (p >= n) return;
    __shared__ int32_t s_idx;
    if (threadIdx.x == 0) {
        const BlockCoord c = pack.coord[p];
        const long long key = pack_key(c.x, c.y, c.z);
        // Pack keys are distinct and nothing else inserts them here, so a
        // key found now was present before this kernel.
        int32_t idx = -1;
        if (find_block(v, c.x, c.y, c.z, key) >= 0) {
            atomicAdd(&counts[0], 1);
        } else {
            idx = find_or_insert<kAllocInsert>(v, c.x, c.y, c.z, key).idx;
            if (idx < 0) atomicAdd(&counts[1], 1);
            else v.block_chunk[idx] = pack.chunk[p];
        }
        s_idx = idx;
    }
    __syncthreads();
    if (s_idx >= 0) copy_block(pool, s_idx, pack, p);
}

BlockSet pool_set(const DevVolume& d) {
    BlockSet b{};
    b.coord = d.block_coord;
    b.chunk = d.block_chunk;
    void* arr[5];
    size_t per[5];
    b.n_arr = (int32_t)voxel_arrays(d.storage, d, arr, per);
    for (int k = 0; k < b.n_arr; ++k) {
        b.arr[k] = static_cast<unsigned char*>(arr[k]);
        b.elem[k] = (int32_t)per[k];
    }
    return b;
}

// Bytes of a pack of n blocks.
int64_t pack_bytes(const BlockSet& like, int64_t n) {
    int64_t total = (int64_t)sizeof(ChunkPackHeader) + n * (int64_t)(sizeof(BlockCoord) + sizeof(int32_t));
    for (int k = 0; k < like.n_arr; ++k) total += n * kBlockVoxels * like.elem[k];
    return total;
}

// Device buffers shaped like the pool, for n blocks (freed by release()).
bool alloc_set(const BlockSet& like, int32_t n, BlockSet& out) {
    out = like;
    out.coord = nullptr;
    out.chunk = nullptr;
    for (int k = 0; k < 5; ++k) out.arr[k] = nullptr;
    if (cudaMalloc(&out.coord, (size_t)n * sizeof(BlockCoord)) != cudaSuccess) return false;
    if (cudaMalloc(&out.chunk, (size_t)n * sizeof(int32_t)) != cudaSuccess) return false;
    for (int k = 0; k < like.n_arr; ++k)
        if (cudaMalloc(&out.arr[k], (size_t)n * kBlockVoxels * like.elem[k]) != cudaSuccess) return false;
    return true;
}

void release(BlockSet& s) {
    cudaFree(s.coord);
    cudaFree(s.chunk);
    for (int k = 0; k < 5; ++k) cudaFree(s.arr[k]);
    s = BlockSet{};
}

}  // namespace

int64_t Volume::evict_bytes(int32_t lo, int32_t hi) {
    if (lo > hi || dv_.slot_index) return -1;  // the pool-order layout only
    const int32_t b = std::min(block_count(), dv_.pool_capacity);  // joins and waits
    std::vector<int32_t> chunk((size_t)b);
    if (b > 0 && (cudaMemcpy(chunk.data(), dv_.block_chunk, (size_t)b * sizeof(int32_t),
                             cudaMemcpyDeviceToHost) != cudaSuccess))
        return -1;
    int64_t n = 0;
    for (int32_t c : chunk) n += (c >= lo && c <= hi) ? 1 : 0;
    return pack_bytes(pool_set(dv_), n);
}

int64_t Volume::evict_chunks(int32_t lo, int32_t hi, void* host, int64_t cap) {
    if (lo > hi || !host || dv_.slot_index) return -1;
    const int32_t b = std::min(block_count(), dv_.pool_capacity);  // joins and waits
    std::vector<int32_t> chunk((size_t)b);
    if (b > 0 && cudaMemcpy(chunk.data(), dv_.block_chunk, (size_t)b * sizeof(int32_t),
                            cudaMemcpyDeviceToHost) != cudaSuccess)
        return -1;
    // New order: the blocks that stay, then the evicted ones, each in pool order.
    std::vector<int32_t> order;
    order.reserve((size_t)b);
    for (int32_t i = 0; i < b; ++i)
        if (!(chunk[i] >= lo && chunk[i] <= hi)) order.push_back(i);
    const int32_t n_keep = (int32_t)order.size();
    for (int32_t i = 0; i < b; ++i)
        if (chunk[i] >= lo && chunk[i] <= hi) order.push_back(i);
    const int32_t n_ev = b - n_keep;
    const BlockSet pool = pool_set(dv_);
    const int64_t need = pack_bytes(pool, n_ev);
    if (cap < need) return -1;

    ChunkPackHeader h{};
    std::memcpy(h.magic, kPackMagic, sizeof(kPackMagic));
    h.version = 1;
    h.storage = dv_.storage;
    h.voxel_size = dv_.voxel_size;
    h.trunc = dv_.trunc;
    h.weight_cap = weight_cap_;
    h.n_blocks = n_ev;
    h.lo = lo;
    h.hi = hi;
    unsigned char* out = static_cast<unsigned char*>(host);
    std::memcpy(out, &h, sizeof(h));
    if (n_ev == 0) return need;

    BlockSet stage{};
    int32_t* d_order = nullptr;
    bool ok = alloc_set(pool, b, stage) && cudaMalloc(&d_order, (size_t)b * sizeof(int32_t)) == cudaSuccess &&
              cudaMemcpyAsync(d_order, order.data(), (size_t)b * sizeof(int32_t), cudaMemcpyHostToDevice,
                              stream_) == cudaSuccess;
    if (ok) {
        gather_blocks_kernel<<<b, kCopyThreads, 0, stream_>>>(pool, stage, d_order, b);
        ok = cudaGetLastError() == cudaSuccess;
    }
    // The blocks that stay, back to the front of the pool.
    ok = ok && cudaMemcpyAsync(pool.coord, stage.coord, (size_t)n_keep * sizeof(BlockCoord),
                               cudaMemcpyDeviceToDevice, stream_) == cudaSuccess;
    ok = ok && cudaMemcpyAsync(pool.chunk, stage.chunk, (size_t)n_keep * sizeof(int32_t),
                               cudaMemcpyDeviceToDevice, stream_) == cudaSuccess;
    for (int k = 0; ok && k < pool.n_arr; ++k) {
        const size_t span = (size_t)kBlockVoxels * pool.elem[k];
        ok = cudaMemcpyAsync(pool.arr[k], stage.arr[k], (size_t)n_keep * span, cudaMemcpyDeviceToDevice,
                             stream_) == cudaSuccess &&
             cudaMemsetAsync(pool.arr[k] + (size_t)n_keep * span, 0, (size_t)n_ev * span, stream_) == cudaSuccess;
    }
    // The table holds the remaining blocks only.
    ok = ok && launch_reset_table(dv_.table, dv_.hash_mask + 1, kEmptyKey, stream_) == cudaSuccess &&
         launch_rebuild_table(dv_, n_keep, stream_) == cudaSuccess;
    // The pack: coordinates, chunk ids, arrays of the evicted blocks.
    unsigned char* p = out + sizeof(h);
    ok = ok && cudaMemcpyAsync(p, stage.coord + n_keep, (size_t)n_ev * sizeof(BlockCoord),
                               cudaMemcpyDeviceToHost, stream_) == cudaSuccess;
    p += (size_t)n_ev * sizeof(BlockCoord);
    ok = ok && cudaMemcpyAsync(p, stage.chunk + n_keep, (size_t)n_ev * sizeof(int32_t), cudaMemcpyDeviceToHost,
                               stream_) == cudaSuccess;
    p += (size_t)n_ev * sizeof(int32_t);
    for (int k = 0; ok && k < pool.n_arr; ++k) {
        const size_t span = (size_t)kBlockVoxels * pool.elem[k];
        ok = cudaMemcpyAsync(p, stage.arr[k] + (size_t)n_keep * span, (size_t)n_ev * span,
                             cudaMemcpyDeviceToHost, stream_) == cudaSuccess;
        p += (size_t)n_ev * span;
    }
    int32_t* hs = reinterpret_cast<int32_t*>(host_small_);
    hs[0] = n_keep;
    ok = ok && cudaMemcpyAsync(dv_.block_count, hs, sizeof(int32_t), cudaMemcpyHostToDevice, stream_) == cudaSuccess &&
         cudaStreamSynchronize(stream_) == cudaSuccess;
    cudaFree(d_order);
    release(stage);
    return ok ? need : -1;
}

int32_t Volume::stream_in(const void* host, int64_t size, int32_t* skipped) {
    if (dv_.slot_index || !host || size < (int64_t)sizeof(ChunkPackHeader)) return 1;
    ChunkPackHeader h;
    std::memcpy(&h, host, sizeof(h));
    if (std::memcmp(h.magic, kPackMagic, sizeof(kPackMagic)) != 0 || h.version != 1) return 1;
    if (h.storage != dv_.storage || h.voxel_size != dv_.voxel_size || h.trunc != dv_.trunc ||
        h.weight_cap != weight_cap_ || h.n_blocks < 0)
        return 1;
    const BlockSet pool = pool_set(dv_);
    if (size < pack_bytes(pool, h.n_blocks)) return 1;
    if (skipped) *skipped = 0;
    const int32_t n = h.n_blocks;
    if (n == 0) return 0;
    join();
    BlockSet pack{};
    int32_t* d_counts = nullptr;
    bool ok = alloc_set(pool, n, pack) && cudaMalloc(&d_counts, 2 * sizeof(int32_t)) == cudaSuccess &&
              cudaMemsetAsync(d_counts, 0, 2 * sizeof(int32_t), stream_) == cudaSuccess;
    const unsigned char* p = static_cast<const unsigned char*>(host) + sizeof(h);
    ok = ok && cudaMemcpyAsync(pack.coord, p, (size_t)n * sizeof(BlockCoord), cudaMemcpyHostToDevice,
                               stream_) == cudaSuccess;
    p += (size_t)n * sizeof(BlockCoord);
    ok = ok && cudaMemcpyAsync(pack.chunk, p, (size_t)n * sizeof(int32_t), cudaMemcpyHostToDevice, stream_) ==
                   cudaSuccess;
    p += (size_t)n * sizeof(int32_t);
    for (int k = 0; ok && k < pool.n_arr; ++k) {
        const size_t bytes = (size_t)n * kBlockVoxels * pool.elem[k];
        ok = cudaMemcpyAsync(pack.arr[k], p, bytes, cudaMemcpyHostToDevice, stream_) == cudaSuccess;
        p += bytes;
    }
    if (ok) {
        stream_in_kernel<<<n, kCopyThreads, 0, stream_>>>(dv_, pool, pack, n, d_counts);
        ok = cudaGetLastError() == cudaSuccess;
    }
    int32_t* hs = reinterpret_cast<int32_t*>(host_small_);
    ok = ok && cudaMemcpyAsync(hs, d_counts, 2 * sizeof(int32_t), cudaMemcpyDeviceToHost, stream_) == cudaSuccess &&
         cudaStreamSynchronize(stream_) == cudaSuccess;
    const int32_t n_skip = ok ? hs[0] : 0, n_full = ok ? hs[1] : 0;
    cudaFree(d_counts);
    release(pack);
    if (!ok) return 3;
    if (skipped) *skipped = n_skip;
    return n_full > 0 ? 2 : 0;
}

}  // namespace osn_b200

extern "C" {

int32_t osn_tsdf_cuda_set_chunk(OsnTsdfCudaVolume* v, int32_t chunk_id) {
    osn_b200::Volume* vol = osn_tsdf_b200_volume_of(v);
    if (!vol) return 1;
    vol->set_chunk(chunk_id);
    return 0;
}

int64_t osn_tsdf_cuda_evict_chunks_bytes(OsnTsdfCudaVolume* v, int32_t lo, int32_t hi) {
    osn_b200::Volume* vol = osn_tsdf_b200_volume_of(v);
    return vol ? vol->evict_bytes(lo, hi) : -1;
}

int64_t osn_tsdf_cuda_evict_chunks(OsnTsdfCudaVolume* v, int32_t lo, int32_t hi, void* host_buffer,
                                   int64_t capacity) {
    osn_b200::Volume* vol = osn_tsdf_b200_volume_of(v);
    return vol ? vol->evict_chunks(lo, hi, host_buffer, capacity) : -1;
}

int32_t osn_tsdf_cuda_stream_in(OsnTsdfCudaVolume* v, const void* host_buffer, int64_t size,
                                int32_t* skipped) {
    osn_b200::Volume* vol = osn_tsdf_b200_volume_of(v);
    return vol ? vol->stream_in(host_buffer, size, skipped) : 1;
}

}  // extern "C"
