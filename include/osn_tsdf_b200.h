/* osn_tsdf_b200: B200-native (sm_100a) hash-blocked TSDF volume behind the
 * reference's CUDA C ABI.
 *
 * The first block below is the reference's CUDA section of
 * cpp/include/osn_tsdf/c_api.h (lines 56-126), re-declared with identical
 * names, argument meanings and return codes, so a caller of the reference's
 * CUDA arm (A3) links against this library instead without a source change.
 * The CPU section of that header (c_api.h:14-46) is the reference's own CPU
 * arm and is not part of this library.
 *
 * Conventions (same as the reference):
 *   - positions are DEVICE pointers owned by the caller, 3 floats per point,
 *     world space; the volume owns every other device allocation;
 *   - calls are asynchronous on the volume's own stream; block_count,
 *     drop_count, extract_mesh and synchronize wait for it;
 *   - nothing throws across the boundary; one host thread per volume.
 *
 * The second block holds extensions with no counterpart in the reference;
 * each says what it adds.
 */
#ifndef OSN_TSDF_B200_H
#define OSN_TSDF_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct OsnTsdfCudaVolume OsnTsdfCudaVolume;

/* Device pointers and parameters describing a volume's storage.
 * Same 104-byte layout as the reference (c_api.h:61-78, size asserted at
 * cpp/src/c_api_cuda.cu:14): table slots are (int64 key, int32 block_idx,
 * int32 pad); tsdf/weight/r/g/b hold weighted SUMS, 512 floats per block at
 * block_idx * 512, voxel (lx,ly,lz) at (lz*8+ly)*8+lx. */
typedef struct {
    void* table;          /* hash_mask+1 live slots, then 2^20 scratch slots (key -2) */
    void* block_count;    /* int32 */
    void* drop_count;     /* uint64 */
    void* block_coord;    /* int32[3] per pool slot */
    void* tsdf;           /* float, weighted sum */
    void* weight;         /* float */
    void* r;
    void* g;
    void* b;
    uint32_t hash_mask;
    uint32_t scratch_base;  /* first scratch slot = hash_mask + 1 */
    int32_t pool_capacity;
    int32_t block_dim;
    float voxel_size_m;
    float trunc_m;
    float weight_cap;
} OsnTsdfDeviceView;

/* ---- reference CUDA section (cpp/include/osn_tsdf/c_api.h:80-126) ---- */

/* c_api.h:80. NULL on invalid parameters or device allocation failure.
 * trunc_m <= 0 selects 4 * voxel_size_m; weight_cap <= 0 disables capping.
 * The table has next_pow2(2 * pool) slots, as in the reference. */
OsnTsdfCudaVolume* osn_tsdf_cuda_create(float voxel_size_m, int32_t pool_capacity_blocks,
                                        float trunc_m, float weight_cap);
/* c_api.h:82 */
void osn_tsdf_cuda_destroy(OsnTsdfCudaVolume* v);
/* c_api.h:83. 1 when every device allocation succeeded. */
int32_t osn_tsdf_cuda_valid(const OsnTsdfCudaVolume* v);
/* c_api.h:86. Returns 0 on success, 1 on a NULL or invalid volume. */
int32_t osn_tsdf_cuda_device_view(const OsnTsdfCudaVolume* v, OsnTsdfDeviceView* out);

/* c_api.h:89-91. Allocate the blocks the batch's truncation bands touch.
 * Returns 0 (queued), 1 on bad arguments (NULL volume or positions, n <= 0),
 * 3 when the kernel launch failed. */
int32_t osn_tsdf_cuda_allocate_blocks(OsnTsdfCudaVolume* v, const float* d_positions,
                                      int32_t n_points, float cam_x, float cam_y, float cam_z,
                                      float radius_m);
/* c_api.h:92-94. Accumulate the batch into allocated blocks: unit weights,
 * grey colour (128), contributions applied as if in (point, band step) order
 * with the weight cap "accept while weight before < cap". Return codes as
 * allocate_blocks. */
int32_t osn_tsdf_cuda_update_voxels(OsnTsdfCudaVolume* v, const float* d_positions,
                                    int32_t n_points, float cam_x, float cam_y, float cam_z,
                                    float radius_m);
/* c_api.h:97-98. Marching-tetrahedra triangle soup into HOST buffers:
 * buffer_posnor holds vert_cap * 6 floats (position, face normal),
 * buffer_rgb vert_cap * 3 bytes or NULL. Returns the vertex count, or -1 if
 * vert_cap was too small or the arguments are invalid. */
int32_t osn_tsdf_cuda_extract_mesh(OsnTsdfCudaVolume* v, float* buffer_posnor, uint8_t* buffer_rgb,
                                   int32_t vert_cap, float min_weight, float iso);
/* c_api.h:106. Back to the just-created state without reallocating. Waits. */
int32_t osn_tsdf_cuda_reset(OsnTsdfCudaVolume* v);
/* c_api.h:110-112. MEASUREMENT: allocate, adding every compare-exchange
 * ATTEMPT to drop_count. Only meaningful on a pool that drops nothing. */
int32_t osn_tsdf_cuda_allocate_counting_cas(OsnTsdfCudaVolume* v, const float* d_positions,
                                            int32_t n_points, float cam_x, float cam_y,
                                            float cam_z, float radius_m);
/* c_api.h:115-117. MEASUREMENT: probe and read, never insert. */
int32_t osn_tsdf_cuda_allocate_no_cas(OsnTsdfCudaVolume* v, const float* d_positions,
                                      int32_t n_points, float cam_x, float cam_y, float cam_z,
                                      float radius_m);
/* c_api.h:120-122. MEASUREMENT: block index = hash slot, hash masked to the
 * pool (which must be a power of two; 2 otherwise); no publication wait. */
int32_t osn_tsdf_cuda_allocate_slot_index(OsnTsdfCudaVolume* v, const float* d_positions,
                                          int32_t n_points, float cam_x, float cam_y, float cam_z,
                                          float radius_m);
/* c_api.h:124-126. Waiting reads of the counters; 0 for a NULL volume. */
int32_t osn_tsdf_cuda_block_count(const OsnTsdfCudaVolume* v);
uint64_t osn_tsdf_cuda_drop_count(const OsnTsdfCudaVolume* v);
void osn_tsdf_cuda_synchronize(const OsnTsdfCudaVolume* v);

/* ---- extensions (no counterpart in the reference) ---------------------- */

/* Voxel storage modes for create_ex.
 *   FP32      the reference's layout (above): float weighted sums in tsdf,
 *             weight, r, g, b; 20 bytes per voxel.
 *   FP16_U16  the MEAN normalised TSDF as IEEE half in tsdf and the weight
 *             as uint16 in weight (4 bytes per voxel); r, g, b are NULL in
 *             the device view (through this ABI every contribution is grey,
 *             so the mean colour of an observed voxel is 128). The running
 *             average (mean * w + batch sum) / (w + accepted) is formed in
 *             FP32 and rounded to half once per batch. Weights saturate at
 *             65535, which is also the cap when weight_cap <= 0 or > 65535.
 *   FP64      the on-device FP64 oracle: double TSDF sums in tsdf, float
 *             weights, no colour arrays; the signed distance of every band
 *             sample is evaluated in double (the samples, blocks and
 *             accepted contributions are those of FP32).
 * Hashing, block coordinates and allocation are identical in every mode. */
#define OSN_TSDF_STORAGE_FP32 0
#define OSN_TSDF_STORAGE_FP16_U16 1
#define OSN_TSDF_STORAGE_FP64 2

/* create with an explicit table size and a storage mode. The reference
 * always sizes the table to next_pow2(2 * pool), which caps its load factor
 * below 0.5; hash_slots (a power of two >= 2, or 0 for the reference sizing)
 * reaches the 0.75 and 0.9 load factors of the irregularity sweep. storage
 * is one of OSN_TSDF_STORAGE_*; NULL for any other value. */
OsnTsdfCudaVolume* osn_tsdf_cuda_create_ex(float voxel_size_m, int32_t pool_capacity_blocks,
                                           float trunc_m, float weight_cap, uint32_t hash_slots,
                                           int32_t storage);

/* Table layouts for create_layout.
 *   POOL        the reference's: a block's pool index comes from a counter
 *               after its key is claimed, published into the slot once its
 *               coordinate is written; a thread that meets a claimed key
 *               waits for the index (bounded).
 *   SLOT_INDEX  the pool is the table: a block's pool index is its table
 *               slot, so a claim publishes everything at once and a thread
 *               that meets the key returns the slot without waiting (the
 *               layout of the reference's slot-index measurement variant,
 *               cpp/src/volume_cuda.cu:194-257, as a production layout). The
 *               pool capacity becomes the table size (hash_slots, or
 *               next_pow2(2 * pool)): about twice the voxel memory. In the
 *               device view block_coord, tsdf, weight, ... are indexed by
 *               slot (only occupied slots -- key >= 0 -- are blocks), not
 *               dense 0..block_count-1; snapshot/restore and chunk eviction
 *               need the POOL layout (they return -1 / 1 here). Results
 *               (blocks, voxels, meshes) are those of the POOL layout. */
#define OSN_TSDF_LAYOUT_POOL 0
#define OSN_TSDF_LAYOUT_SLOT_INDEX 1

/* create_ex with a table layout (OSN_TSDF_LAYOUT_*). No counterpart in the
 * reference. NULL for an unknown layout. */
OsnTsdfCudaVolume* osn_tsdf_cuda_create_layout(float voxel_size_m, int32_t pool_capacity_blocks,
                                               float trunc_m, float weight_cap, uint32_t hash_slots,
                                               int32_t storage, int32_t layout);

/* The volume's table layout, or -1 for a bad handle. */
int32_t osn_tsdf_cuda_layout(const OsnTsdfCudaVolume* v);

/* allocate_blocks then update_voxels on the same points, as the reference's
 * CPU integrate (cpp/src/volume.cpp:301-304), in one pass: blocks are
 * allocated and contributions counted by the same walk. Results are those of
 * the two separate calls. Return codes as allocate_blocks. */
int32_t osn_tsdf_cuda_integrate(OsnTsdfCudaVolume* v, const float* d_positions, int32_t n_points,
                                float cam_x, float cam_y, float cam_z, float radius_m);

/* integrate of several consecutive frames in one call (no counterpart in the
 * reference). Frame k's points are d_positions[frame_begin[k] ..
 * frame_begin[k + 1]) (a DEVICE xyz float array holding all frames' points
 * back to back), seen from the camera at cams_xyz[3k .. 3k + 2];
 * frame_begin (n_frames + 1 entries, frame_begin[0] = 0, non-decreasing) and
 * cams_xyz (3 * n_frames) are HOST arrays, read during the call. At most
 * OSN_TSDF_MAX_FRAMES frames per call.
 * The cap keeps the same contributions as n_frames successive integrate
 * calls (accept while the weight before a contribution is below the cap, in
 * frame, point, step order), so the block set, the weights and the colour
 * sums are identical to theirs; a voxel's stored TSDF takes one rounding per
 * call instead of one per frame. The per-call costs (kernel boundaries, the
 * update tail's pass over the touched blocks, which consecutive frames
 * largely share) are paid once for all the call's frames. FP32 and FP16
 * storage; 2 for the FP64 oracle. Other return codes as integrate. */
#define OSN_TSDF_MAX_FRAMES 32
int32_t osn_tsdf_cuda_integrate_frames(OsnTsdfCudaVolume* v, const float* d_positions,
                                       const int32_t* frame_begin, const float* cams_xyz,
                                       int32_t n_frames, float radius_m);

/* integrate from a depth image, unprojected inside the band walk: pixel
 * (u, v) with depth z (metres along the optical axis, d_depth is a DEVICE
 * float array of height * width in raster order) becomes the world point
 * R [(u - cx) z / fx, (v - cy) z / fy, z] + t in FP64, rounded to float, as
 * crates/tartanair/src/lib.rs:307-340 does on the host; pixels whose depth is
 * non-finite, <= 0 or beyond max_range_m (when > 0) have no point. R (row-
 * major 3x3) and t are the camera-to-world pose (HOST arrays); the camera
 * origin of the walk is (float)t. Results equal integrate() of the host-
 * backprojected valid points in raster order. 4 bytes per pixel cross the
 * bus instead of 12 per point. Return codes as integrate. */
int32_t osn_tsdf_cuda_integrate_depth(OsnTsdfCudaVolume* v, const float* d_depth, int32_t width,
                                      int32_t height, double fx, double fy, double cx, double cy,
                                      const double* cam_to_world_R, const double* cam_to_world_t,
                                      float max_range_m);

/* integrate_depth of several depth images of the same size in one call (no
 * counterpart in the reference): image k occupies d_depth[k * height * width
 * .. (k + 1) * height * width) and is seen from the camera-to-world pose
 * cam_to_world_R[9k .. 9k + 8] (row-major), cam_to_world_t[3k .. 3k + 2]
 * (HOST arrays, read during the call); one set of intrinsics. Results as
 * integrate_frames of the images' backprojected points: the same blocks,
 * weights and colour sums as one integrate_depth call per image, each
 * voxel's TSDF rounded once per call. At most OSN_TSDF_MAX_DEPTH_FRAMES
 * images; FP32 and FP16 storage (2 for the FP64 oracle); other return codes
 * as integrate. */
#define OSN_TSDF_MAX_DEPTH_FRAMES 16
int32_t osn_tsdf_cuda_integrate_depth_frames(OsnTsdfCudaVolume* v, const float* d_depth, int32_t width,
                                             int32_t height, int32_t n_frames, double fx, double fy,
                                             double cx, double cy, const double* cam_to_world_R,
                                             const double* cam_to_world_t, float max_range_m);

/* Extraction into DEVICE buffers (same layout as extract_mesh), skipping the
 * host copy. Returns the vertex count or -1 (overflow / bad arguments).
 * Waits for the count only. */
int32_t osn_tsdf_cuda_extract_mesh_device(OsnTsdfCudaVolume* v, float* d_posnor, uint8_t* d_rgb,
                                          int32_t vert_cap, float min_weight, float iso);

/* Extract the mesh and write it as a raw "OSN1" file (the reference's geometry
 * dump, cpp/bench/bench_arms.cu:506-523; no counterpart in its C ABI):
 * uint32 magic 0x314e534f (the bytes "OSN1"), uint32 vertex count, then the
 * vertices' interleaved position and normal floats (6 per vertex) exactly as
 * extraction produced them, little-endian. Returns the vertex count, -1 on bad
 * arguments or when vert_cap is too small (nothing written), -2 on a file
 * error. Waits. */
int32_t osn_tsdf_cuda_write_mesh_osn1(OsnTsdfCudaVolume* v, const char* path, int32_t vert_cap,
                                      float min_weight, float iso);

/* Snapshot and restore through host memory (checkpoint a volume, or move an
 * idle session out of HBM and back). A snapshot holds the allocated blocks'
 * coordinates and voxel arrays (pool order) and the drop counter; the table
 * is rebuilt on restore, so slot positions may differ while every lookup,
 * update and extraction continues as on the original.
 * snapshot_bytes: bytes a snapshot needs now (waits), -1 on a bad volume.
 * snapshot: writes into host_buffer (capacity bytes); returns the bytes
 * written or -1 (too small, bad volume, CUDA error).
 * restore: replaces the volume's contents with a snapshot taken from a
 * volume with the same voxel size, truncation, weight cap and storage mode;
 * its pool and table must hold the snapshot's blocks. 0 ok, 1 bad snapshot or
 * arguments, 3 CUDA error. All three wait for the volume's stream. */
int64_t osn_tsdf_cuda_snapshot_bytes(OsnTsdfCudaVolume* v);
int64_t osn_tsdf_cuda_snapshot(OsnTsdfCudaVolume* v, void* host_buffer, int64_t capacity);
int32_t osn_tsdf_cuda_restore(OsnTsdfCudaVolume* v, const void* host_buffer, int64_t size);

/* Streaming by chunk id. No counterpart in the reference, which declares a
 * chunk id on every point batch (cpp/include/osn_tsdf/types.hpp:127) but
 * never reads it. Every block carries the chunk id of the last call that
 * allocated or updated it; set_chunk sets the id later calls give (0 at
 * creation; the C++ class takes PointBatch::chunk_id).
 * evict_chunks moves every block whose chunk id lies in [lo, hi] into a host
 * pack (header, coordinates, chunk ids, voxel arrays; evict_chunks_bytes
 * gives its size) and removes it from the volume: the remaining blocks move
 * to the front of the pool in their old order (new pool indices, same
 * contents), the freed pool entries are zeroed and the table is rebuilt, so
 * a scene larger than the pool keeps integrating. Returns the pack's bytes,
 * or -1 (bad range, buffer too small, CUDA error).
 * stream_in inserts a pack's blocks again with their voxels and chunk ids;
 * blocks present again in the volume are left as they are and counted in
 * *skipped. Returns 0, 1 on a bad pack (another volume's voxel size,
 * truncation, cap or storage), 2 when the pool filled (some blocks not
 * restored), 3 on a CUDA error. All wait for the volume's stream. */
int32_t osn_tsdf_cuda_set_chunk(OsnTsdfCudaVolume* v, int32_t chunk_id);
int64_t osn_tsdf_cuda_evict_chunks_bytes(OsnTsdfCudaVolume* v, int32_t lo, int32_t hi);
int64_t osn_tsdf_cuda_evict_chunks(OsnTsdfCudaVolume* v, int32_t lo, int32_t hi, void* host_buffer,
                                   int64_t capacity);
int32_t osn_tsdf_cuda_stream_in(OsnTsdfCudaVolume* v, const void* host_buffer, int64_t size,
                                int32_t* skipped);

/* Device error word, after waiting for the stream: 0 when every bounded
 * wait in the kernels finished in time; bit 0 = a publication wait gave up,
 * bit 1 = an update batch exceeded its scratch. */
uint32_t osn_tsdf_cuda_status(const OsnTsdfCudaVolume* v);

/* Bound on each device-side wait of this volume's later calls (a thread
 * waiting for another to publish the pool index of a block it inserted), in
 * iterations of ~100 ns, 1 .. 2^20 (the default, ~0.1 s). A wait that runs
 * out drops its samples and sets bit 0 of the status word. No counterpart in
 * the reference, whose waits are unbounded (cpp/src/volume_cuda.cu:71-72).
 * Returns 0, or 1 on a bad volume or an out-of-range bound. */
int32_t osn_tsdf_cuda_set_spin_limit(OsnTsdfCudaVolume* v, int32_t iterations);

/* Measured L2 ceiling of the current GPU, for roofline fractions of kernels
 * whose working set stays in L2. No counterpart in the reference. One probe
 * kernel over a fresh device buffer of `bytes` (1 MiB .. 2 GiB; L2-resident
 * well below 126 MB), `iters` operations per thread on a persistent grid of
 * 8 x 256-thread CTAs per SM, timed after a warm-up launch. kind 0:
 * red.add.u64 to pseudo-random words (G ops/s); 1: red.add.u32 (G ops/s);
 * 2: atomic add with return (G ops/s); 3: streamed 16-byte loads through L2
 * (GB/s); 4: pseudo-random 4-byte loads through L2 (G loads/s). Allocates and
 * frees its buffer and synchronises. Returns 0, 1 on bad arguments, 3 on a
 * CUDA error. */
int32_t osn_tsdf_cuda_l2_probe(int32_t kind, int64_t bytes, int32_t iters, double* result);

/* The volume's cudaStream_t, for callers that order their own work after it.
 * In pipelined mode (below) the last calls' update tails may still run on an
 * internal stream: call osn_tsdf_cuda_join first to order work after them. */
void* osn_tsdf_cuda_stream(const OsnTsdfCudaVolume* v);

/* Pipelined updates. When enabled, an integrate/update call's band walk is
 * queued on the volume's stream as usual but its update tail (finish,
 * group, select) runs on an internal stream, so the next call's walk
 * overlaps this call's tail; the per-call scratch alternates between two sets
 * (twice the per-voxel batch state: +12 bytes per voxel). Results are
 * identical. The positions (or depth image) of a call may be reused once the
 * volume's stream has passed the call, as in serial mode; every waiting
 * reader of results (counters, extraction, reset, snapshot, status,
 * synchronize) first waits for the queued tails. Work a caller orders on the
 * volume's stream sees the tails only after osn_tsdf_cuda_join. Returns 0,
 * 1 on a bad volume, 2 for the FP64 oracle storage (not supported: its tail
 * re-reads the points), 3 on an allocation failure (mode unchanged). Waits. */
int32_t osn_tsdf_cuda_set_pipelined(OsnTsdfCudaVolume* v, int32_t enabled);
/* Make the volume's stream wait for every queued update tail (pipelined
 * mode; a no-op otherwise). 0 ok, 1 bad volume. */
int32_t osn_tsdf_cuda_join(OsnTsdfCudaVolume* v);

/* The volume's OSN_TSDF_STORAGE_* mode, or -1 for a NULL or invalid volume. */
int32_t osn_tsdf_cuda_storage(const OsnTsdfCudaVolume* v);

/* MEASUREMENT: one allocate pass that also records, per warp-leader probe
 * sequence, how many slots it visited: hist[min(steps, n_bins-1)] += 1.
 * hist is a HOST array of n_bins uint64 (overwritten). Also allocates. */
int32_t osn_tsdf_cuda_allocate_probe_histogram(OsnTsdfCudaVolume* v, const float* d_positions,
                                               int32_t n_points, float cam_x, float cam_y,
                                               float cam_z, float radius_m, uint64_t* hist,
                                               int32_t n_bins);

/* Per-stage statistics of the last update_voxels call (waits):
 * out[0] voxels whose sums were rewritten, out[1] band records counted
 * (contributions not already excluded by a full voxel),
 * out[2] blocks touched by a band sample,
 * out[3] voxels that crossed the cap inside the batch (ordered selection). */
int32_t osn_tsdf_cuda_last_update_stats(const OsnTsdfCudaVolume* v, int64_t* out4);

/* Largest batch of one update_voxels_noalloc call, counted in records:
 * n_points * (2 * steps + 1) with steps = max(1, ceil(trunc / voxel)). */
#define OSN_TSDF_NOALLOC_MAX_RECORDS (1 << 21)

/* update_voxels that allocates no device memory. No counterpart in the
 * reference. update_voxels may grow its scratch with cudaMalloc (after
 * waiting for the stream) when a batch is larger than any before it; callers
 * that cannot allow that -- serving loops that admit work against a fixed
 * device-memory budget, latency-critical threads that cannot absorb the
 * device-wide synchronisation cudaMalloc/cudaFree imply -- call this
 * instead. Same results as update_voxels.
 * Its scratch is one fixed 36 MiB array inside the library, held on every
 * GPU where the library's code is loaded until the process exits, and shared
 * by all calls: calls whose work overlaps on the GPU race and must be
 * serialised. The calling thread's current device must be the volume's. The
 * first call on a device resolves the array's address (a set-up step) and
 * should come before any stream capture. last_update_stats afterwards reports
 * this call's counters. Returns 0 (queued), 1 on bad arguments (including a
 * current device other than the volume's), 3 on a set-up or launch failure,
 * 4 when n_points * (2*steps+1) exceeds OSN_TSDF_NOALLOC_MAX_RECORDS
 * (nothing is queued; split the batch). */
int32_t osn_tsdf_cuda_update_voxels_noalloc(OsnTsdfCudaVolume* v, const float* d_positions,
                                            int32_t n_points, float cam_x, float cam_y,
                                            float cam_z, float radius_m);

/* ---- batched integrate (no counterpart in the reference) ---------------
 *
 * Many independent volumes ("scenes", each with its own table, pool, voxel
 * size and truncation, one storage mode for all) integrate one frame each
 * per step in one chain of work-queued passes on the batch's stream: a
 * table of the step's scenes is uploaded, then one pass of each kernel
 * (band walk, finish, group, select) covers every scene, its CTAs
 * taking (scene, tile range) work items from atomic queues. Results are
 * bit-identical to integrating each scene alone with osn_tsdf_cuda_integrate.
 *
 * A volume attached to a batch is integrated only through it; before any
 * other call on the volume (counters, extraction, reset, device view),
 * call osn_tsdf_batch_synchronize. At most 64 scenes per batch. */
typedef struct OsnTsdfBatch OsnTsdfBatch;

/* NULL on max_scenes outside [1, 64] or device allocation failure. */
OsnTsdfBatch* osn_tsdf_batch_create(int32_t max_scenes);
void osn_tsdf_batch_destroy(OsnTsdfBatch* b);
/* Attach a volume that will receive frames of up to max_points points (its
 * scratch is sized now; no allocation happens in a step). Waits for the
 * volume's stream. Returns the scene index, or -1 (full, NULL, already
 * attached, storage mode differs from the other scenes, batch too large). */
int32_t osn_tsdf_batch_add(OsnTsdfBatch* b, OsnTsdfCudaVolume* v, int32_t max_points);
/* Detach a scene once the steps queued so far have run (waits for the batch
 * stream); the volume stays valid and its slot is reused by the next add.
 * 0 ok, 1 no such scene, 3 CUDA error. */
int32_t osn_tsdf_batch_remove(OsnTsdfBatch* b, int32_t scene);
/* The next step's frame of one scene: device positions (3 floats per point,
 * kept alive until the step has run), camera origin, far cutoff. Scenes
 * without a frame sit the step out. 0 ok, 1 bad arguments. */
int32_t osn_tsdf_batch_set_frame(OsnTsdfBatch* b, int32_t scene, const float* d_positions,
                                 int32_t n_points, float cam_x, float cam_y, float cam_z,
                                 float radius_m);
/* Queue one step (asynchronous on the batch's stream). 0 ok, 1 bad batch,
 * 3 launch failure. */
int32_t osn_tsdf_batch_step(OsnTsdfBatch* b);
int32_t osn_tsdf_batch_synchronize(OsnTsdfBatch* b);
/* Replay the step's passes from a CUDA graph (captured on the second step
 * with the same scenes and shape). */
int32_t osn_tsdf_batch_set_graph(OsnTsdfBatch* b, int32_t enabled);
/* Run the next 16 * steps_per_shape steps with each candidate shape
 * (band tiles per work item 1/2/4/8, warp-grouped or per-lane block
 * resolution, one or two blocks per finish item), then keep the fastest
 * median. Shapes change speed only, never results. */
int32_t osn_tsdf_batch_autotune(OsnTsdfBatch* b, int32_t steps_per_shape);
/* Fix the shape: tiles_per_item in [1, 8], probe 0 (warp) or 1 (lane),
 * finish_pair 0 or 1. */
int32_t osn_tsdf_batch_set_shape(OsnTsdfBatch* b, int32_t tiles_per_item, int32_t probe,
                                 int32_t finish_pair);
/* Current shape into out3 (tiles_per_item, probe, finish_pair); returns 1
 * while tuning, 0 otherwise, -1 on bad arguments. */
int32_t osn_tsdf_batch_shape(OsnTsdfBatch* b, int32_t* out3);
/* Autotuner record (waits): median step ms of each candidate (-1 if not run)
 * and its shape (3 ints each); returns the number of candidates written. */
int32_t osn_tsdf_batch_tune_results(OsnTsdfBatch* b, double* ms, int32_t* shapes, int32_t n_max);
/* Status words of the batch and its volumes, OR-ed (waits). */
uint32_t osn_tsdf_batch_status(OsnTsdfBatch* b);
void* osn_tsdf_batch_stream(OsnTsdfBatch* b);
int32_t osn_tsdf_batch_size(OsnTsdfBatch* b);

/* Kernel timing. When enabled, every kernel launch of the volume is
 * bracketed by CUDA events on the volume's stream; kernel_times reads (and
 * waits for) the accumulated per-kernel milliseconds and launch counts.
 * Kernel ids: 0 allocate, 1 band (count-and-sum walk; allocates too in
 * integrate), 2 finish (per touched block), 3 group (records of voxels that
 * cross the cap, grouped per voxel), 4 select (ordered cap selection and
 * update of those voxels), 5 extract, 6 reset; id 7 is kept for the
 * numbering and records no launches.
 * Returns the number of ids written. */
int32_t osn_tsdf_cuda_set_timing(OsnTsdfCudaVolume* v, int32_t enabled);
int32_t osn_tsdf_cuda_kernel_times(OsnTsdfCudaVolume* v, double* ms, int64_t* launches,
                                   int32_t n_ids);

#ifdef __cplusplus
}
#endif

#endif /* OSN_TSDF_B200_H */
