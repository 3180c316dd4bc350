/* CPU oracle for the hash-blocked TSDF integrate path.
 *
 * TEST INFRASTRUCTURE ONLY. This is a single-threaded C restatement of the
 * reference's CPU arm (cpp/src/volume.cpp, cpp/src/marching_tets.cpp). It is
 * the checker the parity tests, the smoke check and the CPU-baseline leg of
 * bench.py compare the CUDA library against; no product code path links it.
 *
 * Single-threaded on purpose: the reference's weight cap is a plain read
 * before the atomic adds (cpp/src/volume.cpp:283-291), so with several
 * threads the set of capped contributions depends on scheduling. Run in
 * point order then band-step order, it realises one well-defined semantics:
 * "apply contributions in (point index, step) order, accept while the voxel's
 * weight before the contribution is below the cap".
 *
 * Pinned against the reference itself (oracle/_ref, built from the reference
 * sources by oracle/Makefile) by tests/test_oracle_pin.py: identical block
 * sets, bit-identical voxel arrays and bit-identical meshes.
 */
#ifndef TSDF_ORACLE_H
#define TSDF_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct OracleVolume OracleVolume;

/* hash_slots == 0 selects the reference sizing next_pow2(2 * pool)
 * (cpp/src/volume.cpp:48); otherwise it must be a power of two. */
OracleVolume* oracle_create(float voxel_size_m, int32_t pool_capacity_blocks, float trunc_m,
                            float weight_cap, uint32_t hash_slots);
void oracle_destroy(OracleVolume* v);

int32_t oracle_allocate_blocks(OracleVolume* v, const float* positions, int32_t n,
                               float cam_x, float cam_y, float cam_z, float radius_m);
int32_t oracle_update_voxels(OracleVolume* v, const float* positions, const uint8_t* colors,
                             const float* weights, int32_t n, float cam_x, float cam_y,
                             float cam_z, float radius_m);
int32_t oracle_integrate(OracleVolume* v, const float* positions, const uint8_t* colors,
                         const float* weights, int32_t n, float cam_x, float cam_y, float cam_z,
                         float radius_m);
int32_t oracle_extract_mesh(const OracleVolume* v, float* posnor, uint8_t* rgb, int32_t vert_cap,
                            float min_weight, float iso);

int32_t oracle_block_count(const OracleVolume* v);
uint64_t oracle_drop_count(const OracleVolume* v);
uint32_t oracle_hash_mask(const OracleVolume* v);
float oracle_trunc(const OracleVolume* v);

/* Block coordinates in pool order: out holds 3 * block_count int32. */
int32_t oracle_block_coords(const OracleVolume* v, int32_t* out);
/* Voxel arrays (weighted sums) in pool order, block_count * 512 floats each.
 * Any output pointer may be NULL. */
int32_t oracle_voxels(const OracleVolume* v, float* tsdf, float* weight, float* r, float* g,
                      float* b);
/* Hash table contents: keys (int64) and block indices (int32), hash_mask+1 each. */
int32_t oracle_table(const OracleVolume* v, int64_t* keys, int32_t* block_idx);

/* The reference's analytic test scenes (cpp/tests/analytic_scenes.hpp:19-46),
 * float for float, so the known answers of its tests apply unchanged.
 * sphere: out holds 3 * n_theta * n_phi floats; plane: 3 * n * n floats. */
void oracle_sphere_points(float radius, int32_t n_theta, int32_t n_phi, float* out);
void oracle_plane_points(float z0, float half_extent, int32_t n, float* out);

#ifdef __cplusplus
}
#endif

#endif
