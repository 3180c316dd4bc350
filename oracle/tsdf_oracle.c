/* CPU oracle for the hash-blocked TSDF integrate path -- TEST INFRASTRUCTURE.
 *
 * A single-threaded C restatement of the reference's CPU arm. Each function
 * names the reference lines it follows. Built by oracle/Makefile with
 * -ffp-contract=off on baseline x86-64 (SSE, no FMA), which is how the
 * reference's CPU arm is compiled, so every float operation rounds exactly
 * as the reference's does.
 *
 * Only tests/, the smoke check and the CPU-baseline leg of bench.py load this
 * library, and only as the checker.
 */
#include "tsdf_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

enum { kBlockDim = 8, kBlockVoxels = 512 };
static const int64_t kEmptyKey = -1;
static const int64_t kCoordBias = (int64_t)1 << 20;
static const int kCoordBits = 21;

typedef struct {
    int64_t key;
    int32_t block_idx;
    int32_t pad;
} Entry;

struct OracleVolume {
    float voxel;
    int32_t pool;
    float trunc;
    float cap;
    uint32_t mask;
    Entry* table;
    int32_t* coord; /* 3 per pool slot */
    float *tsdf, *weight, *r, *g, *b;
    int32_t block_count;
    uint64_t drop_count;
};

/* types.hpp:64-69 */
static int64_t pack_coord(int32_t x, int32_t y, int32_t z) {
    const int64_t bx = (int64_t)x + kCoordBias;
    const int64_t by = (int64_t)y + kCoordBias;
    const int64_t bz = (int64_t)z + kCoordBias;
    return (bx << (2 * kCoordBits)) | (by << kCoordBits) | bz;
}

/* types.hpp:150-155 (Teschner et al. multiply-xor spatial hash) */
static uint32_t hash_block(int32_t x, int32_t y, int32_t z, uint32_t mask) {
    const uint32_t h = (uint32_t)x * 73856093u ^ (uint32_t)y * 19349663u ^ (uint32_t)z * 83492791u;
    return h & mask;
}

/* types.hpp:162-165 */
static int32_t floor_div(int32_t a, int32_t b) {
    const int32_t q = a / b;
    return (a % b != 0 && ((a < 0) != (b < 0))) ? q - 1 : q;
}

/* volume.cpp:14-19 */
static uint32_t next_pow2(uint32_t v) {
    if (v < 2) return 2;
    --v;
    v |= v >> 1; v |= v >> 2; v |= v >> 4; v |= v >> 8; v |= v >> 16;
    return v + 1;
}

/* types.hpp:104-106 */
static float config_trunc(float trunc_m, float voxel) { return trunc_m > 0.0f ? trunc_m : 4.0f * voxel; }

/* volume.cpp:41-61 */
OracleVolume* oracle_create(float voxel_size_m, int32_t pool_capacity_blocks, float trunc_m,
                            float weight_cap, uint32_t hash_slots) {
    if (!(voxel_size_m > 0.0f) || pool_capacity_blocks <= 0) return NULL;
    if (hash_slots != 0 && (hash_slots & (hash_slots - 1)) != 0) return NULL;
    OracleVolume* v = (OracleVolume*)calloc(1, sizeof(OracleVolume));
    if (!v) return NULL;
    v->voxel = voxel_size_m;
    v->pool = pool_capacity_blocks;
    v->trunc = config_trunc(trunc_m, voxel_size_m);
    v->cap = weight_cap;
    const uint32_t size = hash_slots ? hash_slots : next_pow2((uint32_t)pool_capacity_blocks * 2u);
    v->mask = size - 1;
    v->table = (Entry*)malloc((size_t)size * sizeof(Entry));
    const size_t n = (size_t)pool_capacity_blocks * kBlockVoxels;
    v->coord = (int32_t*)calloc((size_t)pool_capacity_blocks * 3, sizeof(int32_t));
    v->tsdf = (float*)calloc(n, sizeof(float));
    v->weight = (float*)calloc(n, sizeof(float));
    v->r = (float*)calloc(n, sizeof(float));
    v->g = (float*)calloc(n, sizeof(float));
    v->b = (float*)calloc(n, sizeof(float));
    if (!v->table || !v->coord || !v->tsdf || !v->weight || !v->r || !v->g || !v->b) {
        oracle_destroy(v);
        return NULL;
    }
    for (uint32_t i = 0; i < size; ++i) {
        v->table[i].key = kEmptyKey;
        v->table[i].block_idx = -1;
        v->table[i].pad = 0;
    }
    return v;
}

void oracle_destroy(OracleVolume* v) {
    if (!v) return;
    free(v->table);
    free(v->coord);
    free(v->tsdf);
    free(v->weight);
    free(v->r);
    free(v->g);
    free(v->b);
    free(v);
}

/* volume.cpp:71-92 (single-threaded: an index is always published) */
static int32_t find_block(const OracleVolume* v, int32_t bx, int32_t by, int32_t bz) {
    const int64_t want = pack_coord(bx, by, bz);
    const uint32_t slot = hash_block(bx, by, bz, v->mask);
    const uint32_t size = v->mask + 1;
    for (uint32_t probe = 0; probe < size; ++probe) {
        const Entry* e = &v->table[(slot + probe) & v->mask];
        if (e->key == kEmptyKey) return -1;
        if (e->key == want) return e->block_idx;
    }
    return -1;
}

/* volume.cpp:94-145 */
static int32_t find_or_insert_block(OracleVolume* v, int32_t bx, int32_t by, int32_t bz) {
    const int64_t want = pack_coord(bx, by, bz);
    const uint32_t slot = hash_block(bx, by, bz, v->mask);
    const uint32_t size = v->mask + 1;
    for (uint32_t probe = 0; probe < size; ++probe) {
        Entry* e = &v->table[(slot + probe) & v->mask];
        if (e->key == want) return e->block_idx;
        if (e->key == kEmptyKey) {
            const int32_t idx = v->block_count++;
            if (idx >= v->pool) {
                /* Pool exhausted: release the slot and count the drop. */
                v->block_count--;
                v->drop_count++;
                return -1;
            }
            e->key = want;
            v->coord[(size_t)idx * 3 + 0] = bx;
            v->coord[(size_t)idx * 3 + 1] = by;
            v->coord[(size_t)idx * 3 + 2] = bz;
            e->block_idx = idx;
            return idx;
        }
    }
    v->drop_count++;
    return -1;
}

/* Ray set-up shared by both passes: volume.cpp:154-166 and :209-220.
 * Returns 0 when the point is gated out. */
static int ray_setup(const float* positions, int32_t i, const float cam[3], float radius_sq,
                     float* px, float* py, float* pz, float* dist, float* ux, float* uy,
                     float* uz) {
    *px = positions[(size_t)i * 3 + 0];
    *py = positions[(size_t)i * 3 + 1];
    *pz = positions[(size_t)i * 3 + 2];
    const float dx = *px - cam[0];
    const float dy = *py - cam[1];
    const float dz = *pz - cam[2];
    const float d2 = dx * dx + dy * dy + dz * dz;
    if (radius_sq > 0.0f && d2 > radius_sq) return 0;
    *dist = sqrtf(d2);
    if (!(*dist > 1e-6f)) return 0;
    *ux = dx / *dist;
    *uy = dy / *dist;
    *uz = dz / *dist;
    return 1;
}

/* volume.cpp:147-198 */
int32_t oracle_allocate_blocks(OracleVolume* v, const float* positions, int32_t n, float cam_x,
                               float cam_y, float cam_z, float radius_m) {
    if (!v || !positions || n <= 0) return 1;
    const float cam[3] = {cam_x, cam_y, cam_z};
    const float inv_voxel = 1.0f / v->voxel;
    const float trunc = v->trunc;
    const float radius_sq = radius_m > 0.0f ? radius_m * radius_m : 0.0f;
    const float vs = v->voxel;
    for (int32_t i = 0; i < n; ++i) {
        float px, py, pz, dist, ux, uy, uz;
        if (!ray_setup(positions, i, cam, radius_sq, &px, &py, &pz, &dist, &ux, &uy, &uz)) continue;
        int32_t steps = (int32_t)ceilf(trunc * inv_voxel);
        if (steps < 1) steps = 1;
        for (int32_t s = -steps; s <= steps; ++s) {
            const float t = (float)s * vs;
            const int32_t vx = (int32_t)floorf((px + ux * t) * inv_voxel);
            const int32_t vy = (int32_t)floorf((py + uy * t) * inv_voxel);
            const int32_t vz = (int32_t)floorf((pz + uz * t) * inv_voxel);
            const float cx = ((float)vx + 0.5f) * vs;
            const float cy = ((float)vy + 0.5f) * vs;
            const float cz = ((float)vz + 0.5f) * vs;
            const float ex = cx - cam[0];
            const float ey = cy - cam[1];
            const float ez = cz - cam[2];
            if (dist - sqrtf(ex * ex + ey * ey + ez * ez) < -trunc) continue;
            find_or_insert_block(v, floor_div(vx, kBlockDim), floor_div(vy, kBlockDim),
                                 floor_div(vz, kBlockDim));
        }
    }
    return 0;
}

/* volume.cpp:200-299 */
int32_t oracle_update_voxels(OracleVolume* v, const float* positions, const uint8_t* colors,
                             const float* weights, int32_t n, float cam_x, float cam_y,
                             float cam_z, float radius_m) {
    if (!v || !positions || n <= 0) return 1;
    const float cam[3] = {cam_x, cam_y, cam_z};
    const float inv_voxel = 1.0f / v->voxel;
    const float trunc = v->trunc;
    const float inv_trunc = 1.0f / trunc;
    const float radius_sq = radius_m > 0.0f ? radius_m * radius_m : 0.0f;
    const float wcap = v->cap;
    const float vs = v->voxel;
    for (int32_t i = 0; i < n; ++i) {
        float px, py, pz, dist, ux, uy, uz;
        if (!ray_setup(positions, i, cam, radius_sq, &px, &py, &pz, &dist, &ux, &uy, &uz)) continue;
        const float w_in = weights ? weights[i] : 1.0f;
        float cr = 128.0f, cg = 128.0f, cb = 128.0f;
        if (colors) {
            cr = (float)colors[(size_t)i * 3 + 0];
            cg = (float)colors[(size_t)i * 3 + 1];
            cb = (float)colors[(size_t)i * 3 + 2];
        }
        int32_t steps = (int32_t)ceilf(trunc * inv_voxel);
        if (steps < 1) steps = 1;
        for (int32_t s = -steps; s <= steps; ++s) {
            const float t = (float)s * vs;
            const float sx = px + ux * t;
            const float sy = py + uy * t;
            const float sz = pz + uz * t;
            const int32_t vx = (int32_t)floorf(sx * inv_voxel);
            const int32_t vy = (int32_t)floorf(sy * inv_voxel);
            const int32_t vz = (int32_t)floorf(sz * inv_voxel);
            const int32_t bx = floor_div(vx, kBlockDim);
            const int32_t by = floor_div(vy, kBlockDim);
            const int32_t bz = floor_div(vz, kBlockDim);
            const int32_t bi = find_block(v, bx, by, bz);
            if (bi < 0) continue;
            const float cx = ((float)vx + 0.5f) * vs;
            const float cy = ((float)vy + 0.5f) * vs;
            const float cz = ((float)vz + 0.5f) * vs;
            const float ddx = cx - cam[0];
            const float ddy = cy - cam[1];
            const float ddz = cz - cam[2];
            const float d_voxel = sqrtf(ddx * ddx + ddy * ddy + ddz * ddz);
            const float sdf = dist - d_voxel;
            if (sdf < -trunc) continue;
            float sdf_n = sdf * inv_trunc;
            if (sdf_n < -1.0f) sdf_n = -1.0f;
            if (sdf_n > 1.0f) sdf_n = 1.0f;
            const int32_t lx = vx - bx * kBlockDim;
            const int32_t ly = vy - by * kBlockDim;
            const int32_t lz = vz - bz * kBlockDim;
            const size_t idx = (size_t)bi * kBlockVoxels + (size_t)((lz * kBlockDim + ly) * kBlockDim + lx);
            if (wcap > 0.0f && v->weight[idx] >= wcap) continue;
            v->weight[idx] += w_in;
            v->tsdf[idx] += sdf_n * w_in;
            v->r[idx] += cr * w_in;
            v->g[idx] += cg * w_in;
            v->b[idx] += cb * w_in;
        }
    }
    return 0;
}

/* volume.cpp:301-304 */
int32_t oracle_integrate(OracleVolume* v, const float* positions, const uint8_t* colors,
                         const float* weights, int32_t n, float cam_x, float cam_y, float cam_z,
                         float radius_m) {
    const int32_t rc = oracle_allocate_blocks(v, positions, n, cam_x, cam_y, cam_z, radius_m);
    if (rc) return rc;
    return oracle_update_voxels(v, positions, colors, weights, n, cam_x, cam_y, cam_z, radius_m);
}

/* volume.cpp:306-329 */
static int sample(const OracleVolume* v, int32_t vx, int32_t vy, int32_t vz, float min_weight,
                  float* tsdf_out, float rgb_out[3]) {
    const int32_t bx = floor_div(vx, kBlockDim);
    const int32_t by = floor_div(vy, kBlockDim);
    const int32_t bz = floor_div(vz, kBlockDim);
    const int32_t bi = find_block(v, bx, by, bz);
    if (bi < 0) return 0;
    const int32_t lx = vx - bx * kBlockDim;
    const int32_t ly = vy - by * kBlockDim;
    const int32_t lz = vz - bz * kBlockDim;
    const size_t idx = (size_t)bi * kBlockVoxels + (size_t)((lz * kBlockDim + ly) * kBlockDim + lx);
    const float w = v->weight[idx];
    if (w < min_weight || w <= 0.0f) return 0;
    const float inv_w = 1.0f / w;
    *tsdf_out = v->tsdf[idx] * inv_w;
    rgb_out[0] = v->r[idx] * inv_w;
    rgb_out[1] = v->g[idx] * inv_w;
    rgb_out[2] = v->b[idx] * inv_w;
    return 1;
}

/* marching_tets.cpp:37-46: six tetrahedra around the 0-7 diagonal, corner offsets. */
static const int kTets[6][4] = {
    {0, 5, 1, 7}, {0, 1, 3, 7}, {0, 3, 2, 7}, {0, 6, 4, 7}, {0, 4, 5, 7}, {0, 2, 6, 7},
};
static const int kCorner[8][3] = {
    {0, 0, 0}, {1, 0, 0}, {0, 1, 0}, {1, 1, 0}, {0, 0, 1}, {1, 0, 1}, {0, 1, 1}, {1, 1, 1},
};

typedef struct {
    float p[3];
    float c[3];
} Vtx;

static float clampf(float x, float lo, float hi) { return x < lo ? lo : (hi < x ? hi : x); }

/* marching_tets.cpp:59-80: position-ordered interpolation. */
static Vtx interp(float iso, const float pa[3], const float pb[3], float va, float vb,
                  const float ca[3], const float cb[3]) {
    const int swap = (pb[0] < pa[0]) || (pb[0] == pa[0] && pb[1] < pa[1]) ||
                     (pb[0] == pa[0] && pb[1] == pa[1] && pb[2] < pa[2]);
    const float* p0 = swap ? pb : pa;
    const float* p1 = swap ? pa : pb;
    const float* c0 = swap ? cb : ca;
    const float* c1 = swap ? ca : cb;
    const float v0 = swap ? vb : va;
    const float v1 = swap ? va : vb;
    const float denom = v1 - v0;
    const float t = fabsf(denom) < 1e-12f ? 0.5f : (iso - v0) / denom;
    const float tc = clampf(t, 0.0f, 1.0f);
    Vtx out;
    for (int k = 0; k < 3; ++k) {
        out.p[k] = p0[k] + tc * (p1[k] - p0[k]);
        out.c[k] = c0[k] + tc * (c1[k] - c0[k]);
    }
    return out;
}

/* marching_tets.cpp:84-243, with one worker (block order, then lz, ly, lx). */
int32_t oracle_extract_mesh(const OracleVolume* v, float* posnor, uint8_t* rgb, int32_t vert_cap,
                            float min_weight, float iso) {
    if (!v || !posnor || vert_cap <= 0) return -1;
    const int32_t n_blocks = v->block_count;
    const float vs = v->voxel;
    int32_t n_written = 0;
    int overflow = 0;
    Vtx tri[6];
    for (int32_t bi = 0; bi < n_blocks; ++bi) {
        const int32_t bcx = v->coord[(size_t)bi * 3 + 0];
        const int32_t bcy = v->coord[(size_t)bi * 3 + 1];
        const int32_t bcz = v->coord[(size_t)bi * 3 + 2];
        for (int32_t lz = 0; lz < kBlockDim; ++lz)
            for (int32_t ly = 0; ly < kBlockDim; ++ly)
                for (int32_t lx = 0; lx < kBlockDim; ++lx) {
                    const int32_t vx = bcx * kBlockDim + lx;
                    const int32_t vy = bcy * kBlockDim + ly;
                    const int32_t vz = bcz * kBlockDim + lz;
                    float val[8], pos[8][3], col[8][3];
                    int ok = 1;
                    for (int c = 0; c < 8 && ok; ++c) {
                        float rgbv[3];
                        ok = sample(v, vx + kCorner[c][0], vy + kCorner[c][1], vz + kCorner[c][2],
                                    min_weight, &val[c], rgbv);
                        if (!ok) break;
                        pos[c][0] = ((float)(vx + kCorner[c][0]) + 0.5f) * vs;
                        pos[c][1] = ((float)(vy + kCorner[c][1]) + 0.5f) * vs;
                        pos[c][2] = ((float)(vz + kCorner[c][2]) + 0.5f) * vs;
                        col[c][0] = rgbv[0];
                        col[c][1] = rgbv[1];
                        col[c][2] = rgbv[2];
                    }
                    if (!ok) continue;
                    for (int k = 0; k < 6; ++k) {
                        const int i0 = kTets[k][0], i1 = kTets[k][1], i2 = kTets[k][2], i3 = kTets[k][3];
                        const int code = (val[i0] < iso ? 1 : 0) | (val[i1] < iso ? 2 : 0) |
                                         (val[i2] < iso ? 4 : 0) | (val[i3] < iso ? 8 : 0);
                        int a = -1, b = -1, c = -1, d = -1, quad = 0;
                        switch (code) {
                            case 0x01: case 0x0E: a = i0; b = i1; c = i2; d = i3; break;
                            case 0x02: case 0x0D: a = i1; b = i0; c = i2; d = i3; break;
                            case 0x04: case 0x0B: a = i2; b = i0; c = i1; d = i3; break;
                            case 0x08: case 0x07: a = i3; b = i0; c = i1; d = i2; break;
                            case 0x03: a = i0; b = i1; c = i2; d = i3; quad = 1; break;
                            case 0x0C: a = i2; b = i3; c = i0; d = i1; quad = 1; break;
                            case 0x05: a = i0; b = i2; c = i1; d = i3; quad = 1; break;
                            case 0x0A: a = i1; b = i3; c = i0; d = i2; quad = 1; break;
                            case 0x06: a = i1; b = i2; c = i0; d = i3; quad = 1; break;
                            case 0x09: a = i0; b = i3; c = i1; d = i2; quad = 1; break;
                            default: break;
                        }
                        if (a < 0) continue;
                        int n_tri;
                        if (!quad) {
                            /* Crossings on the three edges from a. */
                            tri[0] = interp(iso, pos[a], pos[b], val[a], val[b], col[a], col[b]);
                            tri[1] = interp(iso, pos[a], pos[c], val[a], val[c], col[a], col[c]);
                            tri[2] = interp(iso, pos[a], pos[d], val[a], val[d], col[a], col[d]);
                            n_tri = 1;
                        } else {
                            /* a,b on one side, c,d on the other: quad ac, ad, bd, bc. */
                            const Vtx ac = interp(iso, pos[a], pos[c], val[a], val[c], col[a], col[c]);
                            const Vtx ad = interp(iso, pos[a], pos[d], val[a], val[d], col[a], col[d]);
                            const Vtx bd = interp(iso, pos[b], pos[d], val[b], val[d], col[b], col[d]);
                            const Vtx bc = interp(iso, pos[b], pos[c], val[b], val[c], col[b], col[c]);
                            tri[0] = ac; tri[1] = ad; tri[2] = bd;
                            tri[3] = ac; tri[4] = bd; tri[5] = bc;
                            n_tri = 2;
                        }
                        const int32_t n_v = n_tri * 3;
                        const int32_t base = n_written;
                        n_written += n_v;
                        if (base + n_v > vert_cap) {
                            overflow = 1;
                            continue;
                        }
                        for (int32_t q = 0; q < n_v; ++q) {
                            float* dst = posnor + (size_t)(base + q) * 6;
                            dst[0] = tri[q].p[0];
                            dst[1] = tri[q].p[1];
                            dst[2] = tri[q].p[2];
                            dst[3] = 0.0f; dst[4] = 0.0f; dst[5] = 0.0f;
                            if (rgb) {
                                uint8_t* cc = rgb + (size_t)(base + q) * 3;
                                cc[0] = (uint8_t)clampf(tri[q].c[0], 0.0f, 255.0f);
                                cc[1] = (uint8_t)clampf(tri[q].c[1], 0.0f, 255.0f);
                                cc[2] = (uint8_t)clampf(tri[q].c[2], 0.0f, 255.0f);
                            }
                        }
                        for (int32_t f = 0; f < n_tri; ++f) {
                            float* v0 = posnor + (size_t)(base + f * 3) * 6;
                            float* v1 = v0 + 6;
                            float* v2 = v0 + 12;
                            const float e1[3] = {v1[0] - v0[0], v1[1] - v0[1], v1[2] - v0[2]};
                            const float e2[3] = {v2[0] - v0[0], v2[1] - v0[1], v2[2] - v0[2]};
                            float nx = e1[1] * e2[2] - e1[2] * e2[1];
                            float ny = e1[2] * e2[0] - e1[0] * e2[2];
                            float nz = e1[0] * e2[1] - e1[1] * e2[0];
                            const float len = sqrtf(nx * nx + ny * ny + nz * nz);
                            if (len > 1e-20f) { nx /= len; ny /= len; nz /= len; }
                            v0[3] = nx; v0[4] = ny; v0[5] = nz;
                            v1[3] = nx; v1[4] = ny; v1[5] = nz;
                            v2[3] = nx; v2[4] = ny; v2[5] = nz;
                        }
                    }
                }
    }
    if (overflow) return -1;
    return n_written;
}

int32_t oracle_block_count(const OracleVolume* v) { return v ? v->block_count : 0; }
uint64_t oracle_drop_count(const OracleVolume* v) { return v ? v->drop_count : 0; }
uint32_t oracle_hash_mask(const OracleVolume* v) { return v ? v->mask : 0; }
float oracle_trunc(const OracleVolume* v) { return v ? v->trunc : 0.0f; }

int32_t oracle_block_coords(const OracleVolume* v, int32_t* out) {
    if (!v || !out) return 1;
    memcpy(out, v->coord, (size_t)v->block_count * 3 * sizeof(int32_t));
    return 0;
}

int32_t oracle_voxels(const OracleVolume* v, float* tsdf, float* weight, float* r, float* g,
                      float* b) {
    if (!v) return 1;
    const size_t n = (size_t)v->block_count * kBlockVoxels * sizeof(float);
    if (tsdf) memcpy(tsdf, v->tsdf, n);
    if (weight) memcpy(weight, v->weight, n);
    if (r) memcpy(r, v->r, n);
    if (g) memcpy(g, v->g, n);
    if (b) memcpy(b, v->b, n);
    return 0;
}

int32_t oracle_table(const OracleVolume* v, int64_t* keys, int32_t* block_idx) {
    if (!v) return 1;
    for (uint32_t i = 0; i <= v->mask; ++i) {
        if (keys) keys[i] = v->table[i].key;
        if (block_idx) block_idx[i] = v->table[i].block_idx;
    }
    return 0;
}

/* analytic_scenes.hpp:19-33: points on a sphere seen from its centre. The
 * float expression order matches the reference so the points are identical. */
void oracle_sphere_points(float radius, int32_t n_theta, int32_t n_phi, float* out) {
    const float pi = (float)3.14159265358979323846;
    size_t k = 0;
    for (int32_t i = 0; i < n_theta; ++i) {
        const float theta = pi * ((float)i + 0.5f) / (float)n_theta;
        for (int32_t j = 0; j < n_phi; ++j) {
            const float phi = 2.0f * pi * (float)j / (float)n_phi;
            out[k++] = radius * sinf(theta) * cosf(phi);
            out[k++] = radius * sinf(theta) * sinf(phi);
            out[k++] = radius * cosf(theta);
        }
    }
}

/* analytic_scenes.hpp:35-46: a z = z0 plane patch. */
void oracle_plane_points(float z0, float half_extent, int32_t n, float* out) {
    size_t k = 0;
    for (int32_t i = 0; i < n; ++i) {
        for (int32_t j = 0; j < n; ++j) {
            out[k++] = -half_extent + 2.0f * half_extent * (float)i / (float)(n - 1);
            out[k++] = -half_extent + 2.0f * half_extent * (float)j / (float)(n - 1);
            out[k++] = z0;
        }
    }
}
