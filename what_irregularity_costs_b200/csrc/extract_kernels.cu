// Extract: marching-tetrahedra triangle soup over every allocated block.
//
// Reference: cpp/src/marching_tets.cpp:31-245 (CPU arm) and
// cpp/src/marching_tets_cuda.cu:33-167 (CUDA arm: one CTA per block, one
// thread per cube, a full hash probe for each of the 8 corners of every cube
// and one global atomic per emitting tetrahedron).
//
// B200 design. One CTA per block, one thread per cube, but the 7 neighbour
// blocks are looked up once per CTA and the 9x9x9 halo of corner samples
// (mean TSDF, validity, mean colour) is staged in shared memory with
// coalesced reads, so the corner loop reads shared memory only. Emission is
// compacted: each thread counts its vertices, a block-wide scan (warp
// shuffles) gives every thread its offset, and one atomic per CTA reserves
// the block's output range, so a block's triangles are contiguous and in a
// fixed order (cube, then tetrahedron).
//
// Arithmetic follows the reference operation for operation, unfused, so a
// volume whose voxels match bit-for-bit extracts bit-identical vertices.
#include <algorithm>

#include "volume.h"

namespace osn_b200 {
namespace {

constexpr int kExtractThreads = 512;
constexpr int kHalo = 9;
constexpr int kHaloCells = kHalo * kHalo * kHalo;

// marching_tets.cpp:37-40: six tetrahedra around the 0-7 diagonal.
constexpr int kTetCorners[6][4] = {
    {0, 5, 1, 7}, {0, 1, 3, 7}, {0, 3, 2, 7}, {0, 6, 4, 7}, {0, 4, 5, 7}, {0, 2, 6, 7},
};

// A tetrahedron's case code (bit i: its corner i is below iso) gives its
// crossing (marching_tets.cpp:165-182): none (0000, 1111), one triangle from
// the corner on its own side (one or three bits set), or a quad split in two
// (two bits set).
constexpr int popc4(int x) { return (x & 1) + ((x >> 1) & 1) + ((x >> 2) & 1) + ((x >> 3) & 1); }
constexpr int tris_of_code(int code) { return (popc4(code) & 1) ? 1 : (popc4(code) == 2 ? 2 : 0); }
constexpr int tet_code(int below, int k) {
    int code = 0;
    for (int i = 0; i < 4; ++i) code |= ((below >> kTetCorners[k][i]) & 1) << i;
    return code;
}

// Tables the kernel stages in shared memory (constant-bank reads with lane-
// dependent indices would serialise):
//   kinds[below]   the six tetrahedra's triangle counts (2 bits each) of a
//                  cube whose corners below iso are the bits of `below`;
//   cases[k][code] tetrahedron k's corners (a, b, c, d) in the order the
//                  case table of marching_tets.cpp:165-182 names them (3 bits
//                  each) and its triangle count (bits 12-13);
//   corners[k]     tetrahedron k's four corners (3 bits each).
struct alignas(4) TetTables {
    uint16_t kinds[256];
    uint16_t cases[6][16];
    uint16_t corners[6];
};
constexpr int case_perm(int code) {  // (a, b, c, d) as positions in the tetrahedron
    switch (code) {
        case 0x01: case 0x0E: case 0x03: return 0 | 1 << 2 | 2 << 4 | 3 << 6;
        case 0x02: case 0x0D: return 1 | 0 << 2 | 2 << 4 | 3 << 6;
        case 0x04: case 0x0B: return 2 | 0 << 2 | 1 << 4 | 3 << 6;
        case 0x08: case 0x07: return 3 | 0 << 2 | 1 << 4 | 2 << 6;
        case 0x0C: return 2 | 3 << 2 | 0 << 4 | 1 << 6;
        case 0x05: return 0 | 2 << 2 | 1 << 4 | 3 << 6;
        case 0x0A: return 1 | 3 << 2 | 0 << 4 | 2 << 6;
        case 0x06: return 1 | 2 << 2 | 0 << 4 | 3 << 6;
        case 0x09: return 0 | 3 << 2 | 1 << 4 | 2 << 6;
        default: return 0;
    }
}
constexpr TetTables make_tet_tables() {
    TetTables t{};
    for (int b = 0; b < 256; ++b) {
        int v = 0;
        for (int k = 0; k < 6; ++k) v |= tris_of_code(tet_code(b, k)) << (2 * k);
        t.kinds[b] = (uint16_t)v;
    }
    for (int k = 0; k < 6; ++k) {
        int c = 0;
        for (int i = 0; i < 4; ++i) c |= kTetCorners[k][i] << (3 * i);
        t.corners[k] = (uint16_t)c;
        for (int code = 0; code < 16; ++code) {
            const int p = case_perm(code);
            int e = 0;
            for (int i = 0; i < 4; ++i) e |= kTetCorners[k][(p >> (2 * i)) & 3] << (3 * i);
            t.cases[k][code] = (uint16_t)(e | tris_of_code(code) << 12);
        }
    }
    return t;
}
__constant__ TetTables c_tet_tables = make_tet_tables();
static_assert(make_tet_tables().kinds[0] == 0 && make_tet_tables().kinds[255] == 0, "no crossing");
static_assert(make_tet_tables().kinds[1] == 0x555, "corner 0 alone: one triangle in every tetrahedron");

// The block's 9^3 corner samples; colours only when the caller wants them.
template <bool COL>
struct Halo {
    float val[kHaloCells];
    float col[COL ? 3 : 1][COL ? kHaloCells : 1];
    unsigned char flag[kHaloCells];  // bit 0: valid sample; bit 1: valid and below iso
};

struct Cube {
    int vx, vy, vz;  // voxel coordinate of corner 0
    int h0;          // halo index of corner 0
    float vs;
};

__device__ __forceinline__ int corner_halo(const Cube& q, int c) {
    return q.h0 + ((c >> 2) & 1) * kHalo * kHalo + ((c >> 1) & 1) * kHalo + (c & 1);
}

// Voxel centre of a corner (marching_tets.cpp:126-128).
__device__ __forceinline__ void corner_pos(const Cube& q, int c, float p[3]) {
    p[0] = __fmul_rn(__fadd_rn((float)(q.vx + (c & 1)), 0.5f), q.vs);
    p[1] = __fmul_rn(__fadd_rn((float)(q.vy + ((c >> 1) & 1)), 0.5f), q.vs);
    p[2] = __fmul_rn(__fadd_rn((float)(q.vz + ((c >> 2) & 1)), 0.5f), q.vs);
}

struct Vert {
    float p[3];
    float c[3];
};

// marching_tets.cpp:59-80: position-ordered interpolation.
template <bool COL>
__device__ __forceinline__ Vert interp(const Halo<COL>& h, const Cube& q, float iso, int ia, int ib) {
    // The corner with the smaller position (x, then y, then z) first. Corner
    // positions are increasing functions of the corner's offset bits on each
    // axis (same cube), so comparing the offsets (x, y, z) as a 3-bit number
    // orders the positions exactly.
    const int ka = ((ia & 1) << 2) | (ia & 2) | ((ia >> 2) & 1);
    const int kb = ((ib & 1) << 2) | (ib & 2) | ((ib >> 2) & 1);
    const bool sw = kb < ka;
    const int i0 = sw ? ib : ia, i1 = sw ? ia : ib;
    float p0[3], p1[3];
    corner_pos(q, i0, p0);
    corner_pos(q, i1, p1);
    const int h0 = corner_halo(q, i0), h1 = corner_halo(q, i1);
    const float v0 = h.val[h0], v1 = h.val[h1];
    const float den = __fsub_rn(v1, v0);
    const float t = fabsf(den) < 1e-12f ? 0.5f : __fdiv_rn(__fsub_rn(iso, v0), den);
    const float tc = fminf(fmaxf(t, 0.0f), 1.0f);
    Vert o;
    for (int k = 0; k < 3; ++k) o.p[k] = __fadd_rn(p0[k], __fmul_rn(tc, __fsub_rn(p1[k], p0[k])));
    if constexpr (COL) {
        for (int k = 0; k < 3; ++k) {
            const float c0 = h.col[k][h0], c1 = h.col[k][h1];
            o.c[k] = __fadd_rn(c0, __fmul_rn(tc, __fsub_rn(c1, c0)));
        }
    }
    return o;
}

// Where a CTA's vertices go: the block's output range is contiguous, so its
// first stage_verts vertices are staged in shared memory (with the range's
// offset inside its 16-byte group, so the copy-out is aligned) and written
// out by the whole CTA with 16-byte streaming stores; any further vertices
// of an unusually dense block go straight to global memory. The instance
// with colours stages fewer (its halo holds the colours too).
template <bool COL>
__host__ __device__ constexpr int stage_verts() { return COL ? 1024 : 1536; }
// A cube emits at most 6 tetrahedra x 2 triangles.
constexpr int kMaxBlockTris = kBlockVoxels * 12;
// Dynamic shared memory of one CTA: the vertex stage (pad + stage_verts * 6
// floats), then the block's triangle list (one 16-bit item per triangle).
template <bool COL>
__host__ __device__ constexpr int extract_dyn_smem() {
    return (4 + stage_verts<COL>() * 6) * 4 + kMaxBlockTris * 2;
}
template <bool COL>
struct VertexSink {
    float* stage;     // shared: [pad + stage_verts * 6]
    int pad;          // floats of the 16-byte group before the block's first vertex
    float* posnor;    // global output
    int64_t base;     // the block's first vertex in the output
    __device__ __forceinline__ float* slot(int local) const {
        return local < stage_verts<COL>() ? stage + pad + local * 6 : posnor + (base + local) * 6;
    }
};

template <bool COL>
__device__ __forceinline__ void emit_triangle(const Vert& a, const Vert& b, const Vert& c,
                                              const VertexSink<COL>& out, uint8_t* rgb, int local) {
    // marching_tets.cpp:206-218: face normal of the emitted triangle.
    const float e1[3] = {__fsub_rn(b.p[0], a.p[0]), __fsub_rn(b.p[1], a.p[1]), __fsub_rn(b.p[2], a.p[2])};
    const float e2[3] = {__fsub_rn(c.p[0], a.p[0]), __fsub_rn(c.p[1], a.p[1]), __fsub_rn(c.p[2], a.p[2])};
    float nx = __fsub_rn(__fmul_rn(e1[1], e2[2]), __fmul_rn(e1[2], e2[1]));
    float ny = __fsub_rn(__fmul_rn(e1[2], e2[0]), __fmul_rn(e1[0], e2[2]));
    float nz = __fsub_rn(__fmul_rn(e1[0], e2[1]), __fmul_rn(e1[1], e2[0]));
    const float len =
        __fsqrt_rn(__fadd_rn(__fadd_rn(__fmul_rn(nx, nx), __fmul_rn(ny, ny)), __fmul_rn(nz, nz)));
    if (len > 1e-20f) {
        nx = __fdiv_rn(nx, len);
        ny = __fdiv_rn(ny, len);
        nz = __fdiv_rn(nz, len);
    }
    const Vert* vs[3] = {&a, &b, &c};
    for (int k = 0; k < 3; ++k) {
        float* dst = out.slot(local + k);
        dst[0] = vs[k]->p[0];
        dst[1] = vs[k]->p[1];
        dst[2] = vs[k]->p[2];
        dst[3] = nx;
        dst[4] = ny;
        dst[5] = nz;
        if constexpr (COL) {
            uint8_t* cc = rgb + (out.base + local + k) * 3;
            cc[0] = (uint8_t)fminf(fmaxf(vs[k]->c[0], 0.0f), 255.0f);
            cc[1] = (uint8_t)fminf(fmaxf(vs[k]->c[1], 0.0f), 255.0f);
            cc[2] = (uint8_t)fminf(fmaxf(vs[k]->c[2], 0.0f), 255.0f);
        }
    }
}

// Resident CTAs per SM the colourless instance is sized for: 4 x 512 threads
// at 32 registers (a few bytes spill), measured 0.38 ms against 0.56 ms at 3
// CTAs and 0.62 ms at 2 on a 14k-block, 8.7M-vertex mesh.
#ifndef OSN_EXTRACT_MIN_BLOCKS
#define OSN_EXTRACT_MIN_BLOCKS 4
#endif
template <int S, bool COL>
__global__ void __launch_bounds__(kExtractThreads, COL ? 1 : OSN_EXTRACT_MIN_BLOCKS)
extract_kernel(DevVolume v, int32_t n_blocks, const int32_t* list, float min_w, float iso, float* out_posnor,
               uint8_t* out_rgb, int32_t cap, int32_t* ctl) {
    __shared__ Halo<COL> h;
    __shared__ uint8_t s_below[kBlockVoxels];
    __shared__ TetTables s_tab;
    extern __shared__ __align__(16) float s_dyn[];
    float* const s_stage = s_dyn;
    uint16_t* const s_items = reinterpret_cast<uint16_t*>(s_dyn + 4 + stage_verts<COL>() * 6);
    __shared__ int s_nb[8];
    __shared__ int s_warp[kExtractThreads / 32];
    __shared__ int s_base, s_total;

    if ((int)blockIdx.x >= n_blocks) return;
    const int b = list ? list[blockIdx.x] : (int)blockIdx.x;  // the block's pool index
    const int t = threadIdx.x;
    const BlockCoord bc = v.block_coord[b];
    if (t < 8) {
        const int dx = t & 1, dy = (t >> 1) & 1, dz = (t >> 2) & 1;
        const int nx = bc.x + dx, ny = bc.y + dy, nz = bc.z + dz;
        s_nb[t] = t == 0 ? b : find_block(v, nx, ny, nz, pack_key(nx, ny, nz));
    }
    for (int k = t; k < (int)(sizeof(TetTables) / 4); k += kExtractThreads)
        reinterpret_cast<uint32_t*>(&s_tab)[k] = reinterpret_cast<const uint32_t*>(&c_tet_tables)[k];
    __syncthreads();

    // Stage the halo: corner samples of this block plus the +x/+y/+z faces,
    // edges and corner of its neighbours (volume.cpp:306-329 per sample).
    for (int k = t; k < kHaloCells; k += kExtractThreads) {
        const int hx = k % kHalo, hy = (k / kHalo) % kHalo, hz = k / (kHalo * kHalo);
        const int nb = s_nb[(hx >> 3) | ((hy >> 3) << 1) | ((hz >> 3) << 2)];
        unsigned char flag = 0;
        h.val[k] = 0.0f;
        if (nb >= 0) {
            const size_t idx = (size_t)nb * kBlockVoxels + (size_t)((((hz & 7) * kBlockDim) + (hy & 7)) * kBlockDim + (hx & 7));
            // Weight and stored TSDF loaded together (one round trip).
            const float w = weight_at<S>(v, idx);
            const float m = mean_from<S>(v, idx, w);
            if (!(w < min_w || w <= 0.0f)) {
                flag = m < iso ? 3 : 1;
                h.val[k] = m;
                if constexpr (COL) {
                    if constexpr (S == kStoreF32) {
                        const float inv = __fdiv_rn(1.0f, w);
                        h.col[0][k] = __fmul_rn(v.r[idx], inv);
                        h.col[1][k] = __fmul_rn(v.g[idx], inv);
                        h.col[2][k] = __fmul_rn(v.b[idx], inv);
                    } else {
                        // No colour arrays: every contribution is grey.
                        h.col[0][k] = 128.0f;
                        h.col[1][k] = 128.0f;
                        h.col[2][k] = 128.0f;
                    }
                }
            }
        }
        h.flag[k] = flag;
    }
    __syncthreads();

    Cube q;
    const int lx = t & 7, ly = (t >> 3) & 7, lz = t >> 6;
    q.vx = bc.x * kBlockDim + lx;
    q.vy = bc.y * kBlockDim + ly;
    q.vz = bc.z * kBlockDim + lz;
    q.h0 = (lz * kHalo + ly) * kHalo + lx;
    q.vs = v.voxel_size;

    unsigned all_ok = 1u;
    unsigned below = 0;  // bit c set when corner c is below iso
#pragma unroll
    for (int c = 0; c < 8; ++c) {
        const unsigned f = h.flag[corner_halo(q, c)];
        all_ok &= f;
        below |= (f >> 1) << c;
    }

    // Triangles of this cube (every corner valid, or none).
    const unsigned kinds = (all_ok & 1u) ? s_tab.kinds[below] : 0u;
    const int n_tri = __popc(kinds & 0x555u) + 2 * __popc(kinds & 0xAAAu);
    s_below[t] = (uint8_t)below;

    // Block-wide exclusive scan of the triangle counts.
    const int lane = t & 31, warp = t >> 5;
    int x = n_tri;
    for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) s_warp[warp] = x;
    __syncthreads();
    if (warp == 0) {
        int w = lane < kExtractThreads / 32 ? s_warp[lane] : 0;
        for (int o = 1; o < 32; o <<= 1) {
            const int y = __shfl_up_sync(0xffffffffu, w, o);
            if (lane >= o) w += y;
        }
        if (lane < kExtractThreads / 32) s_warp[lane] = w;
        if (lane == kExtractThreads / 32 - 1) {
            const int total = 3 * w;  // vertices
            int base = 0;
            if (total > 0) {
                base = atomicAdd(&ctl[0], total);
                if ((int64_t)base + total > (int64_t)cap) {
                    atomicExch(&ctl[1], 1);
                    base = -1;
                }
            }
            s_base = base;
            s_total = total;
        }
    }
    __syncthreads();
    const int total = s_total;
    if (s_base < 0 || total == 0) return;  // uniform across the CTA
    VertexSink<COL> sink;
    sink.stage = s_stage;
    // The caller's buffer is float-aligned, not necessarily 16-byte aligned:
    // the pad is taken from the address of the block's first float.
    sink.pad = (int)((reinterpret_cast<uintptr_t>(out_posnor + (int64_t)s_base * 6) >> 2) & 3);
    sink.posnor = out_posnor;
    sink.base = s_base;

    // The block's triangle list in output order (cube, tetrahedron, triangle):
    // item = cube | tetrahedron << 9 | second triangle of a quad << 12.
    {
        int at = (warp ? s_warp[warp - 1] : 0) + x - n_tri;
        for (int k = 0; k < (n_tri > 0 ? 6 : 0); ++k) {
            const int kind = (int)(kinds >> (2 * k)) & 3;
            for (int m = 0; m < kind; ++m) s_items[at++] = (uint16_t)(t | k << 9 | m << 12);
        }
    }
    __syncthreads();

    // One thread per triangle: the warps stay converged however sparse the
    // surface is within the block.
    const int n_tris = total / 3;
    for (int j = t; j < n_tris; j += kExtractThreads) {
        const int item = s_items[j];
        const int cube = item & (kBlockVoxels - 1), k = (item >> 9) & 7, second = item >> 12;
        Cube qc;
        const int cx = cube & 7, cy = (cube >> 3) & 7, cz = cube >> 6;
        qc.vx = bc.x * kBlockDim + cx;
        qc.vy = bc.y * kBlockDim + cy;
        qc.vz = bc.z * kBlockDim + cz;
        qc.h0 = (cz * kHalo + cy) * kHalo + cx;
        qc.vs = v.voxel_size;
        const unsigned bl = s_below[cube];
        const unsigned tc = s_tab.corners[k];
        const int code = (int)(((bl >> (tc & 7u)) & 1u) | (((bl >> ((tc >> 3) & 7u)) & 1u) << 1) |
                               (((bl >> ((tc >> 6) & 7u)) & 1u) << 2) | (((bl >> (tc >> 9)) & 1u) << 3));
        const unsigned e = s_tab.cases[k][code];
        const int a = (int)(e & 7u), bb = (int)((e >> 3) & 7u), c = (int)((e >> 6) & 7u), d = (int)((e >> 9) & 7u);
        // marching_tets.cpp:142-163: a single triangle (a-b, a-c, a-d), or the
        // quad's two (a-c, a-d, b-d) and (a-c, b-d, b-c).
        int e0a = a, e0b = c, e1a = a, e1b = d, e2a = bb, e2b = d;
        if ((e >> 12) == 1u) {
            e0b = bb;
            e1b = c;
            e2a = a;
        } else if (second) {
            e1a = bb;
            e2b = c;
        }
        const Vert v0 = interp(h, qc, iso, e0a, e0b);
        const Vert v1 = interp(h, qc, iso, e1a, e1b);
        const Vert v2 = interp(h, qc, iso, e2a, e2b);
        emit_triangle<COL>(v0, v1, v2, sink, out_rgb, 3 * j);
    }
    __syncthreads();
    // Copy-out of the staged vertices: 16-byte groups of the output, each
    // wholly inside the block's range stored as one vector, the partial
    // first and last groups float by float.
    const int n_floats = min(total, stage_verts<COL>()) * 6;
    // The 16-byte group holding the block's first float; only floats of the
    // block's range [pad, pad + n_floats) are written.
    float* gbase = reinterpret_cast<float*>(reinterpret_cast<uintptr_t>(out_posnor + (int64_t)s_base * 6) -
                                            4 * (uintptr_t)sink.pad);
    const int groups = (sink.pad + n_floats + 3) >> 2;
    for (int g = t; g < groups; g += kExtractThreads) {
        const int lo = 4 * g;
        if (lo >= sink.pad && lo + 4 <= sink.pad + n_floats) {
            __stcs(reinterpret_cast<float4*>(gbase) + g, reinterpret_cast<const float4*>(s_stage)[g]);
        } else {
            for (int j = max(lo, sink.pad); j < min(lo + 4, sink.pad + n_floats); ++j) gbase[j] = s_stage[j];
        }
    }
}

__global__ void reset_table_kernel(HashEntry* table, uint32_t count, long long key) {
    for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < count; k += gridDim.x * blockDim.x) {
        table[k].key = key;
        table[k].block_idx = -1;
        table[k].pad = 0;
    }
}

// Every occupied slot of the table (slot-index layout: the slot is the
// block's pool index), appended warp by warp.
__global__ void list_blocks_kernel(const HashEntry* table, uint32_t size, int32_t* out, int32_t* count) {
    for (uint32_t base = blockIdx.x * blockDim.x; base < size; base += gridDim.x * blockDim.x) {
        const uint32_t k = base + threadIdx.x;
        bool occ = false;
        if (k < size) {
            const int4 raw = reinterpret_cast<const int4*>(table)[k];
            const long long key = ((long long)(unsigned)raw.y << 32) | (unsigned)raw.x;
            occ = key >= 0 && raw.z == (int)k;
        }
        const unsigned m = __ballot_sync(0xffffffffu, occ);
        int at = 0;
        if ((threadIdx.x & 31) == 0 && m) at = atomicAdd(count, __popc(m));
        at = __shfl_sync(0xffffffffu, at, 0);
        if (occ) out[at + __popc(m & lanemask_lt())] = (int32_t)k;
    }
}

// Zero the voxels of the blocks of a list, one CTA per block.
__global__ void reset_listed_kernel(DevVolume v, const int32_t* list, int32_t n) {
    const int32_t i = blockIdx.x;
    if (i >= n) return;
    const size_t b = (size_t)list[i];
    const float4 z = make_float4(0.f, 0.f, 0.f, 0.f);
    const int n_t = kBlockVoxels * tsdf_bytes(v.storage) / 16;
    const int n_w = kBlockVoxels * weight_bytes(v.storage) / 16;
    for (int k = threadIdx.x; k < n_t; k += blockDim.x) {
        reinterpret_cast<float4*>(v.tsdf)[b * n_t + k] = z;
        if (k < n_w) reinterpret_cast<float4*>(v.weight)[b * n_w + k] = z;
        if (v.storage == kStoreF32) {
            reinterpret_cast<float4*>(v.r)[b * n_t + k] = z;
            reinterpret_cast<float4*>(v.g)[b * n_t + k] = z;
            reinterpret_cast<float4*>(v.b)[b * n_t + k] = z;
        }
    }
}

// Zero the first n_voxels voxels of every array of the volume's storage, 16
// bytes per store (n_voxels is a multiple of 512).
__global__ void reset_voxels_kernel(DevVolume v, size_t n_voxels) {
    const float4 z = make_float4(0.f, 0.f, 0.f, 0.f);
    const size_t n_t = n_voxels * (size_t)tsdf_bytes(v.storage) / 16;
    const size_t n_w = n_voxels * (size_t)weight_bytes(v.storage) / 16;
    const bool rgb = v.storage == kStoreF32;
    for (size_t k = (size_t)blockIdx.x * blockDim.x + threadIdx.x; k < n_t;
         k += (size_t)gridDim.x * blockDim.x) {
        reinterpret_cast<float4*>(v.tsdf)[k] = z;
        if (k < n_w) reinterpret_cast<float4*>(v.weight)[k] = z;
        if (rgb) {
            reinterpret_cast<float4*>(v.r)[k] = z;
            reinterpret_cast<float4*>(v.g)[k] = z;
            reinterpret_cast<float4*>(v.b)[k] = z;
        }
    }
}

}  // namespace

template <int S, bool COL>
static cudaError_t launch_extract_as(const DevVolume& v, int32_t n_blocks, const int32_t* list, float min_w,
                                     float iso, float* posnor, uint8_t* rgb, int32_t cap, int32_t* ctl,
                                     cudaStream_t s) {
    constexpr int dyn = extract_dyn_smem<COL>();
    cudaError_t e = cudaFuncSetAttribute(extract_kernel<S, COL>, cudaFuncAttributeMaxDynamicSharedMemorySize, dyn);
    if (e != cudaSuccess) return e;
    extract_kernel<S, COL><<<n_blocks, kExtractThreads, dyn, s>>>(v, n_blocks, list, min_w, iso, posnor, rgb, cap, ctl);
    return cudaGetLastError();
}

cudaError_t launch_extract(const DevVolume& v, int32_t n_blocks, const int32_t* list, float min_w, float iso,
                           float* posnor, uint8_t* rgb, int32_t cap, int32_t* ctl, cudaStream_t s) {
    if (n_blocks <= 0) return cudaSuccess;
    // Colours in a separate instance: without them the halo holds a quarter
    // of the shared memory and the kernel fewer registers.
    const bool col = rgb != nullptr;
    switch (v.storage) {
        case kStoreF16U16:
            return col ? launch_extract_as<kStoreF16U16, true>(v, n_blocks, list, min_w, iso, posnor, rgb, cap, ctl, s)
                       : launch_extract_as<kStoreF16U16, false>(v, n_blocks, list, min_w, iso, posnor, nullptr, cap, ctl, s);
        case kStoreF64:
            return col ? launch_extract_as<kStoreF64, true>(v, n_blocks, list, min_w, iso, posnor, rgb, cap, ctl, s)
                       : launch_extract_as<kStoreF64, false>(v, n_blocks, list, min_w, iso, posnor, nullptr, cap, ctl, s);
        default:
            return col ? launch_extract_as<kStoreF32, true>(v, n_blocks, list, min_w, iso, posnor, rgb, cap, ctl, s)
                       : launch_extract_as<kStoreF32, false>(v, n_blocks, list, min_w, iso, posnor, nullptr, cap, ctl, s);
    }
}

cudaError_t launch_reset_table(HashEntry* first, uint32_t count, long long key, cudaStream_t s) {
    if (count == 0) return cudaSuccess;
    const int grid = (int)std::min<uint32_t>((count + 255) / 256, 148u * 16u);
    reset_table_kernel<<<grid, 256, 0, s>>>(first, count, key);
    return cudaGetLastError();
}

cudaError_t launch_list_blocks(const DevVolume& v, int32_t* out, int32_t* count, cudaStream_t s) {
    const uint32_t size = v.hash_mask + 1;
    const int grid = (int)std::min<uint32_t>((size + 255) / 256, 148u * 8u);
    list_blocks_kernel<<<grid, 256, 0, s>>>(v.table, size, out, count);
    return cudaGetLastError();
}

cudaError_t launch_reset_voxels(const DevVolume& v, int32_t n_blocks, const int32_t* list, cudaStream_t s) {
    if (n_blocks <= 0) return cudaSuccess;
    if (list) {
        reset_listed_kernel<<<n_blocks, 128, 0, s>>>(v, list, n_blocks);
        return cudaGetLastError();
    }
    const size_t n_voxels = (size_t)n_blocks * kBlockVoxels;
    const size_t n_vec = n_voxels * (size_t)tsdf_bytes(v.storage) / 16;
    const int grid = (int)std::min<size_t>((n_vec + 255) / 256, (size_t)148 * 16);
    reset_voxels_kernel<<<grid, 256, 0, s>>>(v, n_voxels);
    return cudaGetLastError();
}

}  // namespace osn_b200
