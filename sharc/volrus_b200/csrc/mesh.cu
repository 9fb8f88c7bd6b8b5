// volume_to_mesh (src/tools/volume_to_mesh.rs:46-201): marching-cubes
// isosurface of a world-unit f32 grid, with the reference's cell order, vertex
// numbering and vertex positions.
//
// The reference visits the 8^3 cell tiles of every leaf and of its 6 face
// neighbours, tiles in ascending (x, y, z) of origin and cells x-major within a
// tile (volume_to_mesh.rs:58-97); a cell reads its 8 corners with Grid::get,
// flags the edges whose corners classify differently against the isovalue,
// and creates an edge's vertex the first time a processed cell flags it (a
// HashMap edge cache, volume_to_mesh.rs:144-186), so vertex i is the i-th
// first-touched edge in that order, interpolated from the creating cell's
// first endpoint toward its second.  Triangles follow per cell in visit order.
//
// On the GPU:
//   k_mc_cand      the 7 candidate tiles per leaf as x-major 63-bit keys
//   (sort)         two stable 32-bit radix passes (low word, then high word)
//   k_mc_unique    first of each run of equal keys -> sorted tile list; a hash
//                  maps each tile to its rank
//   k_mc_classify  one CTA per tile: 9^3 corner values staged in shared memory,
//                  the case of each cell, and which of its flagged edges it
//                  creates: an edge belongs to up to 4 cells, and the cell
//                  creates it iff none of the other processed cells precedes
//                  it in visit order (decided from the 27 neighbour tiles'
//                  ranks); per-cell word = case | creator mask | in-tile
//                  rank of its first created vertex; per-tile counts
//   (scans)        tile bases of vertices and triangles
//   k_mc_emit      one CTA per tile: creators write their vertex (f64, the
//                  reference's rounding: f32 t, then pa + t * (pb - pa)); the
//                  other flagged edges look up their creator's index; each
//                  cell writes its triangles at its scanned offset
// So the output order needs no sort and no atomics: every index is a prefix
// count in visit order.
//
// Triangle table.  Vertices depend only on the edge table, which is the
// classification rule.  Triangles come from the crate's own 256-case table
// (src/tools/volume_to_mesh.rs:246-503, the classic Lorensen & Cline / Bourke
// table), carried in mc_tri_table.inc with the same corner and edge
// numbering, so each cell emits the same triangles in the same order as the
// crate; a cell's triangles are the table row's triples up to its -1.
#include <algorithm>
#include <cstring>
#include <mutex>

#include "ref_ops.hpp"
#include "sort_reduce.hpp"

namespace vlr {
namespace {

constexpr int kCornerOff[8][3] = {{0, 0, 0}, {1, 0, 0}, {1, 1, 0}, {0, 1, 0}, {0, 0, 1}, {1, 0, 1}, {1, 1, 1}, {0, 1, 1}};
constexpr int kEdgeEnds[12][2] = {{0, 1}, {1, 2}, {2, 3}, {3, 0}, {4, 5}, {5, 6},
                                  {6, 7}, {7, 4}, {0, 4}, {1, 5}, {2, 6}, {3, 7}};
// the crate's triangle table (src/tools/volume_to_mesh.rs:246-503), 16 entries per case, -1 terminated
constexpr int8_t kTriTable[256][16] = {
#include "mc_tri_table.inc"
};

struct McTable {
    int8_t tri[256][16];
    uint8_t ntri[256];
    // the 3 other cells holding edge e: (dx+1) | (dy+1) << 2 | (dz+1) << 4 | e' << 8,
    // e' the edge's index in that cell
    int nb[12][3];
};

McTable build_mc_table() {
    McTable t;
    for (int cs = 0; cs < 256; ++cs) {
        int n = 0;
        while (n < 15 && kTriTable[cs][n] >= 0) n += 3;
        std::memcpy(t.tri[cs], kTriTable[cs], 16);
        t.ntri[cs] = (uint8_t)(n / 3);
    }
    // an edge along axis a with lower corner L lies in the 4 cells at
    // delta = (L_u - du) e_u + (L_w - dw) e_w, du, dw in {0, 1}; in the cell
    // at delta its lower corner is L - delta
    for (int e = 0; e < 12; ++e) {
        const int a = kEdgeEnds[e][0], b = kEdgeEnds[e][1];
        int L[3], axis = 0;
        for (int k = 0; k < 3; ++k) {
            L[k] = std::min(kCornerOff[a][k], kCornerOff[b][k]);
            if (kCornerOff[a][k] != kCornerOff[b][k]) axis = k;
        }
        const int u = (axis + 1) % 3, w = (axis + 2) % 3;
        int q = 0;
        for (int du = 0; du < 2; ++du)
            for (int dw = 0; dw < 2; ++dw) {
                int d[3] = {0, 0, 0};
                d[u] = L[u] - du;
                d[w] = L[w] - dw;
                if (d[u] == 0 && d[w] == 0) continue;
                int M[3];
                for (int k = 0; k < 3; ++k) M[k] = L[k] - d[k];
                int e2 = -1;
                for (int f = 0; f < 12 && e2 < 0; ++f) {
                    int N[3], ax2 = 0;
                    for (int k = 0; k < 3; ++k) {
                        N[k] = std::min(kCornerOff[kEdgeEnds[f][0]][k], kCornerOff[kEdgeEnds[f][1]][k]);
                        if (kCornerOff[kEdgeEnds[f][0]][k] != kCornerOff[kEdgeEnds[f][1]][k]) ax2 = k;
                    }
                    if (ax2 == axis && N[0] == M[0] && N[1] == M[1] && N[2] == M[2]) e2 = f;
                }
                t.nb[e][q++] = (d[0] + 1) | ((d[1] + 1) << 2) | ((d[2] + 1) << 4) | (e2 << 8);
            }
    }
    return t;
}

const McTable& mc_table() {
    static const McTable t = build_mc_table();
    return t;
}

__constant__ int8_t c_mc_tri[256][16];
__constant__ uint8_t c_mc_ntri[256];
__constant__ int c_mc_nb[12][3];
// corner offsets and edge endpoints for device code (same as kCornerOff, kEdgeEnds)
__constant__ int c_corner[8][3] = {{0, 0, 0}, {1, 0, 0}, {1, 1, 0}, {0, 1, 0},
                                   {0, 0, 1}, {1, 0, 1}, {1, 1, 1}, {0, 1, 1}};
__constant__ int c_edge[12][2] = {{0, 1}, {1, 2}, {2, 3}, {3, 0}, {4, 5}, {5, 6},
                                  {6, 7}, {7, 4}, {0, 4}, {1, 5}, {2, 6}, {3, 7}};

std::mutex g_mc_mu;
bool g_mc_ready[128] = {};

// Copies the triangle table into this device's constant memory (once per
// device, with that device current).
int ensure_tables(vlr_ctx* ctx) {
    const int dev = ctx->device;
    if (dev < 0 || dev >= 128) return set_error(ctx, VLR_ERR_INVALID, "device ordinal out of range");
    std::lock_guard<std::mutex> lock(g_mc_mu);
    if (!g_mc_ready[dev]) {
        const McTable& t = mc_table();
        DeviceGuard guard(dev);
        VLR_CUDA(ctx, guard.status);
        VLR_CUDA(ctx, cudaMemcpyToSymbol(c_mc_tri, t.tri, sizeof(t.tri)));
        VLR_CUDA(ctx, cudaMemcpyToSymbol(c_mc_ntri, t.ntri, sizeof(t.ntri)));
        VLR_CUDA(ctx, cudaMemcpyToSymbol(c_mc_nb, t.nb, sizeof(t.nb)));
        g_mc_ready[dev] = true;
    }
    return VLR_OK;
}

constexpr long long kAxisLim = 1ll << kKeyBits;
constexpr uint64_t kBadKey = ~0ull;

// x-major key of a tile (leaf coordinates relative to the grid's hash base):
// ascending keys are ascending (x, y, z), the reference's Coord order.
__host__ __device__ inline uint64_t tile_key(long long lx, long long ly, long long lz, const long long* base) {
    const long long rx = lx - base[0], ry = ly - base[1], rz = lz - base[2];
    if (rx < 0 || ry < 0 || rz < 0 || rx >= kAxisLim || ry >= kAxisLim || rz >= kAxisLim) return kBadKey;
    return ((uint64_t)rx << 42) | ((uint64_t)ry << 21) | (uint64_t)rz;
}

struct TileBase {
    long long b[3];
};

__global__ void k_mc_cand(const int4* __restrict__ origin, int n, TileBase tb, uint64_t* __restrict__ keys,
                          unsigned* __restrict__ lo, unsigned* __restrict__ idx, unsigned* __restrict__ err) {
    const int d[7][3] = {{0, 0, 0}, {-1, 0, 0}, {1, 0, 0}, {0, -1, 0}, {0, 1, 0}, {0, 0, -1}, {0, 0, 1}};
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < 7ll * n;
         i += (long long)gridDim.x * blockDim.x) {
        const int s = (int)(i / 7), j = (int)(i % 7);
        const int4 o = origin[s];
        uint64_t k = tile_key((long long)(o.x >> 3) + d[j][0], (long long)(o.y >> 3) + d[j][1],
                              (long long)(o.z >> 3) + d[j][2], tb.b);
        if (k == kBadKey) atomicOr(err, kErrExtent);
        keys[i] = k;
        lo[i] = (unsigned)k;
        idx[i] = (unsigned)i;
    }
}

__global__ void k_mc_hi(const uint64_t* __restrict__ keys, const unsigned* __restrict__ idx, int n,
                        unsigned* __restrict__ hi) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        hi[i] = (unsigned)(keys[idx[i]] >> 32);
}

__global__ void k_mc_unique(const uint64_t* __restrict__ keys, const unsigned* __restrict__ idx, int n,
                            uint64_t* __restrict__ sorted, int* __restrict__ flag) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const uint64_t k = keys[idx[i]];
        sorted[i] = k;
        flag[i] = (k != kBadKey && (i == 0 || k != keys[idx[i - 1]])) ? 1 : 0;
    }
}

__global__ void k_mc_compact(const uint64_t* __restrict__ sorted, const int* __restrict__ flag,
                             const int* __restrict__ pos, int n, uint64_t* __restrict__ tiles) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        if (flag[i]) tiles[pos[i]] = sorted[i];
}

__global__ void k_mc_hash_clear(uint64_t* key, int* val, int cap) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < cap; i += gridDim.x * blockDim.x) {
        key[i] = kEmptyKey;
        val[i] = -1;
    }
}

__global__ void k_mc_hash_insert(const uint64_t* __restrict__ tiles, int m, uint64_t* hkey, int* hval, int cap,
                                 unsigned* err) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < m; i += gridDim.x * blockDim.x) {
        const uint64_t k = tiles[i];
        const uint32_t msk = (uint32_t)cap - 1u;
        uint32_t p = (uint32_t)mix64(k) & msk;
        bool done = false;
        for (int probe = 0; probe < cap && !done; ++probe) {
            const unsigned long long prev = atomicCAS((unsigned long long*)&hkey[p], kEmptyKey, k);
            if (prev == kEmptyKey || prev == k) {
                hval[p] = i;
                done = true;
            }
            p = (p + 1u) & msk;
        }
        if (!done) atomicOr(err, kErrHashFull);
    }
}

// ---------------------------------------------------------------- cells

struct TileCtx {
    long long o[3];  // voxel origin of the tile
};

// Tile ranks of the 27 neighbour tiles (-1: not processed) and the tile's
// 9^3 corner block (the tile's cells and the +1 layer), shared by both passes.
__device__ inline void stage_tile(const GridView& g, const HashView& th, uint64_t key, const long long* base,
                                  float* s_v, int* s_leaf, int* s_tr, TileCtx& tc) {
    const long long tx = (long long)(key >> 42) + base[0];
    const long long ty = (long long)((key >> 21) & (kAxisLim - 1)) + base[1];
    const long long tz = (long long)(key & (kAxisLim - 1)) + base[2];
    tc.o[0] = tx * 8;
    tc.o[1] = ty * 8;
    tc.o[2] = tz * 8;
    const int t = threadIdx.x;
    if (t < 8) s_leaf[t] = hash_find_leaf(g.hash, tx + (t >> 2), ty + ((t >> 1) & 1), tz + (t & 1));
    if (t >= 32 && t < 32 + 27) {
        const int q = t - 32;
        const uint64_t k = tile_key(tx + q / 9 - 1, ty + (q / 3) % 3 - 1, tz + q % 3 - 1, base);
        s_tr[q] = (k == kBadKey) ? -1 : hash_find(th, k);
    }
    __syncthreads();
    for (int i = t; i < 729; i += blockDim.x) {
        const int x = i / 81, y = (i / 9) % 9, z = i % 9;
        const int slot = s_leaf[((x >> 3) << 2) | ((y >> 3) << 1) | (z >> 3)];
        s_v[i] = slot >= 0 ? g.values[(size_t)slot * kLeafVoxels + voxel_off(x, y, z)] : g.background;
    }
    __syncthreads();
}

// Another cell holding the edge: its tile offset (-1..1 per axis) and local
// cell coordinates; `order` compares it with the current cell in visit order
// (negative: visited earlier).
struct CellRef {
    int toff[3];
    int loc[3];
};

__device__ inline CellRef cell_at(const int* loc, const int* delta) {
    CellRef r;
    for (int k = 0; k < 3; ++k) {
        const int v = loc[k] + delta[k];
        r.toff[k] = v < 0 ? -1 : (v > 7 ? 1 : 0);
        r.loc[k] = v & 7;
    }
    return r;
}

__device__ inline CellRef loc_self(const int* loc) {
    const int zero[3] = {0, 0, 0};
    return cell_at(loc, zero);
}

__device__ inline int tr_index(const int* toff) { return (toff[0] + 1) * 9 + (toff[1] + 1) * 3 + (toff[2] + 1); }

// lexicographic comparison of (tile offset, local cell) pairs
__device__ inline bool visited_before(const CellRef& a, const CellRef& b) {
    for (int k = 0; k < 3; ++k)
        if (a.toff[k] != b.toff[k]) return a.toff[k] < b.toff[k];
    for (int k = 0; k < 3; ++k)
        if (a.loc[k] != b.loc[k]) return a.loc[k] < b.loc[k];
    return false;
}

// The other cell holding edge e of the cell at `loc` listed q-th in c_mc_nb,
// and the edge's index there.
__device__ inline CellRef edge_nb(int e, int q, const int* loc, int& e2) {
    const int code = c_mc_nb[e][q];
    const int delta[3] = {(code & 3) - 1, ((code >> 2) & 3) - 1, ((code >> 4) & 3) - 1};
    e2 = code >> 8;
    return cell_at(loc, delta);
}

// Block-wide exclusive scan of one int per thread (512 threads).
__device__ inline int block_scan512(int v, int* s_w, int* total) {
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    int x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) s_w[w] = x;
    __syncthreads();
    if (w == 0) {
        int s = lane < 16 ? s_w[lane] : 0;
#pragma unroll
        for (int o = 1; o < 16; o <<= 1) {
            const int y = __shfl_up_sync(0xffffffffu, s, o);
            if (lane >= o) s += y;
        }
        if (lane < 16) s_w[lane] = s;
    }
    __syncthreads();
    const int before = (w > 0 ? s_w[w - 1] : 0) + x - v;
    *total = s_w[15];
    __syncthreads();
    return before;
}

__device__ inline int cell_case(const float* s_v, const int* loc, float iso) {
    int ci = 0;
#pragma unroll
    for (int i = 0; i < 8; ++i) {
        const float v = s_v[(loc[0] + c_corner[i][0]) * 81 + (loc[1] + c_corner[i][1]) * 9 + loc[2] + c_corner[i][2]];
        if (v < iso) ci |= 1 << i;
    }
    return ci;
}

__device__ inline unsigned edge_flags(int ci) {
    unsigned m = 0;
#pragma unroll
    for (int e = 0; e < 12; ++e) m |= (unsigned)(((ci >> c_edge[e][0]) ^ (ci >> c_edge[e][1])) & 1) << e;
    return m;
}

__global__ void __launch_bounds__(512) k_mc_classify(GridView g, HashView th, TileBase tb,
                                                    const uint64_t* __restrict__ tiles, float iso,
                                                    uint32_t* __restrict__ words, int* __restrict__ vcount,
                                                    int* __restrict__ tcount) {
    __shared__ float s_v[729];
    __shared__ int s_leaf[8], s_tr[27], s_w[16];
    TileCtx tc;
    stage_tile(g, th, tiles[blockIdx.x], tb.b, s_v, s_leaf, s_tr, tc);
    const int c = threadIdx.x;
    const int loc[3] = {c >> 6, (c >> 3) & 7, c & 7};
    const int ci = cell_case(s_v, loc, iso);
    const unsigned fl = edge_flags(ci);
    // this cell creates a flagged edge iff no other processed cell holding it
    // is visited earlier
    const int zero[3] = {0, 0, 0};
    const CellRef self = cell_at(loc, zero);
    unsigned cm = 0;
    for (int e = 0; e < 12; ++e) {
        if (!((fl >> e) & 1u)) continue;
        bool first = true;
        for (int q = 0; q < 3 && first; ++q) {
            int e2;
            const CellRef c = edge_nb(e, q, loc, e2);
            if (s_tr[tr_index(c.toff)] >= 0 && visited_before(c, self)) first = false;
        }
        if (first) cm |= 1u << e;
    }
    int vt = 0, tt = 0;
    const int vpre = block_scan512(__popc(cm), s_w, &vt);
    block_scan512(c_mc_ntri[ci], s_w, &tt);
    words[(size_t)blockIdx.x * 512 + c] = (uint32_t)ci | (cm << 8) | ((uint32_t)vpre << 20);
    if (c == 0) {
        vcount[blockIdx.x] = vt;
        tcount[blockIdx.x] = tt;
    }
}

__global__ void __launch_bounds__(512) k_mc_emit(GridView g, HashView th, TileBase tb,
                                                const uint64_t* __restrict__ tiles, float iso, double vs,
                                                const uint32_t* __restrict__ words, const int* __restrict__ vbase,
                                                const int* __restrict__ tbase, double* __restrict__ verts,
                                                uint32_t* __restrict__ tris) {
    __shared__ float s_v[729];
    __shared__ int s_leaf[8], s_tr[27], s_w[16];
    TileCtx tc;
    stage_tile(g, th, tiles[blockIdx.x], tb.b, s_v, s_leaf, s_tr, tc);
    const int c = threadIdx.x;
    const int loc[3] = {c >> 6, (c >> 3) & 7, c & 7};
    const uint32_t wd = words[(size_t)blockIdx.x * 512 + c];
    const int ci = (int)(wd & 255u);
    const unsigned cm = (wd >> 8) & 0xfffu;
    const int vpre = (int)(wd >> 20);
    const int nt = c_mc_ntri[ci];
    int tt = 0;
    const int tpre = block_scan512(nt, s_w, &tt);
    if (nt == 0) return;
    const int vb = vbase[blockIdx.x];
    const unsigned fl = edge_flags(ci);
    uint32_t ev[12];
    for (int e = 0; e < 12; ++e) {
        if (!((fl >> e) & 1u)) continue;
        if ((cm >> e) & 1u) {
            const uint32_t vi = (uint32_t)(vb + vpre + __popc(cm & ((1u << e) - 1u)));
            ev[e] = vi;
            const int a = c_edge[e][0], b = c_edge[e][1];
            const float va = s_v[(loc[0] + c_corner[a][0]) * 81 + (loc[1] + c_corner[a][1]) * 9 + loc[2] +
                                 c_corner[a][2]];
            const float vbv = s_v[(loc[0] + c_corner[b][0]) * 81 + (loc[1] + c_corner[b][1]) * 9 + loc[2] +
                                  c_corner[b][2]];
            const float d = __fsub_rn(vbv, va);
            const double t = (fabsf(d) > 1e-10f) ? (double)__fdiv_rn(__fsub_rn(iso, va), d) : 0.5;
#pragma unroll
            for (int k = 0; k < 3; ++k) {
                const double pa = __dmul_rn((double)(tc.o[k] + loc[k] + c_corner[a][k]), vs);
                const double pb = __dmul_rn((double)(tc.o[k] + loc[k] + c_corner[b][k]), vs);
                verts[(size_t)vi * 3 + k] = __dadd_rn(pa, __dmul_rn(t, __dsub_rn(pb, pa)));
            }
        } else {
            // the creator: the earliest processed other cell holding the edge
            int e2 = -1;
            CellRef cr = loc_self(loc);
            bool have = false;
            for (int q = 0; q < 3; ++q) {
                int f;
                const CellRef c = edge_nb(e, q, loc, f);
                if (s_tr[tr_index(c.toff)] < 0) continue;
                if (!have || visited_before(c, cr)) {
                    cr = c;
                    e2 = f;
                    have = true;
                }
            }
            const int rank = s_tr[tr_index(cr.toff)];
            const uint32_t w2 = words[(size_t)rank * 512 + (cr.loc[0] << 6) + (cr.loc[1] << 3) + cr.loc[2]];
            const unsigned cm2 = (w2 >> 8) & 0xfffu;
            ev[e] = (uint32_t)(vbase[rank] + (int)(w2 >> 20) + __popc(cm2 & ((1u << e2) - 1u)));
        }
    }
    const size_t t0 = (size_t)tbase[blockIdx.x] + tpre;
    for (int k = 0; k < nt; ++k)
        for (int j = 0; j < 3; ++j) tris[(t0 + k) * 3 + j] = ev[c_mc_tri[ci][3 * k + j]];
}

__global__ void k_mc_total(const int* cnt, const int* base, int m, long long* out) {
    out[0] = (long long)base[m - 1] + cnt[m - 1];
}

}  // namespace

int volume_to_mesh(vlr_ctx* ctx, const vlr_grid* g, float iso, double* h_verts, size_t cap_v, uint32_t* h_tris,
                   size_t cap_t, size_t* n_verts, size_t* n_tris) {
    *n_verts = 0;
    *n_tris = 0;
    if (g->n == 0) return VLR_OK;
    int rc = ensure_tables(ctx);
    if (rc) return rc;
    cudaStream_t st = ctx->stream;
    const int n7 = 7 * g->n;
    if (g->n > (1 << 27)) return set_error(ctx, VLR_ERR_CAPACITY, "volume_to_mesh: too many leaves");
    TileBase tb;
    for (int a = 0; a < 3; ++a) tb.b[a] = g->base[a];
    const int thr = 256, blocks = ctx->sm_count * 8;
    // candidates and their sort
    const size_t sort_bytes = sort_reduce_scratch_bytes(n7);
    char* buf = nullptr;
    const size_t cand_bytes = (size_t)n7 * (8 + 4 + 4 + 4 + 8 + 4 + 4) + sort_bytes + 256;
    VLR_CUDA(ctx, cudaMallocFromPoolAsync((void**)&buf, cand_bytes, ctx->pool, st));
    char* p = buf;
    uint64_t* keys = (uint64_t*)p;  p += (size_t)n7 * 8;
    uint64_t* sorted = (uint64_t*)p;  p += (size_t)n7 * 8;
    unsigned* lo = (unsigned*)p;  p += (size_t)n7 * 4;
    unsigned* idx = (unsigned*)p;  p += (size_t)n7 * 4;
    int* flag = (int*)p;  p += (size_t)n7 * 4;
    int* pos = (int*)p;  p += (size_t)n7 * 4 + 16;
    void* scratch = (void*)(((uintptr_t)p + 15) & ~(uintptr_t)15);
    auto done = [&](int code) {
        cudaFreeAsync(buf, st);
        return code;
    };
    // 63-bit keys sorted as two stable 32-bit passes carrying the candidate index
    k_mc_cand<<<blocks, thr, 0, st>>>(g->origin, g->n, tb, keys, lo, idx, ctx->d_errword);
    unsigned *k1, *v1, *k2, *v2;
    rc = radix_sort_pairs(ctx, lo, idx, n7, 0xffffffffu, scratch, &k1, &v1);
    if (rc) return done(rc);
    // high words in candidate order of the first pass; the order array moves
    // out of the scratch (if it ended there) before the second pass reuses it
    unsigned* hi = (unsigned*)flag;
    k_mc_hi<<<blocks, thr, 0, st>>>(keys, v1, n7, hi);
    if (v1 != idx) VLR_CUDA(ctx, cudaMemcpyAsync(idx, v1, (size_t)n7 * 4, cudaMemcpyDeviceToDevice, st));
    rc = radix_sort_pairs(ctx, hi, idx, n7, 0x7fffffffu, scratch, &k2, &v2);
    if (rc) return done(rc);
    (void)k1;
    (void)k2;
    // v2 is the final order; flag (the high words) is rewritten here as unique flags
    k_mc_unique<<<blocks, thr, 0, st>>>(keys, v2, n7, sorted, flag);
    rc = scan_exclusive(ctx, flag, pos, n7, pos + n7);
    if (rc) return done(rc);
    int m = 0;
    rc = read_int(ctx, pos + n7, &m);
    if (rc) return done(rc);
    rc = consume_device_errors(ctx, "volume_to_mesh");
    if (rc) return done(rc);
    if (m <= 0) return done(VLR_OK);
    // tile list, tile hash, per-cell words and per-tile counts
    int hcap = 64;
    while (hcap < 2 * m) hcap <<= 1;
    char* buf2 = nullptr;
    const size_t b2 = (size_t)m * 8 + (size_t)hcap * 12 + (size_t)m * 512 * 4 + (size_t)m * 16 + 64 + 256;
    cudaError_t ce = cudaMallocFromPoolAsync((void**)&buf2, b2, ctx->pool, st);
    if (ce != cudaSuccess) return done(check_cuda(ctx, ce, "cudaMallocFromPoolAsync(volume_to_mesh cells)"));
    auto done2 = [&](int code) {
        cudaFreeAsync(buf2, st);
        return done(code);
    };
    p = buf2;
    uint64_t* tiles = (uint64_t*)p;  p += (size_t)m * 8;
    uint64_t* hkey = (uint64_t*)p;  p += (size_t)hcap * 8;
    int* hval = (int*)p;  p += (size_t)hcap * 4;
    uint32_t* words = (uint32_t*)p;  p += (size_t)m * 512 * 4;
    int* vcount = (int*)p;  p += (size_t)m * 4;
    int* tcount = (int*)p;  p += (size_t)m * 4;
    int* vbase = (int*)p;  p += (size_t)m * 4 + 16;
    int* tbase = (int*)p;  p += (size_t)m * 4 + 16;
    long long* totals = (long long*)(((uintptr_t)p + 15) & ~(uintptr_t)15);
    k_mc_compact<<<blocks, thr, 0, st>>>(sorted, flag, pos, n7, tiles);
    k_mc_hash_clear<<<blocks, thr, 0, st>>>(hkey, hval, hcap);
    k_mc_hash_insert<<<blocks, thr, 0, st>>>(tiles, m, hkey, hval, hcap, ctx->d_errword);
    GridView gv = make_view(g);
    HashView th;
    th.key = hkey;
    th.val = hval;
    th.cap = hcap;
    for (int a = 0; a < 3; ++a) th.base[a] = 0;
    VLR_TIMED(ctx, "k_mc_classify",
              k_mc_classify<<<m, 512, 0, st>>>(gv, th, tb, tiles, iso, words, vcount, tcount));
    rc = scan_exclusive(ctx, vcount, vbase, m, vbase + m);
    if (!rc) rc = scan_exclusive(ctx, tcount, tbase, m, tbase + m);
    if (rc) return done2(rc);
    k_mc_total<<<1, 1, 0, st>>>(vcount, vbase, m, totals);
    k_mc_total<<<1, 1, 0, st>>>(tcount, tbase, m, totals + 1);
    long long tot[2] = {0, 0};
    VLR_CUDA(ctx, cudaMemcpyAsync(tot, totals, sizeof(tot), cudaMemcpyDeviceToHost, st));
    VLR_CUDA(ctx, cudaStreamSynchronize(st));
    rc = consume_device_errors(ctx, "volume_to_mesh");
    if (rc) return done2(rc);
    *n_verts = (size_t)tot[0];
    *n_tris = (size_t)tot[1];
    if (tot[0] > 0x7fffffffll || tot[1] > 0x7fffffffll)
        return done2(set_error(ctx, VLR_ERR_CAPACITY, "volume_to_mesh: more than 2^31 vertices or triangles"));
    if ((h_verts && cap_v) || (h_tris && cap_t)) {
        double* d_verts = nullptr;
        uint32_t* d_tris = nullptr;
        ce = cudaMallocFromPoolAsync((void**)&d_verts, (size_t)std::max<long long>(tot[0], 1) * 24, ctx->pool, st);
        if (ce == cudaSuccess)
            ce = cudaMallocFromPoolAsync((void**)&d_tris, (size_t)std::max<long long>(tot[1], 1) * 12, ctx->pool, st);
        if (ce != cudaSuccess) return done2(check_cuda(ctx, ce, "cudaMallocFromPoolAsync(volume_to_mesh output)"));
        VLR_TIMED(ctx, "k_mc_emit",
                  k_mc_emit<<<m, 512, 0, st>>>(gv, th, tb, tiles, iso, g->xf.voxel_size, words, vbase, tbase,
                                               d_verts, d_tris));
        const size_t cv = std::min<size_t>(cap_v, (size_t)tot[0]), ct = std::min<size_t>(cap_t, (size_t)tot[1]);
        ce = cudaGetLastError();
        if (ce != cudaSuccess) {
            cudaFreeAsync(d_verts, st);
            cudaFreeAsync(d_tris, st);
            return done2(check_cuda(ctx, ce, "volume_to_mesh output"));
        }
        int rc2 = VLR_OK;
        if (h_verts && cv) rc2 = d2h_copy(ctx, h_verts, d_verts, cv * 24);
        if (!rc2 && h_tris && ct) rc2 = d2h_copy(ctx, h_tris, d_tris, ct * 12);
        cudaFreeAsync(d_verts, st);
        cudaFreeAsync(d_tris, st);
        if (rc2) return done2(rc2);
        rc = consume_device_errors(ctx, "volume_to_mesh");
        if (rc) return done2(rc);
    }
    return done2(VLR_OK);
}

int mc_triangle_table(int8_t* out) {
    std::memcpy(out, mc_table().tri, sizeof(mc_table().tri));
    return VLR_OK;
}

}  // namespace vlr

extern "C" {

int vlr_volume_to_mesh(vlr_ctx* ctx, const vlr_grid* g, float isovalue, double* vertices, size_t cap_vertices,
                       uint32_t* triangles, size_t cap_triangles, size_t* n_vertices, size_t* n_triangles) {
    using namespace vlr;
    if (!ctx || !g || !n_vertices || !n_triangles) return set_error(ctx, VLR_ERR_INVALID, "null argument");
    if (g->kind != VLR_KIND_F32_WORLD) return set_error(ctx, VLR_ERR_INVALID, "grid is not a world-unit f32 grid");
    return volume_to_mesh(ctx, g, isovalue, vertices, cap_vertices, triangles, cap_triangles, n_vertices,
                          n_triangles);
}

int vlr_mc_triangle_table(int8_t* out) {
    if (!out) return VLR_ERR_INVALID;
    return vlr::mc_triangle_table(out);
}

}  // extern "C"
