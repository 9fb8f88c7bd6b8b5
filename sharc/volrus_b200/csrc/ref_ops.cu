// Reference-semantics kernels: the Sharc.Volrus advection step on flat device
// leaves, bit-exact with the crate's CPU code.
//   k_advect_ref      advect_level_set            src/tools/advection.rs:32-56
//   k_sample_points   sample_trilinear            src/tools/interpolation.rs:11-48
//   k_crossings       find_zero_crossings         src/tools/level_set_track.rs:14-47
//   k_rebuild_window  rebuild_narrow_band         src/tools/level_set_track.rs:80-114
//   k_rebuild_brute   (same, any half-width)
//   k_trim            trim_narrow_band            src/tools/level_set_track.rs:53-68
//   k_sphere          make_level_set_sphere       src/tools/sphere.rs:17-59
// One CTA works on one 8^3 leaf; activity masks are produced with warp ballots.
#include <algorithm>
#include <climits>
#include <cmath>
#include <cstring>
#include <vector>

#include "ref_ops.hpp"
#include "sort_reduce.hpp"

namespace vlr {

// ------------------------------------------------------------- advection

// One CTA per leaf, 128 threads, 4 voxels per thread.  Velocity comes from
// three grids (VelocityField::sample, src/tools/advection.rs:18-24).  The
// output keeps the input's activity mask; inactive voxels read background
// (the leaf is freshly allocated in the reference, src/tree/internal.rs:127-143).
__global__ void __launch_bounds__(128) k_advect_ref(GridView g, GridView vx, GridView vy, GridView vz, double dt,
                                                   float* __restrict__ out_values, uint64_t* __restrict__ out_mask,
                                                   int* __restrict__ nonempty) {
    int slot = blockIdx.x;
    if (slot >= g.n) return;
    int4 o = g.origin[slot];
    const uint64_t* m = g.mask + (size_t)slot * 8;
    int hlx = o.x >> 3, hly = o.y >> 3, hlz = o.z >> 3;
    bool any = false;
    for (int r = 0; r < 4; ++r) {
        int off = threadIdx.x + 128 * r;
        bool on = mask_bit(m, off);
        float outv = g.background;
        if (on) {
            any = true;
            int x = o.x + (off >> 6), y = o.y + ((off >> 3) & 7), z = o.z + (off & 7);
            double w[3];
            index_to_world_ref(g.mat, x, y, z, w);
            double v0 = (double)sample_trilinear_ref(vx, w[0], w[1], w[2]);
            double v1 = (double)sample_trilinear_ref(vy, w[0], w[1], w[2]);
            double v2 = (double)sample_trilinear_ref(vz, w[0], w[1], w[2]);
            double px = __dsub_rn(w[0], __dmul_rn(dt, v0));
            double py = __dsub_rn(w[1], __dmul_rn(dt, v1));
            double pz = __dsub_rn(w[2], __dmul_rn(dt, v2));
            outv = sample_trilinear_ref(g, px, py, pz, slot, hlx, hly, hlz);
        }
        out_values[(size_t)slot * kLeafVoxels + off] = outv;
    }
    if (threadIdx.x < 8) out_mask[(size_t)slot * 8 + threadIdx.x] = m[threadIdx.x];
    int a = __syncthreads_or(any);
    if (threadIdx.x == 0) nonempty[slot] = a;
}

__global__ void k_sample_points(GridView g, const double* __restrict__ pts, int n, float* __restrict__ out) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    out[i] = sample_trilinear_ref(g, pts[3 * i], pts[3 * i + 1], pts[3 * i + 2]);
}

// ------------------------------------------------------- zero crossings

// Value and activity of voxel (x, y, z) given in the local frame of leaf
// `slot` (coordinates may leave the leaf by one voxel).
__device__ inline void local_get(const GridView& g, int slot, int x, int y, int z, float& v, bool& on) {
    int dx = (x < 0) ? -1 : (x > 7 ? 1 : 0);
    int dy = (y < 0) ? -1 : (y > 7 ? 1 : 0);
    int dz = (z < 0) ? -1 : (z > 7 ? 1 : 0);
    int s = slot;
    if (dx | dy | dz) s = g.nbr[slot * kNbr + (dx + 1) * 9 + (dy + 1) * 3 + (dz + 1)];
    if (s < 0) {
        v = g.background;
        on = false;
        return;
    }
    int off = voxel_off(x, y, z);
    v = g.values[(size_t)s * kLeafVoxels + off];
    on = mask_bit(g.mask + (size_t)s * 8, off);
}

// 256 threads, voxels tid and tid+256.  Writes the crossing mask (same bit
// layout as the activity mask) and the per-leaf crossing count.
__global__ void __launch_bounds__(256) k_crossings(GridView g, uint64_t* __restrict__ xmask, int* __restrict__ xcount,
                                                  unsigned long long* __restrict__ total) {
    int slot = blockIdx.x;
    if (slot >= g.n) return;
    const uint64_t* m = g.mask + (size_t)slot * 8;
    int cnt = 0;
    for (int r = 0; r < 2; ++r) {
        int off = threadIdx.x + 256 * r;
        bool cross = false;
        if (mask_bit(m, off)) {
            float val = g.values[(size_t)slot * kLeafVoxels + off];
            if (val == 0.0f) {
                cross = true;
            } else {
                int x = off >> 6, y = (off >> 3) & 7, z = off & 7;
                const int ddx[6] = {1, -1, 0, 0, 0, 0};
                const int ddy[6] = {0, 0, 1, -1, 0, 0};
                const int ddz[6] = {0, 0, 0, 0, 1, -1};
#pragma unroll
                for (int q = 0; q < 6; ++q) {
                    float nv;
                    bool non;
                    local_get(g, slot, x + ddx[q], y + ddy[q], z + ddz[q], nv, non);
                    if (non && __fmul_rn(val, nv) < 0.0f) {
                        cross = true;
                        break;
                    }
                }
            }
        }
        unsigned b = __ballot_sync(0xffffffffu, cross);
        if ((threadIdx.x & 31) == 0) {
            ((unsigned*)xmask)[(size_t)slot * 16 + (off >> 5)] = b;
            cnt += __popc(b);
        }
    }
    __shared__ int s_cnt;
    if (threadIdx.x == 0) s_cnt = 0;
    __syncthreads();
    if ((threadIdx.x & 31) == 0 && cnt) atomicAdd(&s_cnt, cnt);
    __syncthreads();
    if (threadIdx.x == 0) {
        xcount[slot] = s_cnt;
        if (s_cnt) atomicAdd(total, (unsigned long long)s_cnt);
    }
}

// Write crossing coordinates of each leaf at its scanned position.
__global__ void __launch_bounds__(512) k_emit_crossings(GridView g, const uint64_t* __restrict__ xmask,
                                                       const int* __restrict__ pos, int* __restrict__ coords) {
    int slot = blockIdx.x;
    if (slot >= g.n) return;
    int off = threadIdx.x;
    const uint64_t* xm = xmask + (size_t)slot * 8;
    bool on = mask_bit(xm, off);
    // rank of this bit among the leaf's set bits
    int w = off >> 6, b = off & 63;
    int rank = 0;
    for (int q = 0; q < w; ++q) rank += __popcll(xm[q]);
    rank += __popcll(xm[w] & ((b == 0) ? 0ull : (~0ull >> (64 - b))));
    if (on) {
        int4 o = g.origin[slot];
        int j = pos[slot] + rank;
        coords[3 * j] = o.x + (off >> 6);
        coords[3 * j + 1] = o.y + ((off >> 3) & 7);
        coords[3 * j + 2] = o.z + (off & 7);
    }
}

// --------------------------------------------------------------- rebuild

// Nearest crossing by squared index distance inside a cube window of half
// size R <= 8, using the crossing masks of the 27 neighbouring leaves staged
// in shared memory.  A z-row of 8 voxels is one byte of a mask, so each
// (dx, dy) pair of the window is one 24-bit row test.
__global__ void __launch_bounds__(256) k_rebuild_window(GridView g, float* __restrict__ values,
                                                       uint64_t* __restrict__ mask, const uint64_t* __restrict__ xmask,
                                                       int R, float vs, float band, int* __restrict__ nonempty) {
    __shared__ uint64_t s_x[kNbr * 8];
    int slot = blockIdx.x;
    if (slot >= g.n) return;
    for (int t = threadIdx.x; t < kNbr * 8; t += blockDim.x) {
        int d = t >> 3;
        int s = g.nbr[slot * kNbr + d];
        s_x[t] = (s < 0) ? 0ull : xmask[(size_t)s * 8 + (t & 7)];
    }
    __syncthreads();
    const unsigned char* sb = (const unsigned char*)s_x;  // leaf d occupies bytes [64d, 64d+64)
    uint64_t* m = mask + (size_t)slot * 8;
    bool keep_any = false;
    for (int r = 0; r < 2; ++r) {
        int off = threadIdx.x + 256 * r;
        bool on = mask_bit(m, off);
        bool keep = false;
        if (on) {
            int x = off >> 6, y = (off >> 3) & 7, z = off & 7;
            int best = INT_MAX;
            for (int dx = -R; dx <= R; ++dx) {
                int xx = x + dx;
                int lxo = (xx < 0) ? 0 : (xx > 7 ? 2 : 1);
                int xl = xx & 7;
                for (int dy = -R; dy <= R; ++dy) {
                    int dxy = dx * dx + dy * dy;
                    if (dxy >= best) continue;
                    int yy = y + dy;
                    int lyo = (yy < 0) ? 0 : (yy > 7 ? 2 : 1);
                    int yl = yy & 7;
                    int dbase = lxo * 9 + lyo * 3;
                    int byte_idx = xl * 8 + yl;
                    unsigned row = (unsigned)sb[(dbase + 0) * 64 + byte_idx] |
                                   ((unsigned)sb[(dbase + 1) * 64 + byte_idx] << 8) |
                                   ((unsigned)sb[(dbase + 2) * 64 + byte_idx] << 16);
                    int c = z + 8;
                    unsigned lo_mask = (2u << c) - 1u;                      // bits <= c
                    unsigned win = ((c + R + 1 >= 32) ? 0xffffffffu : ((1u << (c + R + 1)) - 1u)) &
                                   ~((c - R <= 0) ? 0u : ((1u << (c - R)) - 1u));
                    unsigned wr = row & win;
                    if (!wr) continue;
                    int dz = 32;
                    unsigned lo = wr & lo_mask;
                    if (lo) dz = c - (31 - __clz(lo));
                    unsigned hi = wr >> c;
                    if (hi) dz = min(dz, __ffs(hi) - 1);
                    int d2 = dxy + dz * dz;
                    if (d2 < best) best = d2;
                }
            }
            if (best != INT_MAX) {
                float old = values[(size_t)slot * kLeafVoxels + off];
                float sign = (old >= 0.0f) ? 1.0f : -1.0f;
                float md = __fsqrt_rn((float)best);
                float nv = __fmul_rn(__fmul_rn(sign, md), vs);
                if (fabsf(nv) < band) {
                    keep = true;
                    values[(size_t)slot * kLeafVoxels + off] = nv;
                }
            }
            if (!keep) values[(size_t)slot * kLeafVoxels + off] = g.background;
        }
        unsigned b = __ballot_sync(0xffffffffu, keep);
        if ((threadIdx.x & 31) == 0) ((unsigned*)m)[off >> 5] = b;
        keep_any |= keep;
    }
    int a = __syncthreads_or(keep_any);
    if (threadIdx.x == 0) nonempty[slot] = a;
}

// Literal form of the reference loop for any half-width: f32 distances to
// every crossing, folded with min.
__global__ void __launch_bounds__(256) k_rebuild_brute(GridView g, float* __restrict__ values,
                                                      uint64_t* __restrict__ mask, const int* __restrict__ cross,
                                                      int n_cross, float vs, float band, int* __restrict__ nonempty) {
    int slot = blockIdx.x;
    if (slot >= g.n) return;
    int4 o = g.origin[slot];
    uint64_t* m = mask + (size_t)slot * 8;
    bool keep_any = false;
    for (int r = 0; r < 2; ++r) {
        int off = threadIdx.x + 256 * r;
        bool keep = false;
        if (mask_bit(m, off)) {
            int x = o.x + (off >> 6), y = o.y + ((off >> 3) & 7), z = o.z + (off & 7);
            float md = 3.402823466e+38f;
            for (int c = 0; c < n_cross; ++c) {
                float dx = __int2float_rn((int)((unsigned)x - (unsigned)cross[3 * c]));
                float dy = __int2float_rn((int)((unsigned)y - (unsigned)cross[3 * c + 1]));
                float dz = __int2float_rn((int)((unsigned)z - (unsigned)cross[3 * c + 2]));
                float d = __fsqrt_rn(__fadd_rn(__fadd_rn(__fmul_rn(dx, dx), __fmul_rn(dy, dy)), __fmul_rn(dz, dz)));
                md = fminf(md, d);
            }
            float old = values[(size_t)slot * kLeafVoxels + off];
            float sign = (old >= 0.0f) ? 1.0f : -1.0f;
            float nv = __fmul_rn(__fmul_rn(sign, md), vs);
            if (fabsf(nv) < band) {
                keep = true;
                values[(size_t)slot * kLeafVoxels + off] = nv;
            } else {
                values[(size_t)slot * kLeafVoxels + off] = g.background;
            }
        }
        unsigned b = __ballot_sync(0xffffffffu, keep);
        if ((threadIdx.x & 31) == 0) ((unsigned*)m)[off >> 5] = b;
        keep_any |= keep;
    }
    int a = __syncthreads_or(keep_any);
    if (threadIdx.x == 0) nonempty[slot] = a;
}

// ------------------------------------------------------------------ trim

__global__ void __launch_bounds__(256) k_trim(GridView g, float* __restrict__ values, uint64_t* __restrict__ mask,
                                             float thr, int* __restrict__ nonempty) {
    int slot = blockIdx.x;
    if (slot >= g.n) return;
    uint64_t* m = mask + (size_t)slot * 8;
    bool keep_any = false;
    for (int r = 0; r < 2; ++r) {
        int off = threadIdx.x + 256 * r;
        bool keep = false;
        if (mask_bit(m, off)) {
            float v = values[(size_t)slot * kLeafVoxels + off];
            if (fabsf(v) >= thr) values[(size_t)slot * kLeafVoxels + off] = g.background;
            else keep = true;
        }
        unsigned b = __ballot_sync(0xffffffffu, keep);
        if ((threadIdx.x & 31) == 0) ((unsigned*)m)[off >> 5] = b;
        keep_any |= keep;
    }
    int a = __syncthreads_or(keep_any);
    if (threadIdx.x == 0) nonempty[slot] = a;
}

// ---------------------------------------------------------------- sphere

// One CTA per candidate leaf of the sphere's index bounding box, leaves
// enumerated x-major (lexicographic origin order).
__global__ void __launch_bounds__(512) k_sphere(int lx0, int ly0, int lz0, int nly, int nlz, int n_cand, int imin,
                                               int jmin, int kmin, int imax, int jmax, int kmax, double radius,
                                               double c0, double c1, double c2, double vs, float bg,
                                               int4* __restrict__ origin, uint64_t* __restrict__ mask,
                                               float* __restrict__ values, int* __restrict__ nonempty) {
    int cand = blockIdx.x;
    if (cand >= n_cand) return;
    int lx = lx0 + cand / (nly * nlz);
    int ly = ly0 + (cand / nlz) % nly;
    int lz = lz0 + cand % nlz;
    int off = threadIdx.x;
    int i = lx * 8 + (off >> 6), j = ly * 8 + ((off >> 3) & 7), k = lz * 8 + (off & 7);
    bool on = false;
    float val = bg;
    if (i >= imin && i <= imax && j >= jmin && j <= jmax && k >= kmin && k <= kmax) {
        double wx = __dsub_rn(__dmul_rn((double)i, vs), c0);
        double wy = __dsub_rn(__dmul_rn((double)j, vs), c1);
        double wz = __dsub_rn(__dmul_rn((double)k, vs), c2);
        double dist = __dsqrt_rn(__dadd_rn(__dadd_rn(__dmul_rn(wx, wx), __dmul_rn(wy, wy)), __dmul_rn(wz, wz)));
        float sdf = __double2float_rn(__dsub_rn(dist, radius));
        if (fabsf(sdf) < bg) {
            on = true;
            val = sdf;
        }
    }
    values[(size_t)cand * kLeafVoxels + off] = val;
    unsigned b = __ballot_sync(0xffffffffu, on);
    if ((off & 31) == 0) ((unsigned*)(mask + (size_t)cand * 8))[off >> 5] = b;
    int a = __syncthreads_or(on);
    if (off == 0) {
        origin[cand] = make_int4(lx * 8, ly * 8, lz * 8, 0);
        nonempty[cand] = a;
    }
}

// ================================================================ host side

GridView make_view(const vlr_grid* g) {
    GridView v;
    v.origin = g->origin;
    v.mask = g->mask;
    v.values = (const float*)g->values;
    v.nbr = g->nbr;
    v.hash.key = g->hkey;
    v.hash.val = g->hval;
    v.hash.cap = g->hcap;
    for (int a = 0; a < 3; ++a) v.hash.base[a] = g->base[a];
    v.n = g->n;
    v.background = g->background;
    v.inv_vs = 1.0 / g->xf.voxel_size;
    for (int a = 0; a < 3; ++a) v.t_origin[a] = g->xf.origin[a];
    for (int q = 0; q < 12; ++q) v.mat[q] = g->xf.affine[q];
    return v;
}

int advect_ref(vlr_ctx* ctx, const vlr_grid* g, const vlr_grid* vx, const vlr_grid* vy, const vlr_grid* vz, double dt,
               vlr_grid* out) {
    out->ctx = ctx;
    out->kind = VLR_KIND_F32_WORLD;
    out->background = g->background;
    // Grid::with_affine keeps the affine and resets the legacy transform to
    // uniform(affine.voxel_size) (src/grid.rs:378-388).
    out->xf = g->xf;
    out->xf.voxel_size = g->xf.affine_voxel_size;
    out->xf.origin[0] = out->xf.origin[1] = out->xf.origin[2] = 0.0;
    for (int a = 0; a < 3; ++a) out->base[a] = g->base[a];
    int rc = grid_alloc(ctx, out, std::max(g->n, 1));
    if (rc) return rc;
    out->n = g->n;
    if (g->n == 0) return grid_index(ctx, out);
    int* nonempty = nullptr;
    VLR_CUDA(ctx, cudaMallocFromPoolAsync(&nonempty, sizeof(int) * g->n, ctx->pool, ctx->stream));
    VLR_CUDA(ctx, cudaMemcpyAsync(out->origin, g->origin, sizeof(int4) * g->n, cudaMemcpyDeviceToDevice, ctx->stream));
    VLR_TIMED(ctx, "k_advect_ref",
              k_advect_ref<<<g->n, 128, 0, ctx->stream>>>(make_view(g), make_view(vx), make_view(vy), make_view(vz),
                                                         dt, (float*)out->values, out->mask, nonempty));
    VLR_CUDA(ctx, cudaGetLastError());
    rc = grid_index(ctx, out);
    if (rc) return rc;
    rc = grid_compact(ctx, out, nonempty);
    if (rc) return rc;
    VLR_CUDA(ctx, cudaFreeAsync(nonempty, ctx->stream));
    return consume_device_errors(ctx, "advect_level_set");
}

int sample_points(vlr_ctx* ctx, const vlr_grid* g, const double* h_pts, size_t n, float* h_out) {
    if (n == 0) return VLR_OK;
    double* d_pts = nullptr;
    float* d_out = nullptr;
    VLR_CUDA(ctx, cudaMallocFromPoolAsync(&d_pts, sizeof(double) * 3 * n, ctx->pool, ctx->stream));
    VLR_CUDA(ctx, cudaMallocFromPoolAsync(&d_out, sizeof(float) * n, ctx->pool, ctx->stream));
    VLR_CUDA(ctx, cudaMemcpyAsync(d_pts, h_pts, sizeof(double) * 3 * n, cudaMemcpyHostToDevice, ctx->stream));
    k_sample_points<<<(unsigned)((n + 255) / 256), 256, 0, ctx->stream>>>(make_view(g), d_pts, (int)n, d_out);
    VLR_CUDA(ctx, cudaGetLastError());
    VLR_CUDA(ctx, cudaMemcpyAsync(h_out, d_out, sizeof(float) * n, cudaMemcpyDeviceToHost, ctx->stream));
    VLR_CUDA(ctx, cudaFreeAsync(d_pts, ctx->stream));
    VLR_CUDA(ctx, cudaFreeAsync(d_out, ctx->stream));
    VLR_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    return VLR_OK;
}

// Crossing masks and counts on the device; *total_out is the crossing count.
int crossings(vlr_ctx* ctx, const vlr_grid* g, uint64_t* d_xmask, int* d_xcount, unsigned long long* d_total,
              unsigned long long* total_out) {
    VLR_CUDA(ctx, cudaMemsetAsync(d_total, 0, sizeof(unsigned long long), ctx->stream));
    if (g->n > 0)
        VLR_TIMED(ctx, "k_crossings",
                  k_crossings<<<g->n, 256, 0, ctx->stream>>>(make_view(g), d_xmask, d_xcount, d_total));
    VLR_CUDA(ctx, cudaGetLastError());
    unsigned long long* h = (unsigned long long*)ctx->pinned;
    VLR_CUDA(ctx, cudaMemcpyAsync(h, d_total, sizeof(unsigned long long), cudaMemcpyDeviceToHost, ctx->stream));
    VLR_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    *total_out = *h;
    return VLR_OK;
}

struct CrossBufs {
    uint64_t* xmask = nullptr;
    int* xcount = nullptr;
    int* pos = nullptr;
    unsigned long long* total = nullptr;
    int* flags = nullptr;
};

static int alloc_cross(vlr_ctx* ctx, int n, CrossBufs& b) {
    size_t need = sizeof(uint64_t) * 8 * (size_t)n + sizeof(int) * (3 * (size_t)n + 8) + 64;
    char* p = nullptr;
    VLR_CUDA(ctx, cudaMallocFromPoolAsync((void**)&p, need, ctx->pool, ctx->stream));
    b.xmask = (uint64_t*)p;
    p += sizeof(uint64_t) * 8 * (size_t)n;
    b.total = (unsigned long long*)p;
    p += 16;
    b.xcount = (int*)p;
    p += sizeof(int) * ((size_t)n + 1);
    b.pos = (int*)p;
    p += sizeof(int) * ((size_t)n + 1);
    b.flags = (int*)p;
    return VLR_OK;
}

// Crossing-list sort on the device: the bounding box of the coordinates, then
// (x, y, z)-major keys of their offsets to it, sorted by two stable 32-bit
// radix passes (low word, then high word) that carry the list index.
__global__ void k_cross_box(const int* __restrict__ c, int n, int* __restrict__ box) {
    int lo[3] = {INT_MAX, INT_MAX, INT_MAX}, hi[3] = {INT_MIN, INT_MIN, INT_MIN};
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        for (int a = 0; a < 3; ++a) {
            lo[a] = min(lo[a], c[3 * i + a]);
            hi[a] = max(hi[a], c[3 * i + a]);
        }
    for (int a = 0; a < 3; ++a) {
        lo[a] = __reduce_min_sync(0xffffffffu, lo[a]);
        hi[a] = __reduce_max_sync(0xffffffffu, hi[a]);
    }
    if ((threadIdx.x & 31) == 0)
        for (int a = 0; a < 3; ++a) {
            atomicMin(&box[a], lo[a]);
            atomicMax(&box[3 + a], hi[a]);
        }
}

__global__ void k_cross_keys(const int* __restrict__ c, int n, int bx, int by, int bz, int bits,
                             uint64_t* __restrict__ keys, unsigned* __restrict__ lo, unsigned* __restrict__ idx) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const uint64_t k = ((uint64_t)(unsigned)(c[3 * i] - bx) << (2 * bits)) |
                           ((uint64_t)(unsigned)(c[3 * i + 1] - by) << bits) | (uint64_t)(unsigned)(c[3 * i + 2] - bz);
        keys[i] = k;
        lo[i] = (unsigned)k;
        idx[i] = (unsigned)i;
    }
}

__global__ void k_cross_hi(const uint64_t* __restrict__ keys, const unsigned* __restrict__ idx, int n,
                           unsigned* __restrict__ hi) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        hi[i] = (unsigned)(keys[idx[i]] >> 32);
}

__global__ void k_cross_gather(const int* __restrict__ c, const unsigned* __restrict__ idx, int n,
                               int* __restrict__ out) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < 3 * n; i += gridDim.x * blockDim.x)
        out[i] = c[3 * idx[i / 3] + i % 3];
}

// Sorts the n crossing coordinates d_c into d_out by (x, y, z) on the device;
// *sorted = false (nothing written) when the box needs keys over 63 bits.
static int sort_crossings_device(vlr_ctx* ctx, const int* d_c, int n, int* d_out, bool* sorted) {
    *sorted = false;
    cudaStream_t st = ctx->stream;
    const size_t sort_bytes = sort_reduce_scratch_bytes(n);
    char* buf = nullptr;
    VLR_CUDA(ctx, cudaMallocFromPoolAsync((void**)&buf, (size_t)n * 20 + sort_bytes + 256, ctx->pool, st));
    auto done = [&](int code) {
        cudaFreeAsync(buf, st);
        return code;
    };
    char* p = buf;
    uint64_t* keys = (uint64_t*)p;  p += (size_t)n * 8;
    unsigned* lo = (unsigned*)p;  p += (size_t)n * 4;
    unsigned* idx = (unsigned*)p;  p += (size_t)n * 4;
    unsigned* hi = (unsigned*)p;  p += (size_t)n * 4;
    int* box = (int*)(((uintptr_t)p + 15) & ~(uintptr_t)15);
    void* scratch = (void*)(((uintptr_t)(box + 8) + 15) & ~(uintptr_t)15);
    const int init[6] = {INT_MAX, INT_MAX, INT_MAX, INT_MIN, INT_MIN, INT_MIN};
    int* hb = static_cast<int*>(ctx->pinned) + 32;
    std::memcpy(hb, init, sizeof(init));
    VLR_CUDA(ctx, cudaMemcpyAsync(box, hb, sizeof(init), cudaMemcpyHostToDevice, st));
    const int blocks = ctx->sm_count * 8;
    k_cross_box<<<blocks, 256, 0, st>>>(d_c, n, box);
    VLR_CUDA(ctx, cudaMemcpyAsync(hb, box, sizeof(init), cudaMemcpyDeviceToHost, st));
    VLR_CUDA(ctx, cudaStreamSynchronize(st));
    int bits = 0;
    for (int a = 0; a < 3; ++a) {
        const long long ext = (long long)hb[3 + a] - hb[a];
        while (bits < 40 && (1ll << bits) <= ext) ++bits;
    }
    if (3 * bits > 63) return done(VLR_OK);
    k_cross_keys<<<blocks, 256, 0, st>>>(d_c, n, hb[0], hb[1], hb[2], bits, keys, lo, idx);
    unsigned *k1, *v1, *k2, *v2;
    int rc = radix_sort_pairs(ctx, lo, idx, n, 0xffffffffu, scratch, &k1, &v1);
    if (rc) return done(rc);
    k_cross_hi<<<blocks, 256, 0, st>>>(keys, v1, n, hi);
    if (v1 != idx) VLR_CUDA(ctx, cudaMemcpyAsync(idx, v1, (size_t)n * 4, cudaMemcpyDeviceToDevice, st));
    rc = radix_sort_pairs(ctx, hi, idx, n, 0x7fffffffu, scratch, &k2, &v2);
    if (rc) return done(rc);
    (void)k1;
    (void)k2;
    k_cross_gather<<<blocks, 256, 0, st>>>(d_c, v2, n, d_out);
    VLR_CUDA(ctx, cudaGetLastError());
    *sorted = true;
    return done(VLR_OK);
}

int find_zero_crossings(vlr_ctx* ctx, const vlr_grid* g, int32_t* h_coords, size_t cap, size_t* count,
                        bool* sorted) {
    *count = 0;
    if (g->n == 0) return VLR_OK;
    CrossBufs b;
    int rc = alloc_cross(ctx, g->n, b);
    if (rc) return rc;
    unsigned long long total = 0;
    rc = crossings(ctx, g, b.xmask, b.xcount, b.total, &total);
    if (rc) return rc;
    *count = (size_t)total;
    if (total > 0 && h_coords && cap > 0) {
        rc = scan_exclusive(ctx, b.xcount, b.pos, g->n, b.pos + g->n);
        if (rc) return rc;
        int* d_coords = nullptr;
        VLR_CUDA(ctx, cudaMallocFromPoolAsync(&d_coords, sizeof(int) * 6 * total, ctx->pool, ctx->stream));
        k_emit_crossings<<<g->n, 512, 0, ctx->stream>>>(make_view(g), b.xmask, b.pos, d_coords);
        VLR_CUDA(ctx, cudaGetLastError());
        // emitted leaf by leaf (leaves in (x, y, z) order, voxels ZYX), which
        // is not the global (x, y, z) order: sorted on the device when the
        // keys fit 63 bits, else by the caller on the host
        bool dev_sorted = false;
        if (sorted) {
            rc = sort_crossings_device(ctx, d_coords, (int)total, d_coords + 3 * total, &dev_sorted);
            if (rc) return rc;
        }
        const int* src = dev_sorted ? d_coords + 3 * total : d_coords;
        size_t m = std::min<size_t>(cap, total);
        VLR_CUDA(ctx, cudaMemcpyAsync(h_coords, src, sizeof(int) * 3 * m, cudaMemcpyDeviceToHost, ctx->stream));
        VLR_CUDA(ctx, cudaFreeAsync(d_coords, ctx->stream));
        VLR_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
        if (sorted) *sorted = dev_sorted;
    }
    VLR_CUDA(ctx, cudaFreeAsync(b.xmask, ctx->stream));
    return VLR_OK;
}

int trim_narrow_band(vlr_ctx* ctx, vlr_grid* g, float half_width) {
    if (g->n == 0) return VLR_OK;
    float vs = (float)g->xf.voxel_size;
    float thr = half_width * vs;
    int* flags = nullptr;
    VLR_CUDA(ctx, cudaMallocFromPoolAsync(&flags, sizeof(int) * g->n, ctx->pool, ctx->stream));
    GridView v = make_view(g);
    VLR_TIMED(ctx, "k_trim", k_trim<<<g->n, 256, 0, ctx->stream>>>(v, (float*)g->values, g->mask, thr, flags));
    VLR_CUDA(ctx, cudaGetLastError());
    int rc = grid_compact(ctx, g, flags);
    if (rc) return rc;
    VLR_CUDA(ctx, cudaFreeAsync(flags, ctx->stream));
    return consume_device_errors(ctx, "trim_narrow_band");
}

int rebuild_narrow_band(vlr_ctx* ctx, vlr_grid* g, float half_width) {
    if (g->n == 0) return VLR_OK;
    float vs = (float)g->xf.voxel_size;
    float band = half_width * vs;
    CrossBufs b;
    int rc = alloc_cross(ctx, g->n, b);
    if (rc) return rc;
    unsigned long long total = 0;
    rc = crossings(ctx, g, b.xmask, b.xcount, b.total, &total);
    if (rc) return rc;
    if (total == 0) {  // no crossings: the grid is returned unchanged (level_set_track.rs:85-87)
        VLR_CUDA(ctx, cudaFreeAsync(b.xmask, ctx->stream));
        return VLR_OK;
    }
    GridView v = make_view(g);
    bool window = std::isfinite(half_width) && vs > 0.0f && half_width <= 9.0f;
    if (window) {
        int R = std::max(0, (int)std::ceil(half_width) - 1);
        VLR_TIMED(ctx, "k_rebuild_window",
                  k_rebuild_window<<<g->n, 256, 0, ctx->stream>>>(v, (float*)g->values, g->mask, b.xmask, R, vs,
                                                                 band, b.flags));
    } else {
        rc = scan_exclusive(ctx, b.xcount, b.pos, g->n, b.pos + g->n);
        if (rc) return rc;
        int* d_coords = nullptr;
        VLR_CUDA(ctx, cudaMallocFromPoolAsync(&d_coords, sizeof(int) * 3 * total, ctx->pool, ctx->stream));
        k_emit_crossings<<<g->n, 512, 0, ctx->stream>>>(v, b.xmask, b.pos, d_coords);
        k_rebuild_brute<<<g->n, 256, 0, ctx->stream>>>(v, (float*)g->values, g->mask, d_coords, (int)total, vs, band,
                                                      b.flags);
        VLR_CUDA(ctx, cudaFreeAsync(d_coords, ctx->stream));
    }
    VLR_CUDA(ctx, cudaGetLastError());
    rc = grid_compact(ctx, g, b.flags);
    if (rc) return rc;
    VLR_CUDA(ctx, cudaFreeAsync(b.xmask, ctx->stream));
    return consume_device_errors(ctx, "rebuild_narrow_band");
}

static int32_t sat_i32(double v) {
    if (std::isnan(v)) return 0;
    if (v <= -2147483648.0) return INT32_MIN;
    if (v >= 2147483647.0) return INT32_MAX;
    return (int32_t)v;
}

int make_sphere(vlr_ctx* ctx, double radius, const double c[3], double vs, double hw, vlr_grid* out) {
    double band = hw * vs;
    float bg = (float)band;
    double extent = radius + band;
    double inv = 1.0 / vs;
    int32_t imin = sat_i32(std::floor((c[0] - extent) * inv));
    int32_t jmin = sat_i32(std::floor((c[1] - extent) * inv));
    int32_t kmin = sat_i32(std::floor((c[2] - extent) * inv));
    int32_t imax = sat_i32(std::ceil((c[0] + extent) * inv));
    int32_t jmax = sat_i32(std::ceil((c[1] + extent) * inv));
    int32_t kmax = sat_i32(std::ceil((c[2] + extent) * inv));
    out->ctx = ctx;
    out->kind = VLR_KIND_F32_WORLD;
    out->background = bg;
    // set_transform(VoxelTransform::uniform(vs)) (src/tools/sphere.rs:36-38)
    std::memset(&out->xf, 0, sizeof(out->xf));
    out->xf.voxel_size = vs;
    out->xf.affine[0] = out->xf.affine[5] = out->xf.affine[10] = vs;
    out->xf.affine_voxel_size = vs;
    if (imin > imax || jmin > jmax || kmin > kmax) {
        out->base[0] = out->base[1] = out->base[2] = -kKeyHalf;
        int rc = grid_alloc(ctx, out, 1);
        if (rc) return rc;
        out->n = 0;
        return grid_index(ctx, out);
    }
    long long lx0 = imin >> 3, ly0 = jmin >> 3, lz0 = kmin >> 3;
    long long nlx = (imax >> 3) - lx0 + 1, nly = (jmax >> 3) - ly0 + 1, nlz = (kmax >> 3) - lz0 + 1;
    long long n_cand = nlx * nly * nlz;
    if (n_cand > (1ll << 26)) return set_error(ctx, VLR_ERR_CAPACITY, "sphere bounding box too large");
    int32_t corner[6] = {imin, jmin, kmin, imax, jmax, kmax};
    int32_t bb[6] = {corner[0], corner[1], corner[2], corner[3], corner[4], corner[5]};
    int rc = choose_base(ctx, bb, 2, out->base);
    if (rc) return rc;
    rc = grid_alloc(ctx, out, (int)n_cand);
    if (rc) return rc;
    out->n = (int)n_cand;
    int* flags = nullptr;
    VLR_CUDA(ctx, cudaMallocFromPoolAsync(&flags, sizeof(int) * n_cand, ctx->pool, ctx->stream));
    k_sphere<<<(unsigned)n_cand, 512, 0, ctx->stream>>>((int)lx0, (int)ly0, (int)lz0, (int)nly, (int)nlz, (int)n_cand,
                                                        imin, jmin, kmin, imax, jmax, kmax, radius, c[0], c[1], c[2],
                                                        vs, bg, out->origin, out->mask, (float*)out->values, flags);
    VLR_CUDA(ctx, cudaGetLastError());
    rc = grid_index(ctx, out);
    if (rc) return rc;
    rc = grid_compact(ctx, out, flags);
    if (rc) return rc;
    VLR_CUDA(ctx, cudaFreeAsync(flags, ctx->stream));
    return consume_device_errors(ctx, "make_level_set_sphere");
}

}  // namespace vlr
