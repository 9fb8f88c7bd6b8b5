// Differentiable advection: frozen-band semi-Lagrangian steps through a dense
// staggered velocity field, with a hand-written adjoint.
//
// Forward, K steps (t_k = t0 + k dt, c_k = cos(pi t_{k+1} / T)):
//   phi_{k+1}(x) = trilinear(phi_k)(x - dt c_k u(x))        for band voxels x
// where u(x) is the trilinear upsample of a staggered (MAC) field V of n^3
// cells of H voxels (component a lives on the faces normal to axis a) and
// every non-band voxel keeps its initial value (+-hw; unallocated leaves read
// the clamped-sign rule).  The map phi_0 -> phi_K is affine on the band, so
// the gradient is exact (up to rounding) wherever floor() does not jump.
//
// Backward, given lambda_K = dL/dphi_K on the band:
//   lambda_k(c) = sum_x lambda_{k+1}(x) w_c(p_k(x))     (transpose of the blend)
//   G(x)      += lambda_{k+1}(x) (-dt c_k) grad trilinear(phi_k)(p_k(x))
//   dL/dphi_0 = lambda_0,  dL/dV = upsample^T G
// The lambda transpose is a gather over the band voxels whose foot cell can
// hold the corner (a window of (2R+2)^3 voxels, R the per-step reach), summed
// in a fixed order; upsample^T goes through a stable radix sort and a
// segmented sum.  No float atomics: deterministic results.  phi_k for the
// backward pass is recomputed from checkpoints taken every C steps (sqrt(K)).
#include <algorithm>
#include <cmath>
#include <cstring>
#include <numeric>
#include <vector>

#include "method_state.hpp"
#include "sort_reduce.hpp"

struct vlr_adjoint {
    vlr_ctx* ctx = nullptr;
    int n_leaves = 0;
    int n_band = 0;
    float hw = 3.0f;
    int4* origin = nullptr;
    int* nbr = nullptr;
    uint64_t* hkey = nullptr;
    int* hval = nullptr;
    int hcap = 0;
    long long base[3] = {0, 0, 0};
    float* phi[2] = {nullptr, nullptr};  // leaf-major, 512 per leaf; phi[0] holds phi_0 layout template
    float* phi_init = nullptr;           // initial full leaves (non-band values are constants)
    int* bidx = nullptr;                 // slot*512 + off -> band index or -1
    int* bvox = nullptr;                 // band index -> slot*512 + off
    float3* ub = nullptr;                // upsampled velocity at band voxels
    float* vel = nullptr;                // staggered field 3 x n^3
    int n_stag = 0;
    double H = 1.0;                      // staggered cell size in voxels
    double dt = 0.0, t0 = 0.0, period = 1.0;
    int steps = 0, chk_every = 1;
    float* checkpoints = nullptr;        // (steps / chk_every + 1) x n_band
    float* segment = nullptr;            // chk_every x n_band (recomputed states)
    float* lam[2] = {nullptr, nullptr};
    float* lam_final = nullptr;          // lam buffer holding dL/dphi_0 after the last backward pass
    // the forward and backward step loops captured as CUDA graphs (dropped
    // when the velocity, hence the reach, changes)
    cudaGraphExec_t fwd_exec = nullptr, bwd_exec = nullptr;
    float* bwd_final = nullptr;          // lam buffer the captured backward loop ends in
    float* gvel = nullptr;               // dL/dV, 3 x n^3
    float3* G = nullptr;
    int reach = 1;                       // displacement bound per step, voxels (ceil of dt max|V|)
    int gather = 0;                      // transpose kernel: 0 by band size and reach, 1 windowed, 2 quad
    int disp = 0;                        // 1: ub holds each band voxel's fixed backtrace displacement
                                         // (a level set's time-independent velocity), step factor 1
    unsigned* foot_pk = nullptr;         // per pool voxel: packed foot offsets of band voxels, 0 elsewhere
    int* lrange = nullptr;               // per leaf: min and max foot offset per axis of its band voxels (6 ints)
    int* wrange = nullptr;               // per leaf: candidate window per axis for its corners (6 ints)
    float4* foot_w = nullptr;            // per pool voxel: (wx, wy, wz, lambda) of band voxels
    unsigned* keys = nullptr;
    float* pvals = nullptr;
    void* scratch = nullptr;
    size_t n_pairs_cap = 0;
};

namespace vlr {

__device__ __forceinline__ int nbx(int c) { return (c < 0) ? 0 : (c > 7 ? 2 : 1); }

// phi at local coordinate (x, y, z) of leaf `slot` (may leave the leaf by one voxel).
__device__ __forceinline__ float adj_read(const float* __restrict__ phi, const int* __restrict__ nbr, int slot, int x,
                                          int y, int z, float hw) {
    int s = nbr[slot * kNbr + nbx(x) * 9 + nbx(y) * 3 + nbx(z)];
    if (s >= 0) return phi[(size_t)s * kLeafVoxels + voxel_off(x, y, z)];
    int cx = min(max(x, 0), 7), cy = min(max(y, 0), 7), cz = min(max(z, 0), 7);
    return copysignf(hw, phi[(size_t)slot * kLeafVoxels + ((cx << 6) | (cy << 3) | cz)]);
}

// Trilinear upsample of component a of the staggered field at voxel point p.
__device__ __forceinline__ float stag_sample(const float* __restrict__ V, int n, float H, int a, float px, float py,
                                             float pz) {
    float g[3] = {px / H, py / H, pz / H};
    for (int q = 0; q < 3; ++q)
        if (q != a) g[q] -= 0.5f;
    int i0[3];
    float w[3];
    for (int q = 0; q < 3; ++q) {
        float f = floorf(g[q]);
        i0[q] = (int)f;
        w[q] = g[q] - f;
    }
    auto at = [&](int i, int j, int k) {
        i = min(max(i, 0), n - 1);
        j = min(max(j, 0), n - 1);
        k = min(max(k, 0), n - 1);
        return V[(size_t)a * n * n * n + ((size_t)i * n + j) * n + k];
    };
    float c00 = at(i0[0], i0[1], i0[2]) * (1 - w[0]) + at(i0[0] + 1, i0[1], i0[2]) * w[0];
    float c01 = at(i0[0], i0[1], i0[2] + 1) * (1 - w[0]) + at(i0[0] + 1, i0[1], i0[2] + 1) * w[0];
    float c10 = at(i0[0], i0[1] + 1, i0[2]) * (1 - w[0]) + at(i0[0] + 1, i0[1] + 1, i0[2]) * w[0];
    float c11 = at(i0[0], i0[1] + 1, i0[2] + 1) * (1 - w[0]) + at(i0[0] + 1, i0[1] + 1, i0[2] + 1) * w[0];
    float c0 = c00 * (1 - w[1]) + c10 * w[1], c1 = c01 * (1 - w[1]) + c11 * w[1];
    return c0 * (1 - w[2]) + c1 * w[2];
}

__global__ void k_adj_upsample(const int* __restrict__ bvox, const int4* __restrict__ origin, int nb,
                               const float* __restrict__ V, int n, float H, float3* __restrict__ ub) {
    for (int b = blockIdx.x * blockDim.x + threadIdx.x; b < nb; b += gridDim.x * blockDim.x) {
        int sv = bvox[b], s = sv >> 9, off = sv & 511;
        int4 o = origin[s];
        float px = (float)(o.x + (off >> 6)), py = (float)(o.y + ((off >> 3) & 7)), pz = (float)(o.z + (off & 7));
        ub[b] = make_float3(stag_sample(V, n, H, 0, px, py, pz), stag_sample(V, n, H, 1, px, py, pz),
                            stag_sample(V, n, H, 2, px, py, pz));
    }
}

// Foot offset, floor and weights of band voxel b at step k.
struct Foot {
    int fx, fy, fz;     // floor of the foot, relative to the voxel
    float wx, wy, wz;   // fractions
};
__device__ __forceinline__ Foot foot_of(float3 u, float s) {
    float ox = s * u.x, oy = s * u.y, oz = s * u.z;  // s = -dt c_k
    Foot f;
    float bx = floorf(ox), by = floorf(oy), bz = floorf(oz);
    f.fx = (int)bx;
    f.fy = (int)by;
    f.fz = (int)bz;
    f.wx = ox - bx;
    f.wy = oy - by;
    f.wz = oz - bz;
    return f;
}

// One forward step over the band voxels, one thread each.  Non-band voxels
// never change, and both state buffers hold phi_0 there (the callers copy it
// into both), so they are not touched.
__global__ void k_adj_forward(const int* __restrict__ bvox, int nb, const int* __restrict__ nbr,
                              const float3* __restrict__ ub, const float* __restrict__ src, float* __restrict__ dst,
                              float s, float hw, unsigned* err) {
    for (int b = blockIdx.x * blockDim.x + threadIdx.x; b < nb; b += gridDim.x * blockDim.x) {
        const int t = bvox[b];
        const int slot = t >> 9, off = t & 511;
        Foot f = foot_of(ub[b], s);
        int x = (off >> 6) + f.fx, y = ((off >> 3) & 7) + f.fy, z = (off & 7) + f.fz;
        if (x < -8 || y < -8 || z < -8 || x > 14 || y > 14 || z > 14) {
            atomicOr(err, kErrReach);
            dst[t] = src[t];
            continue;
        }
        float c000 = adj_read(src, nbr, slot, x, y, z, hw), c100 = adj_read(src, nbr, slot, x + 1, y, z, hw);
        float c010 = adj_read(src, nbr, slot, x, y + 1, z, hw), c110 = adj_read(src, nbr, slot, x + 1, y + 1, z, hw);
        float c001 = adj_read(src, nbr, slot, x, y, z + 1, hw), c101 = adj_read(src, nbr, slot, x + 1, y, z + 1, hw);
        float c011 = adj_read(src, nbr, slot, x, y + 1, z + 1, hw),
              c111 = adj_read(src, nbr, slot, x + 1, y + 1, z + 1, hw);
        float c00 = c000 * (1 - f.wx) + c100 * f.wx, c01 = c001 * (1 - f.wx) + c101 * f.wx;
        float c10 = c010 * (1 - f.wx) + c110 * f.wx, c11 = c011 * (1 - f.wx) + c111 * f.wx;
        float c0 = c00 * (1 - f.wy) + c10 * f.wy, c1 = c01 * (1 - f.wy) + c11 * f.wy;
        dst[t] = c0 * (1 - f.wz) + c1 * f.wz;
    }
}

__global__ void k_adj_gather_band(const int* __restrict__ bvox, int nb, const float* __restrict__ phi,
                                  float* __restrict__ out) {
    for (int b = blockIdx.x * blockDim.x + threadIdx.x; b < nb; b += gridDim.x * blockDim.x) out[b] = phi[bvox[b]];
}

__global__ void k_adj_scatter_band(const int* __restrict__ bvox, int nb, const float* __restrict__ in,
                                   float* __restrict__ phi) {
    for (int b = blockIdx.x * blockDim.x + threadIdx.x; b < nb; b += gridDim.x * blockDim.x) phi[bvox[b]] = in[b];
}

// Band index of the voxel at local (x, y, z) of leaf slot, or n_band (dropped key).
__device__ __forceinline__ unsigned band_key(const int* __restrict__ nbr, const int* __restrict__ bidx, int slot, int x,
                                             int y, int z, unsigned nb) {
    int s = nbr[slot * kNbr + nbx(x) * 9 + nbx(y) * 3 + nbx(z)];
    if (s < 0) return nb;
    int b = bidx[(size_t)s * kLeafVoxels + voxel_off(x, y, z)];
    return b < 0 ? nb : (unsigned)b;
}

// Per step k, for every band voxel x: its foot (floor offsets packed as three
// biased bytes, bit 31 marking a band voxel) and (wx, wy, wz, lambda(x)) in
// pool order, so the gather below reads one word per candidate instead of a
// chain of band-index, velocity and lambda lookups.
__global__ void k_adj_pack(const int* __restrict__ bvox, int nb, const float3* __restrict__ ub,
                           const float* __restrict__ lam, float s, unsigned* __restrict__ foot_pk,
                           float4* __restrict__ foot_w) {
    for (int b = blockIdx.x * blockDim.x + threadIdx.x; b < nb; b += gridDim.x * blockDim.x) {
        const Foot f = foot_of(ub[b], s);
        const int sv = bvox[b];
        foot_pk[sv] = 0x80000000u | ((unsigned)(f.fx + 64) << 14) | ((unsigned)(f.fy + 64) << 7) |
                      (unsigned)(f.fz + 64);
        foot_w[sv] = make_float4(f.wx, f.wy, f.wz, lam[b]);
    }
}

// k_adj_pack for a displacement fixed over the steps (a level set's
// time-independent velocity): the feet and weights of the first step stand,
// so later steps write only lambda, the fourth word of each band voxel's
// foot record.
__global__ void k_adj_pack_lambda(const int* __restrict__ bvox, int nb, const float* __restrict__ lam,
                                  float4* __restrict__ foot_w) {
    float* w = reinterpret_cast<float*>(foot_w);
    for (int b = blockIdx.x * blockDim.x + threadIdx.x; b < nb; b += gridDim.x * blockDim.x)
        w[4 * (size_t)bvox[b] + 3] = lam[b];
}

// Per leaf, the smallest and largest foot offset per axis over its band
// voxels at this step (empty leaves: min > max).  One warp per leaf.
__global__ void k_adj_leafrange(const unsigned* __restrict__ foot_pk, int n_leaves, int* __restrict__ lrange) {
    const int lane = threadIdx.x & 31;
    for (int leaf = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; leaf < n_leaves;
         leaf += (gridDim.x * blockDim.x) >> 5) {
        int lo[3] = {INT_MAX, INT_MAX, INT_MAX}, hi[3] = {INT_MIN, INT_MIN, INT_MIN};
        for (int v = lane; v < kLeafVoxels; v += 32) {
            const unsigned pk = foot_pk[(size_t)leaf * kLeafVoxels + v];
            if (!(pk >> 31)) continue;
            const int f[3] = {(int)((pk >> 14) & 127u) - 64, (int)((pk >> 7) & 127u) - 64, (int)(pk & 127u) - 64};
#pragma unroll
            for (int a = 0; a < 3; ++a) {
                lo[a] = min(lo[a], f[a]);
                hi[a] = max(hi[a], f[a]);
            }
        }
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            lo[a] = __reduce_min_sync(0xffffffffu, lo[a]);
            hi[a] = __reduce_max_sync(0xffffffffu, hi[a]);
        }
        if (lane < 3) {
            lrange[leaf * 6 + lane] = lo[lane];
            lrange[leaf * 6 + 3 + lane] = hi[lane];
        }
    }
}

// Per leaf, the window of candidate offsets dx (per axis) for its corners b:
// a band voxel x = b + dx has b in its foot cell only if dx = -f(x) - {0, 1},
// f(x) its foot offset; x lies in the 27-leaf neighbourhood (|f| <= R < 8),
// so dx runs over [-max f - 1, -min f] taken over the neighbourhood's band
// voxels, within [-1 - R, R].  Empty neighbourhoods get an empty window.
__global__ void k_adj_window(const int* __restrict__ nbr, const int* __restrict__ lrange, int n_leaves, int R,
                             int* __restrict__ wrange) {
    for (int leaf = blockIdx.x * blockDim.x + threadIdx.x; leaf < n_leaves; leaf += gridDim.x * blockDim.x) {
        int lo[3] = {INT_MAX, INT_MAX, INT_MAX}, hi[3] = {INT_MIN, INT_MIN, INT_MIN};
        for (int d = 0; d < kNbr; ++d) {
            const int s = nbr[(size_t)leaf * kNbr + d];
            if (s < 0) continue;
#pragma unroll
            for (int a = 0; a < 3; ++a) {
                lo[a] = min(lo[a], lrange[s * 6 + a]);
                hi[a] = max(hi[a], lrange[s * 6 + 3 + a]);
            }
        }
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            const bool empty = lo[a] > hi[a];
            wrange[leaf * 6 + a] = empty ? 1 : max(-hi[a] - 1, -1 - R);
            wrange[leaf * 6 + 3 + a] = empty ? 0 : min(-lo[a], R);
        }
    }
}

// Adjoint of step k as a gather, one band voxel b per thread:
//   G(b)      += lambda(b) s grad trilinear(phi_k)(p(b))      (b's own foot)
//   lambda'(b) = sum over band voxels x of lambda(x) w_b(p(x))  (b as a corner)
// A step moves a voxel by at most R = reach voxels per axis, so b is a corner
// of x's foot cell only if x lies in b + [-1-R, R]^3; those candidates are
// visited in a fixed order (x, then y, then z ascending), each x's foot taken
// from the same foot_of() as the forward step (through k_adj_pack), so the
// transpose is exact and the sum order is fixed: deterministic, with no sort
// and no float atomics.  RT = 1: the whole window [-2, 1]^3, unrolled.  RT =
// 0: the visit is narrowed to the leaf's window from k_adj_window (offsets
// outside it cannot hold b as a corner), which keeps the order of the
// contributing terms, hence the sums, unchanged; smooth fields leave 2-3
// offsets per axis, against 2R + 2 in the whole window.
template <int RT>
__global__ void k_adj_lambda(const int* __restrict__ bvox, int nb, const int* __restrict__ nbr,
                             const float* __restrict__ phi_k, const unsigned* __restrict__ foot_pk,
                             const float4* __restrict__ foot_w, float s, float hw, const int* __restrict__ wrange,
                             float* __restrict__ lam_out, float3* __restrict__ G) {
    for (int b = blockIdx.x * blockDim.x + threadIdx.x; b < nb; b += gridDim.x * blockDim.x) {
        const int sv = bvox[b], slot = sv >> 9, off = sv & 511;
        const int cx = off >> 6, cy = (off >> 3) & 7, cz = off & 7;
        {
            const unsigned pk = foot_pk[sv];
            const float4 w4 = foot_w[sv];
            const float l = w4.w;
            const int x = cx + (int)((pk >> 14) & 127u) - 64, y = cy + (int)((pk >> 7) & 127u) - 64,
                      z = cz + (int)(pk & 127u) - 64;
            const float wx[2] = {1 - w4.x, w4.x}, wy[2] = {1 - w4.y, w4.y}, wz[2] = {1 - w4.z, w4.z};
            float c[8];
#pragma unroll
            for (int q = 0; q < 8; ++q) c[q] = adj_read(phi_k, nbr, slot, x + (q >> 2), y + ((q >> 1) & 1), z + (q & 1), hw);
            // c[q] with q = i*4 + j*2 + k
            float gx = wy[0] * wz[0] * (c[4] - c[0]) + wy[1] * wz[0] * (c[6] - c[2]) + wy[0] * wz[1] * (c[5] - c[1]) +
                       wy[1] * wz[1] * (c[7] - c[3]);
            float gy = wx[0] * wz[0] * (c[2] - c[0]) + wx[1] * wz[0] * (c[6] - c[4]) + wx[0] * wz[1] * (c[3] - c[1]) +
                       wx[1] * wz[1] * (c[7] - c[5]);
            float gz = wx[0] * wy[0] * (c[1] - c[0]) + wx[1] * wy[0] * (c[5] - c[4]) + wx[0] * wy[1] * (c[3] - c[2]) +
                       wx[1] * wy[1] * (c[7] - c[6]);
            float3 g = G[b];
            g.x += l * s * gx;
            g.y += l * s * gy;
            g.z += l * s * gz;
            G[b] = g;
        }
        const int* nrow = nbr + slot * kNbr;
        int x0 = -2, y0 = -2, z0 = -2, x1 = 1, y1 = 1, z1 = 1;
        if (RT == 0) {
            const int* w6 = wrange + slot * 6;
            x0 = __ldg(&w6[0]);
            y0 = __ldg(&w6[1]);
            z0 = __ldg(&w6[2]);
            x1 = __ldg(&w6[3]);
            y1 = __ldg(&w6[4]);
            z1 = __ldg(&w6[5]);
        }
        float acc = 0.f;
#pragma unroll
        for (int dx = x0; dx <= x1; ++dx) {
            const int x = cx + dx;
#pragma unroll
            for (int dy = y0; dy <= y1; ++dy) {
                const int y = cy + dy;
                const int nb2 = nbx(x) * 9 + nbx(y) * 3;
#pragma unroll
                for (int dz = z0; dz <= z1; ++dz) {
                    const int z = cz + dz;
                    const int ns = __ldg(&nrow[nb2 + nbx(z)]);
                    if (ns < 0) continue;
                    const size_t e = (size_t)ns * kLeafVoxels + voxel_off(x, y, z);
                    const unsigned pk = __ldg(&foot_pk[e]);
                    // corner index of b in x's foot cell: b - (x + floor(offset))
                    const int i = 64 - dx - (int)((pk >> 14) & 127u), j = 64 - dy - (int)((pk >> 7) & 127u),
                              k = 64 - dz - (int)(pk & 127u);
                    if (!(pk >> 31) || (unsigned)i > 1u || (unsigned)j > 1u || (unsigned)k > 1u) continue;
                    const float4 w4 = __ldg(&foot_w[e]);
                    const float wx = i ? w4.x : 1 - w4.x, wy = j ? w4.y : 1 - w4.y, wz = k ? w4.z : 1 - w4.z;
                    acc += w4.w * wx * wy * wz;
                }
            }
        }
        lam_out[b] = acc;
    }
}

// k_adj_lambda<1> for small bands, four lanes per band voxel: lane q of the
// quad visits offset dx = q - 2 of the whole window [-2, 1]^3 (dy, dz
// ascending) and the quad sums its four partial sums in the fixed order
// ((q0 + q1) + q2) + q3; lane 0 adds b's own gradient term.  Deterministic;
// the rounding differs from the one-thread order only in how the partial sums
// associate.  Fills the GPU where one thread per band voxel leaves most warp
// slots empty.
__global__ void k_adj_lambda_quad(const int* __restrict__ bvox, int nb, const int* __restrict__ nbr,
                                  const float* __restrict__ phi_k, const unsigned* __restrict__ foot_pk,
                                  const float4* __restrict__ foot_w, float s, float hw, float* __restrict__ lam_out,
                                  float3* __restrict__ G) {
    const int q = threadIdx.x & 3;
    for (long long gq = (blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 2; gq < nb;
         gq += ((long long)gridDim.x * blockDim.x) >> 2) {
        const int b = (int)gq;
        const int sv = bvox[b], slot = sv >> 9, off = sv & 511;
        const int cx = off >> 6, cy = (off >> 3) & 7, cz = off & 7;
        if (q == 0) {
            const unsigned pk = foot_pk[sv];
            const float4 w4 = foot_w[sv];
            const float l = w4.w;
            const int x = cx + (int)((pk >> 14) & 127u) - 64, y = cy + (int)((pk >> 7) & 127u) - 64,
                      z = cz + (int)(pk & 127u) - 64;
            const float wx[2] = {1 - w4.x, w4.x}, wy[2] = {1 - w4.y, w4.y}, wz[2] = {1 - w4.z, w4.z};
            float c[8];
#pragma unroll
            for (int k = 0; k < 8; ++k) c[k] = adj_read(phi_k, nbr, slot, x + (k >> 2), y + ((k >> 1) & 1), z + (k & 1), hw);
            float gx = wy[0] * wz[0] * (c[4] - c[0]) + wy[1] * wz[0] * (c[6] - c[2]) + wy[0] * wz[1] * (c[5] - c[1]) +
                       wy[1] * wz[1] * (c[7] - c[3]);
            float gy = wx[0] * wz[0] * (c[2] - c[0]) + wx[1] * wz[0] * (c[6] - c[4]) + wx[0] * wz[1] * (c[3] - c[1]) +
                       wx[1] * wz[1] * (c[7] - c[5]);
            float gz = wx[0] * wy[0] * (c[1] - c[0]) + wx[1] * wy[0] * (c[5] - c[4]) + wx[0] * wy[1] * (c[3] - c[2]) +
                       wx[1] * wy[1] * (c[7] - c[6]);
            float3 g = G[b];
            g.x += l * s * gx;
            g.y += l * s * gy;
            g.z += l * s * gz;
            G[b] = g;
        }
        const int* nrow = nbr + slot * kNbr;
        float acc = 0.f;
        const int dx = q - 2;
        const int x = cx + dx;
#pragma unroll
        for (int dy = -2; dy <= 1; ++dy) {
            const int y = cy + dy;
            const int nb2 = nbx(x) * 9 + nbx(y) * 3;
#pragma unroll
            for (int dz = -2; dz <= 1; ++dz) {
                const int z = cz + dz;
                const int ns = __ldg(&nrow[nb2 + nbx(z)]);
                if (ns < 0) continue;
                const size_t e = (size_t)ns * kLeafVoxels + voxel_off(x, y, z);
                const unsigned pk = __ldg(&foot_pk[e]);
                const int i = 64 - dx - (int)((pk >> 14) & 127u), j = 64 - dy - (int)((pk >> 7) & 127u),
                          k = 64 - dz - (int)(pk & 127u);
                if (!(pk >> 31) || (unsigned)i > 1u || (unsigned)j > 1u || (unsigned)k > 1u) continue;
                const float4 w4 = __ldg(&foot_w[e]);
                const float wx = i ? w4.x : 1 - w4.x, wy = j ? w4.y : 1 - w4.y, wz = k ? w4.z : 1 - w4.z;
                acc += w4.w * wx * wy * wz;
            }
        }
        // the quad's lanes are consecutive; sum in lane order
        const unsigned qmask = 0xFu << (threadIdx.x & 28);
        const float a1 = __shfl_sync(qmask, acc, (threadIdx.x & 31 & ~3) + 1);
        const float a2 = __shfl_sync(qmask, acc, (threadIdx.x & 31 & ~3) + 2);
        const float a3 = __shfl_sync(qmask, acc, (threadIdx.x & 31 & ~3) + 3);
        if (q == 0) lam_out[b] = ((acc + a1) + a2) + a3;
    }
}

// Transpose of the upsample: 3 x 8 (node, G_a * weight) pairs per band voxel.
__global__ void k_adj_emit_vel(const int* __restrict__ bvox, const int4* __restrict__ origin, int nb,
                               const float3* __restrict__ G, int n, float H, unsigned* __restrict__ keys,
                               float* __restrict__ vals) {
    for (int b = blockIdx.x * blockDim.x + threadIdx.x; b < nb; b += gridDim.x * blockDim.x) {
        const int sv = bvox[b], s = sv >> 9, off = sv & 511;
        const int4 o = origin[s];
        const float p[3] = {(float)(o.x + (off >> 6)), (float)(o.y + ((off >> 3) & 7)), (float)(o.z + (off & 7))};
        const float3 gg = G[b];
        const float ga[3] = {gg.x, gg.y, gg.z};
        for (int a = 0; a < 3; ++a) {
            float g[3] = {p[0] / H, p[1] / H, p[2] / H};
            for (int q = 0; q < 3; ++q)
                if (q != a) g[q] -= 0.5f;
            int i0[3];
            float w[3];
            for (int q = 0; q < 3; ++q) {
                float fl = floorf(g[q]);
                i0[q] = (int)fl;
                w[q] = g[q] - fl;
            }
            for (int q = 0; q < 8; ++q) {
                int di = q >> 2, dj = (q >> 1) & 1, dk = q & 1;
                int i = min(max(i0[0] + di, 0), n - 1), j = min(max(i0[1] + dj, 0), n - 1),
                    k = min(max(i0[2] + dk, 0), n - 1);
                float wt = (di ? w[0] : 1 - w[0]) * (dj ? w[1] : 1 - w[1]) * (dk ? w[2] : 1 - w[2]);
                size_t e = ((size_t)b * 3 + a) * 8 + q;
                keys[e] = (unsigned)((size_t)a * n * n * n + ((size_t)i * n + j) * n + k);
                vals[e] = ga[a] * wt;
            }
        }
    }
}

__global__ void k_zero3(float3* a, int n) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        a[i] = make_float3(0.f, 0.f, 0.f);
}

__global__ void k_adj_hash_insert(const int4* origin, int n, uint64_t* hkey, int* hval, int hcap, long long b0,
                                  long long b1, long long b2, unsigned* err);
__global__ void k_adj_nbr(const int4* origin, int n, const uint64_t* hkey, const int* hval, int hcap, long long b0,
                          long long b1, long long b2, int* nbr);

__global__ void k_adj_hash_insert(const int4* origin, int n, uint64_t* hkey, int* hval, int hcap, long long b0,
                                  long long b1, long long b2, unsigned* err) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    long long base[3] = {b0, b1, b2};
    int4 o = origin[i];
    uint64_t key = pack_key(o.x >> 3, o.y >> 3, o.z >> 3, base);
    uint32_t m = (uint32_t)hcap - 1u, p = (uint32_t)mix64(key) & m;
    for (int probe = 0; probe < hcap; ++probe) {
        unsigned long long prev =
            atomicCAS((unsigned long long*)&hkey[p], (unsigned long long)kEmptyKey, (unsigned long long)key);
        if (prev == kEmptyKey) {
            hval[p] = i;
            return;
        }
        p = (p + 1u) & m;
    }
    atomicOr(err, kErrHashFull);
}

__global__ void k_adj_nbr(const int4* origin, int n, const uint64_t* hkey, const int* hval, int hcap, long long b0,
                          long long b1, long long b2, int* nbr) {
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n * kNbr) return;
    int i = t / kNbr, d = t % kNbr;
    HashView h{hkey, hval, hcap, {b0, b1, b2}};
    int4 o = origin[i];
    nbr[t] = hash_find_leaf(h, (long long)(o.x >> 3) + d / 9 - 1, (long long)(o.y >> 3) + (d / 3) % 3 - 1,
                            (long long)(o.z >> 3) + d % 3 - 1);
}

}  // namespace vlr

using namespace vlr;

namespace {

int blocks_for(vlr_ctx* ctx, long long n) { return (int)std::max<long long>(1, std::min<long long>((n + 255) / 256, ctx->sm_count * 8ll)); }

void adj_drop_graphs(vlr_adjoint* a) {
    if (a->fwd_exec) cudaGraphExecDestroy(a->fwd_exec);
    if (a->bwd_exec) cudaGraphExecDestroy(a->bwd_exec);
    a->fwd_exec = a->bwd_exec = nullptr;
}

void adj_free(vlr_adjoint* a) {
    adj_drop_graphs(a);
    void* ptrs[] = {a->origin, a->nbr, a->hkey, a->hval, a->phi[0], a->phi[1], a->phi_init, a->bidx, a->bvox,
                    a->ub, a->vel, a->checkpoints, a->segment, a->lam[0], a->lam[1], a->G, a->keys, a->pvals,
                    a->scratch, a->gvel, a->foot_pk, a->foot_w, a->lrange, a->wrange};
    for (void* p : ptrs) cudaFree(p);
}

// Per-axis displacement bound of one step in whole voxels: |s_k u| <= dt max|V|
// (the upsample is a convex combination of V and |cos| <= 1).
int reach_of(const float* vel, size_t nvel, double dt) {
    double m = 0.0;
    for (size_t i = 0; i < nvel; ++i) m = std::max(m, (double)std::fabs(vel[i]));
    return std::max(1, (int)std::ceil(dt * m * (1.0 + 1e-6)));
}

float step_factor(const vlr_adjoint* a, int k) {
    if (a->disp) return 1.0f;  // the displacement already holds -dt and the integrator
    // s_k = -dt cos(pi t_{k+1} / T)
    const double pi = 3.14159265358979323846;
    double t1 = a->t0 + (double)(k + 1) * a->dt;
    return (float)(-a->dt * std::cos(pi * t1 / a->period));
}

int enqueue_forward_step(vlr_ctx* ctx, vlr_adjoint* a, int k, const float* src, float* dst) {
    VLR_TIMED(ctx, "k_adj_forward",
              k_adj_forward<<<blocks_for(ctx, a->n_band), 256, 0, ctx->stream>>>(
                  a->bvox, a->n_band, a->nbr, a->ub, src, dst, step_factor(a, k), a->hw, ctx->d_errword));
    VLR_CUDA(ctx, cudaGetLastError());
    return VLR_OK;
}

// The forward step loop from the initial state (checkpoints every C steps;
// phi_K on the band into lam[1]), enqueued without waiting.
int adj_forward_enqueue(vlr_ctx* ctx, vlr_adjoint* a) {
    cudaStream_t st = ctx->stream;
    const size_t nb = (size_t)a->n_band;
    // both state buffers start as phi_0 (the steps rewrite band voxels only)
    VLR_CUDA(ctx, cudaMemcpyAsync(a->phi[0], a->phi_init, sizeof(float) * 512 * a->n_leaves, cudaMemcpyDeviceToDevice,
                                  st));
    VLR_CUDA(ctx, cudaMemcpyAsync(a->phi[1], a->phi_init, sizeof(float) * 512 * a->n_leaves, cudaMemcpyDeviceToDevice,
                                  st));
    int cur = 0;
    for (int k = 0; k < a->steps; ++k) {
        if (k % a->chk_every == 0)
            k_adj_gather_band<<<blocks_for(ctx, nb), 256, 0, st>>>(a->bvox, (int)nb, a->phi[cur],
                                                                   a->checkpoints + (size_t)(k / a->chk_every) * nb);
        int rc = enqueue_forward_step(ctx, a, k, a->phi[cur], a->phi[1 - cur]);
        if (rc) return rc;
        cur = 1 - cur;
    }
    k_adj_gather_band<<<blocks_for(ctx, nb), 256, 0, st>>>(a->bvox, (int)nb, a->phi[cur], a->lam[1]);
    VLR_CUDA(ctx, cudaGetLastError());
    return VLR_OK;
}

// The backward step loop from lambda_K in lam[1] (recompute from checkpoints,
// gather transpose, G accumulation), enqueued without waiting; records the
// lam buffer it ends in.
int adj_backward_enqueue(vlr_ctx* ctx, vlr_adjoint* a) {
    cudaStream_t st = ctx->stream;
    const size_t nb = (size_t)a->n_band;
    float* lam = a->lam[1];
    k_zero3<<<blocks_for(ctx, nb), 256, 0, st>>>(a->G, (int)nb);
    const int C = a->chk_every;
    for (int seg = (a->steps - 1) / C; seg >= 0; --seg) {
        const int k0 = seg * C, k1 = std::min(a->steps, k0 + C);
        // recompute phi_k0 .. phi_{k1-1} from the checkpoint
        VLR_CUDA(ctx, cudaMemcpyAsync(a->phi[0], a->phi_init, sizeof(float) * 512 * a->n_leaves,
                                      cudaMemcpyDeviceToDevice, st));
        k_adj_scatter_band<<<blocks_for(ctx, nb), 256, 0, st>>>(a->bvox, (int)nb, a->checkpoints + (size_t)seg * nb,
                                                                a->phi[0]);
        VLR_CUDA(ctx, cudaMemcpyAsync(a->phi[1], a->phi[0], sizeof(float) * 512 * a->n_leaves,
                                      cudaMemcpyDeviceToDevice, st));
        int cur = 0;
        for (int k = k0; k < k1; ++k) {
            k_adj_gather_band<<<blocks_for(ctx, nb), 256, 0, st>>>(a->bvox, (int)nb, a->phi[cur],
                                                                   a->segment + (size_t)(k - k0) * nb);
            if (k + 1 < k1) {
                int rc = enqueue_forward_step(ctx, a, k, a->phi[cur], a->phi[1 - cur]);
                if (rc) return rc;
                cur = 1 - cur;
            }
        }
        // adjoint steps k1-1 .. k0: phi_k from the segment (scattered into a full pool)
        for (int k = k1 - 1; k >= k0; --k) {
            k_adj_scatter_band<<<blocks_for(ctx, nb), 256, 0, st>>>(a->bvox, (int)nb,
                                                                    a->segment + (size_t)(k - k0) * nb, a->phi[0]);
            float* lam_out = (lam == a->lam[1]) ? a->lam[0] : a->lam[1];
            const float sk = step_factor(a, k);
            // a fixed displacement keeps the feet, their weights and the
            // leaves' windows of the backward pass's first step
            const bool feet_stand = a->disp && k != a->steps - 1;
            if (feet_stand)
                VLR_TIMED(ctx, "k_adj_pack",
                          k_adj_pack_lambda<<<blocks_for(ctx, nb), 256, 0, st>>>(a->bvox, (int)nb, lam, a->foot_w));
            else
                VLR_TIMED(ctx, "k_adj_pack",
                          k_adj_pack<<<blocks_for(ctx, nb), 256, 0, st>>>(a->bvox, (int)nb, a->ub, lam, sk,
                                                                          a->foot_pk, a->foot_w));
            const int gb = blocks_for(ctx, nb);
            const int nl = a->n_leaves;
            // the narrowed window pays when the whole window is large (reach >= 2)
            // or the band is, where its two small per-leaf passes are cheap
            if (a->gather == 2 || (a->gather == 0 && a->reach == 1 && nb < (1u << 20))) {
                // small band: a quad of lanes per band voxel fills the GPU
                VLR_TIMED(ctx, "k_adj_lambda",
                          k_adj_lambda_quad<<<blocks_for(ctx, 4ll * nb), 256, 0, st>>>(
                              a->bvox, (int)nb, a->nbr, a->phi[0], a->foot_pk, a->foot_w, sk, a->hw, lam_out, a->G));
            } else {
                if (!feet_stand) {
                    VLR_TIMED(ctx, "k_adj_leafrange",
                              k_adj_leafrange<<<blocks_for(ctx, 32ll * nl), 256, 0, st>>>(a->foot_pk, nl, a->lrange));
                    VLR_TIMED(ctx, "k_adj_window",
                              k_adj_window<<<blocks_for(ctx, nl), 256, 0, st>>>(a->nbr, a->lrange, nl, a->reach,
                                                                                a->wrange));
                }
                VLR_TIMED(ctx, "k_adj_lambda",
                          k_adj_lambda<0><<<gb, 256, 0, st>>>(a->bvox, (int)nb, a->nbr, a->phi[0], a->foot_pk,
                                                              a->foot_w, sk, a->hw, a->wrange, lam_out, a->G));
            }
            lam = lam_out;
        }
        (void)cur;
    }
    VLR_CUDA(ctx, cudaGetLastError());
    a->bwd_final = lam;
    return VLR_OK;
}

// Run `enqueue` through a CUDA graph captured on first use (or directly while
// per-kernel timing is on, which brackets launches with events).
template <class F>
int run_captured(vlr_ctx* ctx, cudaGraphExec_t* exec, F&& enqueue) {
    if (ctx->timer.enabled) return enqueue();
    if (!*exec) {
        VLR_CUDA(ctx, cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal));
        const int rc = enqueue();
        cudaGraph_t g = nullptr;
        const cudaError_t e = cudaStreamEndCapture(ctx->stream, &g);
        if (rc) {
            if (g) cudaGraphDestroy(g);
            return rc;
        }
        if (e != cudaSuccess) return check_cuda(ctx, e, "cudaStreamEndCapture");
        const cudaError_t e2 = cudaGraphInstantiate(exec, g, 0);
        cudaGraphDestroy(g);
        if (e2 != cudaSuccess) return check_cuda(ctx, e2, "cudaGraphInstantiate");
    }
    VLR_CUDA(ctx, cudaGraphLaunch(*exec, ctx->stream));
    return VLR_OK;
}

// Level-set adjoint setup, leaves in list order: origins, phi_0 in f32 voxel
// units and the band (active voxel) count of each leaf.
template <typename T>
__global__ void k_adjls_gather(const int* __restrict__ list, int n, const int4* __restrict__ ls_origin,
                               const uint64_t* __restrict__ mask, const T* __restrict__ vals, int4* __restrict__ origin,
                               float* __restrict__ phi, int* __restrict__ cnt) {
    for (int i = blockIdx.x; i < n; i += gridDim.x) {
        const int s = list[i];
        if (threadIdx.x == 0) origin[i] = ls_origin[s];
        for (int t = threadIdx.x; t < kLeafVoxels; t += blockDim.x)
            phi[(size_t)i * kLeafVoxels + t] = to_f(vals[(size_t)s * kLeafVoxels + t]);
        if (threadIdx.x < 32) {
            int c = threadIdx.x < 8 ? __popcll(mask[(size_t)s * 8 + threadIdx.x]) : 0;
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) c += __shfl_xor_sync(0xffffffffu, c, o);
            if (threadIdx.x == 0) cnt[i] = c;
        }
    }
}

// out[b] = phi_0 at band voxel b's coordinate minus (sx, sy, sz), |s| <= 8,
// read with the adjoint's rule for missing leaves.
__global__ void k_adj_shifted(const int* __restrict__ bvox, int nb, const int* __restrict__ nbr,
                              const float* __restrict__ phi, int sx, int sy, int sz, float hw, float* __restrict__ out) {
    for (int b = blockIdx.x * blockDim.x + threadIdx.x; b < nb; b += gridDim.x * blockDim.x) {
        const int sv = bvox[b], slot = sv >> 9, off = sv & 511;
        out[b] = adj_read(phi, nbr, slot, (off >> 6) - sx, ((off >> 3) & 7) - sy, (off & 7) - sz, hw);
    }
}

// Band indices: leaf i's active voxels take pos[i], pos[i] + 1, ... in ZYX order.
__global__ void __launch_bounds__(512) k_adjls_band(const int* __restrict__ list, int n,
                                                   const uint64_t* __restrict__ mask, const int* __restrict__ pos,
                                                   int* __restrict__ bidx, int* __restrict__ bvox) {
    for (int i = blockIdx.x; i < n; i += gridDim.x) {
        const int s = list[i];
        const int t = threadIdx.x, w = t >> 6;
        const uint64_t word = mask[(size_t)s * 8 + w];
        int before = __popcll(word & ((1ull << (t & 63)) - 1ull));
        for (int q = 0; q < w; ++q) before += __popcll(mask[(size_t)s * 8 + q]);
        const size_t v = (size_t)i * kLeafVoxels + t;
        if ((word >> (t & 63)) & 1ull) {
            const int b = pos[i] + before;
            bidx[v] = b;
            bvox[b] = (int)v;
        } else {
            bidx[v] = -1;
        }
    }
}

}  // namespace

extern "C" {

int vlr_adj_create_level_set(vlr_ctx* ctx, vlr_level_set* ls, int steps, int checkpoint_every, vlr_adjoint** out) {
    if (!ctx || !ls || !out) return set_error(ctx, VLR_ERR_INVALID, "null argument");
    if (steps < 1 || checkpoint_every < 1) return set_error(ctx, VLR_ERR_INVALID, "bad adjoint parameters");
    if (ls->n_grids != 1) return set_error(ctx, VLR_ERR_UNSUPPORTED, "level-set adjoint of a single grid only");
    if (ls->vel_kind != MVEL_CONSTANT && ls->vel_kind != MVEL_CURL)
        return set_error(ctx, VLR_ERR_UNSUPPORTED,
                         "level-set adjoint needs a time-independent velocity (constant or curl noise)");
    if (ls->key_bits > kKeyBits) return set_error(ctx, VLR_ERR_EXTENT, "grid too wide for the adjoint's hash");
    *out = nullptr;
    cudaStream_t st = ctx->stream;
    int n = 0;
    int rc = read_int(ctx, ls->scalars, &n);
    if (rc) return rc;
    if (n <= 0) return set_error(ctx, VLR_ERR_INVALID, "empty level set");
    if ((long long)n * kLeafVoxels >= (1ll << 31)) return set_error(ctx, VLR_ERR_CAPACITY, "too many leaves");
    const vlr::MGridParams& P = ls->h_params[0];
    vlr_adjoint* a = new vlr_adjoint();
    a->ctx = ctx;
    a->n_leaves = n;
    a->hw = P.hw;
    a->dt = ls->sp.dt;
    a->t0 = ls->sp.t0;
    a->period = 1.0;
    a->steps = steps;
    a->chk_every = checkpoint_every;
    a->disp = 1;
    for (int k = 0; k < 3; ++k) a->base[k] = P.base[k];
    auto fail = [&](int code) {
        adj_free(a);
        delete a;
        return code;
    };
    const size_t pool = (size_t)n * kLeafVoxels;
    int* cnt = nullptr;  // n + 1 counts, then n + 1 positions
#define ADJ_MALLOC(p, bytes) \
    do { cudaError_t e_ = cudaMalloc(&(p), (bytes)); if (e_ != cudaSuccess) return fail(check_cuda(ctx, e_, "cudaMalloc")); } while (0)
    ADJ_MALLOC(a->origin, sizeof(int4) * n);
    ADJ_MALLOC(a->phi_init, sizeof(float) * pool);
    ADJ_MALLOC(a->bidx, sizeof(int) * pool);
    ADJ_MALLOC(cnt, sizeof(int) * (2 * (size_t)n + 4));
    int* pos = cnt + n + 2;
    const int gb = (int)std::min<long long>(n, (long long)ctx->sm_count * 8);
    if (ls->precision == VLR_PREC_F16)
        k_adjls_gather<__half><<<gb, 256, 0, st>>>(ls->list, n, ls->origin, ls->mask, (const __half*)ls->vals[0],
                                                  a->origin, a->phi_init, cnt);
    else
        k_adjls_gather<float><<<gb, 256, 0, st>>>(ls->list, n, ls->origin, ls->mask, (const float*)ls->vals[0],
                                                 a->origin, a->phi_init, cnt);
    rc = scan_exclusive(ctx, cnt, pos, n, pos + n);
    if (rc) {
        cudaFree(cnt);
        return fail(rc);
    }
    int nb = 0;
    rc = read_int(ctx, pos + n, &nb);
    if (rc || nb <= 0) {
        cudaFree(cnt);
        return fail(rc ? rc : set_error(ctx, VLR_ERR_INVALID, "empty band"));
    }
    a->n_band = nb;
    const int n_chk = steps / checkpoint_every + 1;
    a->hcap = 64;
    while ((size_t)a->hcap < 2 * (size_t)n) a->hcap <<= 1;
    ADJ_MALLOC(a->bvox, sizeof(int) * nb);
    ADJ_MALLOC(a->nbr, sizeof(int) * kNbr * (size_t)n);
    ADJ_MALLOC(a->hkey, sizeof(uint64_t) * a->hcap);
    ADJ_MALLOC(a->hval, sizeof(int) * a->hcap);
    ADJ_MALLOC(a->phi[0], sizeof(float) * pool);
    ADJ_MALLOC(a->phi[1], sizeof(float) * pool);
    ADJ_MALLOC(a->ub, sizeof(float3) * nb);
    ADJ_MALLOC(a->checkpoints, sizeof(float) * (size_t)nb * n_chk);
    ADJ_MALLOC(a->segment, sizeof(float) * (size_t)nb * checkpoint_every);
    ADJ_MALLOC(a->lam[0], sizeof(float) * nb);
    ADJ_MALLOC(a->lam[1], sizeof(float) * nb);
    ADJ_MALLOC(a->G, sizeof(float3) * nb);
    ADJ_MALLOC(a->foot_pk, sizeof(unsigned) * pool);
    ADJ_MALLOC(a->foot_w, sizeof(float4) * pool);
    ADJ_MALLOC(a->lrange, sizeof(int) * 6 * (size_t)n);
    ADJ_MALLOC(a->wrange, sizeof(int) * 6 * (size_t)n);
#undef ADJ_MALLOC
    VLR_CUDA(ctx, cudaMemsetAsync(a->foot_pk, 0, sizeof(unsigned) * pool, st));
    VLR_CUDA(ctx, cudaMemsetAsync(a->hkey, 0xFF, sizeof(uint64_t) * a->hcap, st));  // kEmptyKey
    k_adjls_band<<<gb, 512, 0, st>>>(ls->list, n, ls->mask, pos, a->bidx, a->bvox);
    k_adj_hash_insert<<<(n + 255) / 256, 256, 0, st>>>(a->origin, n, a->hkey, a->hval, a->hcap, a->base[0], a->base[1],
                                                       a->base[2], ctx->d_errword);
    k_adj_nbr<<<(int)(((size_t)n * kNbr + 255) / 256), 256, 0, st>>>(a->origin, n, a->hkey, a->hval, a->hcap,
                                                                      a->base[0], a->base[1], a->base[2], a->nbr);
    unsigned* d_max = reinterpret_cast<unsigned*>(cnt);  // the counts are consumed
    VLR_CUDA(ctx, cudaMemsetAsync(d_max, 0, sizeof(unsigned), st));
    if (ls->vel_kind == MVEL_CURL)
        k_m_feet<MVEL_CURL><<<gb, 128, 0, st>>>(a->origin, n, a->bidx, ls->d_params, ls->d_tab, (float)ls->sp.dt,
                                                ls->sp.integrator, a->ub, d_max, ctx->d_errword);
    else
        k_m_feet<MVEL_CONSTANT><<<gb, 128, 0, st>>>(a->origin, n, a->bidx, ls->d_params, ls->d_tab,
                                                    (float)ls->sp.dt, ls->sp.integrator, a->ub, d_max,
                                                    ctx->d_errword);
    VLR_CUDA(ctx, cudaGetLastError());
    unsigned mbits = 0;
    VLR_CUDA(ctx, cudaMemcpyAsync(&mbits, d_max, sizeof(unsigned), cudaMemcpyDeviceToHost, st));
    cudaError_t e = cudaStreamSynchronize(st);
    cudaFree(cnt);
    if (e != cudaSuccess) return fail(check_cuda(ctx, e, "level-set adjoint setup"));
    rc = consume_device_errors(ctx, "vlr_adj_create_level_set");
    if (rc) return fail(rc);
    float mx;
    std::memcpy(&mx, &mbits, sizeof(mx));
    a->reach = std::max(1, (int)std::ceil((double)mx * (1.0 + 1e-6)));
    if (a->reach > 6) return fail(set_error(ctx, VLR_ERR_REACH, "backtrace displacement exceeds 6 voxels per step"));
    *out = a;
    return VLR_OK;
}

int vlr_adj_set_gather(vlr_ctx* ctx, vlr_adjoint* a, int mode) {
    if (!ctx || !a) return set_error(ctx, VLR_ERR_INVALID, "null argument");
    if (mode < 0 || mode > 2) return set_error(ctx, VLR_ERR_INVALID, "gather mode must be 0, 1 or 2");
    if (mode == 2 && a->reach != 1)
        return set_error(ctx, VLR_ERR_INVALID, "the quad gather covers a reach of one voxel per step only");
    if (mode != a->gather) adj_drop_graphs(a);
    a->gather = mode;
    return VLR_OK;
}

int vlr_adj_shifted_phi0(vlr_ctx* ctx, const vlr_adjoint* a, int sx, int sy, int sz, float* d_out) {
    if (!ctx || !a || !d_out) return set_error(ctx, VLR_ERR_INVALID, "null argument");
    if (sx < -8 || sx > 8 || sy < -8 || sy > 8 || sz < -8 || sz > 8)
        return set_error(ctx, VLR_ERR_INVALID, "shift beyond 8 voxels");
    k_adj_shifted<<<blocks_for(ctx, a->n_band), 256, 0, ctx->stream>>>(a->bvox, a->n_band, a->nbr, a->phi_init, sx,
                                                                        sy, sz, a->hw, d_out);
    VLR_CUDA(ctx, cudaGetLastError());
    return VLR_OK;
}

int vlr_adj_displacement(vlr_ctx* ctx, const vlr_adjoint* a, float* out) {
    if (!ctx || !a || !out) return set_error(ctx, VLR_ERR_INVALID, "null argument");
    if (!a->disp) return set_error(ctx, VLR_ERR_UNSUPPORTED, "not a level-set adjoint");
    VLR_CUDA(ctx, cudaMemcpyAsync(out, a->ub, sizeof(float3) * a->n_band, cudaMemcpyDeviceToHost, ctx->stream));
    VLR_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    return VLR_OK;
}

int vlr_adj_create(vlr_ctx* ctx, const int32_t* origins, const uint64_t* masks, const float* phi, size_t n_leaves,
                   float half_width, const float* vel, int n_stag, double stag_cell, double dt, double period,
                   double t0, int steps, int checkpoint_every, vlr_adjoint** out) {
    if (!ctx || !origins || !masks || !phi || !vel || !out || n_leaves == 0)
        return set_error(ctx, VLR_ERR_INVALID, "null argument");
    if (n_stag < 2 || steps < 1 || checkpoint_every < 1 || !(stag_cell > 0.0) || !(dt > 0.0))
        return set_error(ctx, VLR_ERR_INVALID, "bad adjoint parameters");
    *out = nullptr;
    vlr_adjoint* a = new vlr_adjoint();
    a->ctx = ctx;
    a->n_leaves = (int)n_leaves;
    a->hw = half_width;
    a->n_stag = n_stag;
    a->H = stag_cell;
    a->dt = dt;
    a->period = period;
    a->t0 = t0;
    a->steps = steps;
    a->chk_every = checkpoint_every;
    auto fail = [&](int rc) {
        adj_free(a);
        delete a;
        return rc;
    };
    int rc = choose_base(ctx, origins, n_leaves, a->base);
    if (rc) return fail(rc);
    // band: active voxels, in leaf order then ZYX
    std::vector<int> bidx(n_leaves * 512, -1), bvox;
    for (size_t i = 0; i < n_leaves; ++i)
        for (int off = 0; off < 512; ++off)
            if ((masks[8 * i + (off >> 6)] >> (off & 63)) & 1ull) {
                bidx[i * 512 + off] = (int)bvox.size();
                bvox.push_back((int)(i * 512 + off));
            }
    a->n_band = (int)bvox.size();
    if (a->n_band == 0) return fail(set_error(ctx, VLR_ERR_INVALID, "empty band"));
    const size_t nb = (size_t)a->n_band;
    a->hcap = 64;
    while ((size_t)a->hcap < 2 * n_leaves) a->hcap <<= 1;
    std::vector<int4> o4(n_leaves);
    for (size_t i = 0; i < n_leaves; ++i) o4[i] = make_int4(origins[3 * i], origins[3 * i + 1], origins[3 * i + 2], 0);
    size_t nvel = 3ull * n_stag * n_stag * n_stag;
    int n_chk = steps / checkpoint_every + 1;
    a->n_pairs_cap = std::max(nb * 8, nb * 24);
#define ADJ_MALLOC(p, bytes) \
    do { cudaError_t e_ = cudaMalloc(&(p), (bytes)); if (e_ != cudaSuccess) return fail(check_cuda(ctx, e_, "cudaMalloc")); } while (0)
    ADJ_MALLOC(a->origin, sizeof(int4) * n_leaves);
    ADJ_MALLOC(a->nbr, sizeof(int) * kNbr * n_leaves);
    ADJ_MALLOC(a->hkey, sizeof(uint64_t) * a->hcap);
    ADJ_MALLOC(a->hval, sizeof(int) * a->hcap);
    ADJ_MALLOC(a->phi[0], sizeof(float) * 512 * n_leaves);
    ADJ_MALLOC(a->phi[1], sizeof(float) * 512 * n_leaves);
    ADJ_MALLOC(a->phi_init, sizeof(float) * 512 * n_leaves);
    ADJ_MALLOC(a->bidx, sizeof(int) * 512 * n_leaves);
    ADJ_MALLOC(a->bvox, sizeof(int) * nb);
    ADJ_MALLOC(a->ub, sizeof(float3) * nb);
    ADJ_MALLOC(a->vel, sizeof(float) * nvel);
    ADJ_MALLOC(a->checkpoints, sizeof(float) * nb * n_chk);
    ADJ_MALLOC(a->segment, sizeof(float) * nb * checkpoint_every);
    ADJ_MALLOC(a->lam[0], sizeof(float) * nb);
    ADJ_MALLOC(a->lam[1], sizeof(float) * nb);
    ADJ_MALLOC(a->gvel, sizeof(float) * nvel);
    ADJ_MALLOC(a->foot_pk, sizeof(unsigned) * 512 * n_leaves);
    ADJ_MALLOC(a->foot_w, sizeof(float4) * 512 * n_leaves);
    ADJ_MALLOC(a->lrange, sizeof(int) * 6 * n_leaves);
    ADJ_MALLOC(a->wrange, sizeof(int) * 6 * n_leaves);
    VLR_CUDA(ctx, cudaMemsetAsync(a->foot_pk, 0, sizeof(unsigned) * 512 * n_leaves, ctx->stream));
    ADJ_MALLOC(a->G, sizeof(float3) * nb);
    ADJ_MALLOC(a->keys, sizeof(unsigned) * a->n_pairs_cap);
    ADJ_MALLOC(a->pvals, sizeof(float) * a->n_pairs_cap);
    ADJ_MALLOC(a->scratch, sort_reduce_scratch_bytes((int)a->n_pairs_cap));
#undef ADJ_MALLOC
    cudaStream_t st = ctx->stream;
    VLR_CUDA(ctx, cudaMemcpyAsync(a->origin, o4.data(), sizeof(int4) * n_leaves, cudaMemcpyHostToDevice, st));
    VLR_CUDA(ctx, cudaMemcpyAsync(a->phi_init, phi, sizeof(float) * 512 * n_leaves, cudaMemcpyHostToDevice, st));
    VLR_CUDA(ctx, cudaMemcpyAsync(a->bidx, bidx.data(), sizeof(int) * 512 * n_leaves, cudaMemcpyHostToDevice, st));
    VLR_CUDA(ctx, cudaMemcpyAsync(a->bvox, bvox.data(), sizeof(int) * nb, cudaMemcpyHostToDevice, st));
    a->reach = reach_of(vel, nvel, dt);
    if (a->reach > 6) return fail(set_error(ctx, VLR_ERR_REACH, "dt * max|V| exceeds 6 voxels per step"));
    VLR_CUDA(ctx, cudaMemcpyAsync(a->vel, vel, sizeof(float) * nvel, cudaMemcpyHostToDevice, st));
    std::vector<uint64_t> hk(a->hcap, kEmptyKey);
    VLR_CUDA(ctx, cudaMemcpyAsync(a->hkey, hk.data(), sizeof(uint64_t) * a->hcap, cudaMemcpyHostToDevice, st));
    k_adj_hash_insert<<<(int)((n_leaves + 255) / 256), 256, 0, st>>>(a->origin, (int)n_leaves, a->hkey, a->hval,
                                                                     a->hcap, a->base[0], a->base[1], a->base[2],
                                                                     ctx->d_errword);
    k_adj_nbr<<<(int)((n_leaves * kNbr + 255) / 256), 256, 0, st>>>(a->origin, (int)n_leaves, a->hkey, a->hval, a->hcap,
                                                                    a->base[0], a->base[1], a->base[2], a->nbr);
    k_adj_upsample<<<blocks_for(ctx, nb), 256, 0, st>>>(a->bvox, a->origin, (int)nb, a->vel, n_stag, (float)stag_cell,
                                                        a->ub);
    cudaError_t e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return fail(check_cuda(ctx, e, "adjoint setup"));
    rc = consume_device_errors(ctx, "vlr_adj_create");
    if (rc) return fail(rc);
    *out = a;
    return VLR_OK;
}

int vlr_adj_band(vlr_ctx* ctx, const vlr_adjoint* a, int32_t* coords, size_t cap, size_t* n) {
    if (!ctx || !a || !n) return set_error(ctx, VLR_ERR_INVALID, "null argument");
    *n = (size_t)a->n_band;
    if (!coords) return VLR_OK;
    if (cap < *n) return set_error(ctx, VLR_ERR_CAPACITY, "coordinate buffer too small");
    std::vector<int> bvox(a->n_band);
    std::vector<int4> o4(a->n_leaves);
    VLR_CUDA(ctx, cudaMemcpy(bvox.data(), a->bvox, sizeof(int) * a->n_band, cudaMemcpyDeviceToHost));
    VLR_CUDA(ctx, cudaMemcpy(o4.data(), a->origin, sizeof(int4) * a->n_leaves, cudaMemcpyDeviceToHost));
    for (int b = 0; b < a->n_band; ++b) {
        int s = bvox[b] >> 9, off = bvox[b] & 511;
        coords[3 * b] = o4[s].x + (off >> 6);
        coords[3 * b + 1] = o4[s].y + ((off >> 3) & 7);
        coords[3 * b + 2] = o4[s].z + (off & 7);
    }
    return VLR_OK;
}

int vlr_adj_set_inputs(vlr_ctx* ctx, vlr_adjoint* a, const float* phi0_band, const float* vel) {
    if (!ctx || !a) return set_error(ctx, VLR_ERR_INVALID, "null argument");
    if (vel && a->disp) return set_error(ctx, VLR_ERR_UNSUPPORTED, "a level-set adjoint has no velocity field input");
    cudaStream_t st = ctx->stream;
    if (phi0_band) {
        VLR_CUDA(ctx, cudaMemcpyAsync(a->lam[1], phi0_band, sizeof(float) * a->n_band, cudaMemcpyHostToDevice, st));
        k_adj_scatter_band<<<blocks_for(ctx, a->n_band), 256, 0, st>>>(a->bvox, a->n_band, a->lam[1], a->phi_init);
    }
    if (vel) {
        size_t nvel = 3ull * a->n_stag * a->n_stag * a->n_stag;
        const int reach = reach_of(vel, nvel, a->dt);
        if (reach > 6) return set_error(ctx, VLR_ERR_REACH, "dt * max|V| exceeds 6 voxels per step");
        if (reach != a->reach) adj_drop_graphs(a);
        a->reach = reach;
        VLR_CUDA(ctx, cudaMemcpyAsync(a->vel, vel, sizeof(float) * nvel, cudaMemcpyHostToDevice, st));
        k_adj_upsample<<<blocks_for(ctx, a->n_band), 256, 0, st>>>(a->bvox, a->origin, a->n_band, a->vel, a->n_stag,
                                                                   (float)a->H, a->ub);
    }
    VLR_CUDA(ctx, cudaGetLastError());
    VLR_CUDA(ctx, cudaStreamSynchronize(st));
    return VLR_OK;
}

// Forward K steps from the initial state; checkpoints every C steps; writes
// phi_K on the band (host, n_band floats) when phi_k_band is not null.
int vlr_adj_forward_device(vlr_ctx* ctx, vlr_adjoint* a, float* d_phi_k_band) {
    if (!ctx || !a) return set_error(ctx, VLR_ERR_INVALID, "null argument");
    int rc = run_captured(ctx, &a->fwd_exec, [&]() { return adj_forward_enqueue(ctx, a); });
    if (rc) return rc;
    if (d_phi_k_band)
        VLR_CUDA(ctx, cudaMemcpyAsync(d_phi_k_band, a->lam[1], sizeof(float) * a->n_band, cudaMemcpyDeviceToDevice,
                                      ctx->stream));
    return VLR_OK;
}

int vlr_adj_forward(vlr_ctx* ctx, vlr_adjoint* a, float* phi_k_band) {
    int rc = vlr_adj_forward_device(ctx, a, nullptr);
    if (rc) return rc;
    if (phi_k_band)
        VLR_CUDA(ctx, cudaMemcpyAsync(phi_k_band, a->lam[1], sizeof(float) * a->n_band, cudaMemcpyDeviceToHost,
                                      ctx->stream));
    VLR_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    return consume_device_errors(ctx, "vlr_adj_forward");
}

// Backward pass (vlr_adj_forward must have run): grad_phik_band = dL/dphi_K
// on the band; writes dL/dphi_0 (n_band) and dL/dV (3 n^3), host buffers.
int vlr_adj_backward_device(vlr_ctx* ctx, vlr_adjoint* a, const float* d_grad_phik_band, float* d_grad_phi0_band,
                            float* d_grad_vel) {
    if (!ctx || !a || !d_grad_phik_band) return set_error(ctx, VLR_ERR_INVALID, "null argument");
    if (d_grad_vel && a->disp) return set_error(ctx, VLR_ERR_UNSUPPORTED, "a level-set adjoint has no velocity gradient");
    cudaStream_t st = ctx->stream;
    const size_t nb = (size_t)a->n_band;
    if (d_grad_phik_band != a->lam[1])
        VLR_CUDA(ctx, cudaMemcpyAsync(a->lam[1], d_grad_phik_band, sizeof(float) * nb, cudaMemcpyDeviceToDevice, st));
    int rc = run_captured(ctx, &a->bwd_exec, [&]() { return adj_backward_enqueue(ctx, a); });
    if (rc) return rc;
    float* lam = a->bwd_final;
    a->lam_final = lam;
    if (d_grad_phi0_band)
        VLR_CUDA(ctx, cudaMemcpyAsync(d_grad_phi0_band, lam, sizeof(float) * nb, cudaMemcpyDeviceToDevice, st));
    if (d_grad_vel) {
        size_t nvel = 3ull * a->n_stag * a->n_stag * a->n_stag;
        VLR_TIMED(ctx, "k_adj_emit_vel",
                  k_adj_emit_vel<<<blocks_for(ctx, nb), 256, 0, st>>>(a->bvox, a->origin, (int)nb, a->G, a->n_stag,
                                                                      (float)a->H, a->keys, a->pvals));
        rc = sort_reduce(ctx, a->keys, a->pvals, (int)(nb * 24), (unsigned)nvel + 1, d_grad_vel, (unsigned)nvel,
                         a->scratch);
        if (rc) return rc;
    }
    return VLR_OK;
}

int vlr_adj_backward(vlr_ctx* ctx, vlr_adjoint* a, const float* grad_phik_band, float* grad_phi0_band,
                     float* grad_vel) {
    if (!ctx || !a || !grad_phik_band) return set_error(ctx, VLR_ERR_INVALID, "null argument");
    if (grad_vel && a->disp) return set_error(ctx, VLR_ERR_UNSUPPORTED, "a level-set adjoint has no velocity gradient");
    cudaStream_t st = ctx->stream;
    const size_t nb = (size_t)a->n_band;
    VLR_CUDA(ctx, cudaMemcpyAsync(a->lam[1], grad_phik_band, sizeof(float) * nb, cudaMemcpyHostToDevice, st));
    int rc = vlr_adj_backward_device(ctx, a, a->lam[1], nullptr, grad_vel ? a->gvel : nullptr);
    if (rc) return rc;
    if (grad_phi0_band)
        VLR_CUDA(ctx, cudaMemcpyAsync(grad_phi0_band, a->lam_final, sizeof(float) * nb, cudaMemcpyDeviceToHost, st));
    if (grad_vel)
        VLR_CUDA(ctx, cudaMemcpyAsync(grad_vel, a->gvel, sizeof(float) * 3ull * a->n_stag * a->n_stag * a->n_stag,
                                      cudaMemcpyDeviceToHost, st));
    VLR_CUDA(ctx, cudaStreamSynchronize(st));
    return consume_device_errors(ctx, "vlr_adj_backward");
}

void vlr_adj_destroy(vlr_adjoint* a) {
    if (!a) return;
    if (a->ctx) cudaStreamSynchronize(a->ctx->stream);
    adj_free(a);
    delete a;
}

}  // extern "C"
