// dilate (src/tools/morphology.rs:20-35) on a device grid: `iterations`
// times, every inactive voxel with an active 6-neighbour becomes active and
// takes the value of one of them.
//
// The reference snapshots the active voxels in its tree's iteration order and
// lets each one write its inactive 6-neighbours, first writer wins, so a new
// voxel gets the value of its active neighbour that comes first in that order:
// 128^3 tiles in the root map's order, then leaves in child index order inside
// a tile (x, then y, then z), then voxels in leaf offset order (x*64+y*8+z).
// The root map's order is unspecified (a HashMap); here tiles go in ascending
// (x, y, z) of their origin, one realisation of it (the oracle iterates the
// same way).  The topology does not depend on the order.
//
// Per iteration: k_dil_spill flags leaf faces that hold active voxels next to
// a missing leaf; the host merges the new leaves into the pool's (x, y, z)
// order (they start inactive at the background, as set() allocates them);
// k_dilate then computes every new voxel from the snapshot mask, writing
// values in place (it writes only voxels inactive in the snapshot and reads
// only voxels active in it) and the new mask into scratch.
#include <algorithm>
#include <cstring>
#include <numeric>
#include <vector>

#include "ref_ops.hpp"

using namespace vlr;

namespace vlr {
int grid_add_leaves(vlr_ctx* ctx, vlr_grid* g, const std::vector<int32_t>& origins);
}

namespace {

// neighbour-table index of the 6 face directions -x, +x, -y, +y, -z, +z
__constant__ int kFaceNbr[6] = {4, 22, 10, 16, 12, 14};

__global__ void k_dil_spill(const uint64_t* __restrict__ mask, const int* __restrict__ nbr, int n,
                            unsigned char* __restrict__ flags) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        uint64_t any = 0, y0 = 0, y7 = 0, z0 = 0, z7 = 0;
        uint64_t w[8];
#pragma unroll
        for (int q = 0; q < 8; ++q) {
            w[q] = mask[(size_t)i * 8 + q];
            any |= w[q];
            y0 |= w[q] & 0xFFull;
            y7 |= w[q] & (0xFFull << 56);
            z0 |= w[q] & 0x0101010101010101ull;
            z7 |= w[q] & 0x8080808080808080ull;
        }
        (void)any;
        const bool face[6] = {w[0] != 0, w[7] != 0, y0 != 0, y7 != 0, z0 != 0, z7 != 0};
        unsigned char f = 0;
#pragma unroll
        for (int d = 0; d < 6; ++d)
            if (face[d] && nbr[(size_t)i * kNbr + kFaceNbr[d]] < 0) f |= (unsigned char)(1u << d);
        flags[i] = f;
    }
}

// Old leaf i -> slot dst_old[i]; new leaf j -> slot dst_new[j] (inactive, background).
__global__ void k_dil_merge(int n_old, const int* __restrict__ dst_old, const int4* __restrict__ o_in,
                            const uint64_t* __restrict__ m_in, const float* __restrict__ v_in, int n_new,
                            const int* __restrict__ dst_new, const int4* __restrict__ o_new, float bg,
                            int4* __restrict__ o_out, uint64_t* __restrict__ m_out, float* __restrict__ v_out) {
    for (int i = blockIdx.x; i < n_old + n_new; i += gridDim.x) {
        const bool old = i < n_old;
        const int d = old ? dst_old[i] : dst_new[i - n_old];
        if (threadIdx.x == 0) o_out[d] = old ? o_in[i] : o_new[i - n_old];
        if (threadIdx.x < 8) m_out[(size_t)d * 8 + threadIdx.x] = old ? m_in[(size_t)i * 8 + threadIdx.x] : 0ull;
        for (int t = threadIdx.x; t < kLeafVoxels; t += blockDim.x)
            v_out[(size_t)d * kLeafVoxels + t] = old ? v_in[(size_t)i * kLeafVoxels + t] : bg;
    }
}

// Iteration-order key comparison of two voxels: tile (c >> 7), then leaf in
// tile ((c >> 3) & 15), then voxel in leaf (c & 7), each x then y then z.
__device__ __forceinline__ bool key_less(int ax, int ay, int az, int bx, int by, int bz) {
    const int sh[3] = {7, 3, 0};
    const int mk[3] = {-1, 15, 7};
#pragma unroll
    for (int l = 0; l < 3; ++l) {
        const int a0 = (ax >> sh[l]) & mk[l], b0 = (bx >> sh[l]) & mk[l];
        if (a0 != b0) return a0 < b0;
        const int a1 = (ay >> sh[l]) & mk[l], b1 = (by >> sh[l]) & mk[l];
        if (a1 != b1) return a1 < b1;
        const int a2 = (az >> sh[l]) & mk[l], b2 = (bz >> sh[l]) & mk[l];
        if (a2 != b2) return a2 < b2;
    }
    return false;
}

// One CTA (256 threads) per leaf, 2 voxels per thread.
__global__ void __launch_bounds__(256) k_dilate(const int4* __restrict__ origin, const uint64_t* __restrict__ mask,
                                                const int* __restrict__ nbr, int n, float* __restrict__ values,
                                                uint64_t* __restrict__ mask_out) {
    __shared__ unsigned s_w[16];
    const int lane = threadIdx.x & 31;
    for (int i = blockIdx.x; i < n; i += gridDim.x) {
        const int4 o = origin[i];
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            const int off = threadIdx.x + 256 * h;
            const int x = off >> 6, y = (off >> 3) & 7, z = off & 7;
            const bool was = (mask[(size_t)i * 8 + (off >> 6)] >> (off & 63)) & 1ull;
            bool on = was;
            if (!was) {
                int bx = 0, by = 0, bz = 0, bslot = -1, boff = 0;
#pragma unroll
                for (int d = 0; d < 6; ++d) {
                    const int a = d >> 1, sgn = (d & 1) ? 1 : -1;
                    const int nx = x + (a == 0 ? sgn : 0), ny = y + (a == 1 ? sgn : 0), nz = z + (a == 2 ? sgn : 0);
                    const int slot = (nx >= 0 && nx < 8 && ny >= 0 && ny < 8 && nz >= 0 && nz < 8)
                                         ? i
                                         : nbr[(size_t)i * kNbr + kFaceNbr[d]];
                    if (slot < 0) continue;
                    const int noff = ((nx & 7) << 6) | ((ny & 7) << 3) | (nz & 7);
                    if (!((mask[(size_t)slot * 8 + (noff >> 6)] >> (noff & 63)) & 1ull)) continue;
                    const int gx = o.x + nx, gy = o.y + ny, gz = o.z + nz;
                    if (bslot < 0 || key_less(gx, gy, gz, bx, by, bz)) {
                        bx = gx;
                        by = gy;
                        bz = gz;
                        bslot = slot;
                        boff = noff;
                    }
                }
                if (bslot >= 0) {
                    values[(size_t)i * kLeafVoxels + off] = values[(size_t)bslot * kLeafVoxels + boff];
                    on = true;
                }
            }
            const unsigned b = __ballot_sync(0xffffffffu, on);
            if (lane == 0) s_w[off >> 5] = b;
        }
        __syncthreads();
        if (threadIdx.x < 8)
            mask_out[(size_t)i * 8 + threadIdx.x] =
                (uint64_t)s_w[2 * threadIdx.x] | ((uint64_t)s_w[2 * threadIdx.x + 1] << 32);
        __syncthreads();
    }
}

bool less3(const int32_t* a, const int32_t* b) {
    if (a[0] != b[0]) return a[0] < b[0];
    if (a[1] != b[1]) return a[1] < b[1];
    return a[2] < b[2];
}

int grow_for_dilation(vlr_ctx* ctx, vlr_grid* g) {
    const int n = g->n;
    if (n == 0) return VLR_OK;
    void* scratch = nullptr;
    int rc = ctx_scratch(ctx, (size_t)n * (1 + sizeof(int4)) + 256, &scratch);
    if (rc) return rc;
    unsigned char* d_flags = static_cast<unsigned char*>(scratch);
    k_dil_spill<<<std::min((n + 255) / 256, ctx->sm_count * 8), 256, 0, ctx->stream>>>(g->mask, g->nbr, n, d_flags);
    VLR_CUDA(ctx, cudaGetLastError());
    std::vector<unsigned char> flags(n);
    std::vector<int4> org(n);
    VLR_CUDA(ctx, cudaMemcpyAsync(flags.data(), d_flags, n, cudaMemcpyDeviceToHost, ctx->stream));
    VLR_CUDA(ctx, cudaMemcpyAsync(org.data(), g->origin, sizeof(int4) * n, cudaMemcpyDeviceToHost, ctx->stream));
    VLR_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    static const int kStep[6][3] = {{-8, 0, 0}, {8, 0, 0}, {0, -8, 0}, {0, 8, 0}, {0, 0, -8}, {0, 0, 8}};
    std::vector<int32_t> nw;  // new leaf origins (3 per leaf)
    for (int i = 0; i < n; ++i)
        for (int d = 0; d < 6; ++d)
            if (flags[i] >> d & 1)
                nw.insert(nw.end(), {org[i].x + kStep[d][0], org[i].y + kStep[d][1], org[i].z + kStep[d][2]});
    return grid_add_leaves(ctx, g, nw);
}

}  // namespace

namespace vlr {

// Add leaves at the given origins (3 ints each, any order, repeats and
// origins already present allowed) to a world-unit f32 grid, inactive at the
// background, keeping the pool in (x, y, z) order of origin; rebuilds the
// hash and neighbour table when anything was added.
int grid_add_leaves(vlr_ctx* ctx, vlr_grid* g, const std::vector<int32_t>& origins) {
    const int n = g->n;
    const size_t m0 = origins.size() / 3;
    if (!m0) return VLR_OK;
    std::vector<int4> org(n);
    if (n)
        VLR_CUDA(ctx, cudaMemcpyAsync(org.data(), g->origin, sizeof(int4) * n, cudaMemcpyDeviceToHost, ctx->stream));
    VLR_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    std::vector<int> ord(m0);
    std::iota(ord.begin(), ord.end(), 0);
    std::sort(ord.begin(), ord.end(), [&](int a, int b) { return less3(&origins[3 * a], &origins[3 * b]); });
    std::vector<int32_t> uniq;
    for (size_t k = 0; k < m0; ++k) {
        const int32_t* c = &origins[3 * ord[k]];
        if (k > 0 && !less3(&origins[3 * ord[k - 1]], c)) continue;
        // skip origins the grid already holds (the pool is sorted)
        const int4 key = make_int4(c[0], c[1], c[2], 0);
        const bool present = std::binary_search(org.begin(), org.end(), key, [](const int4& a, const int4& b) {
            if (a.x != b.x) return a.x < b.x;
            if (a.y != b.y) return a.y < b.y;
            return a.z < b.z;
        });
        if (!present) uniq.insert(uniq.end(), c, c + 3);
    }
    const int m = (int)(uniq.size() / 3);
    if (!m) return VLR_OK;
    // merged (x, y, z) order of the old leaves (already sorted) and the new ones
    std::vector<int> dst_old(n), dst_new(m);
    std::vector<int4> o_new(m);
    std::vector<int32_t> all(3 * (size_t)(n + m));
    {
        int a = 0, b = 0, k = 0;
        while (a < n || b < m) {
            const int32_t oa[3] = {a < n ? org[a].x : 0, a < n ? org[a].y : 0, a < n ? org[a].z : 0};
            const bool take_old = b >= m || (a < n && less3(oa, &uniq[3 * b]));
            if (take_old) {
                dst_old[a] = k;
                std::memcpy(&all[3 * k], oa, 12);
                ++a;
            } else {
                dst_new[b] = k;
                o_new[b] = make_int4(uniq[3 * b], uniq[3 * b + 1], uniq[3 * b + 2], 0);
                std::memcpy(&all[3 * k], &uniq[3 * b], 12);
                ++b;
            }
            ++k;
        }
    }
    long long base[3];
    int rc = choose_base(ctx, all.data(), (size_t)(n + m), base);
    if (rc) return rc;
    vlr_grid tmp;
    tmp.ctx = ctx;
    tmp.kind = g->kind;
    rc = grid_alloc(ctx, &tmp, n + m);
    if (rc) return rc;
    // new-leaf origins (int4, 16-byte aligned) first, then the destination indices
    int4* d_onew = nullptr;
    VLR_CUDA(ctx,
             cudaMallocFromPoolAsync(&d_onew, sizeof(int4) * m + sizeof(int) * (n + m), ctx->pool, ctx->stream));
    int* d_idx = reinterpret_cast<int*>(d_onew + m);
    if (n)
        VLR_CUDA(ctx, cudaMemcpyAsync(d_idx, dst_old.data(), sizeof(int) * n, cudaMemcpyHostToDevice, ctx->stream));
    VLR_CUDA(ctx, cudaMemcpyAsync(d_idx + n, dst_new.data(), sizeof(int) * m, cudaMemcpyHostToDevice, ctx->stream));
    VLR_CUDA(ctx, cudaMemcpyAsync(d_onew, o_new.data(), sizeof(int4) * m, cudaMemcpyHostToDevice, ctx->stream));
    k_dil_merge<<<std::min(n + m, ctx->sm_count * 16), 128, 0, ctx->stream>>>(
        n, d_idx, g->origin, g->mask, (const float*)g->values, m, d_idx + n, d_onew, g->background, tmp.origin,
        tmp.mask, (float*)tmp.values);
    VLR_CUDA(ctx, cudaGetLastError());
    VLR_CUDA(ctx, cudaFreeAsync(d_onew, ctx->stream));
    VLR_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    std::swap(g->block, tmp.block);
    std::swap(g->origin, tmp.origin);
    std::swap(g->mask, tmp.mask);
    std::swap(g->values, tmp.values);
    std::swap(g->nbr, tmp.nbr);
    std::swap(g->hkey, tmp.hkey);
    std::swap(g->hval, tmp.hval);
    std::swap(g->hcap, tmp.hcap);
    std::swap(g->cap, tmp.cap);
    grid_free_arrays(&tmp);
    g->n = n + m;
    std::memcpy(g->base, base, sizeof(base));
    return grid_index(ctx, g);
}

}  // namespace vlr

// flood_fill_sign (src/tools/flood_fill.rs:18-107), one CTA per leaf and one
// thread per voxel: the leaf's active-voxel sign counts by CTA-wide counts,
// then each inactive voxel's active 6-neighbours inside the leaf, read from a
// shared-memory snapshot of the leaf, so the result is order independent.
__global__ void __launch_bounds__(512) k_flood_fill(const uint64_t* __restrict__ mask, float* __restrict__ values,
                                                   float bg) {
    __shared__ uint64_t s_m[8];
    __shared__ float s_v[512];
    const size_t leaf = blockIdx.x;
    const int t = threadIdx.x;
    if (t < 8) s_m[t] = mask[leaf * 8 + t];
    const float v = values[leaf * 512 + t];
    s_v[t] = v;
    __syncthreads();
    const bool on = (s_m[t >> 6] >> (t & 63)) & 1ull;
    const int neg = __syncthreads_count(on && v < 0.0f);
    const int act = __syncthreads_count(on);
    if (act == 0 || on) return;
    const float global = neg > act - neg ? -bg : bg;
    const int lx = t >> 6, ly = (t >> 3) & 7, lz = t & 7;
    int ln = 0, lp = 0;
    const int d[6][3] = {{-1, 0, 0}, {1, 0, 0}, {0, -1, 0}, {0, 1, 0}, {0, 0, -1}, {0, 0, 1}};
#pragma unroll
    for (int k = 0; k < 6; ++k) {
        const int nx = lx + d[k][0], ny = ly + d[k][1], nz = lz + d[k][2];
        if (nx < 0 || nx > 7 || ny < 0 || ny > 7 || nz < 0 || nz > 7) continue;
        const int no = (nx << 6) | (ny << 3) | nz;
        if (!((s_m[no >> 6] >> (no & 63)) & 1ull)) continue;
        if (s_v[no] < 0.0f) ++ln;
        else ++lp;
    }
    values[leaf * 512 + t] = (ln + lp > 0) ? (ln > lp ? -bg : bg) : global;
}

extern "C" {

int vlr_dilate(vlr_ctx* ctx, vlr_grid* g, unsigned iterations) {
    if (!ctx || !g) return set_error(ctx, VLR_ERR_INVALID, "null argument");
    if (g->kind != VLR_KIND_F32_WORLD) return set_error(ctx, VLR_ERR_INVALID, "grid is not a world-unit f32 grid");
    for (unsigned it = 0; it < iterations; ++it) {
        int rc = grow_for_dilation(ctx, g);
        if (rc) return rc;
        if (g->n == 0) break;
        void* scratch = nullptr;
        rc = ctx_scratch(ctx, 64ull * g->n, &scratch);
        if (rc) return rc;
        uint64_t* m_new = static_cast<uint64_t*>(scratch);
        k_dilate<<<std::min(g->n, ctx->sm_count * 8), 256, 0, ctx->stream>>>(g->origin, g->mask, g->nbr, g->n,
                                                                             (float*)g->values, m_new);
        VLR_CUDA(ctx, cudaGetLastError());
        VLR_CUDA(ctx, cudaMemcpyAsync(g->mask, m_new, 64ull * g->n, cudaMemcpyDeviceToDevice, ctx->stream));
        VLR_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    }
    return consume_device_errors(ctx, "vlr_dilate");
}

int vlr_flood_fill_sign(vlr_ctx* ctx, vlr_grid* g) {
    if (!ctx || !g) return set_error(ctx, VLR_ERR_INVALID, "null argument");
    if (g->kind != VLR_KIND_F32_WORLD) return set_error(ctx, VLR_ERR_INVALID, "grid is not a world-unit f32 grid");
    if (g->n == 0) return VLR_OK;
    VLR_TIMED(ctx, "k_flood_fill",
              k_flood_fill<<<g->n, 512, 0, ctx->stream>>>(g->mask, (float*)g->values, g->background));
    VLR_CUDA(ctx, cudaGetLastError());
    return VLR_OK;
}

}  // extern "C"
