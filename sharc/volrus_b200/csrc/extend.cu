// extend_velocity (src/tools/level_set_track.rs:115-160) on device grids.
//
// Interface voxels: active in the SDF with |phi| < voxel size (f32).  Band
// voxels: active with voxel size <= |phi| < half_width * voxel size.  Every
// band voxel copies (vx, vy, vz) from its nearest interface voxel by integer
// squared distance, the first such voxel in the SDF's iteration order on a
// tie (min_by_key), and becomes active in each velocity grid (Grid::set),
// allocating the velocity grid's leaf when it is missing.
//
// Search: one CTA per SDF leaf collects the interface voxels of its 27-leaf
// neighbourhood in shared memory and each band voxel takes the minimum over
// them.  Any voxel outside that 24^3 region is at least 9 voxels away, so an
// in-region minimum below 81 is the global one (ties included); band voxels
// without one (or whose neighbourhood holds more interface voxels than the
// shared list) search the whole interface list instead.  Sources are interface
// voxels and targets band voxels, disjoint sets, so the copies are
// independent of order.  Ties use the iteration order of dilate
// (csrc/morphology.cu): 128^3 tiles, leaves in a tile, voxels in a leaf, each
// x then y then z, tiles in ascending origin order.
#include <algorithm>
#include <cstring>
#include <numeric>
#include <vector>

#include "ref_ops.hpp"

using namespace vlr;

namespace {

constexpr int kMaxLocal = 4096;  // interface voxels held per 27-leaf neighbourhood
constexpr int kBuckets = 24;     // 1-voxel distance shells around the leaf centre (a candidate is < 20 away)

// Shell of a candidate (local coordinates packed as in s_cand): the floor of
// its distance from the leaf centre (3.5, 3.5, 3.5).
__device__ __forceinline__ int ev_bucket(unsigned e) {
    const int cx = 2 * ((int)(e & 31u) - 8) - 7, cy = 2 * ((int)((e >> 5) & 31u) - 8) - 7,
              cz = 2 * ((int)(e >> 10) - 8) - 7;
    return min((int)(0.5f * sqrtf((float)(cx * cx + cy * cy + cz * cz))), kBuckets - 1);
}

__device__ __forceinline__ bool ev_key_less(int ax, int ay, int az, int bx, int by, int bz) {
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

// One CTA (256 threads) per leaf: interface and band masks, band count.
__global__ void __launch_bounds__(256) k_ev_classify(const uint64_t* __restrict__ mask, const float* __restrict__ values,
                                                     int n, float vs, float band, uint64_t* __restrict__ imask,
                                                     uint64_t* __restrict__ bmask, int* __restrict__ bcount) {
    __shared__ unsigned s_i[16], s_b[16];
    const int lane = threadIdx.x & 31;
    for (int i = blockIdx.x; i < n; i += gridDim.x) {
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            const int off = threadIdx.x + 256 * h;
            const bool on = (mask[(size_t)i * 8 + (off >> 6)] >> (off & 63)) & 1ull;
            const float a = fabsf(values[(size_t)i * kLeafVoxels + off]);
            const unsigned bi = __ballot_sync(0xffffffffu, on && a < vs);
            const unsigned bb = __ballot_sync(0xffffffffu, on && a >= vs && a < band);
            if (lane == 0) {
                s_i[off >> 5] = bi;
                s_b[off >> 5] = bb;
            }
        }
        __syncthreads();
        if (threadIdx.x < 8) {
            const int q = threadIdx.x;
            imask[(size_t)i * 8 + q] = (uint64_t)s_i[2 * q] | ((uint64_t)s_i[2 * q + 1] << 32);
            const uint64_t b = (uint64_t)s_b[2 * q] | ((uint64_t)s_b[2 * q + 1] << 32);
            bmask[(size_t)i * 8 + q] = b;
            int c = __popcll(b);
#pragma unroll
            for (int d = 1; d < 8; d <<= 1) c += __shfl_xor_sync(0xffu, c, d);
            if (q == 0) bcount[i] = c;
        }
        __syncthreads();
    }
}

// One CTA (256 threads) per leaf: nearest interface voxel of every band voxel
// within the 27-leaf neighbourhood; pairs written at boff[leaf] + rank.
__global__ void __launch_bounds__(256) k_ev_search(const int4* __restrict__ origin, const int* __restrict__ nbr, int n,
                                                   const uint64_t* __restrict__ imask,
                                                   const uint64_t* __restrict__ bmask, const int* __restrict__ boff,
                                                   int4* __restrict__ dst, int4* __restrict__ src,
                                                   int* __restrict__ fb_list, int* __restrict__ fb_count) {
    __shared__ unsigned s_cand[kMaxLocal];  // (x+8) | (y+8) << 5 | (z+8) << 10, local to the leaf
    __shared__ unsigned s_sorted[kMaxLocal];  // the same, grouped by shell
    __shared__ int s_start[kBuckets + 1], s_cur[kBuckets];
    __shared__ int s_n;
    __shared__ uint64_t s_b[8];
    for (int i = blockIdx.x; i < n; i += gridDim.x) {
        if (threadIdx.x == 0) s_n = 0;
        if (threadIdx.x < 8) s_b[threadIdx.x] = bmask[(size_t)i * 8 + threadIdx.x];
        __syncthreads();
        // 27 neighbours x 8 words: one (neighbour, word) per thread
        for (int t = threadIdx.x; t < kNbr * 8; t += blockDim.x) {
            const int d = t >> 3, q = t & 7;
            const int s = nbr[(size_t)i * kNbr + d];
            if (s < 0) continue;
            uint64_t w = imask[(size_t)s * 8 + q];
            if (!w) continue;
            const int dx = d / 9 - 1, dy = (d / 3) % 3 - 1, dz = d % 3 - 1;
            const int pos = atomicAdd(&s_n, __popcll(w));
            int k = 0;
            while (w) {
                const int bit = __ffsll((long long)w) - 1;
                w &= w - 1;
                const int x = 8 * dx + q, y = 8 * dy + (bit >> 3), z = 8 * dz + (bit & 7);
                if (pos + k < kMaxLocal)
                    s_cand[pos + k] = (unsigned)(x + 8) | ((unsigned)(y + 8) << 5) | ((unsigned)(z + 8) << 10);
                ++k;
            }
        }
        __syncthreads();
        const int nc = min(s_n, kMaxLocal);
        const bool overflow = s_n > kMaxLocal;
        // group the candidates by shell: a voxel at distance r from the centre
        // is at least b - r from every candidate of shell b, so once that
        // bound exceeds its best distance the later shells cannot win (the
        // winner is the minimum by (distance, key), whatever the visit order)
        if (threadIdx.x < kBuckets) s_cur[threadIdx.x] = 0;
        __syncthreads();
        for (int c = threadIdx.x; c < nc; c += blockDim.x) atomicAdd(&s_cur[ev_bucket(s_cand[c])], 1);
        __syncthreads();
        if (threadIdx.x == 0) {
            int acc = 0;
            for (int b = 0; b < kBuckets; ++b) {
                const int h = s_cur[b];
                s_start[b] = acc;
                s_cur[b] = acc;
                acc += h;
            }
            s_start[kBuckets] = acc;
        }
        __syncthreads();
        for (int c = threadIdx.x; c < nc; c += blockDim.x) {
            const unsigned e = s_cand[c];
            s_sorted[atomicAdd(&s_cur[ev_bucket(e)], 1)] = e;
        }
        __syncthreads();
        const int4 o = origin[i];
        for (int off = threadIdx.x; off < kLeafVoxels; off += blockDim.x) {
            const int q = off >> 6, bit = off & 63;
            if (!((s_b[q] >> bit) & 1ull)) continue;
            int rank = __popcll(s_b[q] & ((1ull << bit) - 1ull));
            for (int qq = 0; qq < q; ++qq) rank += __popcll(s_b[qq]);
            const int x = q, y = bit >> 3, z = bit & 7;
            int best = INT_MAX, bx = 0, by = 0, bz = 0;
            const float rv = 0.5f * sqrtf((float)((2 * x - 7) * (2 * x - 7) + (2 * y - 7) * (2 * y - 7) +
                                                  (2 * z - 7) * (2 * z - 7)));
            for (int b = 0; b < kBuckets; ++b) {
                // 0.01 voxel of slack covers the rounding of the shell index
                const float lb = (float)b - 0.01f - rv;
                if (lb > 0.f && lb * lb > (float)best) break;
                for (int c = s_start[b]; c < s_start[b + 1]; ++c) {
                    const unsigned e = s_sorted[c];
                    const int cx = (int)(e & 31u) - 8, cy = (int)((e >> 5) & 31u) - 8, cz = (int)(e >> 10) - 8;
                    const int d2 = (cx - x) * (cx - x) + (cy - y) * (cy - y) + (cz - z) * (cz - z);
                    if (d2 < best ||
                        (d2 == best && ev_key_less(o.x + cx, o.y + cy, o.z + cz, o.x + bx, o.y + by, o.z + bz))) {
                        best = d2;
                        bx = cx;
                        by = cy;
                        bz = cz;
                    }
                }
            }
            const int p = boff[i] + rank;
            dst[p] = make_int4(o.x + x, o.y + y, o.z + z, 0);
            src[p] = make_int4(o.x + bx, o.y + by, o.z + bz, 0);
            if (overflow || best >= 81) fb_list[atomicAdd(fb_count, 1)] = p;
        }
        __syncthreads();
    }
}

// Nearest interface voxel over the whole list (64-bit squared distances).
__global__ void k_ev_brute(const int4* __restrict__ iface, int n_iface, const int* __restrict__ fb_list, int n_fb,
                           const int4* __restrict__ dst, int4* __restrict__ src) {
    for (int f = blockIdx.x * blockDim.x + threadIdx.x; f < n_fb; f += gridDim.x * blockDim.x) {
        const int p = fb_list[f];
        const int4 c = dst[p];
        long long best = LLONG_MAX;
        int4 b = iface[0];
        for (int k = 0; k < n_iface; ++k) {
            const int4 s = iface[k];
            const long long dx = (long long)c.x - s.x, dy = (long long)c.y - s.y, dz = (long long)c.z - s.z;
            const long long d2 = dx * dx + dy * dy + dz * dz;
            if (d2 < best || (d2 == best && ev_key_less(s.x, s.y, s.z, b.x, b.y, b.z))) {
                best = d2;
                b = s;
            }
        }
        src[p] = b;
    }
}

// g.set(dst, g.get(src)) for every pair (g holds a leaf for every dst).
__global__ void k_ev_write(GridView g, float* __restrict__ values, unsigned long long* __restrict__ mask,
                           const int4* __restrict__ dst, const int4* __restrict__ src, int n, unsigned* err) {
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < n; p += gridDim.x * blockDim.x) {
        const int4 s = src[p], d = dst[p];
        const int ss = hash_find_leaf(g.hash, s.x >> 3, s.y >> 3, s.z >> 3);
        const float v = ss < 0 ? g.background : g.values[(size_t)ss * kLeafVoxels + voxel_off(s.x, s.y, s.z)];
        const int ds = hash_find_leaf(g.hash, d.x >> 3, d.y >> 3, d.z >> 3);
        if (ds < 0) {
            atomicOr(err, kErrCapacity);
            continue;
        }
        const int off = voxel_off(d.x, d.y, d.z);
        values[(size_t)ds * kLeafVoxels + off] = v;
        atomicOr(&mask[(size_t)ds * 8 + (off >> 6)], 1ull << (off & 63));
    }
}

}  // namespace

extern "C" {

int vlr_extend_velocity(vlr_ctx* ctx, const vlr_grid* sdf, vlr_grid* vx, vlr_grid* vy, vlr_grid* vz,
                        float half_width) {
    if (!ctx || !sdf || !vx || !vy || !vz) return set_error(ctx, VLR_ERR_INVALID, "null argument");
    const vlr_grid* all[4] = {sdf, vx, vy, vz};
    for (int a = 0; a < 4; ++a) {
        if (all[a]->kind != VLR_KIND_F32_WORLD) return set_error(ctx, VLR_ERR_INVALID, "grids must be world-unit f32");
        for (int b = 0; b < a; ++b)
            if (all[a] == all[b]) return set_error(ctx, VLR_ERR_INVALID, "extend_velocity needs four distinct grids");
    }
    const int n = sdf->n;
    if (n == 0) return VLR_OK;
    const float vs = (float)sdf->xf.voxel_size;
    const float band = half_width * vs;
    cudaStream_t st = ctx->stream;
    uint64_t* d_imask = nullptr;
    VLR_CUDA(ctx, cudaMallocFromPoolAsync(&d_imask, 128ull * n + 8ull * n, ctx->pool, st));
    uint64_t* d_bmask = d_imask + 8ull * n;
    int* d_bcount = reinterpret_cast<int*>(d_bmask + 8ull * n);
    int* d_boff = d_bcount + n;
    const int B = std::min(n, ctx->sm_count * 8);
    k_ev_classify<<<B, 256, 0, st>>>(sdf->mask, (const float*)sdf->values, n, vs, band, d_imask, d_bmask, d_bcount);
    VLR_CUDA(ctx, cudaGetLastError());
    std::vector<uint64_t> im(8ull * n);
    std::vector<int> bc(n);
    std::vector<int4> org(n);
    VLR_CUDA(ctx, cudaMemcpyAsync(im.data(), d_imask, 64ull * n, cudaMemcpyDeviceToHost, st));
    VLR_CUDA(ctx, cudaMemcpyAsync(bc.data(), d_bcount, sizeof(int) * n, cudaMemcpyDeviceToHost, st));
    VLR_CUDA(ctx, cudaMemcpyAsync(org.data(), sdf->origin, sizeof(int4) * n, cudaMemcpyDeviceToHost, st));
    VLR_CUDA(ctx, cudaStreamSynchronize(st));
    bool any_iface = false;
    for (size_t k = 0; k < im.size() && !any_iface; ++k) any_iface = im[k] != 0;
    std::vector<int> boff(n);
    long long nb = 0;
    for (int i = 0; i < n; ++i) {
        boff[i] = (int)nb;
        nb += bc[i];
    }
    if (!any_iface || nb == 0) {  // no interface: nothing changes (level_set_track.rs:138-140)
        VLR_CUDA(ctx, cudaFreeAsync(d_imask, st));
        return VLR_OK;
    }
    if (nb > INT32_MAX / 2) return set_error(ctx, VLR_ERR_CAPACITY, "too many band voxels");
    VLR_CUDA(ctx, cudaMemcpyAsync(d_boff, boff.data(), sizeof(int) * n, cudaMemcpyHostToDevice, st));
    int4* d_dst = nullptr;
    VLR_CUDA(ctx, cudaMallocFromPoolAsync(&d_dst, sizeof(int4) * 2 * nb + sizeof(int) * (nb + 1), ctx->pool, st));
    int4* d_src = d_dst + nb;
    int* d_fb = reinterpret_cast<int*>(d_src + nb);
    int* d_fbn = d_fb + nb;
    VLR_CUDA(ctx, cudaMemsetAsync(d_fbn, 0, sizeof(int), st));
    k_ev_search<<<B, 256, 0, st>>>(sdf->origin, sdf->nbr, n, d_imask, d_bmask, d_boff, d_dst, d_src, d_fb, d_fbn);
    VLR_CUDA(ctx, cudaGetLastError());
    int n_fb = 0;
    VLR_CUDA(ctx, cudaMemcpyAsync(&n_fb, d_fbn, sizeof(int), cudaMemcpyDeviceToHost, st));
    VLR_CUDA(ctx, cudaStreamSynchronize(st));
    if (n_fb > 0) {
        // the whole interface list, only for the voxels whose search left the
        // 27-leaf neighbourhood (or whose neighbourhood overflowed)
        std::vector<int4> iface;
        for (int i = 0; i < n; ++i)
            for (int q = 0; q < 8; ++q)
                for (uint64_t w = im[8ull * i + q]; w; w &= w - 1) {
                    const int bit = __builtin_ctzll(w);
                    iface.push_back(make_int4(org[i].x + q, org[i].y + (bit >> 3), org[i].z + (bit & 7), 0));
                }
        int4* d_iface = nullptr;
        VLR_CUDA(ctx, cudaMallocFromPoolAsync(&d_iface, sizeof(int4) * iface.size(), ctx->pool, st));
        VLR_CUDA(ctx, cudaMemcpyAsync(d_iface, iface.data(), sizeof(int4) * iface.size(), cudaMemcpyHostToDevice, st));
        k_ev_brute<<<std::max(1, std::min((n_fb + 127) / 128, ctx->sm_count * 8)), 128, 0, st>>>(
            d_iface, (int)iface.size(), d_fb, n_fb, d_dst, d_src);
        VLR_CUDA(ctx, cudaGetLastError());
        VLR_CUDA(ctx, cudaFreeAsync(d_iface, st));
        // the host list must outlive its copy
        VLR_CUDA(ctx, cudaStreamSynchronize(st));
    }
    // leaves of the band voxels, added to each velocity grid where missing
    std::vector<int32_t> band_leaves;
    for (int i = 0; i < n; ++i)
        if (bc[i]) band_leaves.insert(band_leaves.end(), {org[i].x, org[i].y, org[i].z});
    vlr_grid* vel[3] = {vx, vy, vz};
    int rc = VLR_OK;
    for (int a = 0; a < 3 && !rc; ++a) {
        rc = grid_add_leaves(ctx, vel[a], band_leaves);
        if (rc) break;
        k_ev_write<<<std::min((int)((nb + 255) / 256), ctx->sm_count * 8), 256, 0, st>>>(
            make_view(vel[a]), (float*)vel[a]->values, reinterpret_cast<unsigned long long*>(vel[a]->mask), d_dst,
            d_src, (int)nb, ctx->d_errword);
        cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) rc = check_cuda(ctx, e, "k_ev_write");
    }
    cudaFreeAsync(d_dst, st);
    cudaFreeAsync(d_imask, st);
    if (rc) return rc;
    VLR_CUDA(ctx, cudaStreamSynchronize(st));
    return consume_device_errors(ctx, "vlr_extend_velocity");
}

}  // extern "C"
