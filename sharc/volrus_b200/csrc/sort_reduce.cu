// Deterministic scatter-add: stable LSD radix sort of (u32 key, f32 value)
// pairs followed by a segmented sum in sorted order.  No float atomics: every
// output is a sum taken in a fixed order (the input order of equal keys), so
// results do not depend on thread timing.
//
// Radix sort: 8-bit digits, tiles of 2048 pairs (256 threads x 8, striped).
//   k_rs_hist     per-tile digit counts, digit-major [digit][tile]
//   (scan)        exclusive scan of the counts -> scatter offsets
//   k_rs_scatter  stable rank of each pair within its tile, in 8 rounds of
//                 256: warp ranks come from __match_any_sync on the digit,
//                 earlier warps and rounds from shared-memory counters
// Segmented sum: a thread per segment head walks its run of equal keys.
#include <algorithm>

#include "sort_reduce.hpp"

namespace vlr {

constexpr int kRsThreads = 256;
constexpr int kRsItems = 8;
constexpr int kRsTile = kRsThreads * kRsItems;

__global__ void __launch_bounds__(kRsThreads) k_rs_hist(const unsigned* __restrict__ keys, int n, int shift,
                                                       int n_tiles, int* __restrict__ hist) {
    __shared__ int s_h[256];
    const int tile = blockIdx.x;
    s_h[threadIdx.x] = 0;
    __syncthreads();
#pragma unroll
    for (int i = 0; i < kRsItems; ++i) {
        int p = tile * kRsTile + i * kRsThreads + threadIdx.x;
        if (p < n) atomicAdd(&s_h[(keys[p] >> shift) & 255u], 1);
    }
    __syncthreads();
    hist[threadIdx.x * n_tiles + tile] = s_h[threadIdx.x];
}

__global__ void __launch_bounds__(kRsThreads) k_rs_scatter(const unsigned* __restrict__ keys_in,
                                                          const float* __restrict__ vals_in, int n, int shift,
                                                          int n_tiles, const int* __restrict__ offsets,
                                                          unsigned* __restrict__ keys_out, float* __restrict__ vals_out) {
    __shared__ int s_run[256];               // pairs of each digit placed in earlier rounds
    __shared__ int s_wc[kRsThreads / 32][256];  // per-warp digit counts of the current round
    const int tile = blockIdx.x;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    s_run[threadIdx.x] = 0;
    for (int q = 0; q < kRsThreads / 32; ++q) s_wc[q][threadIdx.x] = 0;
    __syncthreads();
    for (int i = 0; i < kRsItems; ++i) {
        const int p = tile * kRsTile + i * kRsThreads + threadIdx.x;
        const bool valid = p < n;
        unsigned key = valid ? keys_in[p] : 0u;
        float val = valid ? vals_in[p] : 0.f;
        // invalid lanes use digit 256 (never matches a real digit)
        const int digit = valid ? (int)((key >> shift) & 255u) : 256;
        const unsigned peers = __match_any_sync(0xffffffffu, digit);
        const int wrank = __popc(peers & ((1u << lane) - 1u));
        const bool leader = (peers & ((1u << lane) - 1u)) == 0u;
        if (valid && leader) s_wc[w][digit] = __popc(peers);
        __syncthreads();
        if (valid) {
            int before = s_run[digit];
            for (int q = 0; q < w; ++q) before += s_wc[q][digit];
            const int dst = offsets[digit * n_tiles + tile] + before + wrank;
            keys_out[dst] = key;
            vals_out[dst] = val;
        }
        __syncthreads();
        {
            int add = 0;
            for (int q = 0; q < kRsThreads / 32; ++q) {
                add += s_wc[q][threadIdx.x];
                s_wc[q][threadIdx.x] = 0;
            }
            s_run[threadIdx.x] += add;
        }
        __syncthreads();
    }
}

// out[key] = sum of the values of its run (keys sorted; key >= n_out is ignored).
__global__ void k_seg_sum(const unsigned* __restrict__ keys, const float* __restrict__ vals, int n,
                          float* __restrict__ out, unsigned n_out) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const unsigned k = keys[i];
        if (k >= n_out) continue;
        if (i > 0 && keys[i - 1] == k) continue;
        float s = 0.f;
        for (int j = i; j < n && keys[j] == k; ++j) s += vals[j];
        out[k] = s;
    }
}

__global__ void k_fill_f32(float* a, size_t n, float v) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
        a[i] = v;
}

size_t sort_reduce_scratch_bytes(int n) {
    int tiles = (n + kRsTile - 1) / kRsTile;
    size_t pairs = (size_t)n * 8 * 2;            // ping-pong keys + values
    size_t hist = (size_t)256 * tiles * 4 * 2 + 64;  // counts + offsets
    return pairs + hist + 256;
}

int sort_reduce(vlr_ctx* ctx, unsigned* keys, float* vals, int n, unsigned key_limit, float* out, unsigned n_out,
                void* scratch) {
    cudaStream_t st = ctx->stream;
    VLR_TIMED(ctx, "k_fill_f32", k_fill_f32<<<ctx->sm_count * 4, 256, 0, st>>>(out, n_out, 0.f));
    if (n <= 0) return VLR_OK;
    const int tiles = (n + kRsTile - 1) / kRsTile;
    char* p = (char*)scratch;
    unsigned* k2 = (unsigned*)p;
    p += (size_t)n * 4;
    float* v2 = (float*)p;
    p += (size_t)n * 4;
    int* hist = (int*)p;
    p += (size_t)256 * tiles * 4;
    int* offs = (int*)p;
    p += (size_t)256 * tiles * 4 + 64;
    int bits = 1;
    while (bits < 32 && (1ull << bits) <= (unsigned long long)key_limit) ++bits;
    unsigned* ka = keys;
    float* va = vals;
    unsigned* kb = k2;
    float* vb = v2;
    for (int shift = 0; shift < bits; shift += 8) {
        VLR_TIMED(ctx, "k_rs_hist", k_rs_hist<<<tiles, kRsThreads, 0, st>>>(ka, n, shift, tiles, hist));
        int rc = scan_exclusive(ctx, hist, offs, 256 * tiles, offs + 256 * tiles);
        if (rc) return rc;
        VLR_TIMED(ctx, "k_rs_scatter",
                  k_rs_scatter<<<tiles, kRsThreads, 0, st>>>(ka, va, n, shift, tiles, offs, kb, vb));
        std::swap(ka, kb);
        std::swap(va, vb);
    }
    VLR_TIMED(ctx, "k_seg_sum", k_seg_sum<<<ctx->sm_count * 4, 256, 0, st>>>(ka, va, n, out, n_out));
    VLR_CUDA(ctx, cudaGetLastError());
    return VLR_OK;
}

int radix_sort_pairs(vlr_ctx* ctx, unsigned* keys, unsigned* vals, int n, unsigned key_limit, void* scratch,
                     unsigned** keys_out, unsigned** vals_out) {
    cudaStream_t st = ctx->stream;
    *keys_out = keys;
    *vals_out = vals;
    if (n <= 0) return VLR_OK;
    const int tiles = (n + kRsTile - 1) / kRsTile;
    char* p = (char*)scratch;
    unsigned* k2 = (unsigned*)p;
    p += (size_t)n * 4;
    unsigned* v2 = (unsigned*)p;
    p += (size_t)n * 4;
    int* hist = (int*)p;
    p += (size_t)256 * tiles * 4;
    int* offs = (int*)p;
    int bits = 1;
    while (bits < 32 && (1ull << bits) <= (unsigned long long)key_limit) ++bits;
    unsigned *ka = keys, *va = vals, *kb = k2, *vb = v2;
    for (int shift = 0; shift < bits; shift += 8) {
        VLR_TIMED(ctx, "k_rs_hist", k_rs_hist<<<tiles, kRsThreads, 0, st>>>(ka, n, shift, tiles, hist));
        int rc = scan_exclusive(ctx, hist, offs, 256 * tiles, offs + 256 * tiles);
        if (rc) return rc;
        // the payload moves as raw 32-bit words
        VLR_TIMED(ctx, "k_rs_scatter",
                  k_rs_scatter<<<tiles, kRsThreads, 0, st>>>(ka, reinterpret_cast<const float*>(va), n, shift, tiles,
                                                             offs, kb, reinterpret_cast<float*>(vb)));
        std::swap(ka, kb);
        std::swap(va, vb);
    }
    VLR_CUDA(ctx, cudaGetLastError());
    *keys_out = ka;
    *vals_out = va;
    return VLR_OK;
}

}  // namespace vlr
