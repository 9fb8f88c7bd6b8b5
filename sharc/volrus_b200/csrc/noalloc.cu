// find_zero_crossings without any allocation (vlr_find_zero_crossings_noalloc).
//
// Who needs this: callers that cannot call cudaMalloc at the moment they
// need the crossings -- code running inside a CUDA stream capture (an
// allocation there would break the capture), real-time loops that must not
// block in the driver's allocator, and hosts whose device memory is owned by
// another allocator (a caching framework allocator or an engine's fixed
// budget) so that a fresh cudaMalloc may fail.  They pass the grid and
// device output buffers they already own; the scratch memory the kernels need
// (per-leaf crossing masks, counts and offsets) lives in one file-scope
// device array instead of being allocated per call.
//
// Limits and rules:
//   * at most kNoAllocMaxLeaves (65,536) leaves per grid; larger grids are
//     rejected with VLR_ERR_CAPACITY.  The array is 4.5 MiB and every GPU
//     that loads the library holds it until the process exits.
//   * the first call on a device looks up the array's device address
//     (cudaGetSymbolAddress, with that device made current and the caller's
//     current device restored afterwards) and caches it together with the
//     device's CUDA context; make that first call before any stream capture
//     begins.  If the context changes later (a cudaDeviceReset by the host
//     application or another library), the next call looks the address up
//     again instead of writing through a stale pointer.
//   * every call on a device shares the one array, which keeps the previous
//     call's contents: the counter that must start at zero is cleared on each
//     call.  Calls whose kernels overlap on the GPU (two contexts or streams
//     on the same device) race on the array and must be serialised by the
//     caller.
#include <mutex>

#include <cuda.h>

#include "vlr_host.hpp"

namespace vlr {
namespace {

constexpr int kNoAllocMaxLeaves = 65536;
// layout: [total u64 (256 B slot)] [xmask u64[8] per leaf] [count i32 per leaf] [offset i32 per leaf]
constexpr size_t kTotalSlot = 256;
constexpr size_t kXmaskBytes = (size_t)kNoAllocMaxLeaves * 64;
constexpr size_t kCountBytes = (size_t)kNoAllocMaxLeaves * 4;
constexpr size_t kScratchBytes = kTotalSlot + kXmaskBytes + 2 * kCountBytes;

static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

std::mutex g_mu;
struct ScratchSlot {
    void* addr = nullptr;    // device address of g_noalloc_scratch
    CUcontext cu = nullptr;  // the device's context when the address was resolved
};
ScratchSlot g_scratch[128];  // per device ordinal

using PFN_ctx_get_current = CUresult (*)(CUcontext*);

// cuCtxGetCurrent from the driver (through the runtime, so the library links
// only cudart); null if the driver does not offer it.
PFN_ctx_get_current ctx_get_current() {
    static PFN_ctx_get_current fn = [] {
        void* f = nullptr;
        cudaDriverEntryPointQueryResult q{};
        if (cudaGetDriverEntryPointByVersion("cuCtxGetCurrent", &f, 12000, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess)
            f = nullptr;
        return reinterpret_cast<PFN_ctx_get_current>(f);
    }();
    return fn;
}

// Device address of the scratch array on the context's device.  Host code
// may not use the symbol itself as a pointer, so the address is looked up
// with cudaGetSymbolAddress with that device current, then cached with the
// device's CUDA context; a changed context (device reset) is looked up anew.
// The calling thread's current device is restored before returning.
int scratch_address(vlr_ctx* ctx, unsigned char** out) {
    int dev = ctx->device;
    if (dev < 0 || dev >= 128) return set_error(ctx, VLR_ERR_INVALID, "device ordinal out of range");
    PFN_ctx_get_current get_cur = ctx_get_current();
    if (!get_cur) return set_error(ctx, VLR_ERR_CUDA, "cuCtxGetCurrent is not available from the driver");
    std::lock_guard<std::mutex> lock(g_mu);
    DeviceGuard guard(dev);
    VLR_CUDA(ctx, guard.status);
    CUcontext cu = nullptr;
    if (get_cur(&cu) != CUDA_SUCCESS || !cu)
        return set_error(ctx, VLR_ERR_CUDA, "no CUDA context is current on the library's device");
    ScratchSlot& s = g_scratch[dev];
    if (!s.addr || s.cu != cu) {
        void* p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess || !p) return check_cuda(ctx, e, "cudaGetSymbolAddress(g_noalloc_scratch)");
        s.addr = p;
        s.cu = cu;
    }
    *out = (unsigned char*)s.addr;
    return VLR_OK;
}

// Crossing test of find_zero_crossings (src/tools/level_set_track.rs:14-47):
// an active voxel is a crossing if it is exactly zero or some active
// 6-neighbour has a value whose product with it is negative.
__global__ void __launch_bounds__(256) k_noalloc_crossings(GridView g, uint64_t* __restrict__ xmask,
                                                          int* __restrict__ xcount,
                                                          unsigned long long* __restrict__ total) {
    int slot = blockIdx.x;
    if (slot >= g.n) return;
    const uint64_t* m = g.mask + (size_t)slot * 8;
    const float* vals = g.values + (size_t)slot * kLeafVoxels;
    __shared__ int s_cnt;
    if (threadIdx.x == 0) s_cnt = 0;
    __syncthreads();
    for (int r = 0; r < 2; ++r) {
        int off = threadIdx.x + 256 * r;
        bool cross = false;
        if (mask_bit(m, off)) {
            float val = vals[off];
            cross = (val == 0.0f);
            int x = off >> 6, y = (off >> 3) & 7, z = off & 7;
            for (int q = 0; q < 6 && !cross; ++q) {
                int nx = x + (q == 0) - (q == 1), ny = y + (q == 2) - (q == 3), nz = z + (q == 4) - (q == 5);
                int dx = (nx < 0) ? -1 : (nx > 7), dy = (ny < 0) ? -1 : (ny > 7), dz = (nz < 0) ? -1 : (nz > 7);
                int s = (dx | dy | dz) ? g.nbr[slot * kNbr + (dx + 1) * 9 + (dy + 1) * 3 + (dz + 1)] : slot;
                if (s < 0) continue;
                int noff = voxel_off(nx, ny, nz);
                if (!mask_bit(g.mask + (size_t)s * 8, noff)) continue;
                if (__fmul_rn(val, g.values[(size_t)s * kLeafVoxels + noff]) < 0.0f) cross = true;
            }
        }
        unsigned b = __ballot_sync(0xffffffffu, cross);
        if ((threadIdx.x & 31) == 0) {
            ((unsigned*)xmask)[(size_t)slot * 16 + (off >> 5)] = b;
            if (b) atomicAdd(&s_cnt, __popc(b));
        }
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        xcount[slot] = s_cnt;
        if (s_cnt) atomicAdd(total, (unsigned long long)s_cnt);
    }
}

// Exclusive scan of the per-leaf counts by one 1024-thread block (n is at
// most kNoAllocMaxLeaves, so the loop runs at most 64 rounds).
__global__ void __launch_bounds__(1024) k_noalloc_scan(const int* __restrict__ count, int* __restrict__ offset, int n) {
    __shared__ int warp_sums[32];
    __shared__ int carry;
    if (threadIdx.x == 0) carry = 0;
    __syncthreads();
    int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    for (int base = 0; base < n; base += 1024) {
        int i = base + threadIdx.x;
        int v = (i < n) ? count[i] : 0;
        int x = v;
        for (int o = 1; o < 32; o <<= 1) {
            int y = __shfl_up_sync(0xffffffffu, x, o);
            if (lane >= o) x += y;
        }
        if (lane == 31) warp_sums[w] = x;
        __syncthreads();
        if (w == 0) {
            int s = warp_sums[lane];
            int si = s;
            for (int o = 1; o < 32; o <<= 1) {
                int y = __shfl_up_sync(0xffffffffu, si, o);
                if (lane >= o) si += y;
            }
            warp_sums[lane] = si - s;
        }
        __syncthreads();
        if (i < n) offset[i] = carry + warp_sums[w] + x - v;
        __syncthreads();
        if (threadIdx.x == 1023) carry += warp_sums[31] + x;
        __syncthreads();
    }
}

// Coordinates of each crossing at its scanned position; positions at or
// beyond `cap` are not written.  Thread 0 of block 0 stores the total.
__global__ void __launch_bounds__(512) k_noalloc_emit(GridView g, const uint64_t* __restrict__ xmask,
                                                     const int* __restrict__ offset, int* __restrict__ coords,
                                                     unsigned long long cap,
                                                     const unsigned long long* __restrict__ total,
                                                     unsigned long long* __restrict__ out_count) {
    int slot = blockIdx.x;
    if (slot == 0 && threadIdx.x == 0) *out_count = *total;
    if (slot >= g.n) return;
    int off = threadIdx.x;
    const uint64_t* xm = xmask + (size_t)slot * 8;
    if (!mask_bit(xm, off)) return;
    int w = off >> 6, b = off & 63;
    int rank = 0;
    for (int q = 0; q < w; ++q) rank += __popcll(xm[q]);
    if (b) rank += __popcll(xm[w] & (~0ull >> (64 - b)));
    unsigned long long j = (unsigned long long)offset[slot] + (unsigned long long)rank;
    if (j >= cap) return;
    int4 o = g.origin[slot];
    coords[3 * j] = o.x + (off >> 6);
    coords[3 * j + 1] = o.y + ((off >> 3) & 7);
    coords[3 * j + 2] = o.z + (off & 7);
}

GridView view_of(const vlr_grid* g) {
    GridView v{};
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
    return v;
}

}  // namespace
}  // namespace vlr

using namespace vlr;

extern "C" int vlr_find_zero_crossings_noalloc(vlr_ctx* ctx, const vlr_grid* g, int32_t* d_coords, size_t cap,
                                               unsigned long long* d_count) {
    if (!ctx || !g || !d_count || (cap && !d_coords)) return set_error(ctx, VLR_ERR_INVALID, "null argument");
    if (g->kind != VLR_KIND_F32_WORLD) return set_error(ctx, VLR_ERR_INVALID, "grid is not a world-unit f32 grid");
    if (g->n > kNoAllocMaxLeaves)
        return set_error(ctx, VLR_ERR_CAPACITY,
                         "vlr_find_zero_crossings_noalloc: grid has " + std::to_string(g->n) +
                             " leaves, more than the fixed scratch limit of 65536 leaves");
    unsigned char* base = nullptr;
    int rc = scratch_address(ctx, &base);
    if (rc) return rc;
    unsigned long long* total = (unsigned long long*)base;
    uint64_t* xmask = (uint64_t*)(base + kTotalSlot);
    int* count = (int*)(base + kTotalSlot + kXmaskBytes);
    int* offset = (int*)(base + kTotalSlot + kXmaskBytes + kCountBytes);
    // The array keeps the previous call's contents; the total must start at zero.
    VLR_CUDA(ctx, cudaMemsetAsync(total, 0, sizeof(unsigned long long), ctx->stream));
    GridView v = view_of(g);
    if (g->n > 0) {
        k_noalloc_crossings<<<g->n, 256, 0, ctx->stream>>>(v, xmask, count, total);
        k_noalloc_scan<<<1, 1024, 0, ctx->stream>>>(count, offset, g->n);
    }
    k_noalloc_emit<<<g->n > 0 ? g->n : 1, 512, 0, ctx->stream>>>(v, xmask, offset, d_coords,
                                                                 (unsigned long long)cap, total, d_count);
    VLR_CUDA(ctx, cudaGetLastError());
    return VLR_OK;
}
