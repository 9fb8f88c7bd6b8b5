// Leaf-pool management: allocation, hash index, 27-neighbour table, scan and
// order-preserving compaction.  These replace the reference's pointer-chasing
// topology (RootNode HashMap -> InternalNode 16^3 -> boxed LeafNode,
// src/tree/root.rs:55-72, src/tree/internal.rs:88-143) with flat device
// arrays that the stencil kernels index directly.
#include <algorithm>
#include <cstring>
#include <string>

#include "vlr_host.hpp"

namespace vlr {

int set_error(vlr_ctx* ctx, int code, const std::string& msg) {
    if (ctx) ctx->last_error = msg;
    return code;
}

int check_cuda(vlr_ctx* ctx, cudaError_t e, const char* what) {
    int code = (e == cudaErrorMemoryAllocation) ? VLR_ERR_NOMEM : VLR_ERR_CUDA;
    return set_error(ctx, code, std::string(what) + ": " + cudaGetErrorString(e));
}

size_t value_bytes(int kind) { return kind == VLR_KIND_F16_VOXEL ? 2 : 4; }

int ctx_scratch(vlr_ctx* ctx, size_t bytes, void** out) {
    if (bytes > ctx->scratch_bytes) {
        if (ctx->scratch) {
            cudaStreamSynchronize(ctx->stream);
            cudaFree(ctx->scratch);
            ctx->scratch = nullptr;
            ctx->scratch_bytes = 0;
        }
        size_t want = std::max<size_t>(bytes, 1 << 20);
        VLR_CUDA(ctx, cudaMalloc(&ctx->scratch, want));
        ctx->scratch_bytes = want;
    }
    *out = ctx->scratch;
    return VLR_OK;
}

int read_int(vlr_ctx* ctx, const int* d_ptr, int* out) {
    int* h = (int*)ctx->pinned;
    VLR_CUDA(ctx, cudaMemcpyAsync(h, d_ptr, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
    VLR_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    *out = *h;
    return VLR_OK;
}

static cudaEvent_t timer_event(vlr_ctx* ctx) {
    auto& t = ctx->timer;
    if (!t.free_events.empty()) {
        cudaEvent_t e = t.free_events.back();
        t.free_events.pop_back();
        return e;
    }
    cudaEvent_t e = nullptr;
    cudaEventCreate(&e);
    return e;
}

void timer_begin(vlr_ctx* ctx, const char* name) {
    auto& t = ctx->timer;
    if (!t.enabled) return;
    vlr_kernel_timer::Pending p{name, timer_event(ctx), timer_event(ctx)};
    cudaEventRecord(p.a, ctx->stream);
    t.pending.push_back(p);
}

void timer_end(vlr_ctx* ctx) {
    auto& t = ctx->timer;
    if (!t.enabled || t.pending.empty()) return;
    cudaEventRecord(t.pending.back().b, ctx->stream);
}

int timer_collect(vlr_ctx* ctx) {
    auto& t = ctx->timer;
    if (t.pending.empty()) return VLR_OK;
    VLR_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    for (auto& p : t.pending) {
        float ms = 0.0f;
        cudaEventElapsedTime(&ms, p.a, p.b);
        bool found = false;
        for (auto& kv : t.totals)
            if (kv.first == p.name) {
                kv.second.first += ms;
                kv.second.second += 1;
                found = true;
                break;
            }
        if (!found) t.totals.push_back({std::string(p.name), {(double)ms, 1ll}});
        t.free_events.push_back(p.a);
        t.free_events.push_back(p.b);
    }
    t.pending.clear();
    return VLR_OK;
}

int d2h_copy(vlr_ctx* ctx, void* dst, const void* src, size_t bytes) {
    constexpr size_t kChunk = 4u << 20;
    cudaStream_t st = ctx->stream;
    if (!bytes) return VLR_OK;
    cudaPointerAttributes at{};
    const bool pinned_dst = cudaPointerGetAttributes(&at, dst) == cudaSuccess && at.type == cudaMemoryTypeHost;
    cudaGetLastError();  // a pageable pointer may leave an error behind on older drivers
    if (pinned_dst || bytes < 2 * kChunk) {
        VLR_CUDA(ctx, cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, st));
        VLR_CUDA(ctx, cudaStreamSynchronize(st));
        return VLR_OK;
    }
    if (!ctx->stage) {
        VLR_CUDA(ctx, cudaMallocHost(&ctx->stage, 2 * kChunk));
        for (int b = 0; b < 2; ++b) VLR_CUDA(ctx, cudaEventCreateWithFlags(&ctx->stage_ev[b], cudaEventDisableTiming));
    }
    char* stage = static_cast<char*>(ctx->stage);
    char* out = static_cast<char*>(dst);
    const char* in = static_cast<const char*>(src);
    const size_t n = (bytes + kChunk - 1) / kChunk;
    for (size_t k = 0; k <= n; ++k) {
        if (k < n) {  // half k & 1 was emptied by the host copy of chunk k - 2
            const size_t len = std::min(kChunk, bytes - k * kChunk);
            VLR_CUDA(ctx, cudaMemcpyAsync(stage + (k & 1) * kChunk, in + k * kChunk, len, cudaMemcpyDeviceToHost, st));
            VLR_CUDA(ctx, cudaEventRecord(ctx->stage_ev[k & 1], st));
        }
        if (k > 0) {
            const size_t j = k - 1, len = std::min(kChunk, bytes - j * kChunk);
            VLR_CUDA(ctx, cudaEventSynchronize(ctx->stage_ev[j & 1]));
            std::memcpy(out + j * kChunk, stage + (j & 1) * kChunk, len);
        }
    }
    return VLR_OK;
}

int consume_device_errors(vlr_ctx* ctx, const char* what) {
    unsigned* h = (unsigned*)ctx->pinned;
    VLR_CUDA(ctx, cudaMemcpyAsync(h, ctx->d_errword, sizeof(unsigned), cudaMemcpyDeviceToHost, ctx->stream));
    VLR_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    unsigned e = *h;
    if (!e) return VLR_OK;
    VLR_CUDA(ctx, cudaMemsetAsync(ctx->d_errword, 0, sizeof(unsigned), ctx->stream));
    std::string m = std::string(what) + ": device reported";
    int code = VLR_ERR_CUDA;
    if (e & kErrReach) { m += " backtrace outside the staged neighbourhood;"; code = VLR_ERR_REACH; }
    if (e & kErrExtent) { m += " leaf outside the hashable extent;"; code = VLR_ERR_EXTENT; }
    if (e & kErrCapacity) { m += " leaf capacity exceeded;"; code = VLR_ERR_CAPACITY; }
    if (e & kErrHashFull) { m += " hash table full;"; code = VLR_ERR_CAPACITY; }
    if (e & kErrTimeout) { m += " bounded wait timed out;"; code = VLR_ERR_TIMEOUT; }
    if (e & kErrInput) {
        m += " device input failed a check (a leaf origin off the 8-voxel lattice, a leaf listed twice or a list "
             "position out of range);";
        code = VLR_ERR_INVALID;
    }
    return set_error(ctx, code, m);
}

void grid_free_arrays(vlr_grid* g) {
    if (g->block) {
        // stream-ordered: later work on the context stream may reuse the memory
        if (g->ctx && g->ctx->stream) cudaFreeAsync(g->block, g->ctx->stream);
        else cudaFree(g->block);
    }
    g->block = nullptr;
    g->origin = nullptr;
    g->mask = nullptr;
    g->values = nullptr;
    g->nbr = nullptr;
    g->hkey = nullptr;
    g->hval = nullptr;
    g->hcap = 0;
    g->cap = 0;
}

static int next_pow2(long long v) {
    int p = 64;
    while ((long long)p < v && p < (1 << 30)) p <<= 1;
    return p;
}

// The grid's arrays in one allocation from the context's pool (256-byte
// aligned pieces): a step that makes a new grid costs no synchronising
// cudaMalloc.
int grid_alloc(vlr_ctx* ctx, vlr_grid* g, int cap) {
    grid_free_arrays(g);
    if (!g->ctx) g->ctx = ctx;
    int c = std::max(cap, 1);
    size_t vb = value_bytes(g->kind);
    g->hcap = next_pow2(2ll * c);
    auto up = [](size_t b) { return (b + 255) & ~(size_t)255; };
    const size_t s_origin = up(sizeof(int4) * c), s_mask = up(sizeof(uint64_t) * 8 * c),
                 s_values = up(vb * kLeafVoxels * c), s_nbr = up(sizeof(int) * kNbr * (size_t)c),
                 s_hkey = up(sizeof(uint64_t) * g->hcap), s_hval = up(sizeof(int) * g->hcap);
    char* p = nullptr;
    VLR_CUDA(ctx, cudaMallocFromPoolAsync((void**)&p, s_origin + s_mask + s_values + s_nbr + s_hkey + s_hval, ctx->pool,
                                          ctx->stream));
    g->block = p;
    g->origin = (int4*)p;
    p += s_origin;
    g->mask = (uint64_t*)p;
    p += s_mask;
    g->values = p;
    p += s_values;
    g->nbr = (int*)p;
    p += s_nbr;
    g->hkey = (uint64_t*)p;
    p += s_hkey;
    g->hval = (int*)p;
    g->cap = c;
    return VLR_OK;
}

int choose_base(vlr_ctx* ctx, const int32_t* origins, size_t n, long long base[3]) {
    if (n == 0) {
        base[0] = base[1] = base[2] = -kKeyHalf;
        return VLR_OK;
    }
    for (int a = 0; a < 3; ++a) {
        long long lo = LLONG_MAX, hi = LLONG_MIN;
        for (size_t i = 0; i < n; ++i) {
            long long l = (long long)(origins[3 * i + a] >> 3);
            lo = std::min(lo, l);
            hi = std::max(hi, l);
        }
        if (hi - lo >= (1ll << kKeyBits) - 2)
            return set_error(ctx, VLR_ERR_EXTENT, "grid spans more than 2^24 voxels along an axis");
        base[a] = (lo + hi) / 2 - kKeyHalf;
    }
    return VLR_OK;
}

// ---------------------------------------------------------------- kernels

__global__ void k_hash_clear(uint64_t* key, int* val, int cap) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < cap; i += gridDim.x * blockDim.x) {
        key[i] = kEmptyKey;
        val[i] = -1;
    }
}

__global__ void k_hash_insert(const int4* origin, int n, uint64_t* hkey, int* hval, int hcap, long long b0,
                              long long b1, long long b2, unsigned* err) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    long long base[3] = {b0, b1, b2};
    int4 o = origin[i];
    uint64_t key = pack_key(o.x >> 3, o.y >> 3, o.z >> 3, base);
    if (key == kEmptyKey) {
        atomicOr(err, kErrExtent);
        return;
    }
    uint32_t m = (uint32_t)hcap - 1u;
    uint32_t p = (uint32_t)mix64(key) & m;
    for (int probe = 0; probe < hcap; ++probe) {
        unsigned long long prev =
            atomicCAS((unsigned long long*)&hkey[p], (unsigned long long)kEmptyKey, (unsigned long long)key);
        if (prev == kEmptyKey || prev == key) {
            // Duplicates keep the smallest slot (deterministic).
            atomicMin(&hval[p] , i) ;
            return;
        }
        p = (p + 1u) & m;
    }
    atomicOr(err, kErrHashFull);
}

// hval starts at -1 after clear; atomicMin(-1, i) would keep -1, so inserts
// first turn -1 into INT_MAX.
__global__ void k_hash_prep_vals(int* val, int cap) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < cap; i += gridDim.x * blockDim.x) val[i] = INT_MAX;
}

__global__ void k_nbr_build(const int4* origin, int n, const uint64_t* hkey, const int* hval, int hcap, long long b0,
                            long long b1, long long b2, int* nbr, int* dup_flag) {
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    int i = t / kNbr, d = t % kNbr;
    if (i >= n) return;
    HashView h{hkey, hval, hcap, {b0, b1, b2}};
    int4 o = origin[i];
    int dx = d / 9 - 1, dy = (d / 3) % 3 - 1, dz = d % 3 - 1;
    int s = hash_find_leaf(h, (long long)(o.x >> 3) + dx, (long long)(o.y >> 3) + dy, (long long)(o.z >> 3) + dz);
    nbr[i * kNbr + d] = s;
    if (d == 13 && s != i) atomicOr(dup_flag, 1);  // a duplicate origin maps to another slot
}

int grid_index(vlr_ctx* ctx, vlr_grid* g) {
    int hc = g->hcap;
    int thr = 256;
    int blocks = std::min((hc + thr - 1) / thr, ctx->sm_count * 8);
    k_hash_clear<<<blocks, thr, 0, ctx->stream>>>(g->hkey, g->hval, hc);
    k_hash_prep_vals<<<blocks, thr, 0, ctx->stream>>>(g->hval, hc);
    if (g->n > 0) {
        k_hash_insert<<<(g->n + thr - 1) / thr, thr, 0, ctx->stream>>>(g->origin, g->n, g->hkey, g->hval, hc,
                                                                     g->base[0], g->base[1], g->base[2],
                                                                     ctx->d_errword);
        void* sp;
        int rc = ctx_scratch(ctx, sizeof(int), &sp);
        if (rc) return rc;
        int* dup = (int*)sp;
        VLR_CUDA(ctx, cudaMemsetAsync(dup, 0, sizeof(int), ctx->stream));
        long long tot = (long long)g->n * kNbr;
        k_nbr_build<<<(unsigned)((tot + thr - 1) / thr), thr, 0, ctx->stream>>>(
            g->origin, g->n, g->hkey, g->hval, hc, g->base[0], g->base[1], g->base[2], g->nbr, dup);
        VLR_CUDA(ctx, cudaGetLastError());
        int h_dup = 0;
        int r2 = read_int(ctx, dup, &h_dup);
        if (r2) return r2;
        if (h_dup) return set_error(ctx, VLR_ERR_INVALID, "duplicate leaf origin");
    }
    VLR_CUDA(ctx, cudaGetLastError());
    return consume_device_errors(ctx, "grid index");
}

// ------------------------------------------------------------------ scan

// Block-wide exclusive scan of one int per thread (blockDim.x == 1024).
__device__ inline int block_excl_scan(int v, int* warp_sums, int* total) {
    int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    int x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        int y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) warp_sums[w] = x;
    __syncthreads();
    if (w == 0) {
        int s = (lane < (int)(blockDim.x >> 5)) ? warp_sums[lane] : 0;
        int si = s;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            int y = __shfl_up_sync(0xffffffffu, si, o);
            if (lane >= o) si += y;
        }
        warp_sums[lane] = si - s;  // exclusive prefix of warp sums
        if (lane == 31) *total = si;
    }
    __syncthreads();
    int r = x - v + warp_sums[w];
    __syncthreads();
    return r;
}

__global__ void __launch_bounds__(1024) k_scan_block(const int* in, int* out, int n, int* block_sums) {
    __shared__ int ws[32];
    __shared__ int tot;
    int i = blockIdx.x * 1024 + threadIdx.x;
    int v = (i < n) ? in[i] : 0;
    int e = block_excl_scan(v, ws, &tot);
    if (i < n) out[i] = e;
    if (threadIdx.x == 0) block_sums[blockIdx.x] = tot;
}

__global__ void k_scan_add(int* out, int n, const int* block_offsets) {
    int i = blockIdx.x * 1024 + threadIdx.x;
    if (i < n) out[i] += block_offsets[blockIdx.x];
}

__global__ void k_scan_total(const int* in, const int* out, int n, int* total) {
    if (threadIdx.x == 0 && blockIdx.x == 0) *total = (n > 0) ? out[n - 1] + in[n - 1] : 0;
}

// Scratch layout per level: block sums then their scan.
int scan_exclusive(vlr_ctx* ctx, const int* d_in, int* d_out, int n, int* d_total) {
    if (n <= 0) {
        VLR_CUDA(ctx, cudaMemsetAsync(d_total, 0, sizeof(int), ctx->stream));
        return VLR_OK;
    }
    int nb = (n + 1023) / 1024;
    int* sums = nullptr;
    int* sums_scan = nullptr;
    VLR_CUDA(ctx, cudaMallocFromPoolAsync(&sums, sizeof(int) * (nb + 1) * 2, ctx->pool, ctx->stream));
    sums_scan = sums + nb + 1;
    k_scan_block<<<nb, 1024, 0, ctx->stream>>>(d_in, d_out, n, sums);
    if (nb > 1) {
        int* dummy_total = sums_scan + nb;
        int rc = scan_exclusive(ctx, sums, sums_scan, nb, dummy_total);
        if (rc) return rc;
        k_scan_add<<<nb, 1024, 0, ctx->stream>>>(d_out, n, sums_scan);
    }
    k_scan_total<<<1, 32, 0, ctx->stream>>>(d_in, d_out, n, d_total);
    VLR_CUDA(ctx, cudaGetLastError());
    VLR_CUDA(ctx, cudaFreeAsync(sums, ctx->stream));
    return VLR_OK;
}

// ------------------------------------------------------------ compaction

template <typename T>
__global__ void k_compact_leaves(int n, const int* flags, const int* pos, const int4* o_in, const uint64_t* m_in,
                                 const T* v_in, int4* o_out, uint64_t* m_out, T* v_out) {
    int i = blockIdx.x;
    if (i >= n || !flags[i]) return;
    int j = pos[i];
    if (threadIdx.x == 0) o_out[j] = o_in[i];
    if (threadIdx.x < 8) m_out[(size_t)j * 8 + threadIdx.x] = m_in[(size_t)i * 8 + threadIdx.x];
    const uint4* src = (const uint4*)(v_in + (size_t)i * kLeafVoxels);
    uint4* dst = (uint4*)(v_out + (size_t)j * kLeafVoxels);
    constexpr int kVec = kLeafVoxels * sizeof(T) / 16;
    for (int t = threadIdx.x; t < kVec; t += blockDim.x) dst[t] = src[t];
}

int grid_compact(vlr_ctx* ctx, vlr_grid* g, const int* d_flags) {
    if (g->n == 0) return VLR_OK;
    int* pos = nullptr;
    VLR_CUDA(ctx, cudaMallocFromPoolAsync(&pos, sizeof(int) * (g->n + 1), ctx->pool, ctx->stream));
    int* d_total = pos + g->n;
    int rc = scan_exclusive(ctx, d_flags, pos, g->n, d_total);
    if (rc) return rc;
    int total = 0;
    rc = read_int(ctx, d_total, &total);
    if (rc) return rc;
    if (total == g->n) {
        VLR_CUDA(ctx, cudaFreeAsync(pos, ctx->stream));
        return VLR_OK;
    }
    vlr_grid tmp;
    tmp.ctx = ctx;
    tmp.kind = g->kind;
    rc = grid_alloc(ctx, &tmp, std::max(total, 1));
    if (rc) return rc;
    if (g->kind == VLR_KIND_F16_VOXEL)
        k_compact_leaves<__half><<<g->n, 64, 0, ctx->stream>>>(g->n, d_flags, pos, g->origin, g->mask,
                                                              (const __half*)g->values, tmp.origin, tmp.mask,
                                                              (__half*)tmp.values);
    else
        k_compact_leaves<float><<<g->n, 128, 0, ctx->stream>>>(g->n, d_flags, pos, g->origin, g->mask,
                                                              (const float*)g->values, tmp.origin, tmp.mask,
                                                              (float*)tmp.values);
    VLR_CUDA(ctx, cudaGetLastError());
    VLR_CUDA(ctx, cudaFreeAsync(pos, ctx->stream));
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
    g->n = total;
    return grid_index(ctx, g);
}

}  // namespace vlr
