// Re-tracking of the narrow band after each method step, entirely on the
// device and without host synchronisation (so the step can be graph-captured):
//
//   keep      a leaf survives if it has an active voxel or a neighbour's
//             active voxel lies within one voxel of it (dilate26 of the band)
//   propose   a missing leaf touched by a neighbour's spill is proposed in a
//             hash table; atomicMin keeps the proposer that comes first in a
//             fixed direction order seen from the new leaf, so the owner is
//             independent of thread timing
//   relist    survivors keep their list order; each owner's new leaves follow
//             it (exclusive scan of survive + owned counts); slots come from a
//             free stack, new values from the owner by the clamped-sign rule
//   index     hash table and 27-neighbour table rebuilt from the new list
//
// The reference's counterparts are dilate (src/tools/morphology.rs:20-35),
// trim_narrow_band's deactivation (src/tools/level_set_track.rs:53-68) and
// remove_empty_leaves (src/tree/internal.rs:231-247).
#include <algorithm>

#include "method_state.hpp"

namespace vlr {

__device__ __forceinline__ void dir_of(int d, int& dx, int& dy, int& dz) {
    dx = d / 9 - 1;
    dy = (d / 3) % 3 - 1;
    dz = d % 3 - 1;
}

__global__ void k_t_prepare(int* keep, int cap, uint64_t* pkey, int* pval, uint64_t* hkey, int* hval, int hcap) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < max(cap, hcap); i += gridDim.x * blockDim.x) {
        if (i < cap) keep[i] = 0;
        if (i < hcap) {
            pkey[i] = kEmptyKey;
            pval[i] = INT_MAX;
        }
    }
}

__device__ __forceinline__ uint64_t leaf_key(const int4 o, int dx, int dy, int dz, const MGridParams* params,
                                             int bits) {
    const MGridParams& P = params[o.w];
    return mkey((long long)(o.x >> 3) + dx, (long long)(o.y >> 3) + dy, (long long)(o.z >> 3) + dz, o.w, P.base, bits);
}

__global__ void k_t_propose(MLeafArrays A, int* keep, uint64_t* pkey, int* pval, int hcap,
                            const MGridParams* __restrict__ params, int bits, unsigned* err) {
    const int count = *A.count;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < count; i += gridDim.x * blockDim.x) {
        const int s = A.list[i];
        if (A.nonempty[s]) keep[s] = 1;
        unsigned sp = A.spill[s];
        if (!sp) continue;
        const int4 o = A.origin[s];
        while (sp) {
            int d = __ffs(sp) - 1;
            sp &= sp - 1;
            int n = A.nbr[s * kNbr + d];
            if (n >= 0) {
                keep[n] = 1;
                continue;
            }
            int dx, dy, dz;
            dir_of(d, dx, dy, dz);
            uint64_t key = leaf_key(o, dx, dy, dz, params, bits);
            if (key == kEmptyKey) {
                atomicOr(err, kErrExtent);
                continue;
            }
            uint32_t m = (uint32_t)hcap - 1u, p = (uint32_t)mix64(key) & m;
            bool done = false;
            for (int probe = 0; probe < hcap; ++probe) {
                unsigned long long prev = atomicCAS((unsigned long long*)&pkey[p], (unsigned long long)kEmptyKey,
                                                    (unsigned long long)key);
                if (prev == kEmptyKey || prev == key) {
                    atomicMin(&pval[p], kNbr - 1 - d);  // direction of this proposer seen from the new leaf
                    done = true;
                    break;
                }
                p = (p + 1u) & m;
            }
            if (!done) atomicOr(err, kErrHashFull);
        }
    }
}

// Is leaf s (origin o) the owner of its missing neighbour in direction d?
__device__ __forceinline__ bool owns(const int4 o, int d, const uint64_t* pkey, const int* pval, int hcap,
                                     const MGridParams* params, int bits) {
    int dx, dy, dz;
    dir_of(d, dx, dy, dz);
    uint64_t key = leaf_key(o, dx, dy, dz, params, bits);
    return hfind(pkey, pval, hcap, key) == kNbr - 1 - d;
}

__global__ void k_t_count(MLeafArrays A, const int* keep, const uint64_t* pkey, const int* pval, int hcap,
                          const MGridParams* __restrict__ params, int bits, int cap, int* owned) {
    const int count = *A.count;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < cap; i += gridDim.x * blockDim.x) {
        int c = 0;
        if (i < count) {
            const int s = A.list[i];
            c = keep[s] ? 1 : 0;
            unsigned sp = A.spill[s];
            const int4 o = A.origin[s];
            while (sp) {
                int d = __ffs(sp) - 1;
                sp &= sp - 1;
                if (A.nbr[s * kNbr + d] < 0 && owns(o, d, pkey, pval, hcap, params, bits)) ++c;
            }
        }
        owned[i] = c;
    }
}

__global__ void k_t_free(MLeafArrays A, const int* keep, int* free_stack, int* free_top) {
    const int count = *A.count;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < count; i += gridDim.x * blockDim.x) {
        const int s = A.list[i];
        if (!keep[s]) free_stack[atomicAdd(free_top, 1)] = s;
    }
}

// One block per list position: write survivors and owned new leaves to the
// new list; initialise new leaves from their owner's values.
template <typename T>
__global__ void __launch_bounds__(256) k_t_alloc(MLeafArrays A, int4* origin, const int* keep, const int* pos,
                                                const uint64_t* pkey, const int* pval, int hcap,
                                                const MGridParams* __restrict__ params, int bits, int* free_stack,
                                                int* free_top, int* list_new, T* vals, unsigned* err) {
    __shared__ int s_slot;
    const int count = *A.count;
    for (int i = blockIdx.x; i < count; i += gridDim.x) {
        const int s = A.list[i];
        int p = pos[i];
        if (keep[s]) {
            if (threadIdx.x == 0) list_new[p] = s;
            ++p;
        }
        unsigned sp = A.spill[s];
        const int4 o = origin[s];
        const float hw = params[o.w].hw;
        while (sp) {
            int d = __ffs(sp) - 1;
            sp &= sp - 1;
            if (A.nbr[s * kNbr + d] >= 0 || !owns(o, d, pkey, pval, hcap, params, bits)) continue;
            if (threadIdx.x == 0) {
                int t = atomicSub(free_top, 1) - 1;
                if (t < 0) {
                    atomicOr(err, kErrCapacity);
                    s_slot = -1;
                } else {
                    s_slot = free_stack[t];
                }
            }
            __syncthreads();
            const int ns = s_slot;
            __syncthreads();
            if (ns < 0) continue;
            int dx, dy, dz;
            dir_of(d, dx, dy, dz);
            if (threadIdx.x == 0) {
                list_new[p] = ns;
                origin[ns] = make_int4(o.x + 8 * dx, o.y + 8 * dy, o.z + 8 * dz, o.w);
                A.spill[ns] = 0;
                A.nonempty[ns] = 0;
            }
            if (threadIdx.x < 8) {
                A.mask[(size_t)ns * 8 + threadIdx.x] = 0ull;
                A.dmask[(size_t)ns * 8 + threadIdx.x] = 0ull;
            }
            for (int off = threadIdx.x; off < kLeafVoxels; off += blockDim.x) {
                int x = 8 * dx + (off >> 6), y = 8 * dy + ((off >> 3) & 7), z = 8 * dz + (off & 7);
                int cx = min(max(x, 0), 7), cy = min(max(y, 0), 7), cz = min(max(z, 0), 7);
                float v = to_f(vals[(size_t)s * kLeafVoxels + ((cx << 6) | (cy << 3) | cz)]);
                vals[(size_t)ns * kLeafVoxels + off] = from_f<T>(copysignf(hw, v));
            }
            ++p;
        }
    }
}

__global__ void k_t_finalize(int* scalars, const int* list_new, int* list, int cap) {
    const int n = scalars[3];
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < min(n, cap); i += gridDim.x * blockDim.x)
        list[i] = list_new[i];
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        scalars[0] = min(n, cap);
        scalars[1] += 1;
    }
}

__global__ void k_h_clear(uint64_t* hkey, int* hval, int hcap) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < hcap; i += gridDim.x * blockDim.x) {
        hkey[i] = kEmptyKey;
        hval[i] = -1;
    }
}

__global__ void k_h_insert(const int* list, const int* count_ptr, const int4* origin, uint64_t* hkey, int* hval,
                           int hcap, const MGridParams* __restrict__ params, int bits, unsigned* err) {
    const int count = *count_ptr;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < count; i += gridDim.x * blockDim.x) {
        const int s = list[i];
        uint64_t key = leaf_key(origin[s], 0, 0, 0, params, bits);
        if (key == kEmptyKey) {
            atomicOr(err, kErrExtent);
            continue;
        }
        uint32_t m = (uint32_t)hcap - 1u, p = (uint32_t)mix64(key) & m;
        bool done = false;
        for (int probe = 0; probe < hcap; ++probe) {
            unsigned long long prev =
                atomicCAS((unsigned long long*)&hkey[p], (unsigned long long)kEmptyKey, (unsigned long long)key);
            if (prev == kEmptyKey) {
                hval[p] = s;
                done = true;
                break;
            }
            p = (p + 1u) & m;
        }
        if (!done) atomicOr(err, kErrHashFull);
    }
}

__global__ void k_nbr(const int* list, const int* count_ptr, const int4* origin, const uint64_t* hkey,
                      const int* hval, int hcap, const MGridParams* __restrict__ params, int bits, int* nbr) {
    const int count = *count_ptr;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < (long long)count * kNbr;
         t += (long long)gridDim.x * blockDim.x) {
        const int i = (int)(t / kNbr), d = (int)(t % kNbr);
        const int s = list[i];
        int dx, dy, dz;
        dir_of(d, dx, dy, dz);
        nbr[s * kNbr + d] = (d == 13) ? s : hfind(hkey, hval, hcap, leaf_key(origin[s], dx, dy, dz, params, bits));
    }
}

// ------------------------------------------------------- scan (prealloc)

__global__ void __launch_bounds__(1024) k_scan_blk(const int* in, int* out, int n, int* block_sums) {
    __shared__ int ws[32];
    int i = blockIdx.x * 1024 + threadIdx.x;
    int v = (i < n) ? in[i] : 0;
    int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    int x = v;
    for (int o = 1; o < 32; o <<= 1) {
        int y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) ws[w] = x;
    __syncthreads();
    if (w == 0) {
        int s = ws[lane], si = s;
        for (int o = 1; o < 32; o <<= 1) {
            int y = __shfl_up_sync(0xffffffffu, si, o);
            if (lane >= o) si += y;
        }
        ws[lane] = si - s;
        if (lane == 31) block_sums[blockIdx.x] = si;
    }
    __syncthreads();
    if (i < n) out[i] = x - v + ws[w];
}

__global__ void k_scan_addb(int* out, int n, const int* offs) {
    int i = blockIdx.x * 1024 + threadIdx.x;
    if (i < n) out[i] += offs[blockIdx.x];
}

__global__ void k_scan_tot(const int* in, const int* out, int n, int* total) {
    if (threadIdx.x == 0 && blockIdx.x == 0) *total = out[n - 1] + in[n - 1];
}

// Exclusive scan of n ints with scratch laid out level by level.
static void scan_levels(cudaStream_t st, const int* in, int* out, int n, int* total, int* scratch) {
    int nb = (n + 1023) / 1024;
    int* sums = scratch;
    int* sums_scan = scratch + nb;
    k_scan_blk<<<nb, 1024, 0, st>>>(in, out, n, sums);
    if (nb > 1) {
        scan_levels(st, sums, sums_scan, nb, sums_scan + nb, sums_scan + nb + 1);
        k_scan_addb<<<nb, 1024, 0, st>>>(out, n, sums_scan);
    }
    k_scan_tot<<<1, 32, 0, st>>>(in, out, n, total);
}

size_t scan_scratch_ints(int n) {
    size_t s = 0;
    while (true) {
        int nb = (n + 1023) / 1024;
        s += 2 * (size_t)nb + 2;
        if (nb <= 1) break;
        n = nb;
    }
    return s + 16;
}

// ----------------------------------------------------------- orchestration

int ls_enqueue_index(vlr_ctx* ctx, vlr_level_set* ls) {
    cudaStream_t st = ctx->stream;
    const int B = ls->grid_blocks;
    k_h_clear<<<B, 256, 0, st>>>(ls->hkey, ls->hval, ls->hcap);
    k_h_insert<<<B, 256, 0, st>>>(ls->list, ls->scalars, ls->origin, ls->hkey, ls->hval, ls->hcap, ls->d_params,
                                  ls->key_bits, ctx->d_errword);
    k_nbr<<<B, 256, 0, st>>>(ls->list, ls->scalars, ls->origin, ls->hkey, ls->hval, ls->hcap, ls->d_params,
                             ls->key_bits, ls->nbr);
    VLR_CUDA(ctx, cudaGetLastError());
    return VLR_OK;
}

int ls_enqueue_retrack(vlr_ctx* ctx, vlr_level_set* ls) {
    cudaStream_t st = ctx->stream;
    const int B = ls->grid_blocks;
    MLeafArrays A = ls->arrays();
    k_t_prepare<<<B, 256, 0, st>>>(ls->keep, ls->cap, ls->pkey, ls->pval, ls->hkey, ls->hval, ls->hcap);
    VLR_TIMED(ctx, "k_t_propose",
              k_t_propose<<<B, 256, 0, st>>>(A, ls->keep, ls->pkey, ls->pval, ls->hcap, ls->d_params, ls->key_bits,
                                             ctx->d_errword));
    k_t_count<<<B, 256, 0, st>>>(A, ls->keep, ls->pkey, ls->pval, ls->hcap, ls->d_params, ls->key_bits, ls->cap,
                                 ls->owned);
    scan_levels(st, ls->owned, ls->pos, ls->cap, ls->scalars + 3, ls->pos + ls->cap + 1);
    k_t_free<<<B, 256, 0, st>>>(A, ls->keep, ls->free_stack, ls->scalars + 2);
    if (ls->precision == VLR_PREC_F16)
        k_t_alloc<__half><<<B, 256, 0, st>>>(A, ls->origin, ls->keep, ls->pos, ls->pkey, ls->pval, ls->hcap,
                                            ls->d_params, ls->key_bits, ls->free_stack, ls->scalars + 2,
                                            ls->list_new, (__half*)ls->vals[0], ctx->d_errword);
    else
        k_t_alloc<float><<<B, 256, 0, st>>>(A, ls->origin, ls->keep, ls->pos, ls->pkey, ls->pval, ls->hcap,
                                           ls->d_params, ls->key_bits, ls->free_stack, ls->scalars + 2,
                                           ls->list_new, (float*)ls->vals[0], ctx->d_errword);
    k_t_finalize<<<B, 256, 0, st>>>(ls->scalars, ls->list_new, ls->list, ls->cap);
    VLR_CUDA(ctx, cudaGetLastError());
    return ls_enqueue_index(ctx, ls);
}

template <typename T>
static int enqueue_stencils(vlr_ctx* ctx, vlr_level_set* ls) {
    cudaStream_t st = ctx->stream;
    const int B = ls->grid_blocks;
    MLeafArrays A = ls->arrays();
    const T* v0 = (const T*)ls->vals[0];
    T* v1 = (T*)ls->vals[1];
    if (ls->halo == 2)
        VLR_TIMED(ctx, "k_m_advect",
                  k_m_advect<T, 2><<<B, 256, 0, st>>>(A, v0, v1, ls->d_params, ls->d_tab, ls->sp, ctx->d_errword));
    else
        VLR_TIMED(ctx, "k_m_advect",
                  k_m_advect<T, 3><<<B, 256, 0, st>>>(A, v0, v1, ls->d_params, ls->d_tab, ls->sp, ctx->d_errword));
    T* w0 = (T*)ls->vals[0];
    switch (ls->reinit_iters) {
        case 0:
            VLR_TIMED(ctx, "k_m_reinit", k_m_reinit<T, 0><<<B, 256, 0, st>>>(A, v1, w0, ls->d_params));
            break;
        case 1:
            VLR_TIMED(ctx, "k_m_reinit", k_m_reinit<T, 1><<<B, 256, 0, st>>>(A, v1, w0, ls->d_params));
            break;
        default:
            VLR_TIMED(ctx, "k_m_reinit", k_m_reinit<T, 2><<<B, 256, 0, st>>>(A, v1, w0, ls->d_params));
            break;
    }
    VLR_CUDA(ctx, cudaGetLastError());
    return VLR_OK;
}

int ls_enqueue_step(vlr_ctx* ctx, vlr_level_set* ls) {
    int rc = (ls->precision == VLR_PREC_F16) ? enqueue_stencils<__half>(ctx, ls) : enqueue_stencils<float>(ctx, ls);
    if (rc) return rc;
    return ls_enqueue_retrack(ctx, ls);
}

}  // namespace vlr
