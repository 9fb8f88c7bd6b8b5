// Re-tracking of the narrow band after each method step, on the device and
// without host synchronisation (the step is one CUDA graph).  The stencil
// kernels already did two parts: advect cleared the per-step state, reinit
// set keep flags (a leaf survives if it, or a neighbour within one voxel,
// has an active voxel: dilate26 of the band) and proposed missing leaves in
// a hash table where atomicMin keeps the proposer whose direction, seen from
// the new leaf, comes first.  Three kernels finish the step:
//
//   k_t_scanalloc  per list position: survive flag + owned proposals; an
//                  exclusive scan in list order (single pass, decoupled
//                  look-back over 256-position chunks taken by ticket) gives
//                  each survivor its new position, followed by the new leaves
//                  it owns; new leaves take slots from the free stack, slots
//                  of dropped leaves go to a recycle list
//   k_t_finalize   new list, fill of new leaves (clamped-sign rule from the
//                  owner), hash insertion, recycled slots back on the stack
//   k_t_nbr        27-neighbour rows updated where a neighbour was dropped or
//                  is new (the rows of an upload are built whole by k_nbr);
//                  publishes counts
//
// The reference's counterparts are dilate (src/tools/morphology.rs:20-35),
// trim_narrow_band's deactivation (src/tools/level_set_track.rs:53-68) and
// remove_empty_leaves (src/tree/internal.rs:231-247).
#include <algorithm>

#include "method_state.hpp"

namespace vlr {

// scalars: [0] count  [1] step  [2] free top  [3] spare
//          [4] new count  [5] recycled count  [6] new free top  [7] chunk ticket
constexpr int kChunk = 256;
constexpr long long kSpinLimit = 1ll << 22;  // default bound of the look-back wait (about half a second)

__device__ __forceinline__ void dir_of(int d, int& dx, int& dy, int& dz) {
    dx = d / 9 - 1;
    dy = (d / 3) % 3 - 1;
    dz = d % 3 - 1;
}

__device__ __forceinline__ uint64_t leaf_key(const int4 o, int dx, int dy, int dz, const MGridParams* params,
                                             int bits) {
    const MGridParams& P = params[o.w];
    return mkey((long long)(o.x >> 3) + dx, (long long)(o.y >> 3) + dy, (long long)(o.z >> 3) + dz, o.w, P.base, bits);
}

// Status word of a scan chunk: [63..34] tag (step + 1), [33..32] flag
// (1 aggregate, 2 inclusive prefix), [31..0] value.
__device__ __forceinline__ unsigned long long pack_status(unsigned tag, unsigned flag, unsigned value) {
    return ((unsigned long long)(tag & 0x3fffffffu) << 34) | ((unsigned long long)flag << 32) | value;
}

__global__ void __launch_bounds__(kChunk) k_t_scanalloc(MLeafArrays A, int4* origin, const int* keep,
                                                       const uint64_t* __restrict__ pkey, const int* __restrict__ pval,
                                                       int hcap, const MGridParams* __restrict__ params, int bits,
                                                       int* free_stack, int* recycled, int* list_new,
                                                       int* newinfo, unsigned long long* status, int* scalars,
                                                       int cap, unsigned* err) {
    dep_wait();
    dep_launch();
    if (step_aborted(err)) return;
    __shared__ int s_ticket;
    __shared__ int s_warp[kChunk / 32];
    __shared__ int s_prefix;
    const long long spin_limit = wait_limit(err, kSpinLimit);
    const bool hold_first = test_stall(err);
    const int count = scalars[0];
    const unsigned tag = (unsigned)scalars[1] + 1u;
    const int nchunks = (count + kChunk - 1) / kChunk;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    for (;;) {
        if (threadIdx.x == 0) s_ticket = atomicAdd(&scalars[7], 1);
        __syncthreads();
        const int chunk = s_ticket;
        __syncthreads();
        if (chunk >= nchunks) break;
        const int p = chunk * kChunk + threadIdx.x;
        int s = -1, surv = 0, owned = 0;
        unsigned own_bits = 0;
        int4 o = make_int4(0, 0, 0, 0);
        if (p < count) {
            s = A.list[p];
            surv = keep[s] ? 1 : 0;
            if (!surv) recycled[atomicAdd(&scalars[5], 1)] = s;
            unsigned sp = A.spill[s];
            o = origin[s];
            while (sp) {  // absent neighbours only (reinit masked the present ones out)
                int d = __ffs(sp) - 1;
                sp &= sp - 1;
                int dx, dy, dz;
                dir_of(d, dx, dy, dz);
                if (hfind(pkey, pval, hcap, leaf_key(o, dx, dy, dz, params, bits)) == kNbr - 1 - d) {
                    own_bits |= 1u << d;
                    ++owned;
                }
            }
        }
        // block-wide inclusive scan of surv + owned
        int v = surv + owned, x = v;
#pragma unroll
        for (int off = 1; off < 32; off <<= 1) {
            int y = __shfl_up_sync(0xffffffffu, x, off);
            if (lane >= off) x += y;
        }
        if (lane == 31) s_warp[w] = x;
        __syncthreads();
        if (w == 0) {
            int a = (lane < kChunk / 32) ? s_warp[lane] : 0, ai = a;
#pragma unroll
            for (int off = 1; off < 32; off <<= 1) {
                int y = __shfl_up_sync(0xffffffffu, ai, off);
                if (lane >= off) ai += y;
            }
            if (lane < kChunk / 32) s_warp[lane] = ai - a;
            // publish the aggregate, then look back 32 chunks at a time: lane j
            // reads the status of chunk q - j; the walk stops at the nearest
            // chunk holding an inclusive prefix (a virtual one before chunk 0)
            const unsigned total = (unsigned)__shfl_sync(0xffffffffu, ai, kChunk / 32 - 1);
            const unsigned wtag = tag & 0x3fffffffu;
            unsigned prefix = 0;
            if (chunk == 0) {
                // (test hook: withheld, so that every later chunk's wait runs out)
                if (lane == 0 && !hold_first) atomicExch(&status[0], pack_status(tag, 2, total));
            } else {
                if (lane == 0) atomicExch(&status[chunk], pack_status(tag, 1, total));
                int q = chunk - 1;
                long long spins = 0;
                for (;;) {
                    const int idx = q - lane;
                    unsigned flag = 2, val = 0;
                    if (idx >= 0) {
                        const unsigned long long st = *reinterpret_cast<volatile unsigned long long*>(&status[idx]);
                        const bool cur = (unsigned)(st >> 34) == wtag;
                        flag = cur ? (unsigned)(st >> 32) & 3u : 0u;
                        val = (unsigned)st;
                    }
                    const unsigned pmask = __ballot_sync(0xffffffffu, flag == 2);
                    const unsigned invalid = __ballot_sync(0xffffffffu, flag == 0);
                    const int first_p = pmask ? __ffs(pmask) - 1 : 32;
                    const unsigned upto = first_p >= 31 ? 0xffffffffu : ((2u << first_p) - 1u);
                    if (invalid & upto) {
                        if (++spins > spin_limit) {  // bounded wait: report and continue
                            if (lane == 0) atomicOr(err, kErrTimeout);
                            break;
                        }
                        __nanosleep(32);
                        continue;
                    }
                    unsigned add = ((upto >> lane) & 1u) ? val : 0u;
#pragma unroll
                    for (int off = 16; off > 0; off >>= 1) add += __shfl_xor_sync(0xffffffffu, add, off);
                    prefix += add;
                    if (first_p < 32) break;
                    q -= 32;
                }
                if (lane == 0) atomicExch(&status[chunk], pack_status(tag, 2, prefix + total));
            }
            if (lane == 0) {
                s_prefix = (int)prefix;
                if (chunk == nchunks - 1) scalars[4] = (int)(prefix + total);
            }
        }
        __syncthreads();
        int pos = s_prefix + s_warp[w] + x - v;
        if (p < count) {
            if (surv) {
                if (pos < cap) {
                    list_new[pos] = s;
                    newinfo[pos] = -1;
                }
                ++pos;
            }
            while (own_bits) {
                int d = __ffs(own_bits) - 1;
                own_bits &= own_bits - 1;
                int t = atomicSub(&scalars[2], 1) - 1;
                if (t < 0 || pos >= cap) {
                    atomicOr(err, kErrCapacity);
                    if (pos < cap) {
                        newinfo[pos] = -2;  // slot 0 stands in; its values are left alone
                        list_new[pos] = 0;
                    }
                    ++pos;
                    continue;
                }
                int ns = free_stack[t];
                int dx, dy, dz;
                dir_of(d, dx, dy, dz);
                origin[ns] = make_int4(o.x + 8 * dx, o.y + 8 * dy, o.z + 8 * dz, o.w);
                list_new[pos] = ns;
                newinfo[pos] = s * 32 + d;  // owner slot and direction
                A.spill[ns] = 0;
                A.nonempty[ns] = 0;
#pragma unroll
                for (int q = 0; q < 8; ++q) {
                    A.mask[(size_t)ns * 8 + q] = 0ull;
                    A.dmask[(size_t)ns * 8 + q] = 0ull;
                }
                ++pos;
            }
        }
    }
}

// One thread per new-list position, a block's 256 positions at a time: copy
// the list and insert the leaf's hash key; the block's new leaves, queued in
// shared memory, are then filled from their owners one warp each (coalesced
// stores).  The dropped slots go back on the free stack.
template <typename T>
__global__ void __launch_bounds__(256) k_t_finalize(const int* list_new, const int* newinfo, int* list, const int4* origin,
                                                   T* vals, uint64_t* hkey, int* hval, int hcap,
                                                   const MGridParams* __restrict__ params, int bits, int* free_stack,
                                                   const int* recycled, int* scalars, int cap, unsigned* err) {
    dep_wait();
    dep_launch();
    if (step_aborted(err)) return;
    __shared__ int s_q[256];
    __shared__ int s_nq;
    const int n = min(scalars[4], cap);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (threadIdx.x == 0) s_nq = 0;
    __syncthreads();
    for (int base = blockIdx.x * 256; base < n; base += gridDim.x * 256) {
        const int p = base + threadIdx.x;
        if (p < n) {
            const int s = list_new[p];
            const int info = newinfo[p];
            list[p] = s;
            if (info != -2) {
                const uint64_t key = leaf_key(origin[s], 0, 0, 0, params, bits);
                bool done = false;
                if (key != kEmptyKey) {
                    uint32_t m = (uint32_t)hcap - 1u, q = (uint32_t)mix64(key) & m;
                    for (int probe = 0; probe < hcap; ++probe) {
                        const unsigned long long prev = atomicCAS((unsigned long long*)&hkey[q],
                                                                  (unsigned long long)kEmptyKey,
                                                                  (unsigned long long)key);
                        if (prev == kEmptyKey) {
                            hval[q] = s;
                            done = true;
                            break;
                        }
                        q = (q + 1u) & m;
                    }
                }
                if (!done) atomicOr(err, key == kEmptyKey ? kErrExtent : kErrHashFull);
            }
            if (info >= 0) s_q[atomicAdd(&s_nq, 1)] = p;
        }
        __syncthreads();
        const int nq = s_nq;
        for (int j = warp; j < nq; j += 256 / 32) {
            const int q = s_q[j];
            const int s = list_new[q], info = newinfo[q];
            const int owner = info >> 5, d = info & 31;
            int dx, dy, dz;
            dir_of(d, dx, dy, dz);
            const float hw = params[origin[owner].w].hw;
            for (int off = lane; off < kLeafVoxels; off += 32) {
                const int x = 8 * dx + (off >> 6), y = 8 * dy + ((off >> 3) & 7), z = 8 * dz + (off & 7);
                const int cx = min(max(x, 0), 7), cy = min(max(y, 0), 7), cz = min(max(z, 0), 7);
                const float v = to_f(vals[(size_t)owner * kLeafVoxels + ((cx << 6) | (cy << 3) | cz)]);
                vals[(size_t)s * kLeafVoxels + off] = from_f<T>(copysignf(hw, v));
            }
        }
        __syncthreads();
        if (threadIdx.x == 0) s_nq = 0;
        __syncthreads();
    }
    // dropped slots go back on the free stack above the remaining free slots
    const int top = max(scalars[2], 0);
    const int nrec = scalars[5];
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nrec; i += gridDim.x * blockDim.x)
        if (top + i < cap) free_stack[top + i] = recycled[i];
    if (blockIdx.x == 0 && threadIdx.x == 0) scalars[6] = min(top + nrec, cap);
}

// Neighbour rows carried from step to step.  A survivor keeps its slot and
// its position, so its row changes only at a neighbour that was dropped or is
// new (a dropped leaf's slot returns to the free stack after this step's new
// leaves took theirs, so no slot is both).  One warp per dropped leaf: its
// old row names its listed neighbours, and those that survive clear the
// entry that points back at it.  One warp per new leaf (found by a ballot
// over 32 list positions): lane d looks neighbour d up in the hash rebuilt
// by k_t_finalize, writes the new leaf's row and, for a present neighbour,
// the entry that points back at the new leaf (two adjacent new leaves write
// each other's entries with the same values).  Publishes the counts; the
// dropped count is cleared by the next step's advect.
__global__ void k_t_nbr(const int* list, const int* newinfo, const int* recycled, const int* keep, int* scalars,
                        const int4* origin, const uint64_t* hkey, const int* hval, int hcap,
                        const MGridParams* __restrict__ params, int bits, int* nbr, int cap, const unsigned* err) {
    dep_wait();
    dep_launch();
    if (step_aborted(err)) return;
    const int count = min(scalars[4], cap);
    const int nrec = min(scalars[5], cap);
    const int lane = threadIdx.x & 31;
    const int gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, nw = (gridDim.x * blockDim.x) >> 5;
    for (int i = gw; i < nrec; i += nw) {
        const int D = recycled[i];
        if (lane < kNbr && lane != 13) {
            const int M = nbr[(size_t)D * kNbr + lane];
            if (M >= 0 && keep[M]) nbr[(size_t)M * kNbr + (kNbr - 1 - lane)] = -1;
        }
    }
    for (int base = gw * 32; base < count; base += nw * 32) {
        const int p = base + lane;
        unsigned b = __ballot_sync(0xffffffffu, p < count && newinfo[p] >= 0);
        while (b) {
            const int j = __ffs(b) - 1;
            b &= b - 1u;
            const int N = list[base + j];
            if (lane < kNbr) {
                int M = N;
                if (lane != 13) {
                    int dx, dy, dz;
                    dir_of(lane, dx, dy, dz);
                    M = hfind(hkey, hval, hcap, leaf_key(origin[N], dx, dy, dz, params, bits));
                }
                nbr[(size_t)N * kNbr + lane] = M;
                if (M >= 0 && M != N) nbr[(size_t)M * kNbr + (kNbr - 1 - lane)] = N;
            }
        }
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        scalars[0] = count;
        scalars[1] += 1;
        scalars[2] = scalars[6];
    }
}

// ---------------------------------------------- full index (creation/upload)

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
            if (prev == key) {  // the same leaf listed twice
                atomicOr(err, kErrInput);
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
        nbr[(size_t)s * kNbr + d] = (d == 13) ? s : hfind(hkey, hval, hcap, leaf_key(origin[s], dx, dy, dz, params, bits));
    }
}

size_t scan_scratch_ints(int n) { return (size_t)((n + kChunk - 1) / kChunk) * 2 + 16; }

// ----------------------------------------------------------- orchestration

// Launch one kernel of the step with programmatic stream serialization (its
// CTAs may be scheduled while the previous kernel drains; the kernel itself
// waits for that kernel's results with dep_wait()).
template <typename... KArgs, typename... Args>
static cudaError_t pdl_launch(void (*kernel)(KArgs...), int grid, int block, size_t smem, cudaStream_t st,
                              Args... args) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)grid);
    cfg.blockDim = dim3((unsigned)block);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, kernel, args...);
}

MTopo topo_of(vlr_level_set* ls) {
    MTopo t;
    t.keep = ls->keep;
    t.cap = ls->cap;
    t.pkey = ls->pkey;
    t.pval = ls->pval;
    t.hkey = ls->hkey;
    t.hval = ls->hval;
    t.hcap = ls->hcap;
    t.scalars = ls->scalars;
    t.key_bits = ls->key_bits;
    return t;
}

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
    // status words of the look-back scan live after the scan positions in `pos`
    unsigned long long* status = reinterpret_cast<unsigned long long*>(ls->pos);
    VLR_TIMED(ctx, "k_t_scanalloc",
              VLR_CUDA(ctx, pdl_launch(k_t_scanalloc, B, kChunk, 0, st, A, ls->origin, (const int*)ls->keep,
                                       (const uint64_t*)ls->pkey, (const int*)ls->pval, ls->hcap,
                                       (const MGridParams*)ls->d_params, ls->key_bits, ls->free_stack, ls->owned,
                                       ls->list_new, ls->newinfo, status, ls->scalars, ls->cap, ctx->d_errword)));
    if (ls->precision == VLR_PREC_F16)
        VLR_TIMED(ctx, "k_t_finalize",
                  VLR_CUDA(ctx, pdl_launch(k_t_finalize<__half>, B, 256, 0, st, (const int*)ls->list_new,
                                           (const int*)ls->newinfo, ls->list, (const int4*)ls->origin,
                                           (__half*)ls->vals[0], ls->hkey, ls->hval, ls->hcap,
                                           (const MGridParams*)ls->d_params, ls->key_bits, ls->free_stack,
                                           (const int*)ls->owned, ls->scalars, ls->cap, ctx->d_errword)));
    else
        VLR_TIMED(ctx, "k_t_finalize",
                  VLR_CUDA(ctx, pdl_launch(k_t_finalize<float>, B, 256, 0, st, (const int*)ls->list_new,
                                           (const int*)ls->newinfo, ls->list, (const int4*)ls->origin,
                                           (float*)ls->vals[0], ls->hkey, ls->hval, ls->hcap,
                                           (const MGridParams*)ls->d_params, ls->key_bits, ls->free_stack,
                                           (const int*)ls->owned, ls->scalars, ls->cap, ctx->d_errword)));
    VLR_TIMED(ctx, "k_t_nbr",
              VLR_CUDA(ctx, pdl_launch(k_t_nbr, B, 256, 0, st, (const int*)ls->list, (const int*)ls->newinfo,
                                       (const int*)ls->owned, (const int*)ls->keep, ls->scalars,
                                       (const int4*)ls->origin, (const uint64_t*)ls->hkey, (const int*)ls->hval,
                                       ls->hcap, (const MGridParams*)ls->d_params, ls->key_bits, ls->nbr, ls->cap,
                                       (const unsigned*)ctx->d_errword)));
    VLR_CUDA(ctx, cudaGetLastError());
    return VLR_OK;
}

// ------------------------------------------------------ stencil launches

// The launch shape of a stencil kernel (threads per CTA, persistent CTAs per
// SM, staging mode) is chosen by ls_autotune_step; until then the kernels run
// at 256 threads with every SM filled to the occupancy limit and cp.async
// staging.

template <typename T, int H, int VK>
static int launch_advect_vk(vlr_ctx* ctx, vlr_level_set* ls, const MLeafArrays& A, const MTopo& topo, int blocks) {
    const size_t smem = advect_smem_bytes(sizeof(T) == 2, H);
    VLR_CUDA(ctx, cudaFuncSetAttribute(k_m_advect<T, H, VK>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    VLR_TIMED(ctx, "k_m_advect",
              VLR_CUDA(ctx, pdl_launch(k_m_advect<T, H, VK>, blocks, kAdvectThreads, smem, ctx->stream, A,
                                       (const T*)ls->vals[0], (T*)ls->vals[1], (const MGridParams*)ls->d_params,
                                       (const float2*)ls->d_tab, ls->sp, topo, ctx->d_errword)));
    return VLR_OK;
}

template <typename T, int H>
static int launch_advect_h(vlr_ctx* ctx, vlr_level_set* ls, const MLeafArrays& A, const MTopo& topo, int blocks) {
    switch (ls->vel_kind) {
        case MVEL_CONSTANT: return launch_advect_vk<T, H, MVEL_CONSTANT>(ctx, ls, A, topo, blocks);
        case MVEL_VORTEX: return launch_advect_vk<T, H, MVEL_VORTEX>(ctx, ls, A, topo, blocks);
        case MVEL_CURL: return launch_advect_vk<T, H, MVEL_CURL>(ctx, ls, A, topo, blocks);
        default: return launch_advect_vk<T, H, -1>(ctx, ls, A, topo, blocks);
    }
}

template <typename T>
static int launch_advect(vlr_ctx* ctx, vlr_level_set* ls, StencilShape sh) {
    MLeafArrays A = ls->arrays();
    MTopo topo = topo_of(ls);
    return ls->halo == 2 ? launch_advect_h<T, 2>(ctx, ls, A, topo, sh.blocks)
                         : launch_advect_h<T, 3>(ctx, ls, A, topo, sh.blocks);
}

template <typename T, int NIT, int FIX>
static int launch_reinit_fix(vlr_ctx* ctx, vlr_level_set* ls, const MLeafArrays& A, const MTopo& topo, int blocks) {
    const size_t smem = reinit_smem_bytes(sizeof(T) == 2, NIT, FIX);
    VLR_CUDA(ctx, cudaFuncSetAttribute(k_m_reinit<T, NIT, FIX>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)smem));
    VLR_TIMED(ctx, "k_m_reinit",
              VLR_CUDA(ctx, pdl_launch(k_m_reinit<T, NIT, FIX>, blocks, kReinitThreads, smem, ctx->stream, A,
                                       (const T*)ls->vals[1], (T*)ls->vals[0], (const MGridParams*)ls->d_params,
                                       topo, ctx->d_errword)));
    return VLR_OK;
}

template <typename T, int NIT>
static int launch_reinit_nit(vlr_ctx* ctx, vlr_level_set* ls, const MLeafArrays& A, const MTopo& topo, int blocks) {
    return ls->sp.reinit_mode == 1 ? launch_reinit_fix<T, NIT, 1>(ctx, ls, A, topo, blocks)
                                   : launch_reinit_fix<T, NIT, 0>(ctx, ls, A, topo, blocks);
}

template <typename T>
static int launch_reinit(vlr_ctx* ctx, vlr_level_set* ls, StencilShape sh) {
    MLeafArrays A = ls->arrays();
    MTopo topo = topo_of(ls);
    switch (ls->reinit_iters) {
        case 0: return launch_reinit_nit<T, 0>(ctx, ls, A, topo, sh.blocks);
        case 1: return launch_reinit_nit<T, 1>(ctx, ls, A, topo, sh.blocks);
        default: return launch_reinit_nit<T, 2>(ctx, ls, A, topo, sh.blocks);
    }
}

// Occupancy limit (CTAs per SM) of the advect kernel; every velocity kind
// instantiates the same staging, so the mixed-kind kernel stands for the
// register and shared-memory footprint.
template <typename T>
static int advect_occupancy(vlr_ctx* ctx, vlr_level_set* ls, int* per_sm) {
    *per_sm = 0;
    const size_t smem = advect_smem_bytes(sizeof(T) == 2, ls->halo);
    if (ls->halo == 2) {
        VLR_CUDA(ctx, cudaFuncSetAttribute(k_m_advect<T, 2, -1>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                           (int)smem));
        VLR_CUDA(ctx, cudaOccupancyMaxActiveBlocksPerMultiprocessor(per_sm, k_m_advect<T, 2, -1>, kAdvectThreads,
                                                                    smem));
    } else {
        VLR_CUDA(ctx, cudaFuncSetAttribute(k_m_advect<T, 3, -1>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                           (int)smem));
        VLR_CUDA(ctx, cudaOccupancyMaxActiveBlocksPerMultiprocessor(per_sm, k_m_advect<T, 3, -1>, kAdvectThreads,
                                                                    smem));
    }
    return VLR_OK;
}

// Occupancy limit (CTAs per SM) of the reinit kernel (its 2-iteration
// instance at the level set's reinitialisation mode stands for all).
template <typename T>
static int reinit_occupancy(vlr_ctx* ctx, vlr_level_set* ls, int* per_sm) {
    *per_sm = 0;
    const int fix = ls->sp.reinit_mode == 1;
    const size_t smem = reinit_smem_bytes(sizeof(T) == 2, 2, fix);
    if (fix) {
        VLR_CUDA(ctx, cudaFuncSetAttribute(k_m_reinit<T, 2, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                           (int)smem));
        VLR_CUDA(ctx, cudaOccupancyMaxActiveBlocksPerMultiprocessor(per_sm, k_m_reinit<T, 2, 1>, kReinitThreads,
                                                                    smem));
    } else {
        VLR_CUDA(ctx, cudaFuncSetAttribute(k_m_reinit<T, 2, 0>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                           (int)smem));
        VLR_CUDA(ctx, cudaOccupancyMaxActiveBlocksPerMultiprocessor(per_sm, k_m_reinit<T, 2, 0>, kReinitThreads,
                                                                    smem));
    }
    return VLR_OK;
}

// Candidate launch shapes of a stencil kernel (128 threads per CTA): the
// occupancy limit, 3/4 and 1/2 of it, in persistent CTAs over all SMs.
template <typename T>
static int stencil_candidates(vlr_ctx* ctx, vlr_level_set* ls, int which, std::vector<StencilShape>& out) {
    out.clear();
    int occ = 0;
    int rc = which == 0 ? advect_occupancy<T>(ctx, ls, &occ) : reinit_occupancy<T>(ctx, ls, &occ);
    if (rc) return rc;
    int prev = -1;
    for (int per_sm : {occ, (3 * occ + 3) / 4, (occ + 1) / 2}) {
        if (per_sm < 1 || per_sm == prev) continue;
        prev = per_sm;
        out.push_back(StencilShape{which == 0 ? kAdvectThreads : kReinitThreads, per_sm * ctx->sm_count, 0});
    }
    if (out.empty()) return set_error(ctx, VLR_ERR_CUDA, "stencil kernel does not fit on an SM");
    return VLR_OK;
}

// The shape used when none has been chosen: occupancy-limited.
template <typename T>
static int default_shape(vlr_ctx* ctx, vlr_level_set* ls, int which, StencilShape* sh) {
    int occ = 0;
    int rc = which == 0 ? advect_occupancy<T>(ctx, ls, &occ) : reinit_occupancy<T>(ctx, ls, &occ);
    if (rc) return rc;
    if (occ < 1) return set_error(ctx, VLR_ERR_CUDA, "stencil kernel does not fit on an SM");
    *sh = StencilShape{which == 0 ? kAdvectThreads : kReinitThreads, occ * ctx->sm_count, 0};
    return VLR_OK;
}

template <typename T>
static int enqueue_stencils(vlr_ctx* ctx, vlr_level_set* ls) {
    if (!ls->adv_shape.nt) {
        int rc = default_shape<T>(ctx, ls, 0, &ls->adv_shape);
        if (rc) return rc;
    }
    if (!ls->re_shape.nt) {
        int rc = default_shape<T>(ctx, ls, 1, &ls->re_shape);
        if (rc) return rc;
    }
    int rc = launch_advect<T>(ctx, ls, ls->adv_shape);
    if (rc) return rc;
    rc = launch_reinit<T>(ctx, ls, ls->re_shape);
    if (rc) return rc;
    VLR_CUDA(ctx, cudaGetLastError());
    return VLR_OK;
}

// Times every candidate shape of one stencil kernel on the current inputs
// (two rounds; the second round's time counts, so the first round warms the
// caches for all candidates alike) and keeps the fastest.
template <typename T>
static int tune_one(vlr_ctx* ctx, vlr_level_set* ls, int which, StencilShape* best) {
    std::vector<StencilShape> cand;
    int rc = stencil_candidates<T>(ctx, ls, which, cand);
    if (rc) return rc;
    const int n = (int)cand.size();
    std::vector<cudaEvent_t> ev(2 * n);
    for (auto& e : ev) VLR_CUDA(ctx, cudaEventCreate(&e));
    ls->tune_log[which].clear();
    for (int round = 0; round < 2 && !rc; ++round)
        for (int i = 0; i < n && !rc; ++i) {
            if (round) VLR_CUDA(ctx, cudaEventRecord(ev[2 * i], ctx->stream));
            rc = which == 0 ? launch_advect<T>(ctx, ls, cand[i]) : launch_reinit<T>(ctx, ls, cand[i]);
            if (round && !rc) VLR_CUDA(ctx, cudaEventRecord(ev[2 * i + 1], ctx->stream));
        }
    if (!rc) {
        cudaError_t e = cudaStreamSynchronize(ctx->stream);
        if (e != cudaSuccess) rc = check_cuda(ctx, e, "autotune");
    }
    float best_ms = 0.f;
    for (int i = 0; i < n && !rc; ++i) {
        float ms = 0.f;
        cudaError_t e = cudaEventElapsedTime(&ms, ev[2 * i], ev[2 * i + 1]);
        if (e != cudaSuccess) {
            rc = check_cuda(ctx, e, "autotune timing");
            break;
        }
        ls->tune_log[which].push_back(TuneEntry{cand[i], ms});
        if (i == 0 || ms < best_ms) {
            best_ms = ms;
            *best = cand[i];
        }
    }
    for (auto& e : ev) cudaEventDestroy(e);
    return rc;
}

template <typename T>
static int autotune_stencils(vlr_ctx* ctx, vlr_level_set* ls) {
    StencilShape a{}, r{};
    int rc = tune_one<T>(ctx, ls, 0, &a);
    if (rc) return rc;
    // the inputs of the last advect launch stand (every candidate wrote the same)
    ls->adv_shape = a;
    rc = tune_one<T>(ctx, ls, 1, &r);
    if (rc) return rc;
    ls->re_shape = r;
    return VLR_OK;
}

int ls_autotune_step(vlr_ctx* ctx, vlr_level_set* ls) {
    int rc = (ls->precision == VLR_PREC_F16) ? autotune_stencils<__half>(ctx, ls) : autotune_stencils<float>(ctx, ls);
    if (rc) return rc;
    ls->tuned = true;
    return ls_enqueue_retrack(ctx, ls);
}

int ls_enqueue_step(vlr_ctx* ctx, vlr_level_set* ls) {
    int rc = (ls->precision == VLR_PREC_F16) ? enqueue_stencils<__half>(ctx, ls) : enqueue_stencils<float>(ctx, ls);
    if (rc) return rc;
    return ls_enqueue_retrack(ctx, ls);
}

}  // namespace vlr
