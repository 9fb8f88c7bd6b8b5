// In-place edits of a single-grid level set's leaf pool, for a grid divided
// over devices: each rank keeps its owned leaves resident in its pool and, per
// step, reads the leaves its neighbours need (vlr_ls_gather_device), adds the
// ghost leaves it receives and, after the step, drops what it does not own
// and adds what other ranks computed for it (vlr_ls_edit_device).  Values
// travel in the pool's own type (FP16 for an FP16 level set), so a ghost leaf
// is bit-identical to its owner's copy and no value is converted on the way.
//
// The crate has no counterpart (its step is serial over one in-memory tree);
// the leaf records are those of src/nano/layout.rs:89-170 (origin, value
// mask, 512 values in ZYX order).
#include <cuda_fp16.h>

#include "method_state.hpp"

using namespace vlr;

namespace {

// keep[i] = 1 for the list positions that stay.
__global__ void k_edit_flags(const uint8_t* __restrict__ drop, int n, int* __restrict__ keep) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) keep[i] = drop[i] ? 0 : 1;
}

// Kept positions move to list_new[kpos[i]] in list order; dropped slots are
// pushed on the free stack above its top, in list order.
__global__ void k_edit_compact(const int* __restrict__ list, const int* __restrict__ keep,
                               const int* __restrict__ kpos, int n, int* __restrict__ list_new,
                               int* __restrict__ free_stack, const int* __restrict__ scalars) {
    const int top = scalars[2];
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        if (keep[i]) list_new[kpos[i]] = list[i];
        else free_stack[top + (i - kpos[i])] = list[i];
    }
}

// The new list: kept leaves, then n_add leaves in slots popped off the free
// stack (lowest first), their records copied in.  A pool without room for
// them flags kErrCapacity and changes nothing (k_edit_finish then leaves the
// count and the stack top as they were).
__device__ __forceinline__ bool edit_room(const int* kpos, int n, int n_add, const int* scalars, int cap, int* kept,
                                          int* top) {
    *kept = kpos[n];
    *top = scalars[2] + (n - *kept);  // after the pushes of k_edit_compact
    return *kept + n_add <= cap && n_add <= *top;
}

template <typename T>
__global__ void k_edit_append(const int* __restrict__ list_new, const int* __restrict__ kpos, int n,
                              const int32_t* __restrict__ o3, const uint64_t* __restrict__ masks,
                              const T* __restrict__ phi, int n_add, int* __restrict__ list,
                              const int* __restrict__ free_stack, int4* __restrict__ origin,
                              uint64_t* __restrict__ mask, T* __restrict__ vals, const int* __restrict__ scalars,
                              int cap, unsigned* err) {
    int kept, top;
    if (!edit_room(kpos, n, n_add, scalars, cap, &kept, &top)) {
        if (blockIdx.x == 0 && threadIdx.x == 0) atomicOr(err, kErrCapacity);
        return;
    }
    const long long total = (long long)kept + n_add;
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total; i += stride) {
        if (i < kept) {
            list[i] = list_new[i];
        } else {
            const int j = (int)(i - kept);
            const int s = free_stack[top - 1 - j];
            list[i] = s;
            const int x = o3[3 * j], y = o3[3 * j + 1], z = o3[3 * j + 2];
            if ((x | y | z) & 7) atomicOr(err, kErrInput);
            origin[s] = make_int4(x, y, z, 0);
        }
    }
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < (long long)n_add * kLeafVoxels;
         t += stride) {
        const int j = (int)(t / kLeafVoxels), v = (int)(t % kLeafVoxels);
        const int s = free_stack[top - 1 - j];
        vals[(size_t)s * kLeafVoxels + v] = phi[t];
        if (v < 8) mask[(size_t)s * 8 + v] = masks[(size_t)j * 8 + v];
    }
}

__global__ void k_edit_finish(const int* __restrict__ kpos, int n, int n_add, int* __restrict__ scalars, int cap) {
    int kept, top;
    if (threadIdx.x == 0 && edit_room(kpos, n, n_add, scalars, cap, &kept, &top)) {
        scalars[0] = kept + n_add;
        scalars[2] = top - n_add;
    }
}

// Records at list positions pos[i] (or i when pos is null); values and masks
// only where their outputs are given.
template <typename T>
__global__ void k_gather_pos(const int* __restrict__ list, const int* __restrict__ pos, int n,
                             const int4* __restrict__ origin, const uint64_t* __restrict__ mask,
                             const T* __restrict__ vals, int32_t* __restrict__ o3, uint64_t* __restrict__ m_out,
                             T* __restrict__ v_out) {
    const int W = v_out ? kLeafVoxels : 8;  // work items per leaf
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < (long long)n * W;
         t += (long long)gridDim.x * blockDim.x) {
        const int i = (int)(t / W), v = (int)(t % W);
        const int s = list[pos ? pos[i] : i];
        if (v_out) v_out[t] = vals[(size_t)s * kLeafVoxels + v];
        if (v < 8 && m_out) m_out[(size_t)i * 8 + v] = mask[(size_t)s * 8 + v];
        if (v < 3) {
            const int4 o = origin[s];
            o3[3 * i + v] = v == 0 ? o.x : (v == 1 ? o.y : o.z);
        }
    }
}

// Positions out of [0, count) flag kErrInput.
__global__ void k_check_pos(const int* __restrict__ pos, int n, const int* __restrict__ scalars, unsigned* err) {
    const int count = scalars[0];
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        if (pos[i] < 0 || pos[i] >= count) atomicOr(err, kErrInput);
}

int list_count(vlr_ctx* ctx, const vlr_level_set* ls, int* n) {
    return read_int(ctx, ls->scalars, n);
}

}  // namespace

extern "C" {

int vlr_ls_gather_device(vlr_ctx* ctx, const vlr_level_set* ls, const int32_t* d_pos, size_t n,
                         int32_t* d_origins, uint64_t* d_masks, void* d_phi) {
    if (!ctx || !ls || (n && !d_origins)) return set_error(ctx, VLR_ERR_INVALID, "null argument");
    if (ls->n_grids != 1) return set_error(ctx, VLR_ERR_UNSUPPORTED, "pool edits serve single-grid level sets only");
    int count = 0;
    int rc = list_count(ctx, ls, &count);
    if (rc) return rc;
    if (!d_pos && n > (size_t)count) return set_error(ctx, VLR_ERR_INVALID, "more leaves asked for than listed");
    if (n > (size_t)(1 << 30)) return set_error(ctx, VLR_ERR_INVALID, "too many positions");
    if (n == 0) return VLR_OK;
    const int B = ls->grid_blocks;
    if (d_pos) {
        k_check_pos<<<B, 256, 0, ctx->stream>>>(d_pos, (int)n, ls->scalars, ctx->d_errword);
        VLR_CUDA(ctx, cudaGetLastError());
        VLR_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
        rc = consume_device_errors(ctx, "vlr_ls_gather_device");
        if (rc) return rc;
    }
    if (ls->precision == VLR_PREC_F16)
        k_gather_pos<__half><<<B, 256, 0, ctx->stream>>>(ls->list, d_pos, (int)n, ls->origin, ls->mask,
                                                         (const __half*)ls->vals[0], d_origins, d_masks,
                                                         (__half*)d_phi);
    else
        k_gather_pos<float><<<B, 256, 0, ctx->stream>>>(ls->list, d_pos, (int)n, ls->origin, ls->mask,
                                                        (const float*)ls->vals[0], d_origins, d_masks,
                                                        (float*)d_phi);
    VLR_CUDA(ctx, cudaGetLastError());
    VLR_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    return VLR_OK;
}

int vlr_ls_edit_device(vlr_ctx* ctx, vlr_level_set* ls, const uint8_t* d_drop, size_t n_list,
                       const int32_t* d_origins, const uint64_t* d_masks, const void* d_phi, size_t n_add) {
    if (!ctx || !ls) return set_error(ctx, VLR_ERR_INVALID, "null argument");
    if (n_add && (!d_origins || !d_masks || !d_phi)) return set_error(ctx, VLR_ERR_INVALID, "null leaf arrays");
    if (ls->n_grids != 1) return set_error(ctx, VLR_ERR_UNSUPPORTED, "pool edits serve single-grid level sets only");
    if (ls->state_lost)
        return set_error(ctx, VLR_ERR_INVALID, "the level set's state is undefined after a failed step: upload first");
    int count = 0;
    int rc = list_count(ctx, ls, &count);
    if (rc) return rc;
    if (n_list != (size_t)count)
        return set_error(ctx, VLR_ERR_INVALID, "drop flags must cover exactly the listed leaves");
    if (n_list && !d_drop) return set_error(ctx, VLR_ERR_INVALID, "null drop flags");
    if (n_add > (size_t)ls->cap) return set_error(ctx, VLR_ERR_CAPACITY, "more leaves than the level set's capacity");
    const int n = (int)n_list;
    const int B = ls->grid_blocks;
    cudaStream_t st = ctx->stream;
    // keep flags (cap ints) and their scan with its total (cap + 1 ints) live
    // in per-step scratch of the pool that carries nothing between steps
    int* keep = ls->keep;
    int* kpos = ls->owned;
    if (n) {
        k_edit_flags<<<B, 256, 0, st>>>(d_drop, n, keep);
        VLR_CUDA(ctx, cudaGetLastError());
    }
    rc = scan_exclusive(ctx, keep, kpos, n, kpos + n);
    if (rc) return rc;
    // room for the added leaves, checked before anything changes
    int kept = 0, top = 0;
    rc = read_int(ctx, kpos + n, &kept);
    if (!rc) rc = read_int(ctx, ls->scalars + 2, &top);
    if (rc) return rc;
    if ((size_t)kept + n_add > (size_t)ls->cap || n_add > (size_t)top + (size_t)(n - kept))
        return set_error(ctx, VLR_ERR_CAPACITY, "the pool has no room for the added leaves");
    if (n) {
        k_edit_compact<<<B, 256, 0, st>>>(ls->list, keep, kpos, n, ls->list_new, ls->free_stack, ls->scalars);
        VLR_CUDA(ctx, cudaGetLastError());
    }
    if (ls->precision == VLR_PREC_F16)
        k_edit_append<__half><<<B, 256, 0, st>>>(ls->list_new, kpos, n, d_origins, d_masks, (const __half*)d_phi,
                                                 (int)n_add, ls->list, ls->free_stack, ls->origin, ls->mask,
                                                 (__half*)ls->vals[0], ls->scalars, ls->cap, ctx->d_errword);
    else
        k_edit_append<float><<<B, 256, 0, st>>>(ls->list_new, kpos, n, d_origins, d_masks, (const float*)d_phi,
                                                (int)n_add, ls->list, ls->free_stack, ls->origin, ls->mask,
                                                (float*)ls->vals[0], ls->scalars, ls->cap, ctx->d_errword);
    k_edit_finish<<<1, 32, 0, st>>>(kpos, n, (int)n_add, ls->scalars, ls->cap);
    VLR_CUDA(ctx, cudaGetLastError());
    rc = ls_enqueue_index(ctx, ls);
    if (rc) return rc;
    VLR_CUDA(ctx, cudaStreamSynchronize(st));
    rc = consume_device_errors(ctx, "vlr_ls_edit_device");
    // a device error (an added origin off the lattice or outside the hashable
    // range, a repeated leaf) leaves the pool undefined until the next upload
    if (rc) ls->state_lost = true;
    return rc;
}

}  // extern "C"
