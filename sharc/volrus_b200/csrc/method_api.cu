// Host side of the narrow-band method: creation (device sphere generator or
// uploaded leaves), per-grid velocity tables, graph-captured steps,
// download and the FP64 volume.  C entry points vlr_ls_* (include/volrus_b200.h).
#include <algorithm>
#include <climits>
#include <cmath>
#include <cstring>
#include <numeric>
#include <vector>

#include "method_state.hpp"
#include "sort_reduce.hpp"

namespace vlr {

size_t scan_scratch_ints(int n);

static int next_pow2i(long long v) {
    int p = 64;
    while ((long long)p < v && p < (1 << 30)) p <<= 1;
    return p;
}

void ls_free(vlr_level_set* ls) {
    for (cudaEvent_t& e : ls->slab_ev) {
        if (e) cudaEventDestroy(e);
        e = nullptr;
    }
    for (cudaStream_t& s : ls->slab_stream) {
        if (s) cudaStreamDestroy(s);
        s = nullptr;
    }
    if (ls->graph_exec) cudaGraphExecDestroy(ls->graph_exec);
    if (ls->graph) cudaGraphDestroy(ls->graph);
    ls->graph_exec = nullptr;
    ls->graph = nullptr;
    void* ptrs[] = {ls->origin, ls->mask, ls->dmask, ls->vals[0], ls->vals[1], ls->nbr, ls->spill, ls->nonempty,
                    ls->keep, ls->list, ls->list_new, ls->owned, ls->pos, ls->free_stack, ls->scalars, ls->hkey,
                    ls->hval, ls->pkey, ls->pval, ls->d_params, ls->d_tab, ls->d_partial, ls->d_sum,
                    ls->newinfo};
    for (void* p : ptrs) cudaFree(p);
    ls->newinfo = nullptr;
    cudaFree(ls->staging);
    ls->staging = nullptr;
    ls->staging_bytes = 0;
    ls->origin = nullptr;
    ls->mask = ls->dmask = nullptr;
    ls->vals[0] = ls->vals[1] = nullptr;
    ls->nbr = ls->nonempty = ls->keep = ls->list = ls->list_new = ls->owned = ls->pos = ls->free_stack = nullptr;
    ls->spill = nullptr;
    ls->scalars = nullptr;
    ls->hkey = ls->pkey = nullptr;
    ls->hval = ls->pval = nullptr;
    ls->d_params = nullptr;
    ls->d_tab = nullptr;
    ls->d_partial = ls->d_sum = nullptr;
}

int ls_alloc(vlr_ctx* ctx, vlr_level_set* ls, int cap) {
    ls->cap = cap;
    size_t vb = (ls->precision == VLR_PREC_F16) ? 2 : 4;
    ls->hcap = next_pow2i(2ll * cap);
    {
        // refuse up front what cannot fit, rather than filling the device first
        const size_t c = (size_t)cap, h = (size_t)ls->hcap;
        const size_t need = c * (16 + 64 + 64 + 2 * vb * kLeafVoxels + 4 * kNbr + 4 * 9 + 8) +
                            4 * scan_scratch_ints(cap) + h * 24 + 256;
        size_t free_b = 0, total_b = 0;
        if (cudaMemGetInfo(&free_b, &total_b) == cudaSuccess && need > free_b)
            return set_error(ctx, VLR_ERR_NOMEM,
                             "level set of " + std::to_string(cap) + " slots needs " + std::to_string(need >> 20) +
                                 " MiB, more than the device's free " + std::to_string(free_b >> 20) + " MiB");
    }
    VLR_CUDA(ctx, cudaMalloc(&ls->origin, sizeof(int4) * cap));
    VLR_CUDA(ctx, cudaMalloc(&ls->mask, 64ull * cap));
    VLR_CUDA(ctx, cudaMalloc(&ls->dmask, 64ull * cap));
    VLR_CUDA(ctx, cudaMalloc(&ls->vals[0], vb * kLeafVoxels * cap));
    VLR_CUDA(ctx, cudaMalloc(&ls->vals[1], vb * kLeafVoxels * cap));
    VLR_CUDA(ctx, cudaMalloc(&ls->nbr, sizeof(int) * kNbr * (size_t)cap));
    VLR_CUDA(ctx, cudaMalloc(&ls->spill, sizeof(unsigned) * cap));
    VLR_CUDA(ctx, cudaMalloc(&ls->nonempty, sizeof(int) * cap));
    VLR_CUDA(ctx, cudaMalloc(&ls->keep, sizeof(int) * cap));
    VLR_CUDA(ctx, cudaMalloc(&ls->list, sizeof(int) * cap));
    VLR_CUDA(ctx, cudaMalloc(&ls->list_new, sizeof(int) * cap));
    VLR_CUDA(ctx, cudaMalloc(&ls->owned, sizeof(int) * (cap + 1)));
    VLR_CUDA(ctx, cudaMalloc(&ls->pos, sizeof(int) * (cap + 1 + scan_scratch_ints(cap))));
    VLR_CUDA(ctx, cudaMemsetAsync(ls->pos, 0, sizeof(int) * (cap + 1 + scan_scratch_ints(cap)), ctx->stream));
    VLR_CUDA(ctx, cudaMalloc(&ls->newinfo, sizeof(int) * cap));
    VLR_CUDA(ctx, cudaMemsetAsync(ls->newinfo, 0xff, sizeof(int) * cap, ctx->stream));  // -1: no new leaf
    VLR_CUDA(ctx, cudaMalloc(&ls->free_stack, sizeof(int) * cap));
    VLR_CUDA(ctx, cudaMalloc(&ls->scalars, sizeof(int) * 8));
    VLR_CUDA(ctx, cudaMalloc(&ls->hkey, sizeof(uint64_t) * ls->hcap));
    VLR_CUDA(ctx, cudaMalloc(&ls->hval, sizeof(int) * ls->hcap));
    VLR_CUDA(ctx, cudaMalloc(&ls->pkey, sizeof(uint64_t) * ls->hcap));
    VLR_CUDA(ctx, cudaMalloc(&ls->pval, sizeof(int) * ls->hcap));
    VLR_CUDA(ctx, cudaMalloc(&ls->d_partial, sizeof(double) * cap));
    VLR_CUDA(ctx, cudaMalloc(&ls->d_sum, sizeof(double) * 2));
    VLR_CUDA(ctx, cudaMemsetAsync(ls->scalars, 0, sizeof(int) * 8, ctx->stream));
    VLR_CUDA(ctx, cudaMemsetAsync(ls->spill, 0, sizeof(unsigned) * cap, ctx->stream));
    VLR_CUDA(ctx, cudaMemsetAsync(ls->nonempty, 0, sizeof(int) * cap, ctx->stream));
    // list entries past a failed allocation must still name valid slots
    VLR_CUDA(ctx, cudaMemsetAsync(ls->list_new, 0, sizeof(int) * cap, ctx->stream));
    VLR_CUDA(ctx, cudaMemsetAsync(ls->list, 0, sizeof(int) * cap, ctx->stream));
    ls->grid_blocks = ctx->sm_count * 4;  // stencil kernels keep 4 CTAs of 256 threads per SM
    return VLR_OK;
}

// Largest displacement per step along one axis (voxels) for the field.
static double speed_bound(const vlr_velocity_desc* v) {
    if (v->kind == VLR_VEL_CONSTANT)
        return std::max({std::fabs(v->constant[0]), std::fabs(v->constant[1]), std::fabs(v->constant[2])});
    if (v->kind == VLR_VEL_VORTEX) return 2.0 / v->voxel_size;
    double b = 0.0;
    for (int o = 0; o < v->octaves; ++o) b += 2.0 * std::fabs(v->amp[o] * v->wavenumber[o]);
    return b;
}

// Per-grid parameters and sin/cos tables (computed in f64, stored as f32 pairs).
static int grid_params(vlr_ctx* ctx, const vlr_method_desc* m, const vlr_velocity_desc* v, const int32_t bb_lo[3],
                       const int32_t bb_hi[3], int key_bits, MGridParams& P, std::vector<float2>& tab) {
    std::memset(&P, 0, sizeof(P));
    P.hw = m->half_width;
    P.vel_kind = v->kind;
    int32_t lo[3], hi[3];
    for (int a = 0; a < 3; ++a) {
        if (v->domain_lo[a] <= v->domain_hi[a]) {
            lo[a] = v->domain_lo[a];
            hi[a] = v->domain_hi[a];
        } else if (v->kind == VLR_VEL_VORTEX && v->voxel_size > 0.0) {
            // the deformation field lives on the unit cube: index box of [0, 1] + 16 voxels
            lo[a] = (int32_t)std::floor(-v->w0[a] / v->voxel_size) - 16;
            hi[a] = (int32_t)std::ceil((1.0 - v->w0[a]) / v->voxel_size) + 16;
        } else {
            lo[a] = bb_lo[a] - 256;
            hi[a] = bb_hi[a] + 256;
        }
        long long centre = ((long long)(bb_lo[a] >> 3) + (long long)(bb_hi[a] >> 3)) / 2;
        P.base[a] = centre - (1ll << (key_bits - 1));
    }
    const double pi = 3.14159265358979323846;
    auto add_family = [&](int f, double dphi, const double ph[3], const double scale[3], const double offs[3]) {
        P.dphi[f] = (float)dphi;
        for (int a = 0; a < 3; ++a) {
            P.tab_off[f][a] = (int)tab.size();
            for (int32_t i = lo[a]; i <= hi[a]; ++i) {
                double ang = scale[a] * (offs[a] + dphi / scale[a] * i) + ph[a];
                tab.push_back(make_float2((float)std::sin(ang), (float)std::cos(ang)));
            }
        }
    };
    for (int a = 0; a < 3; ++a) {
        P.tab_lo[a] = lo[a];
        P.tab_len[a] = hi[a] - lo[a] + 1;
        if (P.tab_len[a] <= 0 || P.tab_len[a] > (1 << 25))
            return set_error(ctx, VLR_ERR_INVALID, "velocity domain box empty or too large");
    }
    if (v->kind == VLR_VEL_CONSTANT) {
        for (int a = 0; a < 3; ++a) P.c[a] = (float)v->constant[a];
        for (int a = 0; a < 3; ++a) P.tab_len[a] = 0;
    } else if (v->kind == VLR_VEL_VORTEX) {
        if (!(v->voxel_size > 0.0) || !(v->period != 0.0))
            return set_error(ctx, VLR_ERR_INVALID, "vortex needs voxel_size > 0 and period != 0");
        P.vel_scale = (float)(1.0 / v->voxel_size);
        P.pi_over_T = (float)(pi / v->period);
        // angle(i) = pi * (w0 + vs * i)
        double ph[3] = {0, 0, 0}, sc[3] = {pi, pi, pi}, of[3] = {v->w0[0], v->w0[1], v->w0[2]};
        add_family(0, pi * v->voxel_size, ph, sc, of);
    } else if (v->kind == VLR_VEL_CURL) {
        if (v->octaves < 1 || v->octaves > kMaxOctaves) return set_error(ctx, VLR_ERR_INVALID, "curl octaves 1..4");
        P.octaves = v->octaves;
        for (int o = 0; o < v->octaves; ++o) {
            P.ak[o] = (float)(v->amp[o] * v->wavenumber[o]);
            for (int a = 0; a < 3; ++a) P.e[o][a] = (float)v->dir[o][a];
            // angle(i) = k * i + phase
            double sc[3] = {1, 1, 1}, of[3] = {0, 0, 0};
            add_family(o, v->wavenumber[o], v->phase[o], sc, of);
        }
    } else {
        return set_error(ctx, VLR_ERR_INVALID, "unknown velocity kind");
    }
    return VLR_OK;
}

// Per-grid parameters and tables for n grids (bounding boxes in index units);
// all grids of a level set share dt, integrator, reinitialisation and halo.
int ls_setup_grids(vlr_ctx* ctx, vlr_level_set* ls, const vlr_method_desc* m, const vlr_velocity_desc* const* vels,
                   const int32_t (*bb_lo)[3], const int32_t (*bb_hi)[3], int n) {
    if (m->integrator < 1 || m->integrator > 3) return set_error(ctx, VLR_ERR_INVALID, "integrator must be 1, 2 or 3");
    if (m->reinit_iters < 0 || m->reinit_iters > 2)
        return set_error(ctx, VLR_ERR_UNSUPPORTED, "reinit_iters must be 0, 1 or 2");
    if (!(m->half_width > 0.0f) || m->half_width > 7.0f)
        return set_error(ctx, VLR_ERR_INVALID, "half_width must be in (0, 7] voxels");
    if (!(m->dt > 0.0)) return set_error(ctx, VLR_ERR_INVALID, "dt must be positive");
    double disp = 0.0;
    for (int g = 0; g < n; ++g) disp = std::max(disp, speed_bound(vels[g]) * m->dt);
    if (disp <= 1.0) ls->halo = 2;
    else if (disp <= 2.0) ls->halo = 3;
    else return set_error(ctx, VLR_ERR_REACH, "velocity * dt exceeds 2 voxels per step (CFL); reduce dt");
    ls->reinit_iters = m->reinit_iters;
    ls->n_grids = n;
    ls->vel_kind = n > 0 ? vels[0]->kind : -1;
    for (int g = 1; g < n; ++g)
        if (vels[g]->kind != ls->vel_kind) ls->vel_kind = -1;
    ls->sp.dt = (float)m->dt;
    ls->sp.t0 = (float)m->t0;
    ls->sp.integrator = m->integrator;
    ls->sp.n_grids = n;
    ls->sp.key_bits = ls->key_bits;
    if (m->reinit_mode != 0 && m->reinit_mode != 1)
        return set_error(ctx, VLR_ERR_INVALID, "reinit_mode must be 0 (plain Godunov) or 1 (subcell fix)");
    ls->sp.reinit_mode = m->reinit_mode;
    std::vector<float2> tab;
    ls->h_params.resize(n);
    for (int g = 0; g < n; ++g) {
        MGridParams& P = ls->h_params[g];
        int rc = grid_params(ctx, m, vels[g], bb_lo[g], bb_hi[g], ls->key_bits, P, tab);
        if (rc) return rc;
        // curl octaves whose table angles double from one octave to the next
        // rotate by double-angle formulas from octave 0's series
        P.doubling = (P.vel_kind == MVEL_CURL && P.octaves >= 2) ? 1 : 0;
        for (int o = 1; o < P.octaves && P.doubling; ++o)
            if (P.dphi[o] != 2.0f * P.dphi[o - 1]) P.doubling = 0;
        // rotation angles stay below dphi * disp; the shortest series exact to
        // well below f32 resolution at that angle is used
        double max_angle = 0.0, gdisp = speed_bound(vels[g]) * m->dt;
        for (int f = 0; f < (P.doubling ? 1 : kMaxOctaves); ++f)
            max_angle = std::max(max_angle, std::fabs((double)P.dphi[f]) * gdisp);
        P.series = max_angle < 0.004 ? 0 : (max_angle < 0.05 ? 1 : 2);
    }
    VLR_CUDA(ctx, cudaMalloc(&ls->d_params, sizeof(MGridParams) * n));
    VLR_CUDA(ctx, cudaMemcpy(ls->d_params, ls->h_params.data(), sizeof(MGridParams) * n, cudaMemcpyHostToDevice));
    size_t nt = std::max<size_t>(tab.size(), 1);
    VLR_CUDA(ctx, cudaMalloc(&ls->d_tab, sizeof(float2) * nt));
    if (!tab.empty())
        VLR_CUDA(ctx, cudaMemcpy(ls->d_tab, tab.data(), sizeof(float2) * tab.size(), cudaMemcpyHostToDevice));
    return VLR_OK;
}

static int setup_common(vlr_ctx* ctx, vlr_level_set* ls, const vlr_method_desc* m, const vlr_velocity_desc* v,
                        const int32_t bb_lo[3], const int32_t bb_hi[3]) {
    const vlr_velocity_desc* vs[1] = {v};
    int32_t lo[1][3] = {{bb_lo[0], bb_lo[1], bb_lo[2]}}, hi[1][3] = {{bb_hi[0], bb_hi[1], bb_hi[2]}};
    return ls_setup_grids(ctx, ls, m, vs, lo, hi, 1);
}

__global__ void k_iota(int* a, int n) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) a[i] = i;
}

// free stack = slots [n, cap) (pops take the lowest slots first), list = 0..n-1,
// count = n; `step` keeps its value unless reset.
__global__ void k_init_lists(int* list, int* free_stack, int* scalars, int n, int cap, int reset_step) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < cap; i += gridDim.x * blockDim.x) {
        if (i < n) list[i] = i;
        if (i < cap - n) free_stack[i] = cap - 1 - i;
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        scalars[0] = n;
        if (reset_step) scalars[1] = 0;
        scalars[2] = cap - n;
        for (int q = 3; q < 8; ++q) scalars[q] = 0;
    }
}

int ls_init_lists(vlr_ctx* ctx, vlr_level_set* ls, int n, bool reset_step) {
    k_init_lists<<<ls->grid_blocks, 256, 0, ctx->stream>>>(ls->list, ls->free_stack, ls->scalars, n, ls->cap,
                                                           reset_step ? 1 : 0);
    VLR_CUDA(ctx, cudaGetLastError());
    int rc = ls_enqueue_index(ctx, ls);
    if (rc) return rc;
    VLR_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    rc = consume_device_errors(ctx, "method grid index");
    if (rc == VLR_OK) ls->state_lost = false;  // a complete new state
    return rc;
}

// Staging buffer of at least `bytes` owned by the level set.
static int ls_staging(vlr_ctx* ctx, vlr_level_set* ls, size_t bytes, void** out) {
    if (bytes > ls->staging_bytes) {
        cudaStreamSynchronize(ctx->stream);
        cudaFree(ls->staging);
        ls->staging = nullptr;
        ls->staging_bytes = 0;
        VLR_CUDA(ctx, cudaMalloc(&ls->staging, bytes));
        ls->staging_bytes = bytes;
    }
    *out = ls->staging;
    return VLR_OK;
}

template <typename T>
__global__ void k_pick(const int* flags, const int* pos, int n, const int4* o_in, const uint64_t* m_in,
                       const T* v_in, int4* o_out, uint64_t* m_out, T* v_out) {
    for (int i = blockIdx.x; i < n; i += gridDim.x) {
        if (!flags[i]) continue;
        int j = pos[i];
        if (threadIdx.x == 0) o_out[j] = o_in[i];
        if (threadIdx.x < 8) m_out[(size_t)j * 8 + threadIdx.x] = m_in[(size_t)i * 8 + threadIdx.x];
        for (int t = threadIdx.x; t < kLeafVoxels; t += blockDim.x)
            v_out[(size_t)j * kLeafVoxels + t] = v_in[(size_t)i * kLeafVoxels + t];
    }
}

template <typename T>
__global__ void k_from_f32(const float* in, T* out, size_t n) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
        out[i] = from_f<T>(in[i]);
}

__global__ void k_gather_origins(const int* list, int n, const int4* origin, int4* o_out) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) o_out[i] = origin[list[i]];
}

// Masks and f32 values of the leaves at list positions sel[0..k) in that
// order (output order), one CTA per leaf.
template <typename T>
__global__ void k_gather_sel(const int* list, const int* sel, int k, const uint64_t* mask, const T* vals,
                             uint64_t* m_out, float* v_out) {
    for (int i = blockIdx.x; i < k; i += gridDim.x) {
        const int s = list[sel[i]];
        if (threadIdx.x < 8) m_out[(size_t)i * 8 + threadIdx.x] = mask[(size_t)s * 8 + threadIdx.x];
        for (int t = threadIdx.x; t < kLeafVoxels; t += blockDim.x)
            v_out[(size_t)i * kLeafVoxels + t] = to_f(vals[(size_t)s * kLeafVoxels + t]);
    }
}

// Output order of a host step without a host round trip: for up to
// kDevSortLeaves listed leaves of a single grid, their (x, y, z) keys (leaf
// coordinates relative to the grid's hash base, bits each, so key order is
// the lexicographic order of the origins) are ranked on the device: a leaf's
// rank is the number of smaller keys (the keys are distinct: origins are
// unique), counted by kRankLanes lanes per leaf across the whole GPU, and the
// leaf's list position and origin are written at its rank.  More leaves:
// *status = 0 and the host sorts instead.
constexpr int kDevSortLeaves = 8192;
constexpr int kRankLanes = 16;

__global__ void k_rank_keys(const int* __restrict__ list, const int* __restrict__ count,
                            const int4* __restrict__ origin, long long b0, long long b1, long long b2, int bits,
                            unsigned long long* __restrict__ keys, int* __restrict__ status) {
    const int n = *count;
    if (blockIdx.x == 0 && threadIdx.x == 0) *status = (n <= kDevSortLeaves) ? 1 : 0;
    if (n > kDevSortLeaves) return;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const int4 o = origin[list[i]];
        keys[i] = ((unsigned long long)((o.x >> 3) - b0) << (2 * bits)) |
                  ((unsigned long long)((o.y >> 3) - b1) << bits) | (unsigned long long)((o.z >> 3) - b2);
    }
}

__global__ void __launch_bounds__(256) k_rank_scatter(const int* __restrict__ list, const int* __restrict__ count,
                                                      const int4* __restrict__ origin,
                                                      const unsigned long long* __restrict__ keys,
                                                      int* __restrict__ sel, int32_t* __restrict__ o3) {
    const int n = *count;
    if (n > kDevSortLeaves) return;
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if ((t & ~31) / kRankLanes >= n) return;  // whole warps past the last leaf
    const int i = t / kRankLanes, s = t % kRankLanes;
    const unsigned long long ki = i < n ? keys[i] : 0ull;
    int less = 0;
#pragma unroll 4
    for (int j = s; j < n; j += kRankLanes) less += (__ldg(&keys[j]) < ki) ? 1 : 0;
#pragma unroll
    for (int d = 1; d < kRankLanes; d <<= 1) less += __shfl_xor_sync(0xffffffffu, less, d);
    if (s == 0 && i < n) {
        sel[less] = i;
        const int4 o = origin[list[i]];
        o3[3 * less] = o.x;
        o3[3 * less + 1] = o.y;
        o3[3 * less + 2] = o.z;
    }
}

// k_gather_sel with the count and the sort status read on the device.
template <typename T>
__global__ void k_gather_sel_dev(const int* list, const int* sel, const int* count, const int* status,
                                 const uint64_t* mask, const T* vals, uint64_t* m_out, float* v_out) {
    if (!*status) return;
    const int k = *count;
    for (int i = blockIdx.x; i < k; i += gridDim.x) {
        const int s = list[sel[i]];
        if (threadIdx.x < 8) m_out[(size_t)i * 8 + threadIdx.x] = mask[(size_t)s * 8 + threadIdx.x];
        for (int t = threadIdx.x; t < kLeafVoxels; t += blockDim.x)
            v_out[(size_t)i * kLeafVoxels + t] = to_f(vals[(size_t)s * kLeafVoxels + t]);
    }
}

__global__ void k_count_active(const int* list, const int* count_ptr, const uint64_t* mask,
                               unsigned long long* out) {
    int n = *count_ptr;
    unsigned long long c = 0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n * 8; i += gridDim.x * blockDim.x)
        c += __popcll(mask[(size_t)list[i >> 3] * 8 + (i & 7)]);
    for (int o = 16; o > 0; o >>= 1) c += __shfl_down_sync(0xffffffffu, c, o);
    if ((threadIdx.x & 31) == 0 && c) atomicAdd(out, c);
}

}  // namespace vlr

using namespace vlr;

namespace {

int create_sphere_impl(vlr_ctx* ctx, vlr_level_set* ls, const vlr_method_desc* m, const vlr_velocity_desc* vel,
                       double radius, const double c[3], double vs, const double w0[3]) {
    double hw = (double)m->half_width;
    int32_t lo[3], hi[3];
    for (int a = 0; a < 3; ++a) {
        double ci = (c[a] - w0[a]) / vs, ri = radius / vs;
        lo[a] = (int32_t)std::floor(ci - ri - hw - 2.0);
        hi[a] = (int32_t)std::ceil(ci + ri + hw + 2.0);
    }
    long long nl[3];
    for (int a = 0; a < 3; ++a) nl[a] = (long long)(hi[a] >> 3) - (lo[a] >> 3) + 1;
    long long n_cand = nl[0] * nl[1] * nl[2];
    if (n_cand > (1ll << 26)) return set_error(ctx, VLR_ERR_CAPACITY, "sphere bounding box too large");
    int rc = setup_common(ctx, ls, m, vel, lo, hi);
    if (rc) return rc;
    size_t vb = (ls->precision == VLR_PREC_F16) ? 2 : 4;
    int4* o_tmp = nullptr;
    uint64_t* m_tmp = nullptr;
    void* v_tmp = nullptr;
    int* touched = nullptr;
    int* pos = nullptr;
    DeviceTemps temps;  // freed on every return
    VLR_CUDA(ctx, cudaMalloc(&o_tmp, sizeof(int4) * n_cand));
    temps.track(o_tmp);
    VLR_CUDA(ctx, cudaMalloc(&m_tmp, 64ull * n_cand));
    temps.track(m_tmp);
    VLR_CUDA(ctx, cudaMalloc(&v_tmp, vb * kLeafVoxels * n_cand));
    temps.track(v_tmp);
    VLR_CUDA(ctx, cudaMalloc(&touched, sizeof(int) * (n_cand + 1)));
    temps.track(touched);
    VLR_CUDA(ctx, cudaMalloc(&pos, sizeof(int) * (n_cand + 1)));
    temps.track(pos);
    int blocks = std::min<long long>(n_cand, (long long)ctx->sm_count * 16);
    if (ls->precision == VLR_PREC_F16)
        k_m_sphere<__half><<<blocks, 256, 0, ctx->stream>>>(lo[0] >> 3, lo[1] >> 3, lo[2] >> 3, (int)nl[1], (int)nl[2],
                                                            (int)n_cand, radius, c[0], c[1], c[2], vs, w0[0], w0[1],
                                                            w0[2], hw, o_tmp, m_tmp, (__half*)v_tmp, touched);
    else
        k_m_sphere<float><<<blocks, 256, 0, ctx->stream>>>(lo[0] >> 3, lo[1] >> 3, lo[2] >> 3, (int)nl[1], (int)nl[2],
                                                           (int)n_cand, radius, c[0], c[1], c[2], vs, w0[0], w0[1],
                                                           w0[2], hw, o_tmp, m_tmp, (float*)v_tmp, touched);
    VLR_CUDA(ctx, cudaGetLastError());
    rc = scan_exclusive(ctx, touched, pos, (int)n_cand, pos + n_cand);
    if (rc) return rc;
    int n = 0;
    rc = read_int(ctx, pos + n_cand, &n);
    if (rc) return rc;
    int cap = m->capacity ? (int)std::min<size_t>(m->capacity, (size_t)1 << 30) : 2 * n + 4096;
    if (cap < n) return set_error(ctx, VLR_ERR_CAPACITY, "capacity below the initial leaf count");
    rc = ls_alloc(ctx, ls, cap);
    if (rc) return rc;
    if (ls->precision == VLR_PREC_F16)
        k_pick<__half><<<blocks, 256, 0, ctx->stream>>>(touched, pos, (int)n_cand, o_tmp, m_tmp, (const __half*)v_tmp,
                                                        ls->origin, ls->mask, (__half*)ls->vals[0]);
    else
        k_pick<float><<<blocks, 256, 0, ctx->stream>>>(touched, pos, (int)n_cand, o_tmp, m_tmp, (const float*)v_tmp,
                                                       ls->origin, ls->mask, (float*)ls->vals[0]);
    VLR_CUDA(ctx, cudaGetLastError());
    VLR_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    return ls_init_lists(ctx, ls, n, true);
}

// Replace the state with n host leaves (origins i32[3], masks, phi f32 voxel
// units), staged through one pinned-free device buffer.
__global__ void k_unpack_upload(const int32_t* o3, int n, int4* origin) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        origin[i] = make_int4(o3[3 * i], o3[3 * i + 1], o3[3 * i + 2], 0);
}

// Enqueue the replacement of a level set's state by host leaves (no wait).
int upload_enqueue(vlr_ctx* ctx, vlr_level_set* ls, const int32_t* origins, const uint64_t* masks, const float* phi,
                   size_t n, bool reset_step) {
    if (n > (size_t)ls->cap) return set_error(ctx, VLR_ERR_CAPACITY, "more leaves than the level set's capacity");
    for (size_t i = 0; i < 3 * n; ++i)
        if (origins[i] & 7) return set_error(ctx, VLR_ERR_INVALID, "leaf origin not a multiple of 8");
    size_t vbytes = sizeof(float) * kLeafVoxels * n;
    void* stg = nullptr;
    int rc = ls_staging(ctx, ls, vbytes + 12 * n + 16, &stg);
    if (rc) return rc;
    float* tmp = (float*)stg;
    int32_t* o3 = (int32_t*)((char*)stg + vbytes);
    VLR_CUDA(ctx, cudaMemcpyAsync(o3, origins, 12 * n, cudaMemcpyHostToDevice, ctx->stream));
    VLR_CUDA(ctx, cudaMemcpyAsync(ls->mask, masks, 64 * n, cudaMemcpyHostToDevice, ctx->stream));
    k_unpack_upload<<<ls->grid_blocks, 256, 0, ctx->stream>>>(o3, (int)n, ls->origin);
    if (ls->precision == VLR_PREC_F16) {
        VLR_CUDA(ctx, cudaMemcpyAsync(tmp, phi, vbytes, cudaMemcpyHostToDevice, ctx->stream));
        k_from_f32<__half><<<ls->grid_blocks, 256, 0, ctx->stream>>>(tmp, (__half*)ls->vals[0], kLeafVoxels * n);
    } else {
        VLR_CUDA(ctx, cudaMemcpyAsync(ls->vals[0], phi, vbytes, cudaMemcpyHostToDevice, ctx->stream));
    }
    VLR_CUDA(ctx, cudaGetLastError());
    k_init_lists<<<ls->grid_blocks, 256, 0, ctx->stream>>>(ls->list, ls->free_stack, ls->scalars, (int)n, ls->cap,
                                                           reset_step ? 1 : 0);
    VLR_CUDA(ctx, cudaGetLastError());
    rc = ls_enqueue_index(ctx, ls);
    if (rc == VLR_OK) ls->state_lost = false;  // a complete new state is on its way
    return rc;
}

// Device-resident leaves: origins i32[3] -> the pool's int4 origins (origins
// not on the 8-voxel lattice flag kErrInput), f32 values -> the pool's type.
__global__ void k_upload_dev_origins(const int32_t* o3, int n, int4* origin, unsigned* err) {
    unsigned bad = 0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const int x = o3[3 * i], y = o3[3 * i + 1], z = o3[3 * i + 2];
        bad |= (unsigned)((x | y | z) & 7);
        origin[i] = make_int4(x, y, z, 0);
    }
    if (bad) atomicOr(err, kErrInput);
}

// The listed leaves in list order into device buffers (origins i32[3], masks,
// f32 values), one CTA per leaf.
template <typename T>
__global__ void k_export_dev(const int* list, const int* count, const int4* origin, const uint64_t* mask,
                             const T* vals, int32_t* o3, uint64_t* m_out, float* v_out) {
    const int n = *count;
    for (int i = blockIdx.x; i < n; i += gridDim.x) {
        const int s = list[i];
        if (threadIdx.x < 3) {
            const int4 o = origin[s];
            o3[3 * i + threadIdx.x] = threadIdx.x == 0 ? o.x : (threadIdx.x == 1 ? o.y : o.z);
        }
        if (threadIdx.x < 8) m_out[(size_t)i * 8 + threadIdx.x] = mask[(size_t)s * 8 + threadIdx.x];
        for (int t = threadIdx.x; t < kLeafVoxels; t += blockDim.x)
            v_out[(size_t)i * kLeafVoxels + t] = to_f(vals[(size_t)s * kLeafVoxels + t]);
    }
}

int upload_impl(vlr_ctx* ctx, vlr_level_set* ls, const int32_t* origins, const uint64_t* masks, const float* phi,
                size_t n, bool reset_step) {
    int rc = upload_enqueue(ctx, ls, origins, masks, phi, n, reset_step);
    if (rc) return rc;
    VLR_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    return consume_device_errors(ctx, "method grid index");
}

int create_leaves_impl(vlr_ctx* ctx, vlr_level_set* ls, const vlr_method_desc* m, const vlr_velocity_desc* vel,
                       const int32_t* origins, const uint64_t* masks, const float* phi, size_t n) {
    if (n == 0) return set_error(ctx, VLR_ERR_INVALID, "no leaves");
    int32_t lo[3] = {INT32_MAX, INT32_MAX, INT32_MAX}, hi[3] = {INT32_MIN, INT32_MIN, INT32_MIN};
    for (size_t i = 0; i < n; ++i)
        for (int a = 0; a < 3; ++a) {
            if (origins[3 * i + a] & 7) return set_error(ctx, VLR_ERR_INVALID, "leaf origin not a multiple of 8");
            lo[a] = std::min(lo[a], origins[3 * i + a]);
            hi[a] = std::max(hi[a], origins[3 * i + a] + 7);
        }
    for (int a = 0; a < 3; ++a)
        if (((long long)hi[a] - lo[a]) >> 3 >= (1ll << (ls->key_bits - 1)) - 4)
            return set_error(ctx, VLR_ERR_EXTENT, "grid spans more than 2^24 voxels along an axis");
    int rc = setup_common(ctx, ls, m, vel, lo, hi);
    if (rc) return rc;
    int cap = m->capacity ? (int)std::min<size_t>(m->capacity, (size_t)1 << 30) : 2 * (int)n + 4096;
    if ((size_t)cap < n) return set_error(ctx, VLR_ERR_CAPACITY, "capacity below the leaf count");
    rc = ls_alloc(ctx, ls, cap);
    if (rc) return rc;
    return upload_impl(ctx, ls, origins, masks, phi, n, true);
}

int capture_step(vlr_ctx* ctx, vlr_level_set* ls) {
    if (ls->graph_exec) return VLR_OK;
    VLR_CUDA(ctx, cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal));
    int rc = ls_enqueue_step(ctx, ls);
    cudaGraph_t g = nullptr;
    cudaError_t e = cudaStreamEndCapture(ctx->stream, &g);
    if (rc) {
        if (g) cudaGraphDestroy(g);
        return rc;
    }
    if (e != cudaSuccess) return check_cuda(ctx, e, "cudaStreamEndCapture");
    ls->graph = g;
    VLR_CUDA(ctx, cudaGraphInstantiate(&ls->graph_exec, g, 0));
    return VLR_OK;
}

void drop_graph(vlr_level_set* ls) {
    if (ls->graph_exec) cudaGraphExecDestroy(ls->graph_exec);
    if (ls->graph) cudaGraphDestroy(ls->graph);
    ls->graph_exec = nullptr;
    ls->graph = nullptr;
}

// One step: the autotuning step first (launch shapes not chosen yet, run with
// the kernel timers paused), then graph replays (direct launches while the
// per-kernel timers are on).
int enqueue_one_step(vlr_ctx* ctx, vlr_level_set* ls) {
    if (ls->state_lost)
        return set_error(ctx, VLR_ERR_INVALID,
                         "the level set's state is undefined after a step failed with VLR_ERR_TIMEOUT or "
                         "VLR_ERR_CAPACITY: upload a state first");
    if (ls->autotune && !ls->tuned) {
        const bool timing = ctx->timer.enabled;
        ctx->timer.enabled = false;
        drop_graph(ls);
        int rc = ls_autotune_step(ctx, ls);
        ctx->timer.enabled = timing;
        return rc;
    }
    if (ctx->timer.enabled) return ls_enqueue_step(ctx, ls);
    int rc = capture_step(ctx, ls);
    if (rc) return rc;
    VLR_CUDA(ctx, cudaGraphLaunch(ls->graph_exec, ctx->stream));
    return VLR_OK;
}

// Leaves of one grid (grid < 0: all) of a level set holding n listed leaves,
// sorted by (grid, x, y, z), into host buffers.
// Leaf keys of list positions 0..n-1 of a single grid (leaf coordinates
// relative to the hash base, `bits` each: key order is the origins'
// lexicographic order), their low words and the identity permutation.
__global__ void k_leaf_keys(const int* __restrict__ list, int n, const int4* __restrict__ origin, long long b0,
                            long long b1, long long b2, int bits, unsigned long long* __restrict__ keys,
                            unsigned* __restrict__ lo, unsigned* __restrict__ idx) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const int4 o = origin[list[i]];
        const unsigned long long k = ((unsigned long long)((o.x >> 3) - b0) << (2 * bits)) |
                                     ((unsigned long long)((o.y >> 3) - b1) << bits) |
                                     (unsigned long long)((o.z >> 3) - b2);
        keys[i] = k;
        lo[i] = (unsigned)k;
        idx[i] = (unsigned)i;
    }
}

__global__ void k_leaf_keys_hi(const unsigned long long* __restrict__ keys, const unsigned* __restrict__ perm, int n,
                               unsigned* __restrict__ hi) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        hi[i] = (unsigned)(keys[perm[i]] >> 32);
}

// Origins (i32[3]) of the list positions perm[0..n) in that order.
__global__ void k_sorted_origins(const int* __restrict__ list, const unsigned* __restrict__ perm, int n,
                                 const int4* __restrict__ origin, int32_t* __restrict__ o3) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const int4 o = origin[list[perm[i]]];
        o3[3 * i] = o.x;
        o3[3 * i + 1] = o.y;
        o3[3 * i + 2] = o.z;
    }
}

// The sorted download of all leaves of a single grid with the order made on
// the device: 64-bit leaf keys sorted by two stable 32-bit radix passes (low
// word, then high word), then origins, masks and f32 values gathered in that
// order and copied once into the caller's buffers.
int download_sorted_device(vlr_ctx* ctx, const vlr_level_set* ls, size_t n, int32_t* origins, uint64_t* masks,
                           float* phi) {
    cudaStream_t st = ctx->stream;
    const int nn = (int)n;
    const size_t sort_bytes = sort_reduce_scratch_bytes(nn);
    const size_t vbytes = sizeof(float) * kLeafVoxels * n;
    char* buf = nullptr;
    VLR_CUDA(ctx, cudaMallocFromPoolAsync((void**)&buf, vbytes + n * (8 + 4 * 3 + 12 + 64) + sort_bytes + 512,
                                          ctx->pool, st));
    auto done = [&](int code) {
        cudaFreeAsync(buf, st);
        return code;
    };
    char* q = buf;
    float* v = (float*)q;  q += vbytes;
    unsigned long long* keys = (unsigned long long*)q;  q += n * 8;
    uint64_t* mm = (uint64_t*)q;  q += n * 64;
    unsigned* lo = (unsigned*)q;  q += n * 4;
    unsigned* idx = (unsigned*)q;  q += n * 4;
    unsigned* hi = (unsigned*)q;  q += n * 4;
    int32_t* o3 = (int32_t*)q;  q += n * 12;
    void* scratch = (void*)(((uintptr_t)q + 255) & ~(uintptr_t)255);
    const vlr::MGridParams& P = ls->h_params[0];
    const int B = ctx->sm_count * 8;
    k_leaf_keys<<<B, 256, 0, st>>>(ls->list, nn, ls->origin, P.base[0], P.base[1], P.base[2], ls->key_bits, keys, lo,
                                   idx);
    unsigned *k1, *v1, *k2, *v2;
    int rc = radix_sort_pairs(ctx, lo, idx, nn, 0xffffffffu, scratch, &k1, &v1);
    if (rc) return done(rc);
    k_leaf_keys_hi<<<B, 256, 0, st>>>(keys, v1, nn, hi);
    if (v1 != idx) VLR_CUDA(ctx, cudaMemcpyAsync(idx, v1, n * 4, cudaMemcpyDeviceToDevice, st));
    rc = radix_sort_pairs(ctx, hi, idx, nn, 0x7fffffffu, scratch, &k2, &v2);
    if (rc) return done(rc);
    (void)k1;
    (void)k2;
    const int* sel = (const int*)v2;
    if (origins) k_sorted_origins<<<B, 256, 0, st>>>(ls->list, v2, nn, ls->origin, o3);
    if (masks || phi) {
        const int G = (int)std::min<size_t>(n, (size_t)ctx->sm_count * 8);
        if (ls->precision == VLR_PREC_F16)
            k_gather_sel<__half><<<G, 256, 0, st>>>(ls->list, sel, nn, ls->mask, (const __half*)ls->vals[0], mm, v);
        else
            k_gather_sel<float><<<G, 256, 0, st>>>(ls->list, sel, nn, ls->mask, (const float*)ls->vals[0], mm, v);
    }
    VLR_CUDA(ctx, cudaGetLastError());
    if (origins && (rc = d2h_copy(ctx, origins, o3, n * 12))) return done(rc);
    if (masks && (rc = d2h_copy(ctx, masks, mm, n * 64))) return done(rc);
    if (phi && (rc = d2h_copy(ctx, phi, v, vbytes))) return done(rc);
    VLR_CUDA(ctx, cudaStreamSynchronize(st));
    return done(VLR_OK);
}

int download_n(vlr_ctx* ctx, const vlr_level_set* ls, size_t n, int grid, int32_t* grid_ids, int32_t* origins,
               uint64_t* masks, float* phi, size_t cap_leaves, size_t* n_out) {
    int rc = VLR_OK;
    *n_out = 0;
    if (grid < 0 && n > cap_leaves) return set_error(ctx, VLR_ERR_CAPACITY, "output buffers too small");
    if (!n) return VLR_OK;
    if (grid < 0 && !grid_ids && ls->n_grids == 1 && 3 * ls->key_bits <= 63 && n <= (size_t)INT_MAX / 16) {
        rc = download_sorted_device(ctx, ls, n, origins, masks, phi);
        if (rc == VLR_OK) *n_out = n;
        return rc;
    }
    // origins in list order -> host, output order sorted by (grid, x, y, z)
    // there; masks and values are then gathered on the device in that order
    // and copied once, straight into the caller's buffers
    void* stg = nullptr;
    size_t vbytes = sizeof(float) * kLeafVoxels * n;
    rc = ls_staging(ctx, const_cast<vlr_level_set*>(ls), vbytes + 84 * n + 256, &stg);
    if (rc) return rc;
    float* v = (float*)stg;
    int4* o = (int4*)((char*)stg + vbytes);
    uint64_t* mm = (uint64_t*)((char*)stg + vbytes + 16 * n);
    int* dsel = (int*)((char*)stg + vbytes + 80 * n);
    k_gather_origins<<<ls->grid_blocks, 256, 0, ctx->stream>>>(ls->list, (int)n, ls->origin, o);
    std::vector<int4> ho(n);
    VLR_CUDA(ctx, cudaMemcpyAsync(ho.data(), o, sizeof(int4) * n, cudaMemcpyDeviceToHost, ctx->stream));
    VLR_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    std::vector<int> order(n);
    std::iota(order.begin(), order.end(), 0);
    std::sort(order.begin(), order.end(), [&](int a, int b) {
        const int4 &A = ho[a], &B2 = ho[b];
        if (A.w != B2.w) return A.w < B2.w;
        if (A.x != B2.x) return A.x < B2.x;
        if (A.y != B2.y) return A.y < B2.y;
        return A.z < B2.z;
    });
    std::vector<int> sel;
    sel.reserve(n);
    for (size_t i = 0; i < n; ++i)
        if (grid < 0 || ho[order[i]].w == grid) sel.push_back(order[i]);
    const size_t k = sel.size();
    if (k > cap_leaves) return set_error(ctx, VLR_ERR_CAPACITY, "output buffers too small");
    for (size_t i = 0; i < k; ++i) {
        const int4 q = ho[sel[i]];
        if (grid_ids) grid_ids[i] = q.w;
        if (origins) {
            origins[3 * i] = q.x;
            origins[3 * i + 1] = q.y;
            origins[3 * i + 2] = q.z;
        }
    }
    if (k && (masks || phi)) {
        VLR_CUDA(ctx, cudaMemcpyAsync(dsel, sel.data(), sizeof(int) * k, cudaMemcpyHostToDevice, ctx->stream));
        const int B = (int)std::min<size_t>(k, (size_t)ctx->sm_count * 8);
        if (ls->precision == VLR_PREC_F16)
            k_gather_sel<__half><<<B, 256, 0, ctx->stream>>>(ls->list, dsel, (int)k, ls->mask,
                                                             (const __half*)ls->vals[0], mm, v);
        else
            k_gather_sel<float><<<B, 256, 0, ctx->stream>>>(ls->list, dsel, (int)k, ls->mask,
                                                            (const float*)ls->vals[0], mm, v);
        VLR_CUDA(ctx, cudaGetLastError());
        if (masks) VLR_CUDA(ctx, cudaMemcpyAsync(masks, mm, 64 * k, cudaMemcpyDeviceToHost, ctx->stream));
        if (phi)
            VLR_CUDA(ctx, cudaMemcpyAsync(phi, v, sizeof(float) * kLeafVoxels * k, cudaMemcpyDeviceToHost,
                                          ctx->stream));
        VLR_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    }
    *n_out = k;
    return VLR_OK;
}

// ------------------------------------------------- host step over x-slabs
//
// A host step of a large single-grid state whose host leaves are sorted by x
// (the order every download writes) runs as a pipeline over slabs of
// consecutive x.  Slab s owns the leaves with x in [X_s, X_{s+1}); it steps
// them together with the input leaves within kSlabRing voxels in x on either
// side, and keeps the outputs whose x lies in its own range.  A step reads
// within 5 voxels of a voxel (a backtrace of at most 3 voxels, two one-voxel
// reinitialisation sweeps), so the new values and mask of a leaf, whether
// the re-track keeps or allocates it, and the neighbour that fills a new leaf
// depend only on the input leaves within one leaf of it; those lie inside
// the slab's input for every output the slab keeps, so each kept output is
// bit for bit the one-pass step's (the kernels compute a leaf the same way
// whatever else is listed).  The kept outputs of a slab, sorted by (x, y, z),
// are one contiguous run of the sorted result.
//
// Copies: every slab's input goes up on one stream in slab order; slab s
// steps as soon as its input (its leaves and its ring) is on the device; its
// kept outputs go down on another stream while the next slab steps and later
// input goes up, so the copies in both directions overlap each other and the
// steps.  At the end the sorted result is loaded back into the pool, so the
// level set holds the stepped state as after a one-pass host step.
constexpr int kSlabRing = 16;                   // voxels: two leaves of input beside a slab
constexpr size_t kSlabLeavesAuto = 1u << 17;    // automatic count: one slab per this many leaves
constexpr unsigned long long kSlabOther = 0x7fffffffffffffffull;  // key of a leaf the slab does not keep

// Keys of the listed leaves (as k_leaf_keys) for those with x in [xlo, xhi),
// kSlabOther for the others (sorted after every kept leaf), and the number
// of kept leaves added to *kept.
__global__ void k_slab_keys(const int* __restrict__ list, const int* __restrict__ count,
                            const int4* __restrict__ origin, long long b0, long long b1, long long b2, int bits,
                            long long xlo, long long xhi, unsigned long long* __restrict__ keys,
                            unsigned* __restrict__ lo, unsigned* __restrict__ idx, int* __restrict__ kept) {
    const int n = *count;
    int c = 0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const int4 o = origin[list[i]];
        unsigned long long k = kSlabOther;
        if (o.x >= xlo && o.x < xhi) {
            k = ((unsigned long long)((o.x >> 3) - b0) << (2 * bits)) |
                ((unsigned long long)((o.y >> 3) - b1) << bits) | (unsigned long long)((o.z >> 3) - b2);
            ++c;
        }
        keys[i] = k;
        lo[i] = (unsigned)k;
        idx[i] = (unsigned)i;
    }
    for (int d = 16; d > 0; d >>= 1) c += __shfl_down_sync(0xffffffffu, c, d);
    if ((threadIdx.x & 31) == 0 && c) atomicAdd(kept, c);
}

// Origins, masks and f32 values of the first min(*kept, room) sorted list
// positions sel[i], one CTA per leaf.
template <typename T>
__global__ void k_gather_slab(const int* __restrict__ list, const unsigned* __restrict__ sel,
                              const int* __restrict__ kept, int room, const int4* __restrict__ origin,
                              const uint64_t* __restrict__ mask, const T* __restrict__ vals, int32_t* __restrict__ o3,
                              uint64_t* __restrict__ m_out, float* __restrict__ v_out) {
    const int k = min(*kept, room);
    for (int i = blockIdx.x; i < k; i += gridDim.x) {
        const int s = list[sel[i]];
        if (threadIdx.x < 3) {
            const int4 o = origin[s];
            o3[3 * i + threadIdx.x] = threadIdx.x == 0 ? o.x : (threadIdx.x == 1 ? o.y : o.z);
        }
        if (threadIdx.x < 8) m_out[(size_t)i * 8 + threadIdx.x] = mask[(size_t)s * 8 + threadIdx.x];
        for (int t = threadIdx.x; t < kLeafVoxels; t += blockDim.x)
            v_out[(size_t)i * kLeafVoxels + t] = to_f(vals[(size_t)s * kLeafVoxels + t]);
    }
}

__global__ void k_set_step(int* scalars, const int* step) { scalars[1] = *step; }

bool host_pinned(const void* p) {
    cudaPointerAttributes at{};
    const bool ok = cudaPointerGetAttributes(&at, p) == cudaSuccess && at.type == cudaMemoryTypeHost;
    cudaGetLastError();
    return ok;
}

// Leaves [n_first, n_first + n) of a device copy of host records (o3, masks,
// f32 values) as the pool's state, index enqueued; no wait.
int load_pool(vlr_ctx* ctx, vlr_level_set* ls, const int32_t* o3, const uint64_t* masks, const float* phi, size_t n) {
    cudaStream_t st = ctx->stream;
    if (n) {
        k_unpack_upload<<<ls->grid_blocks, 256, 0, st>>>(o3, (int)n, ls->origin);
        VLR_CUDA(ctx, cudaMemcpyAsync(ls->mask, masks, 64 * n, cudaMemcpyDeviceToDevice, st));
        if (ls->precision == VLR_PREC_F16)
            k_from_f32<__half><<<ls->grid_blocks, 256, 0, st>>>(phi, (__half*)ls->vals[0], kLeafVoxels * n);
        else
            VLR_CUDA(ctx, cudaMemcpyAsync(ls->vals[0], phi, sizeof(float) * kLeafVoxels * n, cudaMemcpyDeviceToDevice,
                                          st));
    }
    k_init_lists<<<ls->grid_blocks, 256, 0, st>>>(ls->list, ls->free_stack, ls->scalars, (int)n, ls->cap, 0);
    VLR_CUDA(ctx, cudaGetLastError());
    return ls_enqueue_index(ctx, ls);
}

// The slabs of a host step, or false when the one-pass path serves it (a
// small or unsorted state, pageable buffers, one slab asked for).
struct SlabPlan {
    std::vector<size_t> first;    // owned leaves of slab s: [first[s], first[s + 1])
    std::vector<long long> x;     // owned x range of slab s: [x[s], x[s + 1])
    std::vector<size_t> lo, hi;   // stepped input of slab s: [lo[s], hi[s])
};

bool plan_slabs(const vlr_level_set* ls, const int32_t* origins, size_t n, SlabPlan* p) {
    int S = ls->host_slabs;
    if (S == 1 || n < 2 || n > (size_t)ls->cap) return false;
    if (S == 0) S = (int)std::min<size_t>(kHostSlabsMax, n / kSlabLeavesAuto);
    S = std::min(S, kHostSlabsMax);
    if (S < 2) return false;
    for (size_t i = 0; i < n; ++i) {
        if ((origins[3 * i] | origins[3 * i + 1] | origins[3 * i + 2]) & 7) return false;  // the one pass reports it
        if (i && origins[3 * i] < origins[3 * i - 3]) return false;
    }
    auto xat = [&](size_t i) { return (long long)origins[3 * i]; };
    auto lower = [&](long long x) {  // first leaf with x at or above
        size_t a = 0, b = n;
        while (a < b) {
            const size_t m = a + (b - a) / 2;
            if (xat(m) < x) a = m + 1;
            else b = m;
        }
        return a;
    };
    p->first.assign(1, 0);
    for (int s = 1; s < S; ++s) {
        const size_t j = lower(xat((size_t)s * n / S));
        if (j > p->first.back() && j < n) p->first.push_back(j);
    }
    p->first.push_back(n);
    const int ns = (int)p->first.size() - 1;
    if (ns < 2) return false;
    p->x.assign(ns + 1, 0);
    p->x[0] = LLONG_MIN;
    p->x[ns] = LLONG_MAX;
    for (int s = 1; s < ns; ++s) p->x[s] = xat(p->first[s]);
    p->lo.resize(ns);
    p->hi.resize(ns);
    for (int s = 0; s < ns; ++s) {
        p->lo[s] = s == 0 ? 0 : lower(p->x[s] - kSlabRing);
        p->hi[s] = s == ns - 1 ? n : lower(p->x[s + 1] + kSlabRing);
    }
    return true;
}

// VLR_OK for cudaSuccess, else the error recorded on the context.
int cuda_rc(vlr_ctx* ctx, cudaError_t e, const char* what) {
    return e == cudaSuccess ? VLR_OK : check_cuda(ctx, e, what);
}

int step_host_slabs(vlr_ctx* ctx, vlr_level_set* ls, const SlabPlan& P, const int32_t* origins,
                    const uint64_t* masks, const float* phi, size_t n, int32_t* out_o, uint64_t* out_m,
                    float* out_v, size_t cap_leaves, size_t* n_out) {
    cudaStream_t st = ctx->stream;
    const int ns = (int)P.first.size() - 1;
    for (cudaStream_t& s : ls->slab_stream)
        if (!s) VLR_CUDA(ctx, cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
    for (cudaEvent_t& e : ls->slab_ev)
        if (!e) VLR_CUDA(ctx, cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    cudaStream_t up = ls->slab_stream[0], down = ls->slab_stream[1];
    cudaEvent_t* ev_up = ls->slab_ev;                      // [ns]: slab s's input is on the device
    cudaEvent_t* ev_out = ls->slab_ev + kHostSlabsMax;     // [ns]: slab s's kept outputs are gathered
    cudaEvent_t ev_ready = ls->slab_ev[2 * kHostSlabsMax];  // buffers allocated
    cudaEvent_t ev_down = ls->slab_ev[2 * kHostSlabsMax + 1];
    const size_t cap_out = std::min(cap_leaves, (size_t)ls->cap);
    const size_t cmax = (size_t)ls->cap;
    const size_t rec = sizeof(float) * kLeafVoxels + 64 + 12;
    const size_t sort_bytes = sort_reduce_scratch_bytes((int)cmax);
    const size_t bytes = n * rec + cap_out * rec + cmax * (8 + 12) + sort_bytes + 2 * kHostSlabsMax * sizeof(int) +
                         16 * 256;  // each of the 12 pieces below starts on a 256-byte boundary
    char* buf = nullptr;
    VLR_CUDA(ctx, cudaMallocFromPoolAsync((void**)&buf, bytes, ctx->pool, st));
    char* q = buf;
    auto take = [&](size_t b) {
        char* r = q;
        q += (b + 255) & ~(size_t)255;
        return r;
    };
    float* in_v = (float*)take(n * 4 * kLeafVoxels);
    uint64_t* in_m = (uint64_t*)take(n * 64);
    int32_t* in_o = (int32_t*)take(n * 12);
    float* out_sv = (float*)take(cap_out * 4 * kLeafVoxels);
    uint64_t* out_sm = (uint64_t*)take(cap_out * 64);
    int32_t* out_so = (int32_t*)take(cap_out * 12);
    unsigned long long* keys = (unsigned long long*)take(cmax * 8);
    unsigned* klo = (unsigned*)take(cmax * 4);
    unsigned* kidx = (unsigned*)take(cmax * 4);
    unsigned* khi = (unsigned*)take(cmax * 4);
    // [0, ns) kept per slab, [kHostSlabsMax] step at entry
    int* d_small = (int*)take(2 * kHostSlabsMax * sizeof(int));
    void* scratch = take(sort_bytes);
    int* h_count = static_cast<int*>(ctx->pinned) + 64;                  // pool count after slab s's step
    int* h_kept = static_cast<int*>(ctx->pinned) + 64 + kHostSlabsMax;   // outputs slab s keeps
    unsigned* h_err = static_cast<unsigned*>(ctx->pinned) + 64 + 2 * kHostSlabsMax;

    int rc = VLR_OK;
    auto finish = [&](int code) {
        // nothing may still read or write the buffers when they go back to the pool
        cudaEventRecord(ev_down, down);
        cudaStreamWaitEvent(st, ev_down, 0);
        cudaEventRecord(ev_down, up);
        cudaStreamWaitEvent(st, ev_down, 0);
        cudaFreeAsync(buf, st);
        if (code) {
            cudaStreamSynchronize(st);
            ls->state_lost = true;
        }
        return code;
    };
    if ((rc = cuda_rc(ctx, cudaMemsetAsync(d_small, 0, 2 * kHostSlabsMax * sizeof(int), st), "cudaMemsetAsync")) ||
        (rc = cuda_rc(ctx, cudaMemcpyAsync(d_small + kHostSlabsMax, ls->scalars + 1, sizeof(int),
                                           cudaMemcpyDeviceToDevice, st), "cudaMemcpyAsync")) ||
        (rc = cuda_rc(ctx, cudaEventRecord(ev_ready, st), "cudaEventRecord")) ||
        (rc = cuda_rc(ctx, cudaStreamWaitEvent(up, ev_ready, 0), "cudaStreamWaitEvent")) ||
        (rc = cuda_rc(ctx, cudaStreamWaitEvent(down, ev_ready, 0), "cudaStreamWaitEvent")))
        return finish(rc);
    // every slab's input, in slab order
    size_t done = 0;
    for (int s = 0; s < ns; ++s) {
        const size_t a = done, b = P.hi[s];
        if (b > a) {
            const size_t k = b - a;
            if ((rc = cuda_rc(ctx, cudaMemcpyAsync(in_o + 3 * a, origins + 3 * a, 12 * k, cudaMemcpyHostToDevice,
                                                      up), "slab input copy")) ||
                (rc = cuda_rc(ctx, cudaMemcpyAsync(in_m + 8 * a, masks + 8 * a, 64 * k, cudaMemcpyHostToDevice,
                                                      up), "slab input copy")) ||
                (rc = cuda_rc(ctx, cudaMemcpyAsync(in_v + kLeafVoxels * a, phi + kLeafVoxels * a,
                                                      sizeof(float) * kLeafVoxels * k, cudaMemcpyHostToDevice, up),
                                 "slab input copy")))
                return finish(rc);
            done = b;
        }
        if ((rc = cuda_rc(ctx, cudaEventRecord(ev_up[s], up), "cudaEventRecord"))) return finish(rc);
    }
    const vlr::MGridParams& G = ls->h_params[0];
    const int B = ctx->sm_count * 8;
    size_t off = 0;  // kept outputs of the slabs before
    std::vector<size_t> offs(ns, 0);
    auto copy_down = [&](int s) -> int {
        const size_t k = (size_t)h_kept[s], o = offs[s];
        if (o + k > cap_out) return set_error(ctx, VLR_ERR_CAPACITY, "output buffers too small");
        if (!k) return VLR_OK;
        VLR_CUDA(ctx, cudaStreamWaitEvent(down, ev_out[s], 0));
        VLR_CUDA(ctx, cudaMemcpyAsync(out_o + 3 * o, out_so + 3 * o, 12 * k, cudaMemcpyDeviceToHost, down));
        VLR_CUDA(ctx, cudaMemcpyAsync(out_m + 8 * o, out_sm + 8 * o, 64 * k, cudaMemcpyDeviceToHost, down));
        VLR_CUDA(ctx, cudaMemcpyAsync(out_v + kLeafVoxels * o, out_sv + kLeafVoxels * o,
                                      sizeof(float) * kLeafVoxels * k, cudaMemcpyDeviceToHost, down));
        return VLR_OK;
    };
    for (int s = 0; s < ns; ++s) {
        // slab s: its input as the pool's state, the step counter and the scan
        // status words as at entry, one step, its pool count to the host
        const size_t a = P.lo[s], m = P.hi[s] - P.lo[s];
        if ((rc = cuda_rc(ctx, cudaStreamWaitEvent(st, ev_up[s], 0), "cudaStreamWaitEvent")) ||
            (rc = load_pool(ctx, ls, in_o + 3 * a, in_m + 8 * a, in_v + kLeafVoxels * a, m)))
            return finish(rc);
        k_set_step<<<1, 1, 0, st>>>(ls->scalars, d_small + kHostSlabsMax);
        if ((rc = cuda_rc(ctx, cudaMemsetAsync(ls->pos, 0, sizeof(int) * (ls->cap + 1 + scan_scratch_ints(ls->cap)),
                                                  st), "cudaMemsetAsync")) ||
            (rc = enqueue_one_step(ctx, ls)) ||
            (rc = cuda_rc(ctx, cudaMemcpyAsync(h_count + s, ls->scalars, sizeof(int), cudaMemcpyDeviceToHost, st),
                             "count read-back")) ||
            (rc = cuda_rc(ctx, cudaMemcpyAsync(h_err, ctx->d_errword, sizeof(unsigned), cudaMemcpyDeviceToHost, st),
                             "error read-back")))
            return finish(rc);
        // the previous slab's kept outputs go down while this slab steps
        if (s > 0) {
            if ((rc = cuda_rc(ctx, cudaEventSynchronize(ev_out[s - 1]), "cudaEventSynchronize"))) return finish(rc);
            off += (size_t)h_kept[s - 1];
            if ((rc = copy_down(s - 1))) return finish(rc);
        }
        if ((rc = cuda_rc(ctx, cudaStreamSynchronize(st), "cudaStreamSynchronize"))) return finish(rc);
        const int c = h_count[s];
        if (*h_err || c < 0 || c > ls->cap) {
            rc = consume_device_errors(ctx, "vlr_ls_step_host");
            return finish(rc ? rc : set_error(ctx, VLR_ERR_CUDA, "slab step left an inconsistent leaf count"));
        }
        // its kept outputs, sorted by (x, y, z), gathered after those of the slabs before
        offs[s] = off;
        if (c) {
            k_slab_keys<<<B, 256, 0, st>>>(ls->list, ls->scalars, ls->origin, G.base[0], G.base[1], G.base[2],
                                           ls->key_bits, P.x[s], P.x[s + 1], keys, klo, kidx, d_small + s);
            unsigned *k1, *v1, *k2, *v2;
            if ((rc = radix_sort_pairs(ctx, klo, kidx, c, 0xffffffffu, scratch, &k1, &v1))) return finish(rc);
            k_leaf_keys_hi<<<B, 256, 0, st>>>(keys, v1, c, khi);
            if (v1 != kidx &&
                (rc = cuda_rc(ctx, cudaMemcpyAsync(kidx, v1, (size_t)c * 4, cudaMemcpyDeviceToDevice, st),
                                 "cudaMemcpyAsync")))
                return finish(rc);
            if ((rc = radix_sort_pairs(ctx, khi, kidx, c, 0x7fffffffu, scratch, &k2, &v2))) return finish(rc);
            (void)k1;
            (void)k2;
            const size_t o = std::min(off, cap_out);
            const int room = (int)(cap_out - o);
            if (ls->precision == VLR_PREC_F16)
                k_gather_slab<__half><<<B, 256, 0, st>>>(ls->list, v2, d_small + s, room, ls->origin, ls->mask,
                                                         (const __half*)ls->vals[0], out_so + 3 * o, out_sm + 8 * o,
                                                         out_sv + kLeafVoxels * o);
            else
                k_gather_slab<float><<<B, 256, 0, st>>>(ls->list, v2, d_small + s, room, ls->origin, ls->mask,
                                                        (const float*)ls->vals[0], out_so + 3 * o, out_sm + 8 * o,
                                                        out_sv + kLeafVoxels * o);
            if ((rc = cuda_rc(ctx, cudaGetLastError(), "slab gather"))) return finish(rc);
        }
        if ((rc = cuda_rc(ctx, cudaMemcpyAsync(h_kept + s, d_small + s, sizeof(int), cudaMemcpyDeviceToHost, st),
                             "kept read-back")) ||
            (rc = cuda_rc(ctx, cudaEventRecord(ev_out[s], st), "cudaEventRecord")))
            return finish(rc);
    }
    if ((rc = cuda_rc(ctx, cudaEventSynchronize(ev_out[ns - 1]), "cudaEventSynchronize")) ||
        (rc = copy_down(ns - 1)))
        return finish(rc);
    const size_t total = offs[ns - 1] + (size_t)h_kept[ns - 1];
    // the stepped state back into the pool (its step counter is already one
    // past the entry value), while the last outputs go down
    if ((rc = load_pool(ctx, ls, out_so, out_sm, out_sv, total))) return finish(rc);
    rc = finish(VLR_OK);
    if (rc) return rc;
    rc = consume_device_errors(ctx, "vlr_ls_step_host");
    if (rc) {
        ls->state_lost = true;
        return rc;
    }
    *n_out = total;
    return VLR_OK;
}


}  // namespace

extern "C" {

int vlr_ls_create_sphere(vlr_ctx* ctx, const vlr_method_desc* m, const vlr_velocity_desc* vel, double radius,
                         const double center[3], double voxel_size, const double w0[3], vlr_level_set** out) {
    if (!ctx || !m || !vel || !center || !out) return set_error(ctx, VLR_ERR_INVALID, "null argument");
    if (!(voxel_size > 0.0) || !(radius > 0.0)) return set_error(ctx, VLR_ERR_INVALID, "radius and voxel_size > 0");
    *out = nullptr;
    vlr_level_set* ls = new vlr_level_set();
    ls->ctx = ctx;
    ls->precision = m->precision == VLR_PREC_F16 ? VLR_PREC_F16 : VLR_PREC_F32;
    double zero[3] = {0, 0, 0};
    int rc = create_sphere_impl(ctx, ls, m, vel, radius, center, voxel_size, w0 ? w0 : zero);
    if (rc) {
        vlr_ls_destroy(ls);
        return rc;
    }
    *out = ls;
    return VLR_OK;
}

int vlr_ls_create_from_leaves(vlr_ctx* ctx, const vlr_method_desc* m, const vlr_velocity_desc* vel,
                              const int32_t* origins, const uint64_t* masks, const float* phi, size_t n_leaves,
                              vlr_level_set** out) {
    if (!ctx || !m || !vel || !origins || !masks || !phi || !out) return set_error(ctx, VLR_ERR_INVALID, "null argument");
    *out = nullptr;
    vlr_level_set* ls = new vlr_level_set();
    ls->ctx = ctx;
    ls->precision = m->precision == VLR_PREC_F16 ? VLR_PREC_F16 : VLR_PREC_F32;
    int rc = create_leaves_impl(ctx, ls, m, vel, origins, masks, phi, n_leaves);
    if (rc) {
        vlr_ls_destroy(ls);
        return rc;
    }
    *out = ls;
    return VLR_OK;
}

int vlr_ls_enqueue(vlr_ctx* ctx, vlr_level_set* ls, int n_steps) {
    if (!ctx || !ls) return set_error(ctx, VLR_ERR_INVALID, "null argument");
    for (int i = 0; i < n_steps; ++i) {
        int rc = enqueue_one_step(ctx, ls);
        if (rc) return rc;
    }
    return VLR_OK;
}

int vlr_ctx_check(vlr_ctx* ctx) {
    if (!ctx) return VLR_ERR_INVALID;
    VLR_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    return consume_device_errors(ctx, "vlr_ctx_check");
}

int vlr_ls_step(vlr_ctx* ctx, vlr_level_set* ls, int n_steps) {
    if (!ctx || !ls) return set_error(ctx, VLR_ERR_INVALID, "null argument");
    for (int i = 0; i < n_steps; ++i) {
        int rc = enqueue_one_step(ctx, ls);
        if (rc) return rc;
    }
    VLR_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    const int rc = consume_device_errors(ctx, "vlr_ls_step");
    if (rc == VLR_ERR_TIMEOUT || rc == VLR_ERR_CAPACITY) ls->state_lost = true;
    return rc;
}

int vlr_ls_set_launch_shape(vlr_ctx* ctx, vlr_level_set* ls, int advect_threads, int advect_ctas, int advect_staging,
                            int reinit_threads, int reinit_ctas, int reinit_staging) {
    if (!ctx || !ls) return set_error(ctx, VLR_ERR_INVALID, "null argument");
    drop_graph(ls);
    if (advect_threads == 0) {
        ls->autotune = true;
        ls->tuned = false;
        return VLR_OK;
    }
    if (advect_threads != kAdvectThreads || advect_staging != 0 || reinit_threads != kReinitThreads ||
        reinit_staging != 0 || advect_ctas < 1 || reinit_ctas < 1)
        return set_error(ctx, VLR_ERR_INVALID, "launch shape: 128 threads, staging 0 and CTAs > 0 for both kernels");
    ls->adv_shape = StencilShape{advect_threads, advect_ctas, advect_staging};
    ls->re_shape = StencilShape{reinit_threads, reinit_ctas, reinit_staging};
    ls->autotune = false;
    ls->tuned = true;
    return VLR_OK;
}

int vlr_ls_get_launch_shape(vlr_ctx* ctx, const vlr_level_set* ls, int shape[6], int* n_timed, float* log,
                            int cap_log) {
    if (!ctx || !ls || !shape) return set_error(ctx, VLR_ERR_INVALID, "null argument");
    shape[0] = ls->adv_shape.nt;
    shape[1] = ls->adv_shape.blocks;
    shape[2] = ls->adv_shape.stage;
    shape[3] = ls->re_shape.nt;
    shape[4] = ls->re_shape.blocks;
    shape[5] = ls->re_shape.stage;
    int k = 0;
    for (int w = 0; w < 2; ++w)
        for (const TuneEntry& e : ls->tune_log[w]) {
            if (log && k < cap_log) {
                log[5 * k] = (float)w;
                log[5 * k + 1] = (float)e.shape.nt;
                log[5 * k + 2] = (float)e.shape.blocks;
                log[5 * k + 3] = (float)e.shape.stage;
                log[5 * k + 4] = e.ms * 1000.0f;
            }
            ++k;
        }
    if (n_timed) *n_timed = k;
    return VLR_OK;
}

int vlr_ls_info(vlr_ctx* ctx, const vlr_level_set* ls, size_t* n_leaves, uint64_t* n_active, double* time) {
    if (!ctx || !ls) return set_error(ctx, VLR_ERR_INVALID, "null argument");
    int sc[8];
    VLR_CUDA(ctx, cudaMemcpyAsync(sc, ls->scalars, sizeof(sc), cudaMemcpyDeviceToHost, ctx->stream));
    VLR_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    if (n_leaves) *n_leaves = (size_t)sc[0];
    if (time) *time = (double)ls->sp.t0 + (double)sc[1] * (double)ls->sp.dt;
    if (n_active) {
        unsigned long long* d = (unsigned long long*)ls->d_sum;
        VLR_CUDA(ctx, cudaMemsetAsync(d, 0, sizeof(unsigned long long), ctx->stream));
        k_count_active<<<ls->grid_blocks, 256, 0, ctx->stream>>>(ls->list, ls->scalars, ls->mask, d);
        unsigned long long h = 0;
        VLR_CUDA(ctx, cudaMemcpyAsync(&h, d, sizeof(h), cudaMemcpyDeviceToHost, ctx->stream));
        VLR_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
        *n_active = h;
    }
    return VLR_OK;
}

int vlr_ls_download(vlr_ctx* ctx, const vlr_level_set* ls, int32_t* origins, uint64_t* masks, float* phi,
                    size_t cap_leaves) {
    size_t n_out = 0;
    return vlr_ls_download_grid(ctx, ls, -1, nullptr, origins, masks, phi, cap_leaves, &n_out);
}

int vlr_ls_download_grid(vlr_ctx* ctx, const vlr_level_set* ls, int grid, int32_t* grid_ids, int32_t* origins,
                         uint64_t* masks, float* phi, size_t cap_leaves, size_t* n_out) {
    if (!ctx || !ls || !n_out) return set_error(ctx, VLR_ERR_INVALID, "null argument");
    *n_out = 0;
    size_t n = 0;
    int rc = vlr_ls_info(ctx, ls, &n, nullptr, nullptr);
    if (rc) return rc;
    return download_n(ctx, ls, n, grid, grid_ids, origins, masks, phi, cap_leaves, n_out);
}

int vlr_ls_step_host(vlr_ctx* ctx, vlr_level_set* ls, const int32_t* origins, const uint64_t* masks, const float* phi,
                     size_t n_leaves, int n_steps, int32_t* out_origins, uint64_t* out_masks, float* out_phi,
                     size_t cap_leaves, size_t* n_out) {
    if (!ctx || !ls || !origins || !masks || !phi || !n_out) return set_error(ctx, VLR_ERR_INVALID, "null argument");
    if (ls->n_grids != 1) return set_error(ctx, VLR_ERR_UNSUPPORTED, "host steps replace single-grid states only");
    *n_out = 0;
    // large x-sorted states in pinned buffers: one step as a pipeline over x-slabs
    SlabPlan plan;
    if (n_steps == 1 && 3 * ls->key_bits <= 63 && out_origins && out_masks && out_phi && host_pinned(origins) &&
        host_pinned(masks) && host_pinned(phi) && host_pinned(out_origins) && host_pinned(out_masks) &&
        host_pinned(out_phi) && plan_slabs(ls, origins, n_leaves, &plan))
        return step_host_slabs(ctx, ls, plan, origins, masks, phi, n_leaves, out_origins, out_masks, out_phi,
                               cap_leaves, n_out);
    // staging for the device-sorted download (sized first, so the upload
    // never regrows it while its copies are in flight)
    const size_t kv = (size_t)kDevSortLeaves;
    const size_t dl_bytes = kv * (sizeof(float) * kLeafVoxels + 64 + 12 + 4 + 8) + 256;
    void* stg = nullptr;
    int rc = ls_staging(ctx, ls, std::max(dl_bytes, sizeof(float) * kLeafVoxels * n_leaves + 12 * n_leaves + 16),
                        &stg);
    if (rc) return rc;
    rc = upload_enqueue(ctx, ls, origins, masks, phi, n_leaves, false);
    if (rc) return rc;
    for (int i = 0; i < n_steps; ++i) {
        rc = enqueue_one_step(ctx, ls);
        if (rc) return rc;
    }
    int* h = static_cast<int*>(ctx->pinned) + 16;
    if (3 * ls->key_bits > 63) {  // keys too wide for the device sort: the host sorts
        VLR_CUDA(ctx, cudaMemcpyAsync(h, ls->scalars, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
        rc = consume_device_errors(ctx, "vlr_ls_step_host");
        if (rc == VLR_ERR_TIMEOUT || rc == VLR_ERR_CAPACITY) ls->state_lost = true;
        if (rc) return rc;
        return download_n(ctx, ls, (size_t)h[0], -1, nullptr, out_origins, out_masks, out_phi, cap_leaves, n_out);
    }
    float* v = (float*)ls->staging;
    uint64_t* mm = (uint64_t*)((char*)ls->staging + kv * sizeof(float) * kLeafVoxels);
    int32_t* o3 = (int32_t*)((char*)mm + kv * 64);
    int* dsel = (int*)((char*)o3 + kv * 12);
    int* dstatus = (int*)((char*)dsel + kv * 4);
    unsigned long long* dkeys = reinterpret_cast<unsigned long long*>(((uintptr_t)(dstatus + 4) + 15) & ~(uintptr_t)15);
    const vlr::MGridParams& P = ls->h_params[0];
    k_rank_keys<<<ctx->sm_count, 256, 0, ctx->stream>>>(ls->list, ls->scalars, ls->origin, P.base[0], P.base[1],
                                                        P.base[2], ls->key_bits, dkeys, dstatus);
    k_rank_scatter<<<kDevSortLeaves * kRankLanes / 256, 256, 0, ctx->stream>>>(ls->list, ls->scalars, ls->origin,
                                                                               dkeys, dsel, o3);
    const int B = ctx->sm_count * 8;
    if (ls->precision == VLR_PREC_F16)
        k_gather_sel_dev<__half><<<B, 256, 0, ctx->stream>>>(ls->list, dsel, ls->scalars, dstatus, ls->mask,
                                                             (const __half*)ls->vals[0], mm, v);
    else
        k_gather_sel_dev<float><<<B, 256, 0, ctx->stream>>>(ls->list, dsel, ls->scalars, dstatus, ls->mask,
                                                            (const float*)ls->vals[0], mm, v);
    VLR_CUDA(ctx, cudaGetLastError());
    // copies of the records [lo, hi) of the sorted output into the caller's buffers
    auto copy_out = [&](size_t lo, size_t hi) -> int {
        if (hi <= lo) return VLR_OK;
        const size_t k = hi - lo;
        if (out_origins)
            VLR_CUDA(ctx, cudaMemcpyAsync(out_origins + 3 * lo, o3 + 3 * lo, 12 * k, cudaMemcpyDeviceToHost,
                                          ctx->stream));
        if (out_masks)
            VLR_CUDA(ctx, cudaMemcpyAsync(out_masks + 8 * lo, mm + 8 * lo, 64 * k, cudaMemcpyDeviceToHost, ctx->stream));
        if (out_phi)
            VLR_CUDA(ctx, cudaMemcpyAsync(out_phi + kLeafVoxels * lo, v + kLeafVoxels * lo,
                                          sizeof(float) * kLeafVoxels * k, cudaMemcpyDeviceToHost, ctx->stream));
        return VLR_OK;
    };
    // the output holds about as many leaves as the input: copy that many
    // before the count is known, so the copies overlap the count's round trip
    const size_t guess = std::min(std::min(n_leaves, cap_leaves), kv);
    rc = copy_out(0, guess);
    if (rc) return rc;
    // leaf count, sort status and device errors in one round trip
    VLR_CUDA(ctx, cudaMemcpyAsync(h, ls->scalars, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
    VLR_CUDA(ctx, cudaMemcpyAsync(h + 1, dstatus, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
    rc = consume_device_errors(ctx, "vlr_ls_step_host");
    if (rc == VLR_ERR_TIMEOUT || rc == VLR_ERR_CAPACITY) ls->state_lost = true;
    if (rc) return rc;
    const size_t n = (size_t)h[0];
    if (!h[1]) return download_n(ctx, ls, n, -1, nullptr, out_origins, out_masks, out_phi, cap_leaves, n_out);
    if (n > cap_leaves) return set_error(ctx, VLR_ERR_CAPACITY, "output buffers too small");
    if (n > guess) {
        rc = copy_out(guess, n);
        if (rc) return rc;
        VLR_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    }
    *n_out = n;
    return VLR_OK;
}

int vlr_ls_upload(vlr_ctx* ctx, vlr_level_set* ls, const int32_t* origins, const uint64_t* masks, const float* phi,
                  size_t n_leaves) {
    if (!ctx || !ls || !origins || !masks || !phi) return set_error(ctx, VLR_ERR_INVALID, "null argument");
    if (ls->n_grids != 1) return set_error(ctx, VLR_ERR_UNSUPPORTED, "upload replaces single-grid states only");
    return upload_impl(ctx, ls, origins, masks, phi, n_leaves, false);
}

int vlr_ls_upload_device(vlr_ctx* ctx, vlr_level_set* ls, const int32_t* d_origins, const uint64_t* d_masks,
                         const float* d_phi, size_t n_leaves) {
    if (!ctx || !ls || (n_leaves && (!d_origins || !d_masks || !d_phi)))
        return set_error(ctx, VLR_ERR_INVALID, "null argument");
    if (ls->n_grids != 1) return set_error(ctx, VLR_ERR_UNSUPPORTED, "upload replaces single-grid states only");
    if (n_leaves > (size_t)ls->cap) return set_error(ctx, VLR_ERR_CAPACITY, "more leaves than the level set's capacity");
    const int n = (int)n_leaves;
    if (n) {
        k_upload_dev_origins<<<ls->grid_blocks, 256, 0, ctx->stream>>>(d_origins, n, ls->origin, ctx->d_errword);
        VLR_CUDA(ctx, cudaMemcpyAsync(ls->mask, d_masks, 64 * n_leaves, cudaMemcpyDeviceToDevice, ctx->stream));
        if (ls->precision == VLR_PREC_F16)
            k_from_f32<__half><<<ls->grid_blocks, 256, 0, ctx->stream>>>(d_phi, (__half*)ls->vals[0],
                                                                          kLeafVoxels * n_leaves);
        else
            VLR_CUDA(ctx, cudaMemcpyAsync(ls->vals[0], d_phi, sizeof(float) * kLeafVoxels * n_leaves,
                                          cudaMemcpyDeviceToDevice, ctx->stream));
        VLR_CUDA(ctx, cudaGetLastError());
    }
    // origins are checked before the index is built from them
    int rc = consume_device_errors(ctx, "vlr_ls_upload_device");
    if (rc) return rc;
    return ls_init_lists(ctx, ls, n, false);
}

int vlr_ls_download_device(vlr_ctx* ctx, const vlr_level_set* ls, int32_t* d_origins, uint64_t* d_masks,
                           float* d_phi, size_t cap_leaves, size_t* n_out) {
    if (!ctx || !ls || !n_out || !d_origins || !d_masks || !d_phi)
        return set_error(ctx, VLR_ERR_INVALID, "null argument");
    *n_out = 0;
    size_t n = 0;
    int rc = vlr_ls_info(ctx, ls, &n, nullptr, nullptr);
    if (rc) return rc;
    if (n > cap_leaves) return set_error(ctx, VLR_ERR_CAPACITY, "output buffers too small");
    if (n) {
        const int B = (int)std::min<size_t>(n, (size_t)ctx->sm_count * 8);
        if (ls->precision == VLR_PREC_F16)
            k_export_dev<__half><<<B, 256, 0, ctx->stream>>>(ls->list, ls->scalars, ls->origin, ls->mask,
                                                             (const __half*)ls->vals[0], d_origins, d_masks, d_phi);
        else
            k_export_dev<float><<<B, 256, 0, ctx->stream>>>(ls->list, ls->scalars, ls->origin, ls->mask,
                                                            (const float*)ls->vals[0], d_origins, d_masks, d_phi);
        VLR_CUDA(ctx, cudaGetLastError());
        VLR_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    }
    *n_out = n;
    return VLR_OK;
}

int vlr_ls_volume_partials(vlr_ctx* ctx, vlr_level_set* ls, const double ref[3], double* d_partials,
                           size_t cap, size_t* n_out) {
    if (!ctx || !ls || !d_partials || !n_out) return set_error(ctx, VLR_ERR_INVALID, "null argument");
    *n_out = 0;
    size_t n = 0;
    int rc = vlr_ls_info(ctx, ls, &n, nullptr, nullptr);
    if (rc) return rc;
    if (n > cap) return set_error(ctx, VLR_ERR_CAPACITY, "partials buffer too small");
    double r[3] = {0, 0, 0};
    if (ref) std::memcpy(r, ref, sizeof(r));
    MLeafArrays A = ls->arrays();
    if (ls->precision == VLR_PREC_F16)
        k_m_volume<__half><<<ls->grid_blocks, 256, 0, ctx->stream>>>(A, (const __half*)ls->vals[0], ls->d_params,
                                                                     r[0], r[1], r[2], d_partials);
    else
        k_m_volume<float><<<ls->grid_blocks, 256, 0, ctx->stream>>>(A, (const float*)ls->vals[0], ls->d_params, r[0],
                                                                    r[1], r[2], d_partials);
    VLR_CUDA(ctx, cudaGetLastError());
    VLR_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    *n_out = n;
    return VLR_OK;
}

int vlr_ls_set_step(vlr_ctx* ctx, vlr_level_set* ls, int step) {
    if (!ctx || !ls) return set_error(ctx, VLR_ERR_INVALID, "null argument");
    if (step < 0) return set_error(ctx, VLR_ERR_INVALID, "step must be >= 0");
    if (!ls->scalars) return set_error(ctx, VLR_ERR_INVALID, "level set has no state");
    // the look-back scan tags its status words with step + 1: clear them so no
    // word of an earlier step can carry the tag of a step to come
    VLR_CUDA(ctx, cudaMemsetAsync(ls->pos, 0, sizeof(int) * (ls->cap + 1 + scan_scratch_ints(ls->cap)), ctx->stream));
    VLR_CUDA(ctx, cudaMemcpyAsync(ls->scalars + 1, &step, sizeof(int), cudaMemcpyHostToDevice, ctx->stream));
    VLR_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    return VLR_OK;
}

int vlr_ls_set_host_slabs(vlr_ctx* ctx, vlr_level_set* ls, int slabs) {
    if (!ctx || !ls) return set_error(ctx, VLR_ERR_INVALID, "null argument");
    if (slabs < 0) return set_error(ctx, VLR_ERR_INVALID, "slabs must be >= 0");
    ls->host_slabs = std::min(slabs, kHostSlabsMax);
    return VLR_OK;
}

int vlr_ls_volume(vlr_ctx* ctx, vlr_level_set* ls, const double ref[3], double* volume) {
    if (!ctx || !ls || !volume) return set_error(ctx, VLR_ERR_INVALID, "null argument");
    double r[3] = {0, 0, 0};
    if (ref) std::memcpy(r, ref, sizeof(r));
    MLeafArrays A = ls->arrays();
    if (ls->precision == VLR_PREC_F16)
        VLR_TIMED(ctx, "k_m_volume",
                  k_m_volume<__half><<<ls->grid_blocks, 256, 0, ctx->stream>>>(A, (const __half*)ls->vals[0],
                                                                               ls->d_params, r[0], r[1], r[2],
                                                                               ls->d_partial));
    else
        VLR_TIMED(ctx, "k_m_volume",
                  k_m_volume<float><<<ls->grid_blocks, 256, 0, ctx->stream>>>(A, (const float*)ls->vals[0],
                                                                              ls->d_params, r[0], r[1], r[2],
                                                                              ls->d_partial));
    k_reduce_fixed<<<1, 1024, 0, ctx->stream>>>(ls->d_partial, ls->scalars, ls->d_sum);
    VLR_CUDA(ctx, cudaGetLastError());
    VLR_CUDA(ctx, cudaMemcpyAsync(volume, ls->d_sum, sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    VLR_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    return VLR_OK;
}

void vlr_ls_destroy(vlr_level_set* ls) {
    if (!ls) return;
    if (ls->ctx) cudaStreamSynchronize(ls->ctx->stream);
    ls_free(ls);
    delete ls;
}

}  // extern "C"
