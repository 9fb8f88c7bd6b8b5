// advect_particles / advect_particles_euler (src/tools/advection.rs:58-110)
// on particle positions: RK4 (or forward Euler) through a VelocityField of
// three grids.  VelocityField::sample is three sample_trilinear calls widened
// to f64 (src/tools/advection.rs:16-24); the position arithmetic is f64 in the
// reference's order, with explicitly rounded operations so nothing is
// contracted into an FMA.
//
// vlr_advect_points is the whole crate call: the position update followed by
// PointDataGrid::rebin (src/points/point_grid.rs:258-266), which drains every
// leaf and re-inserts each particle into the leaf of
// AffineMap::world_to_index(position) aligned to 8.  The crate drains its
// leaves in HashMap order; here leaves are drained in ascending (x, y, z)
// origin order, so with particles handed in that binned order the re-binned
// grid is a stable sort of the particles by their new leaf.  On the GPU:
//   k_points_move    position update, then the new leaf per particle as three
//                    order-preserving 29-bit keys (one per axis)
//   (sort)           three stable radix sorts of (key, particle index): z,
//                    then y, then x, the keys of each pass gathered in the
//                    order the previous pass left (k_gather_keys)
//   k_points_emit    particles gathered into sorted order; a flag where the
//                    leaf changes
//   (scan)           leaf ranks; k_points_leaves writes each leaf's origin and
//                    first particle
#include <algorithm>

#include "ref_ops.hpp"
#include "sort_reduce.hpp"

namespace vlr {
namespace {

struct V3 {
    double x, y, z;
};

__device__ __forceinline__ V3 vsample(const GridView& vx, const GridView& vy, const GridView& vz, const V3& p) {
    return V3{(double)sample_trilinear_ref(vx, p.x, p.y, p.z), (double)sample_trilinear_ref(vy, p.x, p.y, p.z),
              (double)sample_trilinear_ref(vz, p.x, p.y, p.z)};
}

__device__ __forceinline__ V3 scale(double s, const V3& v) {
    return V3{__dmul_rn(s, v.x), __dmul_rn(s, v.y), __dmul_rn(s, v.z)};
}

// pos + k * f (k * f rounded first, as `pos[a] + k[a] * 0.5` evaluates)
__device__ __forceinline__ V3 axpy(const V3& pos, const V3& k, double f) {
    return V3{__dadd_rn(pos.x, __dmul_rn(k.x, f)), __dadd_rn(pos.y, __dmul_rn(k.y, f)),
              __dadd_rn(pos.z, __dmul_rn(k.z, f))};
}

// pos + (k1 + 2 k2 + 2 k3 + k4) / 6, summed left to right
__device__ __forceinline__ double rk4_comb(double p, double k1, double k2, double k3, double k4) {
    const double s = __dadd_rn(__dadd_rn(__dadd_rn(k1, __dmul_rn(2.0, k2)), __dmul_rn(2.0, k3)), k4);
    return __dadd_rn(p, __ddiv_rn(s, 6.0));
}

__global__ void k_advect_particles(GridView vx, GridView vy, GridView vz, double* __restrict__ pos, int n, double dt,
                                   int rk4) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const V3 p{pos[3 * i], pos[3 * i + 1], pos[3 * i + 2]};
        V3 out;
        if (rk4) {
            const V3 k1 = scale(dt, vsample(vx, vy, vz, p));
            const V3 k2 = scale(dt, vsample(vx, vy, vz, axpy(p, k1, 0.5)));
            const V3 k3 = scale(dt, vsample(vx, vy, vz, axpy(p, k2, 0.5)));
            const V3 k4 = scale(dt, vsample(vx, vy, vz, axpy(p, k3, 1.0)));
            out = V3{rk4_comb(p.x, k1.x, k2.x, k3.x, k4.x), rk4_comb(p.y, k1.y, k2.y, k3.y, k4.y),
                     rk4_comb(p.z, k1.z, k2.z, k3.z, k4.z)};
        } else {
            const V3 v = vsample(vx, vy, vz, p);
            out = V3{__dadd_rn(p.x, __dmul_rn(dt, v.x)), __dadd_rn(p.y, __dmul_rn(dt, v.y)),
                     __dadd_rn(p.z, __dmul_rn(dt, v.z))};
        }
        pos[3 * i] = out.x;
        pos[3 * i + 1] = out.y;
        pos[3 * i + 2] = out.z;
    }
}

// f64::round (half away from zero) then Rust's saturating `as i32`.
__device__ __forceinline__ int32_t round_to_i32(double f) {
    const double r = round(f);
    if (r != r) return 0;
    if (r >= 2147483647.0) return 2147483647;
    if (r <= -2147483648.0) return INT32_MIN;
    return (int32_t)r;
}

struct InvRows {
    double r[12];  // rows 0..2 of the world -> index 4x4 map
};

// Leaf origin coordinate (a multiple of 8) -> order-preserving key below 2^29.
__device__ __forceinline__ unsigned leaf_key(int32_t v) { return ((unsigned)v >> 3) ^ (1u << 28); }
__device__ __forceinline__ int32_t key_leaf(unsigned k) { return (int32_t)((k ^ (1u << 28)) << 3); }

__global__ void k_points_move(GridView vx, GridView vy, GridView vz, vlr_particle* __restrict__ pts, int n,
                              double dt, int rk4, InvRows inv, unsigned* __restrict__ kx, unsigned* __restrict__ ky,
                              unsigned* __restrict__ kz, unsigned* __restrict__ idx) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        double* pp = pts[i].position;
        const V3 p{pp[0], pp[1], pp[2]};
        V3 out;
        if (rk4) {
            const V3 k1 = scale(dt, vsample(vx, vy, vz, p));
            const V3 k2 = scale(dt, vsample(vx, vy, vz, axpy(p, k1, 0.5)));
            const V3 k3 = scale(dt, vsample(vx, vy, vz, axpy(p, k2, 0.5)));
            const V3 k4 = scale(dt, vsample(vx, vy, vz, axpy(p, k3, 1.0)));
            out = V3{rk4_comb(p.x, k1.x, k2.x, k3.x, k4.x), rk4_comb(p.y, k1.y, k2.y, k3.y, k4.y),
                     rk4_comb(p.z, k1.z, k2.z, k3.z, k4.z)};
        } else {
            const V3 v = vsample(vx, vy, vz, p);
            out = V3{__dadd_rn(p.x, __dmul_rn(dt, v.x)), __dadd_rn(p.y, __dmul_rn(dt, v.y)),
                     __dadd_rn(p.z, __dmul_rn(dt, v.z))};
        }
        pp[0] = out.x;
        pp[1] = out.y;
        pp[2] = out.z;
        // AffineMap::world_to_index: a*x + b*y + c*z + d, left to right, then aligned(3)
        unsigned* keys[3] = {kx, ky, kz};
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            const double* r = inv.r + 4 * a;
            const double f = __dadd_rn(__dadd_rn(__dadd_rn(__dmul_rn(r[0], out.x), __dmul_rn(r[1], out.y)),
                                                 __dmul_rn(r[2], out.z)),
                                       r[3]);
            keys[a][i] = leaf_key(round_to_i32(f) & ~7);
        }
        idx[i] = (unsigned)i;
    }
}

__global__ void k_gather_keys(const unsigned* __restrict__ keys, const unsigned* __restrict__ perm, int n,
                              unsigned* __restrict__ out) {
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += gridDim.x * blockDim.x) out[j] = keys[perm[j]];
}

__global__ void k_points_emit(const vlr_particle* __restrict__ in, const unsigned* __restrict__ perm,
                              const unsigned* __restrict__ kx, const unsigned* __restrict__ ky,
                              const unsigned* __restrict__ kz, int n, vlr_particle* __restrict__ out,
                              int* __restrict__ head) {
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += gridDim.x * blockDim.x) {
        const unsigned i = perm[j];
        out[j] = in[i];
        int h = 1;
        if (j > 0) {
            const unsigned q = perm[j - 1];
            h = (kx[i] != kx[q]) | (ky[i] != ky[q]) | (kz[i] != kz[q]);
        }
        head[j] = h;
    }
}

__global__ void k_points_leaves(const unsigned* __restrict__ perm, const unsigned* __restrict__ kx,
                                const unsigned* __restrict__ ky, const unsigned* __restrict__ kz,
                                const int* __restrict__ head, const int* __restrict__ rank, int n,
                                int32_t* __restrict__ origins, uint32_t* __restrict__ start) {
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += gridDim.x * blockDim.x) {
        if (!head[j]) continue;
        const int l = rank[j];
        const unsigned i = perm[j];
        origins[3 * l] = key_leaf(kx[i]);
        origins[3 * l + 1] = key_leaf(ky[i]);
        origins[3 * l + 2] = key_leaf(kz[i]);
        start[l] = (uint32_t)j;
    }
}

}  // namespace
}  // namespace vlr

using namespace vlr;

extern "C" {

int vlr_advect_particles(vlr_ctx* ctx, const vlr_grid* vx, const vlr_grid* vy, const vlr_grid* vz, double* positions,
                         size_t n, double dt, int rk4) {
    if (!ctx || !vx || !vy || !vz || (n && !positions)) return set_error(ctx, VLR_ERR_INVALID, "null argument");
    if (vx->kind != VLR_KIND_F32_WORLD || vy->kind != VLR_KIND_F32_WORLD || vz->kind != VLR_KIND_F32_WORLD)
        return set_error(ctx, VLR_ERR_INVALID, "velocity grids must be world-unit f32 grids");
    if (n == 0) return VLR_OK;
    if (n > (size_t)INT32_MAX / 3) return set_error(ctx, VLR_ERR_CAPACITY, "too many particles");
    double* d = nullptr;
    VLR_CUDA(ctx, cudaMallocFromPoolAsync(&d, sizeof(double) * 3 * n, ctx->pool, ctx->stream));
    VLR_CUDA(ctx, cudaMemcpyAsync(d, positions, sizeof(double) * 3 * n, cudaMemcpyHostToDevice, ctx->stream));
    const int blocks = (int)std::min<size_t>((n + 255) / 256, (size_t)ctx->sm_count * 16);
    k_advect_particles<<<blocks, 256, 0, ctx->stream>>>(make_view(vx), make_view(vy), make_view(vz), d, (int)n, dt,
                                                        rk4 ? 1 : 0);
    VLR_CUDA(ctx, cudaGetLastError());
    VLR_CUDA(ctx, cudaMemcpyAsync(positions, d, sizeof(double) * 3 * n, cudaMemcpyDeviceToHost, ctx->stream));
    VLR_CUDA(ctx, cudaFreeAsync(d, ctx->stream));
    VLR_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    return consume_device_errors(ctx, "vlr_advect_particles");
}

int vlr_advect_points(vlr_ctx* ctx, const vlr_grid* vx, const vlr_grid* vy, const vlr_grid* vz,
                      const double world_to_index[12], vlr_particle* particles, size_t n, double dt, int rk4,
                      int32_t* leaf_origins, uint32_t* leaf_start, size_t cap_leaves, size_t* n_leaves) {
    if (!ctx || !vx || !vy || !vz || !world_to_index || !n_leaves || (n && !particles) || !leaf_start ||
        (cap_leaves && !leaf_origins))
        return set_error(ctx, VLR_ERR_INVALID, "null argument");
    if (vx->kind != VLR_KIND_F32_WORLD || vy->kind != VLR_KIND_F32_WORLD || vz->kind != VLR_KIND_F32_WORLD)
        return set_error(ctx, VLR_ERR_INVALID, "velocity grids must be world-unit f32 grids");
    *n_leaves = 0;
    if (n == 0) {
        leaf_start[0] = 0;
        return VLR_OK;
    }
    if (n > ((size_t)1 << 28)) return set_error(ctx, VLR_ERR_CAPACITY, "more than 2^28 particles in one call");
    const int nn = (int)n;
    cudaStream_t st = ctx->stream;
    InvRows inv;
    for (int i = 0; i < 12; ++i) inv.r[i] = world_to_index[i];
    // one stream-ordered block: particles in and out, keys, permutation, flags, ranks, sort scratch
    const size_t pb = sizeof(vlr_particle) * n, wb = sizeof(unsigned) * n;
    const size_t sb = sort_reduce_scratch_bytes(nn);
    auto al = [](size_t b) { return (b + 255) & ~(size_t)255; };
    const size_t total = 2 * al(pb) + 8 * al(wb) + al(sizeof(int) * 2) + al(sb) + al(sizeof(int32_t) * 3 * n) +
                         al(sizeof(uint32_t) * (n + 1));
    char* blk = nullptr;
    if (cudaMallocFromPoolAsync((void**)&blk, total, ctx->pool, st) != cudaSuccess) {
        cudaGetLastError();
        return set_error(ctx, VLR_ERR_NOMEM, "vlr_advect_points: device allocation failed");
    }
    char* q = blk;
    auto take = [&](size_t b) {
        char* r = q;
        q += al(b);
        return r;
    };
    vlr_particle* d_in = (vlr_particle*)take(pb);
    vlr_particle* d_out = (vlr_particle*)take(pb);
    unsigned* kx = (unsigned*)take(wb);
    unsigned* ky = (unsigned*)take(wb);
    unsigned* kz = (unsigned*)take(wb);
    unsigned* idx = (unsigned*)take(wb);
    unsigned* kbuf = (unsigned*)take(wb);
    unsigned* pbuf = (unsigned*)take(wb);
    int* head = (int*)take(wb);
    int* rank = (int*)take(wb);
    int* d_total = (int*)take(sizeof(int) * 2);
    void* scratch = take(sb);
    int32_t* d_org = (int32_t*)take(sizeof(int32_t) * 3 * n);
    uint32_t* d_start = (uint32_t*)take(sizeof(uint32_t) * (n + 1));
    int rc = VLR_OK;
    auto fail = [&](int code) {
        cudaFreeAsync(blk, st);
        return code;
    };
    const int blocks = (int)std::min<size_t>((n + 255) / 256, (size_t)ctx->sm_count * 16);
    if (cudaMemcpyAsync(d_in, particles, pb, cudaMemcpyHostToDevice, st) != cudaSuccess)
        return fail(check_cuda(ctx, cudaGetLastError(), "particle upload"));
    VLR_TIMED(ctx, "k_points_move",
              k_points_move<<<blocks, 256, 0, st>>>(make_view(vx), make_view(vy), make_view(vz), d_in, nn, dt,
                                                    rk4 ? 1 : 0, inv, kx, ky, kz, idx));
    // stable sorts by z, then y, then x: lexicographic (x, y, z), ties in input
    // order.  A sort may leave its result in its scratch, which the next sort
    // reuses, so each pass's permutation is first moved to pbuf.
    const unsigned lim = (1u << 29) - 1u;
    unsigned *ko = nullptr, *perm = nullptr;
    if (cudaMemcpyAsync(kbuf, kz, wb, cudaMemcpyDeviceToDevice, st) != cudaSuccess)
        return fail(check_cuda(ctx, cudaGetLastError(), "key copy"));
    rc = radix_sort_pairs(ctx, kbuf, idx, nn, lim, scratch, &ko, &perm);
    if (rc) return fail(rc);
    const unsigned* axis_keys[2] = {ky, kx};
    for (int pass = 0; pass < 2; ++pass) {
        if (perm != pbuf && cudaMemcpyAsync(pbuf, perm, wb, cudaMemcpyDeviceToDevice, st) != cudaSuccess)
            return fail(check_cuda(ctx, cudaGetLastError(), "permutation copy"));
        k_gather_keys<<<blocks, 256, 0, st>>>(axis_keys[pass], pbuf, nn, kbuf);
        rc = radix_sort_pairs(ctx, kbuf, pbuf, nn, lim, scratch, &ko, &perm);
        if (rc) return fail(rc);
    }
    VLR_TIMED(ctx, "k_points_emit",
              k_points_emit<<<blocks, 256, 0, st>>>(d_in, perm, kx, ky, kz, nn, d_out, head));
    rc = scan_exclusive(ctx, head, rank, nn, d_total);
    if (rc) return fail(rc);
    k_points_leaves<<<blocks, 256, 0, st>>>(perm, kx, ky, kz, head, rank, nn, d_org, d_start);
    if (cudaGetLastError() != cudaSuccess) return fail(check_cuda(ctx, cudaGetLastError(), "k_points_leaves"));
    int leaves = 0;
    rc = read_int(ctx, d_total, &leaves);
    if (rc) return fail(rc);
    *n_leaves = (size_t)leaves;
    if ((size_t)leaves > cap_leaves) {
        fail(VLR_OK);
        return set_error(ctx, VLR_ERR_CAPACITY,
                         "vlr_advect_points: " + std::to_string(leaves) + " leaves exceed cap_leaves");
    }
    VLR_CUDA(ctx, cudaMemcpyAsync(particles, d_out, pb, cudaMemcpyDeviceToHost, st));
    VLR_CUDA(ctx, cudaMemcpyAsync(leaf_origins, d_org, sizeof(int32_t) * 3 * leaves, cudaMemcpyDeviceToHost, st));
    VLR_CUDA(ctx, cudaMemcpyAsync(leaf_start, d_start, sizeof(uint32_t) * leaves, cudaMemcpyDeviceToHost, st));
    VLR_CUDA(ctx, cudaStreamSynchronize(st));
    leaf_start[leaves] = (uint32_t)n;
    cudaFreeAsync(blk, st);
    return consume_device_errors(ctx, "vlr_advect_points");
}

}  // extern "C"
