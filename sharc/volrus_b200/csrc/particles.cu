// advect_particles / advect_particles_euler (src/tools/advection.rs:58-110)
// on particle positions: RK4 (or forward Euler) through a VelocityField of
// three grids.  VelocityField::sample is three sample_trilinear calls widened
// to f64 (src/tools/advection.rs:16-24); the position arithmetic is f64 in the
// reference's order, with explicitly rounded operations so nothing is
// contracted into an FMA.  The PointDataGrid's re-binning of particles into
// leaves (src/points) stays with the caller: positions in, positions out.
#include "ref_ops.hpp"

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

}  // extern "C"
