// Non-stencil kernels of the narrow-band METHOD (the stencils are in
// method_stencil.cu).  One CTA works on one 8^3 leaf; CTAs stride over the
// ordered leaf list, whose length lives in device memory.
//
//   k_m_volume     FP64 smeared-delta surface integral, one partial per leaf
//   k_reduce_fixed fixed-order FP64 reduction of the partials
//   k_m_sphere     initial state of a sphere (f64 SDF as the oracle computes it)
#include "method_kernels.hpp"

namespace vlr {

constexpr int kThreads = 256;

// Leaf offset index (0..26) of the neighbour holding local coordinate c in [-8, 15].
__device__ __forceinline__ int nb_axis(int c) { return (c < 0) ? 0 : (c > 7 ? 2 : 1); }

// -------------------------------------------------------------- volume

// delta_eps(phi) (p - ref) . grad phi per active voxel with |phi| < eps, summed
// per leaf in a fixed order (FP64).
template <typename T>
__global__ void __launch_bounds__(kThreads) k_m_volume(MLeafArrays A, const T* __restrict__ vals,
                                                      const MGridParams* __restrict__ params, double r0, double r1,
                                                      double r2, double* __restrict__ partial) {
    __shared__ double s_red[kThreads];
    __shared__ int s_nbr[kNbr];
    const int count = *A.count;
    const double pi = 3.14159265358979323846, eps = 1.5;
    for (int li = blockIdx.x; li < count; li += gridDim.x) {
        const int slot = A.list[li];
        const int4 o = A.origin[slot];
        const float hw = params[o.w].hw;
        if (threadIdx.x < kNbr) s_nbr[threadIdx.x] = A.nbr[(size_t)slot * kNbr + threadIdx.x];
        __syncthreads();
        double acc = 0.0;
        for (int r = 0; r < 2; ++r) {
            const int off = threadIdx.x + kThreads * r;
            if (!mask_bit(A.mask + (size_t)slot * 8, off)) continue;
            double p = (double)to_f(vals[(size_t)slot * kLeafVoxels + off]);
            if (fabs(p) >= eps) continue;
            const int x = off >> 6, y = (off >> 3) & 7, z = off & 7;
            auto rd = [&](int xx, int yy, int zz) -> double {
                int s = s_nbr[nb_axis(xx) * 9 + nb_axis(yy) * 3 + nb_axis(zz)];
                if (s < 0) return (double)copysignf(hw, (float)p);
                return (double)to_f(vals[(size_t)s * kLeafVoxels + voxel_off(xx, yy, zz)]);
            };
            double gx = 0.5 * (rd(x + 1, y, z) - rd(x - 1, y, z));
            double gy = 0.5 * (rd(x, y + 1, z) - rd(x, y - 1, z));
            double gz = 0.5 * (rd(x, y, z + 1) - rd(x, y, z - 1));
            double delta = (1.0 + cos(pi * p / eps)) / (2.0 * eps);
            acc += delta * (((double)(o.x + x) - r0) * gx + ((double)(o.y + y) - r1) * gy + ((double)(o.z + z) - r2) * gz);
        }
        s_red[threadIdx.x] = acc;
        __syncthreads();
        for (int w = kThreads / 2; w > 0; w >>= 1) {
            if (threadIdx.x < w) s_red[threadIdx.x] += s_red[threadIdx.x + w];
            __syncthreads();
        }
        if (threadIdx.x == 0) partial[li] = s_red[0] / 3.0;
        __syncthreads();
    }
}

// Fixed-order reduction of n doubles by one block (deterministic).
__global__ void __launch_bounds__(1024) k_reduce_fixed(const double* __restrict__ in, const int* __restrict__ n_ptr,
                                                      double* __restrict__ out) {
    __shared__ double s[1024];
    int n = *n_ptr;
    double a = 0.0;
    for (int i = threadIdx.x; i < n; i += 1024) a += in[i];
    s[threadIdx.x] = a;
    __syncthreads();
    for (int w = 512; w > 0; w >>= 1) {
        if (threadIdx.x < w) s[threadIdx.x] += s[threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x == 0) *out = s[0];
}

// ---------------------------------------------------------------- init

// Sphere initial state: candidate leaf c of the box [lo, lo + n) (leaf units);
// phi = (|w0 + vs p - centre| - r) / vs in f64 (same expression as the oracle).
template <typename T>
__global__ void __launch_bounds__(kThreads) k_m_sphere(int lx0, int ly0, int lz0, int ny, int nz, int n_cand,
                                                      double r, double c0, double c1, double c2, double vs,
                                                      double w00, double w01, double w02, double hwd, int4* origin,
                                                      uint64_t* mask, T* vals, int* touched) {
    __shared__ int s_touch;
    for (int cand = blockIdx.x; cand < n_cand; cand += gridDim.x) {
        int lx = lx0 + cand / (ny * nz), ly = ly0 + (cand / nz) % ny, lz = lz0 + cand % nz;
        if (threadIdx.x == 0) s_touch = 0;
        __syncthreads();
        auto phi_at = [&](int x, int y, int z) -> double {
            double dx = __dsub_rn(__dadd_rn(w00, __dmul_rn(vs, (double)x)), c0);
            double dy = __dsub_rn(__dadd_rn(w01, __dmul_rn(vs, (double)y)), c1);
            double dz = __dsub_rn(__dadd_rn(w02, __dmul_rn(vs, (double)z)), c2);
            double d = __dsqrt_rn(__dadd_rn(__dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy)), __dmul_rn(dz, dz)));
            return __ddiv_rn(__dsub_rn(d, r), vs);
        };
        bool t_any = false;
        for (int t = threadIdx.x; t < 1000; t += kThreads) {
            int x = t / 100 - 1, y = (t / 10) % 10 - 1, z = t % 10 - 1;
            if (fabs(phi_at(lx * 8 + x, ly * 8 + y, lz * 8 + z)) < hwd) t_any = true;
        }
        if (t_any) s_touch = 1;
        __syncthreads();
        for (int rr = 0; rr < 2; ++rr) {
            int off = threadIdx.x + kThreads * rr;
            double p = phi_at(lx * 8 + (off >> 6), ly * 8 + ((off >> 3) & 7), lz * 8 + (off & 7));
            bool on = fabs(p) < hwd;
            float v = on ? (float)p : copysignf((float)hwd, (float)p);
            vals[(size_t)cand * kLeafVoxels + off] = from_f<T>(v);
            unsigned b = __ballot_sync(0xffffffffu, on);
            if ((threadIdx.x & 31) == 0) ((unsigned*)(mask + (size_t)cand * 8))[off >> 5] = b;
        }
        if (threadIdx.x == 0) {
            origin[cand] = make_int4(lx * 8, ly * 8, lz * 8, 0);
            touched[cand] = s_touch;
        }
        __syncthreads();
    }
}

// ------------------------------------------------------- instantiations

#define VLR_INST_T(T)                                                                                            \
    template __global__ void k_m_volume<T>(MLeafArrays, const T*, const MGridParams*, double, double, double,      \
                                           double*);                                                             \
    template __global__ void k_m_sphere<T>(int, int, int, int, int, int, double, double, double, double, double,   \
                                           double, double, double, double, int4*, uint64_t*, T*, int*);
VLR_INST_T(float)
VLR_INST_T(__half)

}  // namespace vlr
