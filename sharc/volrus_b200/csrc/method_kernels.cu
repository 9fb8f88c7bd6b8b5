// Kernels of the narrow-band METHOD step.  One CTA works on one 8^3 leaf
// (persistent: CTAs stride over the ordered leaf list, whose length lives in
// device memory so that a whole step can be captured in a CUDA graph).
//
//   k_m_advect     dilation of the activity mask (26-neighbourhood) and the
//                  semi-Lagrangian backtrace (Euler / RK2 / SSP-RK3) of every
//                  dilated voxel, trilinear sampling from a (8+2H)^3 halo tile
//                  of the previous values staged in shared memory
//   k_m_reinit     NIT (0..2) Jacobi iterations of Godunov-upwind
//                  reinitialisation fused in one pass (the first iteration is
//                  evaluated on the 10^3 box around the leaf), then trim to
//                  |phi| < hw, new activity mask and the 26-direction spill
//                  mask used by re-tracking
//   k_m_volume     FP64 smeared-delta surface integral, one partial per leaf
#include "method_kernels.hpp"

namespace vlr {

constexpr int kThreads = 256;

// Leaf offset index (0..26) of the neighbour holding local coordinate c in [-8, 15].
__device__ __forceinline__ int nb_axis(int c) { return (c < 0) ? 0 : (c > 7 ? 2 : 1); }

// --------------------------------------------------------------- advect

template <typename T, int H>
__global__ void __launch_bounds__(kThreads) k_m_advect(MLeafArrays A, const T* __restrict__ src, T* __restrict__ dst,
                                                      const MGridParams* __restrict__ params,
                                                      const float2* __restrict__ tab, MStepParams sp,
                                                      unsigned* __restrict__ err) {
    constexpr int E = 8 + 2 * H;
    __shared__ float s_tile[E * E * E];
    __shared__ int s_nbr[kNbr];
    __shared__ uint64_t s_m[kNbr * 8];
    __shared__ unsigned char s_D[64];
    const int count = *A.count;
    const int step = *A.step;
    const float t1 = sp.t0 + (float)(step + 1) * sp.dt;
    unsigned bad = 0;
    for (int li = blockIdx.x; li < count; li += gridDim.x) {
        const int slot = A.list[li];
        const int4 o = A.origin[slot];
        const MGridParams& P = params[o.w];
        if (threadIdx.x < kNbr) s_nbr[threadIdx.x] = A.nbr[slot * kNbr + threadIdx.x];
        __syncthreads();
        for (int t = threadIdx.x; t < kNbr * 8; t += kThreads) {
            int s = s_nbr[t >> 3];
            s_m[t] = (s < 0) ? 0ull : A.mask[(size_t)s * 8 + (t & 7)];
        }
        const T* csrc = src + (size_t)slot * kLeafVoxels;
        for (int t = threadIdx.x; t < E * E * E; t += kThreads) {
            int sz = t % E, sy = (t / E) % E, sx = t / (E * E);
            int x = sx - H, y = sy - H, z = sz - H;
            int d = nb_axis(x) * 9 + nb_axis(y) * 3 + nb_axis(z);
            int s = s_nbr[d];
            float v;
            if (s >= 0) {
                v = to_f(src[(size_t)s * kLeafVoxels + voxel_off(x, y, z)]);
            } else {
                int cx = min(max(x, 0), 7), cy = min(max(y, 0), 7), cz = min(max(z, 0), 7);
                v = copysignf(P.hw, to_f(csrc[(cx << 6) | (cy << 3) | cz]));
            }
            s_tile[t] = v;
        }
        __syncthreads();
        // D = dilate26(M): one thread per z-row (x, y); 10-bit rows z = -1..8.
        if (threadIdx.x < 64) {
            int x = threadIdx.x >> 3, y = threadIdx.x & 7;
            unsigned acc = 0;
            for (int dx = -1; dx <= 1; ++dx)
                for (int dy = -1; dy <= 1; ++dy) {
                    int xx = x + dx, yy = y + dy;
                    int base = nb_axis(xx) * 9 + nb_axis(yy) * 3;
                    int bi = ((xx & 7) << 3) | (yy & 7);
                    const unsigned char* m0 = (const unsigned char*)&s_m[(base + 0) * 8];
                    const unsigned char* m1 = (const unsigned char*)&s_m[(base + 1) * 8];
                    const unsigned char* m2 = (const unsigned char*)&s_m[(base + 2) * 8];
                    acc |= ((unsigned)m0[bi] >> 7) | ((unsigned)m1[bi] << 1) | (((unsigned)m2[bi] & 1u) << 9);
                }
            s_D[threadIdx.x] = (unsigned char)(((acc | (acc << 1) | (acc >> 1)) >> 1) & 0xffu);
        }
        __syncthreads();
        const float dt = sp.dt;
        float ct1 = 1.f, ct2 = 1.f, ct3 = 1.f;
        if (P.vel_kind == MVEL_VORTEX) {
            ct1 = cosf(P.pi_over_T * t1);
            ct2 = cosf(P.pi_over_T * (t1 - 0.5f * dt));
            ct3 = cosf(P.pi_over_T * (t1 - dt));
        }
        for (int r = 0; r < 2; ++r) {
            const int off = threadIdx.x + kThreads * r;
            const int x = off >> 6, y = (off >> 3) & 7, z = off & 7;
            const int ct = ((x + H) * E + (y + H)) * E + (z + H);
            float out;
            if ((s_D[off >> 3] >> (off & 7)) & 1) {
                const int ix = o.x + x, iy = o.y + y, iz = o.z + z;
                float fx, fy, fz;
                float3 k1 = velocity<false>(P, tab, ix, iy, iz, 0.f, 0.f, 0.f, ct1, bad);
                if (sp.integrator == 1) {
                    fx = -dt * k1.x;
                    fy = -dt * k1.y;
                    fz = -dt * k1.z;
                } else if (sp.integrator == 2) {
                    float3 k2 = velocity<true>(P, tab, ix, iy, iz, -0.5f * dt * k1.x, -0.5f * dt * k1.y,
                                               -0.5f * dt * k1.z, ct2, bad);
                    fx = -dt * k2.x;
                    fy = -dt * k2.y;
                    fz = -dt * k2.z;
                } else {
                    const float h = -dt;
                    float ax = h * k1.x, ay = h * k1.y, az = h * k1.z;              // X1 - x
                    float3 k2 = velocity<true>(P, tab, ix, iy, iz, ax, ay, az, ct3, bad);
                    float bx = 0.25f * (ax + h * k2.x), by = 0.25f * (ay + h * k2.y), bz = 0.25f * (az + h * k2.z);  // X2 - x
                    float3 k3 = velocity<true>(P, tab, ix, iy, iz, bx, by, bz, ct2, bad);
                    fx = (2.0f / 3.0f) * (bx + h * k3.x);
                    fy = (2.0f / 3.0f) * (by + h * k3.y);
                    fz = (2.0f / 3.0f) * (bz + h * k3.z);
                }
                float px = (float)(x + H) + fx, py = (float)(y + H) + fy, pz = (float)(z + H) + fz;
                float bxf = floorf(px), byf = floorf(py), bzf = floorf(pz);
                float wx = px - bxf, wy = py - byf, wz = pz - bzf;
                int i = (int)bxf, j = (int)byf, k = (int)bzf;
                if (i < 0 || j < 0 || k < 0 || i > E - 2 || j > E - 2 || k > E - 2 || !(px == px) || !(py == py) ||
                    !(pz == pz)) {
                    bad = 1u;
                    i = min(max(i, 0), E - 2);
                    j = min(max(j, 0), E - 2);
                    k = min(max(k, 0), E - 2);
                    wx = fminf(fmaxf(wx, 0.f), 1.f);
                    wy = fminf(fmaxf(wy, 0.f), 1.f);
                    wz = fminf(fmaxf(wz, 0.f), 1.f);
                }
                const float* q = &s_tile[(i * E + j) * E + k];
                float c000 = q[0], c001 = q[1], c010 = q[E], c011 = q[E + 1];
                float c100 = q[E * E], c101 = q[E * E + 1], c110 = q[E * E + E], c111 = q[E * E + E + 1];
                float c00 = c000 * (1.f - wx) + c100 * wx, c01 = c001 * (1.f - wx) + c101 * wx;
                float c10 = c010 * (1.f - wx) + c110 * wx, c11 = c011 * (1.f - wx) + c111 * wx;
                float c0 = c00 * (1.f - wy) + c10 * wy, c1 = c01 * (1.f - wy) + c11 * wy;
                out = c0 * (1.f - wz) + c1 * wz;
            } else {
                out = copysignf(P.hw, s_tile[ct]);
            }
            dst[(size_t)slot * kLeafVoxels + off] = from_f<T>(out);
        }
        if (threadIdx.x < 8) A.dmask[(size_t)slot * 8 + threadIdx.x] = ((const uint64_t*)s_D)[threadIdx.x];
        __syncthreads();
    }
    if (bad) atomicOr(err, kErrReach);
}

// -------------------------------------------------------------- reinit

__device__ __forceinline__ float godunov_g(float p, float xm, float xp, float ym, float yp, float zm, float zp, float s) {
    float am[3] = {p - xm, p - ym, p - zm};
    float ap[3] = {xp - p, yp - p, zp - p};
    float g2 = 0.f;
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        float u, w;
        if (s >= 0.f) {
            u = fmaxf(am[a], 0.f);
            w = fminf(ap[a], 0.f);
        } else {
            u = fminf(am[a], 0.f);
            w = fmaxf(ap[a], 0.f);
        }
        g2 += fmaxf(u * u, w * w);
    }
    return sqrtf(g2);
}

// NaN marks a voxel of an unallocated leaf; a 6-neighbour stencil reads it as
// copysign(hw, phi(centre)).
__device__ __forceinline__ float nb(float v, float centre, float hw) { return (v != v) ? copysignf(hw, centre) : v; }

template <typename T, int NIT>
__global__ void __launch_bounds__(kThreads) k_m_reinit(MLeafArrays A, const T* __restrict__ src, T* __restrict__ dst,
                                                      const MGridParams* __restrict__ params) {
    constexpr int E = 12;  // phi1 tile: leaf + 2-voxel ring
    constexpr int F = 10;  // phi2 tile and D rows: leaf + 1-voxel ring
    __shared__ float s_p1[E * E * E];
    __shared__ float s_p2[F * F * F];
    __shared__ unsigned short s_D[F * F];  // bit z+1 = dilated-mask bit of voxel z in [-1, 8]
    __shared__ int s_nbr[kNbr];
    __shared__ unsigned char s_M[64];
    const int count = *A.count;
    for (int li = blockIdx.x; li < count; li += gridDim.x) {
        const int slot = A.list[li];
        const int4 o = A.origin[slot];
        const float hw = params[o.w].hw;
        if (threadIdx.x < kNbr) s_nbr[threadIdx.x] = A.nbr[slot * kNbr + threadIdx.x];
        __syncthreads();
        for (int t = threadIdx.x; t < E * E * E; t += kThreads) {
            int x = t / (E * E) - 2, y = (t / E) % E - 2, z = t % E - 2;
            int s = s_nbr[nb_axis(x) * 9 + nb_axis(y) * 3 + nb_axis(z)];
            s_p1[t] = (s >= 0) ? to_f(src[(size_t)s * kLeafVoxels + voxel_off(x, y, z)]) : __int_as_float(0x7fc00000);
        }
        for (int t = threadIdx.x; t < F * F; t += kThreads) {
            int x = t / F - 1, y = t % F - 1;
            int base = nb_axis(x) * 9 + nb_axis(y) * 3;
            int bi = ((x & 7) << 3) | (y & 7);
            unsigned row = 0;
            int s0 = s_nbr[base], s1 = s_nbr[base + 1], s2 = s_nbr[base + 2];
            if (s0 >= 0) row |= (unsigned)(((const unsigned char*)(A.dmask + (size_t)s0 * 8))[bi] >> 7);
            if (s1 >= 0) row |= (unsigned)((const unsigned char*)(A.dmask + (size_t)s1 * 8))[bi] << 1;
            if (s2 >= 0) row |= ((unsigned)((const unsigned char*)(A.dmask + (size_t)s2 * 8))[bi] & 1u) << 9;
            s_D[t] = (unsigned short)row;
        }
        __syncthreads();
        if (NIT == 2) {
            // first iteration on the 10^3 box
            for (int t = threadIdx.x; t < F * F * F; t += kThreads) {
                int xr = t / (F * F), yr = (t / F) % F, zr = t % F;
                int c = ((xr + 1) * E + (yr + 1)) * E + (zr + 1);
                float p = s_p1[c];
                float q = p;
                if ((s_D[xr * F + yr] >> zr) & 1u) {
                    float s = p * rsqrtf(p * p + 1.0f);
                    float G = godunov_g(p, nb(s_p1[c - E * E], p, hw), nb(s_p1[c + E * E], p, hw),
                                        nb(s_p1[c - E], p, hw), nb(s_p1[c + E], p, hw), nb(s_p1[c - 1], p, hw),
                                        nb(s_p1[c + 1], p, hw), s);
                    q = p - 0.5f * s * (G - 1.0f);
                }
                s_p2[t] = q;
            }
            __syncthreads();
        }
        bool any = false;
        for (int r = 0; r < 2; ++r) {
            const int off = threadIdx.x + kThreads * r;
            const int x = off >> 6, y = (off >> 3) & 7, z = off & 7;
            const bool inD = (s_D[(x + 1) * F + (y + 1)] >> (z + 1)) & 1u;
            const int c1 = ((x + 2) * E + (y + 2)) * E + (z + 2);
            float p1 = s_p1[c1];
            float v;
            if (NIT == 0) {
                v = p1;
            } else if (NIT == 1) {
                v = p1;
                if (inD) {
                    float s = p1 * rsqrtf(p1 * p1 + 1.0f);
                    float G = godunov_g(p1, nb(s_p1[c1 - E * E], p1, hw), nb(s_p1[c1 + E * E], p1, hw),
                                        nb(s_p1[c1 - E], p1, hw), nb(s_p1[c1 + E], p1, hw), nb(s_p1[c1 - 1], p1, hw),
                                        nb(s_p1[c1 + 1], p1, hw), s);
                    v = p1 - 0.5f * s * (G - 1.0f);
                }
            } else {
                const int c2 = ((x + 1) * F + (y + 1)) * F + (z + 1);
                float p2 = s_p2[c2];
                v = p2;
                if (inD) {
                    float s = p1 * rsqrtf(p1 * p1 + 1.0f);
                    float G = godunov_g(p2, nb(s_p2[c2 - F * F], p2, hw), nb(s_p2[c2 + F * F], p2, hw),
                                        nb(s_p2[c2 - F], p2, hw), nb(s_p2[c2 + F], p2, hw), nb(s_p2[c2 - 1], p2, hw),
                                        nb(s_p2[c2 + 1], p2, hw), s);
                    v = p2 - 0.5f * s * (G - 1.0f);
                }
            }
            bool on = inD && fabsf(v) < hw;
            if (!on) v = copysignf(hw, v);
            dst[(size_t)slot * kLeafVoxels + off] = from_f<T>(v);
            unsigned b = __ballot_sync(0xffffffffu, on);
            if ((threadIdx.x & 31) == 0) ((unsigned*)(A.mask + (size_t)slot * 8))[off >> 5] = b;
            if ((threadIdx.x & 31) == 0) ((unsigned*)s_M)[off >> 5] = b;
            any |= on;
        }
        __syncthreads();
        // spill mask: bit d (leaf offset (dx,dy,dz)) set if an active voxel lies on
        // the boundary layer facing that neighbour.
        if (threadIdx.x < kNbr) {
            int d = threadIdx.x;
            int dx = d / 9 - 1, dy = (d / 3) % 3 - 1, dz = d % 3 - 1;
            unsigned zsel = (dz < 0) ? 0x01u : (dz > 0 ? 0x80u : 0xffu);
            int x0 = (dx < 0) ? 0 : (dx > 0 ? 7 : 0), x1 = (dx < 0) ? 0 : 7;
            int y0 = (dy < 0) ? 0 : (dy > 0 ? 7 : 0), y1 = (dy < 0) ? 0 : 7;
            bool sp = false;
            for (int x = x0; x <= x1 && !sp; ++x)
                for (int y = y0; y <= y1; ++y)
                    if (s_M[x * 8 + y] & zsel) {
                        sp = true;
                        break;
                    }
            unsigned bits = __ballot_sync(0x07ffffffu, sp && d != 13);
            if (d == 0) A.spill[slot] = bits;
        }
        int a = __syncthreads_or(any);
        if (threadIdx.x == 0) A.nonempty[slot] = a;
    }
}

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
        if (threadIdx.x < kNbr) s_nbr[threadIdx.x] = A.nbr[slot * kNbr + threadIdx.x];
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
    template __global__ void k_m_advect<T, 2>(MLeafArrays, const T*, T*, const MGridParams*, const float2*,        \
                                              MStepParams, unsigned*);                                           \
    template __global__ void k_m_advect<T, 3>(MLeafArrays, const T*, T*, const MGridParams*, const float2*,        \
                                              MStepParams, unsigned*);                                           \
    template __global__ void k_m_reinit<T, 0>(MLeafArrays, const T*, T*, const MGridParams*);                      \
    template __global__ void k_m_reinit<T, 1>(MLeafArrays, const T*, T*, const MGridParams*);                      \
    template __global__ void k_m_reinit<T, 2>(MLeafArrays, const T*, T*, const MGridParams*);                      \
    template __global__ void k_m_volume<T>(MLeafArrays, const T*, const MGridParams*, double, double, double,      \
                                           double*);                                                             \
    template __global__ void k_m_sphere<T>(int, int, int, int, int, int, double, double, double, double, double,   \
                                           double, double, double, double, int4*, uint64_t*, T*, int*);
VLR_INST_T(float)
VLR_INST_T(__half)

}  // namespace vlr
