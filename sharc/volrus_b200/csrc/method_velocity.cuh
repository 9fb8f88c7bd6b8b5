// Velocity evaluation and semi-Lagrangian backtrace of the METHOD step,
// shared by the advect kernel and by the frozen-band adjoint's displacement
// kernel (k_m_feet), so that the adjoint differentiates exactly the step the
// forward takes.
//
// Analytic velocities are evaluated at integer voxel coordinate i plus an f32
// offset: per-axis (sin, cos) table entries at i (built on the host in f64)
// are rotated by the small angle dphi * offset, whose sine and cosine come
// from a Taylor series (the series order is chosen per grid from the largest
// angle a step can reach, so every order used is exact to well below f32
// resolution); curl-noise octaves whose wavenumbers double reuse octave 0's
// rotation through the double-angle formulas.
#pragma once
#include "method.cuh"

namespace vlr {

// Rotation series orders (MGridParams::series): the largest rotation angle a
// step reaches is below 0.004 rad (order 0), 0.05 rad (order 1) or 1 rad (2).
enum : int { kSeriesMicro = 0, kSeriesTiny = 1, kSeriesFull = 2 };

// Per-grid velocity constants held in registers for a leaf.  ae[o] is octave
// o's amplitude times its potential direction (a_o e_o).
struct VelConst {
    int kind;
    int octaves;
    int doubling;  // curl: octave o's table angle per voxel is 2^o times octave 0's
    float c[3];
    float scale;  // vortex: vel_scale
    float dphi[kMaxOctaves];
    float ae[kMaxOctaves][3];
};

__device__ __forceinline__ VelConst vel_const(const MGridParams& P) {
    VelConst V;
    V.kind = P.vel_kind;
    V.octaves = P.octaves;
    V.doubling = P.doubling;
    V.scale = P.vel_scale;
#pragma unroll
    for (int a = 0; a < 3; ++a) V.c[a] = P.c[a];
#pragma unroll
    for (int o = 0; o < kMaxOctaves; ++o) {
        V.dphi[o] = P.dphi[o];
#pragma unroll
        for (int a = 0; a < 3; ++a) V.ae[o][a] = P.ak[o] * P.e[o][a];
    }
    return V;
}

// sin and cos of a rotation angle d for series order SER:
//   micro (|d| < 0.004): d - d^3/6 and 1 - d^2/2   (errors < 1e-14, 1.1e-11)
//   tiny  (|d| < 0.05):  to d^5 and d^4            (error < 3e-10)
//   full  (|d| < 1):     to d^9 and d^10           (error < 3e-9)
template <int SER>
__device__ __forceinline__ void series_sincos(float d, float& s, float& c) {
    const float d2 = d * d;
    if constexpr (SER == kSeriesMicro) {
        s = __fmaf_rn(-(d * d2), 1.0f / 6.0f, d);
        c = __fmaf_rn(-0.5f, d2, 1.0f);
    } else if constexpr (SER == kSeriesTiny) {
        s = d * (1.0f - d2 * (1.0f / 6.0f) * (1.0f - d2 * (1.0f / 20.0f)));
        c = 1.0f - d2 * 0.5f * (1.0f - d2 * (1.0f / 12.0f));
    } else {
        s = d * (1.0f - d2 * (1.0f / 6.0f) *
                            (1.0f - d2 * (1.0f / 20.0f) * (1.0f - d2 * (1.0f / 42.0f) * (1.0f - d2 * (1.0f / 72.0f)))));
        c = 1.0f - d2 * 0.5f *
                       (1.0f - d2 * (1.0f / 12.0f) *
                                   (1.0f - d2 * (1.0f / 30.0f) * (1.0f - d2 * (1.0f / 56.0f) * (1.0f - d2 * (1.0f / 90.0f)))));
    }
}

// (sin, cos) of (table angle + rotation angle) from the table pair and the
// rotation's sine and cosine.
__device__ __forceinline__ float2 rot(float2 t, float sd, float cd) {
    return make_float2(__fmaf_rn(t.y, sd, t.x * cd), __fmaf_rn(-t.x, sd, t.y * cd));
}

template <int SER>
__device__ __forceinline__ float2 rotate(float2 t, float d) {
    float sd, cd;
    series_sincos<SER>(d, sd, cd);
    return rot(t, sd, cd);
}

// Curl-noise octave o's contribution a_o (grad f_o x e_o) from its rotated
// (sin, cos) pairs per axis; grad f_o / a_o = (cx sy sz, sx cy sz, sx sy cz).
__device__ __forceinline__ void curl_octave(const VelConst& V, int o, float2 X, float2 Y, float2 Z, float3& u) {
    const float gx = X.y * (Y.x * Z.x), gy = X.x * (Y.y * Z.x), gz = X.x * (Y.x * Z.y);
    u.x = __fmaf_rn(gy, V.ae[o][2], __fmaf_rn(-gz, V.ae[o][1], u.x));
    u.y = __fmaf_rn(gz, V.ae[o][0], __fmaf_rn(-gx, V.ae[o][2], u.y));
    u.z = __fmaf_rn(gx, V.ae[o][1], __fmaf_rn(-gy, V.ae[o][0], u.z));
}

// Octave count of a curl field: OC > 0 fixes it at compile time, OC = 0
// takes V.octaves.
template <int OC>
__device__ __forceinline__ bool octave_on(const VelConst& V, int o) {
    return OC > 0 ? (o < OC) : (o < V.octaves);
}

// Velocity (voxels per unit time) at local voxel (lx, ly, lz) + offset, from
// the leaf's staged sin/cos tables (tab[family][axis][local coordinate]).
// kOff = false: no offset (voxel centre).  `ct` is the vortex time factor.
template <int VK, int OC, int SER, bool kOff>
__device__ __forceinline__ float3 leaf_velocity(const VelConst& V, const float2 (*tab)[3][8], int lx, int ly, int lz,
                                                float ox, float oy, float oz, float ct) {
    const int kind = (VK >= 0) ? VK : V.kind;
    if (kind == MVEL_CONSTANT) return make_float3(V.c[0], V.c[1], V.c[2]);
    if (kind == MVEL_VORTEX) {
        float2 X = tab[0][0][lx], Y = tab[0][1][ly], Z = tab[0][2][lz];
        if (kOff) {
            X = rotate<SER>(X, V.dphi[0] * ox);
            Y = rotate<SER>(Y, V.dphi[0] * oy);
            Z = rotate<SER>(Z, V.dphi[0] * oz);
        }
        // u = 2 sin^2(pi x) sin(2 pi y) sin(2 pi z), v = -sin(2 pi x) sin^2(pi y) sin(2 pi z),
        // w = -sin(2 pi x) sin(2 pi y) sin^2(pi z), times cos(pi t / T), world units / voxel size
        const float k = V.scale * ct;
        const float sycy = Y.x * Y.y, szcz = Z.x * Z.y, sxcx = X.x * X.y;
        return make_float3(8.0f * k * X.x * X.x * sycy * szcz, -4.0f * k * sxcx * Y.x * Y.x * szcz,
                           -4.0f * k * sxcx * sycy * Z.x * Z.x);
    }
    float3 u = make_float3(0.f, 0.f, 0.f);
    if (kOff && V.doubling) {
        // octave o rotates by 2^o times octave 0's angle: one series per axis,
        // then sin 2a = 2 sin a cos a, cos 2a = 1 - 2 sin^2 a between octaves
        float sx, cx, sy, cy, sz, cz;
        series_sincos<SER>(V.dphi[0] * ox, sx, cx);
        series_sincos<SER>(V.dphi[0] * oy, sy, cy);
        series_sincos<SER>(V.dphi[0] * oz, sz, cz);
#pragma unroll
        for (int o = 0; o < kMaxOctaves; ++o) {
            if (octave_on<OC>(V, o)) {
                curl_octave(V, o, rot(tab[o][0][lx], sx, cx), rot(tab[o][1][ly], sy, cy), rot(tab[o][2][lz], sz, cz),
                            u);
                if (octave_on<OC>(V, o + 1)) {
                    float t = sx + sx;
                    float n = t * cx;
                    cx = __fmaf_rn(-t, sx, 1.0f);
                    sx = n;
                    t = sy + sy;
                    n = t * cy;
                    cy = __fmaf_rn(-t, sy, 1.0f);
                    sy = n;
                    t = sz + sz;
                    n = t * cz;
                    cz = __fmaf_rn(-t, sz, 1.0f);
                    sz = n;
                }
            }
        }
        return u;
    }
#pragma unroll
    for (int o = 0; o < kMaxOctaves; ++o) {
        if (octave_on<OC>(V, o)) {
            float2 X = tab[o][0][lx], Y = tab[o][1][ly], Z = tab[o][2][lz];
            if (kOff) {
                X = rotate<SER>(X, V.dphi[o] * ox);
                Y = rotate<SER>(Y, V.dphi[o] * oy);
                Z = rotate<SER>(Z, V.dphi[o] * oz);
            }
            curl_octave(V, o, X, Y, Z, u);
        }
    }
    return u;
}

// Backtrace displacement (voxels) of local voxel (x, y, z) over one step:
// Euler (integrator 1), RK2 midpoint (2) or SSP-RK3 (3), velocities from the
// leaf's staged sin/cos tables at the stage times' cosine factors.
template <int VK, int OC, int SER>
__device__ __forceinline__ float3 backtrace(const VelConst& V, const float2 (*s_tab)[3][8], int x, int y, int z,
                                            float dt, int integrator, float ct1, float ct2, float ct3) {
    float fx, fy, fz;
    const float3 k1 = leaf_velocity<VK, OC, SER, false>(V, s_tab, x, y, z, 0.f, 0.f, 0.f, ct1);
    if (integrator == 1) {
        fx = -dt * k1.x;
        fy = -dt * k1.y;
        fz = -dt * k1.z;
    } else if (integrator == 2) {
        const float3 k2 = leaf_velocity<VK, OC, SER, true>(V, s_tab, x, y, z, -0.5f * dt * k1.x, -0.5f * dt * k1.y,
                                                           -0.5f * dt * k1.z, ct2);
        fx = -dt * k2.x;
        fy = -dt * k2.y;
        fz = -dt * k2.z;
    } else {
        const float h = -dt;
        const float ax = h * k1.x, ay = h * k1.y, az = h * k1.z;
        const float3 k2 = leaf_velocity<VK, OC, SER, true>(V, s_tab, x, y, z, ax, ay, az, ct3);
        const float bx = 0.25f * __fmaf_rn(h, k2.x, ax), by = 0.25f * __fmaf_rn(h, k2.y, ay),
                    bz = 0.25f * __fmaf_rn(h, k2.z, az);
        const float3 k3 = leaf_velocity<VK, OC, SER, true>(V, s_tab, x, y, z, bx, by, bz, ct2);
        fx = (2.0f / 3.0f) * __fmaf_rn(h, k3.x, bx);
        fy = (2.0f / 3.0f) * __fmaf_rn(h, k3.y, by);
        fz = (2.0f / 3.0f) * __fmaf_rn(h, k3.z, bz);
    }
    return make_float3(fx, fy, fz);
}

// The backtrace instance for a grid's octave count (3 fixed at compile time,
// else taken at run time) and series order; uniform over a leaf.
template <int VK>
__device__ __forceinline__ float3 backtrace_any(const VelConst& V, int series, const float2 (*s_tab)[3][8], int x,
                                                int y, int z, float dt, int integrator, float ct1, float ct2,
                                                float ct3) {
    const bool oc3 = V.octaves == 3;
    if (series == kSeriesMicro)
        return oc3 ? backtrace<VK, 3, kSeriesMicro>(V, s_tab, x, y, z, dt, integrator, ct1, ct2, ct3)
                   : backtrace<VK, 0, kSeriesMicro>(V, s_tab, x, y, z, dt, integrator, ct1, ct2, ct3);
    if (series == kSeriesTiny)
        return oc3 ? backtrace<VK, 3, kSeriesTiny>(V, s_tab, x, y, z, dt, integrator, ct1, ct2, ct3)
                   : backtrace<VK, 0, kSeriesTiny>(V, s_tab, x, y, z, dt, integrator, ct1, ct2, ct3);
    return oc3 ? backtrace<VK, 3, kSeriesFull>(V, s_tab, x, y, z, dt, integrator, ct1, ct2, ct3)
               : backtrace<VK, 0, kSeriesFull>(V, s_tab, x, y, z, dt, integrator, ct1, ct2, ct3);
}

}  // namespace vlr
