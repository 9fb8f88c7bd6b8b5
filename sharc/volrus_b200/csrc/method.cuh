// Device-side definitions of the narrow-band level-set METHOD step
// (semi-Lagrangian RK backtrace with analytic velocity, Godunov-upwind
// reinitialisation, dilation re-tracking).  Values are stored in voxel units
// as f32 or f16; arithmetic is f32.  Positions are split into an integer
// voxel coordinate plus an f32 offset: analytic velocities read per-axis
// sin/cos tables at the integer coordinate (built on the host in f64) and
// rotate them by the small angle of the offset, so sub-voxel accuracy does
// not degrade with the coordinate's magnitude (domains up to 2^24 voxels).
//
// Missing-leaf rule: a voxel of an unallocated leaf, read by a computation
// centred on leaf C, holds copysign(hw, phi_C[clamp(p - origin_C, 0, 7)]).
// For 6-neighbour stencils this is copysign(hw, phi(centre voxel)).
#pragma once
#include <cstdint>
#include <cuda_fp16.h>

#include "vlr_common.cuh"

namespace vlr {

enum : int { MVEL_CONSTANT = 0, MVEL_VORTEX = 1, MVEL_CURL = 2 };
constexpr int kMaxOctaves = 4;

// Per-grid parameters of a method grid (a batch holds one per grid).
struct MGridParams {
    float hw;              // narrow-band half width (voxels)
    int vel_kind;
    float c[3];            // constant velocity, voxels per unit time
    float vel_scale;       // vortex: 1 / voxel_size (world -> index units)
    float pi_over_T;       // vortex: pi / period
    int octaves;           // curl noise
    float ak[kMaxOctaves];     // amplitude * wavenumber per octave
    float e[kMaxOctaves][3];   // potential direction per octave
    float dphi[kMaxOctaves];   // table angle per voxel per family (vortex: pi*vs; curl: k_o)
    int tab_off[kMaxOctaves][3];  // first float2 of family f, axis a
    int tab_lo[3];         // index coordinate of table entry 0 (per axis)
    int tab_len[3];
    int full_series;       // 1: rotation angles may reach 1 rad (full Taylor series); 0: below 0.05 rad
    int doubling;          // curl: dphi[o] = 2^o dphi[0] exactly (rotations by double-angle formulas)
    long long base[3];     // hash key base (leaf coordinates)
};

// sin and cos of |d| < 0.05 (Taylor to d^5 / d^4, error < 3e-10).
__device__ __forceinline__ void tiny_sincos(float d, float& s, float& c) {
    float d2 = d * d;
    s = d * (1.0f - d2 * (1.0f / 6.0f) * (1.0f - d2 * (1.0f / 20.0f)));
    c = 1.0f - d2 * 0.5f * (1.0f - d2 * (1.0f / 12.0f));
}

// Step-wide parameters (shared by all grids of a batch).
struct MStepParams {
    float dt;
    float t0;
    int integrator;        // 1 Euler, 2 RK2 midpoint, 3 SSP-RK3
    int n_grids;
    int key_bits;          // bits per axis in a hash key (21 for one grid, 18 for batches)
    int reinit_mode;       // 0 plain Godunov, 1 Godunov with the subcell fix at cut voxels
};

__device__ __forceinline__ float to_f(float v) { return v; }
__device__ __forceinline__ float to_f(__half v) { return __half2float(v); }
template <typename T> __device__ __forceinline__ T from_f(float v);
template <> __device__ __forceinline__ float from_f<float>(float v) { return v; }
template <> __device__ __forceinline__ __half from_f<__half>(float v) { return __float2half_rn(v); }

// sin and cos of a small angle |d| < 1 (Taylor to d^9 / d^10, error < 3e-9).
__device__ __forceinline__ void small_sincos(float d, float& s, float& c) {
    float d2 = d * d;
    s = d * (1.0f - d2 * (1.0f / 6.0f) * (1.0f - d2 * (1.0f / 20.0f) * (1.0f - d2 * (1.0f / 42.0f) * (1.0f - d2 * (1.0f / 72.0f)))));
    c = 1.0f - d2 * 0.5f * (1.0f - d2 * (1.0f / 12.0f) * (1.0f - d2 * (1.0f / 30.0f) * (1.0f - d2 * (1.0f / 56.0f) * (1.0f - d2 * (1.0f / 90.0f)))));
}

// (sin, cos) of the table angle at integer coordinate i (axis a, family f),
// rotated by dphi * off.  Sets *bad if i lies outside the table.
template <bool kOffset>
__device__ __forceinline__ float2 table_sc(const MGridParams& P, const float2* __restrict__ tab, int f, int a, int i,
                                           float off, unsigned& bad) {
    int k = i - P.tab_lo[a];
    if (k < 0 || k >= P.tab_len[a]) {
        bad = 1u;
        k = min(max(k, 0), P.tab_len[a] - 1);
    }
    float2 t = __ldg(&tab[P.tab_off[f][a] + k]);
    if (!kOffset) return t;
    float sd, cd;
    small_sincos(P.dphi[f] * off, sd, cd);
    return make_float2(t.x * cd + t.y * sd, t.y * cd - t.x * sd);
}

// Velocity in voxels per unit time at position (ix + ox, iy + oy, iz + oz).
// `ct` is the vortex time factor cos(pi t / T).
template <bool kOffset>
__device__ __forceinline__ float3 velocity(const MGridParams& P, const float2* __restrict__ tab, int ix, int iy, int iz,
                                           float ox, float oy, float oz, float ct, unsigned& bad) {
    if (P.vel_kind == MVEL_CONSTANT) return make_float3(P.c[0], P.c[1], P.c[2]);
    if (P.vel_kind == MVEL_VORTEX) {
        float2 X = table_sc<kOffset>(P, tab, 0, 0, ix, ox, bad);
        float2 Y = table_sc<kOffset>(P, tab, 0, 1, iy, oy, bad);
        float2 Z = table_sc<kOffset>(P, tab, 0, 2, iz, oz, bad);
        float k = P.vel_scale * ct;
        // u = 2 sin^2(pi x) sin(2 pi y) sin(2 pi z), v = -sin(2 pi x) sin^2(pi y) sin(2 pi z),
        // w = -sin(2 pi x) sin(2 pi y) sin^2(pi z), times cos(pi t / T), world units / voxel size
        float sycy = Y.x * Y.y, szcz = Z.x * Z.y, sxcx = X.x * X.y;
        return make_float3(8.0f * k * X.x * X.x * sycy * szcz, -4.0f * k * sxcx * Y.x * Y.x * szcz,
                           -4.0f * k * sxcx * sycy * Z.x * Z.x);
    }
    float3 u = make_float3(0.f, 0.f, 0.f);
    for (int o = 0; o < P.octaves; ++o) {
        float2 X = table_sc<kOffset>(P, tab, o, 0, ix, ox, bad);
        float2 Y = table_sc<kOffset>(P, tab, o, 1, iy, oy, bad);
        float2 Z = table_sc<kOffset>(P, tab, o, 2, iz, oz, bad);
        float a = P.ak[o];
        float gx = a * X.y * Y.x * Z.x, gy = a * X.x * Y.y * Z.x, gz = a * X.x * Y.x * Z.y;
        const float* e = P.e[o];
        u.x += gy * e[2] - gz * e[1];
        u.y += gz * e[0] - gx * e[2];
        u.z += gx * e[1] - gy * e[0];
    }
    return u;
}

// Programmatic dependent launch: the kernels of a step are launched with
// programmatic stream serialization, so a kernel's CTAs may be scheduled while
// the previous kernel drains.  dep_wait() blocks until the previous kernel has
// completed and its writes are visible (a no-op for an ordinary launch);
// dep_launch() lets the next kernel's CTAs be scheduled as this kernel's CTAs
// retire.
__device__ __forceinline__ void dep_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void dep_launch() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }

// Error word layout (vlr_ctx::d_errword): [0] error bits of the current
// operation (kErr*), [1] spare, [2] test hook: non-zero makes the look-back
// scan's first chunk withhold its prefix, [3] bound of the device-side waits
// in polls (0: each wait's own default).
//
// A step whose bounded wait gave up, or whose leaf pool or hash overflowed,
// is abandoned: every later kernel of the step, and of any step enqueued
// after it, returns at once while that bit is set, so nothing works on a
// half-built topology (the host reports VLR_ERR_TIMEOUT or VLR_ERR_CAPACITY
// and requires a new state before the next step).
__device__ __forceinline__ bool step_aborted(const unsigned* err) {
    return (*reinterpret_cast<const volatile unsigned*>(err) & (kErrTimeout | kErrCapacity | kErrHashFull)) != 0u;
}
__device__ __forceinline__ long long wait_limit(const unsigned* err, long long dflt) {
    const unsigned v = reinterpret_cast<const volatile unsigned*>(err)[3];
    return v ? (long long)v : dflt;
}
__device__ __forceinline__ bool test_stall(const unsigned* err) {
    return reinterpret_cast<const volatile unsigned*>(err)[2] != 0u;
}

// Hash lookup of a leaf coordinate within a grid (key packs the grid id).
__device__ __forceinline__ uint64_t mkey(long long lx, long long ly, long long lz, int gid, const long long* base,
                                         int bits) {
    long long rx = lx - base[0], ry = ly - base[1], rz = lz - base[2];
    long long lim = 1ll << bits;
    if (rx < 0 || ry < 0 || rz < 0 || rx >= lim || ry >= lim || rz >= lim) return kEmptyKey;
    return (uint64_t)rx | ((uint64_t)ry << bits) | ((uint64_t)rz << (2 * bits)) | ((uint64_t)gid << (3 * bits));
}

__device__ __forceinline__ int hfind(const uint64_t* __restrict__ hkey, const int* __restrict__ hval, int hcap,
                                     uint64_t key) {
    if (key == kEmptyKey) return -1;
    uint32_t m = (uint32_t)hcap - 1u;
    uint32_t p = (uint32_t)mix64(key) & m;
    for (int probe = 0; probe < hcap; ++probe) {
        uint64_t k = hkey[p];
        if (k == key) return hval[p];
        if (k == kEmptyKey) return -1;
        p = (p + 1u) & m;
    }
    return -1;
}

}  // namespace vlr
