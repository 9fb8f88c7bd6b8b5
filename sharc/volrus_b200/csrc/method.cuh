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
    int series;            // rotation series order: 0 angles below 0.004 rad, 1 below 0.05 rad, 2 below 1 rad
    int doubling;          // curl: dphi[o] = 2^o dphi[0] exactly (rotations by double-angle formulas)
    long long base[3];     // hash key base (leaf coordinates)
};

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
