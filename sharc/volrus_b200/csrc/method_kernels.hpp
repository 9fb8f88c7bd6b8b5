// Declarations shared by the method kernels and their host orchestration.
#pragma once
#include <cuda.h>  // CUtensorMap (a plain 128-byte struct; no driver library is linked)

#include "method.cuh"

namespace vlr {

// Slot-indexed leaf arrays of a method grid plus its ordered leaf list.
struct MLeafArrays {
    const int* list;     // list[i] = slot of the i-th leaf in processing order
    const int* count;    // device scalar: number of list entries
    const int* step;     // device scalar: steps taken since creation
    const int4* origin;  // {x, y, z, grid id}
    uint64_t* mask;      // activity
    uint64_t* dmask;     // dilated activity of the current step (written by advect)
    const int* nbr;      // 27 neighbour slots per slot
    unsigned* spill;     // 27-bit mask per slot of absent neighbours the band spills into (written by reinit)
    int* nonempty;       // 1 if the slot has an active voxel after the step
};

// Per-step topology state touched by the stencil kernels: advect clears it,
// reinit records keep flags and new-leaf proposals.
struct MTopo {
    int* keep;           // cap: leaf survives this step
    int cap;
    uint64_t* pkey;      // proposal table: key -> min owner direction
    int* pval;
    uint64_t* hkey;      // leaf hash, rebuilt each step
    int* hval;
    int hcap;
    int* scalars;        // [7] chunk ticket of the look-back scan
    int key_bits;
};

// Tensor maps of a stencil kernel's source value pool for staging mode 1, one
// box shape per map, with ey = (i & 1 ? 8 : H) and ex = (i & 2 ? 8 : H):
//   maps 0-3: 3-D view (yz, x, slot) of the pool, where yz = y * 8 + z runs
//             over the 64 contiguous values of an x-plane; box {ey * 8, ex, 1}
//             (whole z-rows, so a box row is ey * 8 contiguous values)
//   maps 4-7: 4-D view (z, y, x, slot); box {4, ey, ex, 1} (the f32 z-halves)
// f16 pools use maps 0-3, f32 pools 0-7.
struct StageMaps {
    CUtensorMap m[8];
};

// Staging of the stencil kernels' halo tiles (ST): 0 = asynchronous 16-byte
// copies by every thread (cp.async), 1 = one tensor copy per present
// neighbour leaf (cp.async.bulk.tensor, TMA) completing on an mbarrier.
// VK: velocity kind of every grid (MVEL_*), or -1 when a batch mixes kinds.
// NT: threads per CTA (128 or 256); the result depends neither on NT, on ST
// nor on the grid size.
template <typename T, int H, int VK, int NT, int ST>
__global__ void k_m_advect(MLeafArrays A, const T* __restrict__ src, T* __restrict__ dst,
                           const MGridParams* __restrict__ params, const float2* __restrict__ tab, MStepParams sp,
                           MTopo topo, unsigned* __restrict__ err, const __grid_constant__ StageMaps maps);
// Dynamic shared memory of the stencil kernels (bytes).
size_t advect_smem_bytes(int precision_f16, int halo, int stage);
size_t reinit_smem_bytes(int precision_f16, int stage);
template <typename T, int NIT, int NT, int ST>
__global__ void k_m_reinit(MLeafArrays A, const T* __restrict__ src, T* __restrict__ dst,
                           const MGridParams* __restrict__ params, MTopo topo, int mode, unsigned* __restrict__ err,
                           const __grid_constant__ StageMaps maps);
// Backtrace displacement (voxels) of the voxels of n leaves with bidx >= 0
// over one step of a time-independent velocity (VK = MVEL_CONSTANT or
// MVEL_CURL), k_m_advect's arithmetic; *maxabs collects the largest component
// magnitude (float bits).  128 threads per CTA.
template <int VK>
__global__ void k_m_feet(const int4* __restrict__ origin, int n, const int* __restrict__ bidx,
                         const MGridParams* __restrict__ params, const float2* __restrict__ tab, float dt,
                         int integrator, float3* __restrict__ disp, unsigned* __restrict__ maxabs,
                         unsigned* __restrict__ err);
template <typename T>
__global__ void k_m_volume(MLeafArrays A, const T* __restrict__ vals, const MGridParams* __restrict__ params,
                           double r0, double r1, double r2, double* __restrict__ partial);
__global__ void k_reduce_fixed(const double* __restrict__ in, const int* __restrict__ n_ptr, double* __restrict__ out);
template <typename T>
__global__ void k_m_sphere(int lx0, int ly0, int lz0, int ny, int nz, int n_cand, double r, double c0, double c1,
                           double c2, double vs, double w00, double w01, double w02, double hwd, int4* origin,
                           uint64_t* mask, T* vals, int* touched);

}  // namespace vlr
