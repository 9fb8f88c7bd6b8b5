// Declarations shared by the method kernels and their host orchestration.
#pragma once

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

constexpr int kAdvectThreads = 128;
constexpr int kReinitThreads = 128;
// The advect kernel (method_advect.cu): 128 threads per CTA, persistent over
// the leaf list.  VK: velocity kind of every grid (MVEL_*), or -1 when a batch
// mixes kinds.  The result depends neither on the grid size nor on VK.
template <typename T, int H, int VK>
__global__ void k_m_advect(MLeafArrays A, const T* __restrict__ src, T* __restrict__ dst,
                           const MGridParams* __restrict__ params, const float2* __restrict__ tab, MStepParams sp,
                           MTopo topo, unsigned* __restrict__ err);
// The reinitialisation kernel (method_reinit.cu): NIT iterations (0..2),
// FIX = 1 with the subcell fix at cut voxels; 128 threads per CTA.
template <typename T, int NIT, int FIX>
__global__ void k_m_reinit(MLeafArrays A, const T* __restrict__ src, T* __restrict__ dst,
                           const MGridParams* __restrict__ params, MTopo topo, unsigned* __restrict__ err);
// Dynamic shared memory of the stencil kernels (bytes).
size_t advect_smem_bytes(int precision_f16, int halo);
size_t reinit_smem_bytes(int precision_f16, int nit, int fix);
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
