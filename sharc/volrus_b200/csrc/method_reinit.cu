// The reinitialisation kernel of the METHOD step: NIT (0..2) Jacobi
// iterations of Godunov-upwind reinitialisation fused in one pass (the first
// iteration runs on the 10^3 box around the leaf so that the second needs no
// exchange), trim to |phi| < hw, the new activity mask, and the re-tracking
// bookkeeping: keep flags and proposals of missing neighbour leaves the band
// spills into.
//
// One CTA of 128 threads works on one 8^3 leaf at a time and strides over the
// ordered leaf list (persistent).  Per leaf:
//
//   stage      the advected field around the leaf, 2-voxel halo, row-packed
//              as in the advect kernel (tile row (x, y) holds z in [-4, 12)),
//              and the 27 neighbours' dilated masks arrive by cp.async one
//              leaf ahead into the other of two buffers.  The pieces of
//              absent leaves are set to NaN when the copies are issued, so
//              the stage is complete at its barrier; a 6-neighbour stencil
//              reads NaN as copysign(hw, its centre value), which needs no
//              work in the common case (see godunov_update_raw).
//   phase 1    warp 0 compacts the box voxels of D for iteration 1 (the
//              10^3 box around the leaf without its edges and corners, which
//              iteration 2 never reads) and keeps their bit words; warp 1
//              compacts the leaf's voxels of D; warps 1-3 issue the next
//              leaf's copies and write every voxel's outside-D result
//              copysign(hw, value) to global memory (coalesced).
//   phase 2    iteration 1 on the box list, consecutive voxels on
//              consecutive lanes (bank-conflict-free stage reads), into phi2.
//   phase 3    iteration 2 (or the only one) on the leaf list, its
//              neighbours from phi2 where the box bit is set and from the
//              stage (phi1) elsewhere; trim, stores over the outside-D
//              results, activity bits into a shared mask.
//   phase 4    mask out, spill toward absent neighbours, keep flags and
//              proposals (hash of the missing leaf, atomicMin of the
//              proposer's direction), by warp 3 during the next leaf's
//              phase 1 (its mask words, neighbour row, slot and origin kept
//              in shared memory), after the loop for the CTA's last leaf.
//
// Three CTA barriers per leaf (two without iteration 1).  Neighbour rows
// are loaded one leaf before the iteration that stores them, so no global
// load waits in front of a barrier.  Every leaf is computed by one CTA with
// the same arithmetic whatever the grid size; side effects on shared
// per-step state are idempotent (flags set to 1, atomicMin), so relaunching
// the kernel on the same inputs leaves the step's result unchanged.
#include "method_kernels.hpp"

namespace vlr {
namespace {

constexpr int kNT = kReinitThreads;
constexpr int kNW = kNT / 32;
constexpr int kH = 2;                            // halo of the stage
constexpr int kE = 8 + 2 * kH;                   // 12: stage rows per axis
constexpr int kF = 10;                           // phi2 box and D rows: leaf + 1-voxel ring
constexpr int kBox = kF * kF * kF;               // 1000 voxels of the phi2 box

__device__ __forceinline__ int nb_axis(int c) { return (c < 0) ? 0 : (c > 7 ? 2 : 1); }
__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void cp_async16(void* dst, const void* src) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(smem_u32(dst)), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async8(void* dst, const void* src) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(smem_u32(dst)), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }

// Staged row layout (as in the advect kernel): RP values, z = 0 at Z0.
template <typename T>
struct Row {
    static constexpr int RP = sizeof(T) == 2 ? 24 : 16;
    static constexpr int Z0 = sizeof(T) == 2 ? 8 : 4;
};

// One piece of a stage row: 8 values (full: the own z range) or 4 (a half
// row of a z neighbour) of leaf slot sl from value `off`, by asynchronous
// copy; NaN when the leaf is absent.
template <typename T>
__device__ __forceinline__ void stage_piece(int sl, const T* __restrict__ vals, int off, T* dst, bool full) {
    if (sl < 0) {
        if constexpr (sizeof(T) == 2) {
            const uint64_t nan4 = 0x7e007e007e007e00ull;
            uint64_t* o = reinterpret_cast<uint64_t*>(dst);
            o[0] = nan4;
            if (full) o[1] = nan4;
        } else {
            const unsigned nan = 0x7fc00000u;
            uint4* o = reinterpret_cast<uint4*>(dst);
            o[0] = make_uint4(nan, nan, nan, nan);
            if (full) o[1] = make_uint4(nan, nan, nan, nan);
        }
        return;
    }
    const T* src = vals + (size_t)sl * kLeafVoxels + off;
    if constexpr (sizeof(T) == 2) {
        if (full) cp_async16(dst, src);
        else cp_async8(dst, src);
    } else {
        cp_async16(dst, src);
        if (full) cp_async16(dst + 4, src + 4);
    }
}

// One leaf's stage, one tile row (x, y) at a time with its three pieces from
// the z-lower, own and z-upper leaves of that column (NaN for absent leaves),
// and the 27 dilated masks (zero for absent leaves), by a group of ns
// threads, this thread being number t.
template <typename T>
__device__ __forceinline__ void issue_stage(const int* s_nb, const T* __restrict__ vals,
                                            const uint64_t* __restrict__ masks, T* stage, uint64_t* s_m, int t,
                                            int ns) {
    constexpr int RP = Row<T>::RP, Z0 = Row<T>::Z0;
    for (int r = t; r < kE * kE; r += ns) {
        const int rx = r / kE;
        const int x = rx - kH, y = r - rx * kE - kH;
        const int d0 = nb_axis(x) * 9 + nb_axis(y) * 3;
        const int g = ((x & 7) << 6) | ((y & 7) << 3);
        T* row = stage + r * RP;
        stage_piece<T>(s_nb[d0], vals, g + 4, row + Z0 - 4, false);
        stage_piece<T>(s_nb[d0 + 1], vals, g, row + Z0, true);
        stage_piece<T>(s_nb[d0 + 2], vals, g, row + Z0 + 8, false);
    }
    for (int u = t; u < kNbr * 4; u += ns) {
        const int d = u >> 2, q = u & 3;
        const int sl = s_nb[d];
        if (sl >= 0) cp_async16(s_m + d * 8 + 2 * q, masks + (size_t)sl * 8 + 2 * q);
        else *reinterpret_cast<uint4*>(s_m + d * 8 + 2 * q) = make_uint4(0u, 0u, 0u, 0u);
    }
    cp_async_commit();
}

// Stage value at local voxel (x, y, z), x, y, z in [-2, 10).
template <typename T>
__device__ __forceinline__ const T* at(const T* stage, int x, int y, int z) {
    return stage + ((x + kH) * kE + (y + kH)) * Row<T>::RP + Row<T>::Z0 + z;
}

// Godunov upwind |grad phi| for the sign of s.  Per axis the upwind one-sided
// differences are u = max(sg (p - phi_-), 0) and w = max(sg (p - phi_+), 0),
// sg = +-1 the sign of s, and the axis term is max(u, w)^2, the same value as
// the sign-split form max(max(a-, 0)^2, min(a+, 0)^2) for s >= 0 and its
// mirror for s < 0, without the sign branch.  max(u, w) is evaluated as
// max(sg p - min(sg phi_-, sg phi_+), 0): negation is exact and rounding is
// monotone, so this is the same value, and fminf drops a NaN neighbour just
// as fmaxf drops its NaN difference.  The correctly rounded sqrtf keeps a
// full deformation period's FP32 topology equal to the FP64 run's (an
// rsqrtf-based magnitude measured two voxels flipping at the band's edge).
__device__ __forceinline__ float godunov_g(float p, float xm, float xp, float ym, float yp, float zm, float zp, float s) {
    const float sg = (s >= 0.f) ? 1.f : -1.f;
    const float q = sg * p;
    const float mx = fmaxf(q - fminf(sg * xm, sg * xp), 0.f);
    const float my = fmaxf(q - fminf(sg * ym, sg * yp), 0.f);
    const float mz = fmaxf(q - fminf(sg * zm, sg * zp), 0.f);
    // squares rounded before the sums (no contraction)
    float g2 = __fmul_rn(mx, mx) + __fmul_rn(my, my);
    g2 += __fmul_rn(mz, mz);
    return sqrtf(g2);
}

// NaN marks a voxel of an unallocated leaf; a 6-neighbour stencil reads it as
// copysign(hw, phi(centre)).
__device__ __forceinline__ float nbv(float v, float centre, float hw) { return (v != v) ? copysignf(hw, centre) : v; }

struct Nb6 {
    float xm, xp, ym, yp, zm, zp;
};

// The 6 neighbours of the value at c (axis strides SX, SY, 1), NaNs resolved
// against the centre value p.
template <typename T, int SX, int SY>
__device__ __forceinline__ Nb6 load_nb6(const T* c, float p, float hw) {
    return Nb6{nbv(to_f(c[-SX]), p, hw), nbv(to_f(c[SX]), p, hw), nbv(to_f(c[-SY]), p, hw),
               nbv(to_f(c[SY]), p, hw),  nbv(to_f(c[-1]), p, hw), nbv(to_f(c[1]), p, hw)};
}

// The 6 neighbours of the value at c as stored (NaN for an unallocated leaf).
template <typename T, int SX, int SY>
__device__ __forceinline__ Nb6 load_nb6_raw(const T* c) {
    return Nb6{to_f(c[-SX]), to_f(c[SX]), to_f(c[-SY]), to_f(c[SY]), to_f(c[-1]), to_f(c[1])};
}

__device__ __forceinline__ float godunov_update(float p, const Nb6& n, float s) {
    const float G = godunov_g(p, n.xm, n.xp, n.ym, n.yp, n.zm, n.zp, s);
    return p - 0.5f * s * (G - 1.0f);
}

// godunov_update with raw neighbours, NaN marking an unallocated leaf.  The
// missing-leaf value copysign(hw, p) gives an upwind term max(<= 0, 0) = 0
// whenever |p| <= hw and p's sign bit matches the upwind sign of s, and
// fmaxf gives the same 0 for the NaN itself, so the NaNs are resolved only
// outside that case: bit for bit the update of the resolved neighbours.
__device__ __forceinline__ float godunov_update_raw(float p, Nb6 n, float s, float hw) {
    if (!(fabsf(p) <= hw && (signbit(p) != 0) == (s < 0.f)))
        n = Nb6{nbv(n.xm, p, hw), nbv(n.xp, p, hw), nbv(n.ym, p, hw),
                nbv(n.yp, p, hw), nbv(n.zm, p, hw), nbv(n.zp, p, hw)};
    return godunov_update(p, n, s);
}

// Subcell fix of the reinitialisation (Russo & Smereka, J. Comput. Phys. 163,
// 2000): if the 6-neighbourhood of phi0 (the field before reinitialisation)
// changes sign at this voxel, the distance to the interface estimated as
// phi0 / |grad phi0| (per axis the largest of the central and the two
// one-sided differences, at least 1e-6); NaN otherwise.  Cut voxels relax
// toward it, phi <- phi - 1/2 (sign(phi0) |phi| - d), instead of taking the
// Godunov update, so reinitialisation does not move the interface.
__device__ __forceinline__ float cut_distance(float p, const Nb6& n) {
    const bool cut = (p * n.xm < 0.f) | (p * n.xp < 0.f) | (p * n.ym < 0.f) | (p * n.yp < 0.f) |
                     (p * n.zm < 0.f) | (p * n.zp < 0.f);
    if (!cut) return __int_as_float(0x7fc00000);
    const float mx = fmaxf(fmaxf(fabsf(n.xp - n.xm) * 0.5f, fabsf(n.xp - p)), fmaxf(fabsf(p - n.xm), 1e-6f));
    const float my = fmaxf(fmaxf(fabsf(n.yp - n.ym) * 0.5f, fabsf(n.yp - p)), fmaxf(fabsf(p - n.ym), 1e-6f));
    const float mz = fmaxf(fmaxf(fabsf(n.zp - n.zm) * 0.5f, fabsf(n.zp - p)), fmaxf(fabsf(p - n.zm), 1e-6f));
    return p / sqrtf(mx * mx + my * my + mz * mz);
}

__device__ __forceinline__ float cut_relax(float phi, float phi0, float d) {
    return phi - 0.5f * (copysignf(fabsf(phi), phi0) - d);
}

// 10-bit row of the dilated mask along z in [-1, 9) at (x, y) in [-1, 9)^2,
// from the 27 neighbour masks (bit i = z + 1).
__device__ __forceinline__ unsigned d_row(const uint64_t* s_m, int x, int y) {
    const int base = nb_axis(x) * 9 + nb_axis(y) * 3;
    const int bi = ((x & 7) << 3) | (y & 7);
    const unsigned char* m = (const unsigned char*)s_m;
    return ((unsigned)m[base * 64 + bi] >> 7) | ((unsigned)m[(base + 1) * 64 + bi] << 1) |
           (((unsigned)m[(base + 2) * 64 + bi] & 1u) << 9);
}

// Bits [32 l, 32 l + 32) of the box's voxels of D in flat order t = (bx *
// 10 + by) * 10 + bz (b = voxel + 1): the dilated mask on the 10^3 box
// without its edges and corners, which the second iteration never reads.
__device__ __forceinline__ unsigned box_word(const uint64_t* s_m, int l) {
    const int t0 = 32 * l;
    if (t0 >= kBox) return 0u;
    unsigned w = 0u;
    const int r1 = min(t0 + 31, kBox - 1) / kF;
    for (int r = t0 / kF; r <= r1; ++r) {
        const int bx = r / kF, by = r - bx * kF;
        const int edges = (bx == 0 || bx == kF - 1) + (by == 0 || by == kF - 1);
        const unsigned keep = edges == 0 ? 0x3FFu : (edges == 1 ? 0x1FEu : 0u);
        const unsigned rb = d_row(s_m, bx - 1, by - 1) & keep;
        const int sh = r * kF - t0;  // in [-9, 31]
        w |= sh >= 0 ? (rb << sh) : (rb >> -sh);
    }
    return w;
}

// Inclusive warp scan of c.
__device__ __forceinline__ int warp_incl_scan(int c, int lane) {
    int incl = c;
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
        const int y = __shfl_up_sync(0xffffffffu, incl, off);
        if (lane >= off) incl += y;
    }
    return incl;
}

// copysign(hw, value) of every voxel of the leaf, row by row into the output
// (coalesced); the voxels of D are overwritten in phase 2.
template <typename T>
__device__ __forceinline__ void write_outside(const T* stage, T* __restrict__ out, float hw, int t) {
    if (t >= 64) return;
    const int x = t >> 3, y = t & 7;
    const T* crow = at(stage, x, y, 0);
    if constexpr (sizeof(T) == 2) {
        const uint64_t h = __half_as_ushort(__float2half_rn(hw)) & 0x7fffu;
        const uint64_t hw4 = h | (h << 16) | (h << 32) | (h << 48);
        const uint64_t* c = reinterpret_cast<const uint64_t*>(crow);
        const uint64_t a = hw4 | (c[0] & 0x8000800080008000ull), b = hw4 | (c[1] & 0x8000800080008000ull);
        *reinterpret_cast<uint4*>(out + t * 8) =
            make_uint4((unsigned)a, (unsigned)(a >> 32), (unsigned)b, (unsigned)(b >> 32));
    } else {
        const unsigned hb = __float_as_uint(hw) & 0x7fffffffu;
        const uint4* c = reinterpret_cast<const uint4*>(crow);
        uint4* o = reinterpret_cast<uint4*>(out + t * 8);
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            const uint4 v = c[h];
            o[h] = make_uint4(hb | (v.x & 0x80000000u), hb | (v.y & 0x80000000u), hb | (v.z & 0x80000000u),
                              hb | (v.w & 0x80000000u));
        }
    }
}

// Phase 4 of a leaf, by one warp: its mask words to global memory, the
// spill toward absent neighbours, keep flags and re-tracking proposals.
// sM: the leaf's 16 mask words in shared memory; nb: the leaf's neighbour
// slot for the lane's direction (-1 absent).
__device__ __forceinline__ void spill_and_propose(const unsigned* sM, int slot, int4 o, int nb, int lane,
                                                  const MLeafArrays& A, const MTopo& topo,
                                                  const MGridParams* __restrict__ params, unsigned* err) {
    if (lane < 16) reinterpret_cast<unsigned*>(A.mask + (size_t)slot * 8)[lane] = sM[lane];
    // spill mask from 64-bit (x*8+y) plane masks of z = 0, z = 7 and any z
    const unsigned char* B = (const unsigned char*)sM;
    const unsigned b0 = B[lane], b1 = B[lane + 32];
    const uint64_t z0 = (uint64_t)__ballot_sync(0xffffffffu, b0 & 1u) |
                        ((uint64_t)__ballot_sync(0xffffffffu, b1 & 1u) << 32);
    const uint64_t z7 = (uint64_t)__ballot_sync(0xffffffffu, b0 & 0x80u) |
                        ((uint64_t)__ballot_sync(0xffffffffu, b1 & 0x80u) << 32);
    const uint64_t za = (uint64_t)__ballot_sync(0xffffffffu, b0 != 0u) |
                        ((uint64_t)__ballot_sync(0xffffffffu, b1 != 0u) << 32);
    bool spl = false;
    if (lane < kNbr && lane != 13) {
        const int dx = lane / 9 - 1, dy = (lane / 3) % 3 - 1, dz = lane % 3 - 1;
        const uint64_t plane = dz < 0 ? z0 : (dz > 0 ? z7 : za);
        const uint64_t xs = dx < 0 ? 0xFFull : (dx > 0 ? (0xFFull << 56) : ~0ull);
        const uint64_t ys = dy < 0 ? 0x0101010101010101ull : (dy > 0 ? 0x8080808080808080ull : ~0ull);
        spl = (plane & xs & ys) != 0ull;
    }
    // spill toward absent neighbours only: those are the proposals the
    // allocation scan resolves (present ones are kept right here)
    const unsigned sbits = __ballot_sync(0xffffffffu, spl && nb < 0);
    if (lane == 0) {
        A.spill[slot] = sbits;
        A.nonempty[slot] = (za != 0ull) ? 1 : 0;
        if (za != 0ull) topo.keep[slot] = 1;
    }
    // re-tracking proposals: an existing neighbour touched by the spill
    // survives; a missing one is proposed, keeping the proposer whose
    // direction seen from the new leaf comes first (atomicMin).
    if (spl) {
        if (nb >= 0) {
            topo.keep[nb] = 1;
        } else {
            const int dx = lane / 9 - 1, dy = (lane / 3) % 3 - 1, dz = lane % 3 - 1;
            const MGridParams& P = params[o.w];
            const uint64_t key = mkey((long long)(o.x >> 3) + dx, (long long)(o.y >> 3) + dy,
                                      (long long)(o.z >> 3) + dz, o.w, P.base, topo.key_bits);
            bool done = false;
            if (key != kEmptyKey) {
                uint32_t m = (uint32_t)topo.hcap - 1u, pp = (uint32_t)mix64(key) & m;
                for (int probe = 0; probe < topo.hcap; ++probe) {
                    const unsigned long long prev = atomicCAS((unsigned long long*)&topo.pkey[pp],
                                                              (unsigned long long)kEmptyKey, (unsigned long long)key);
                    if (prev == kEmptyKey || prev == key) {
                        atomicMin(&topo.pval[pp], kNbr - 1 - lane);
                        done = true;
                        break;
                    }
                    pp = (pp + 1u) & m;
                }
            }
            if (!done) atomicOr(err, key == kEmptyKey ? kErrExtent : kErrHashFull);
        }
    }
}

}  // namespace

template <typename T, int NIT, int FIX>
struct ReinitLayout {
    static constexpr size_t stage = (size_t)kE * kE * Row<T>::RP * sizeof(T);
    static constexpr size_t masks = (size_t)kNbr * 64;
    static constexpr size_t p2 = NIT == 2 ? (size_t)kBox * 4 : 0;               // phi2 on the 10^3 box
    static constexpr size_t dist = (NIT == 2 && FIX) ? (size_t)kBox * 4 : 0;    // cut distances
    static constexpr size_t bytes = 2 * stage + 2 * masks + p2 + dist;
    static_assert(stage % 16 == 0, "16-byte aligned buffers");
};

template <typename T, int NIT, int FIX>
__global__ void __launch_bounds__(kNT, 8) k_m_reinit(MLeafArrays A, const T* __restrict__ src, T* __restrict__ dst,
                                                     const MGridParams* __restrict__ params, MTopo topo,
                                                     unsigned* __restrict__ err) {
    dep_wait();
    dep_launch();
    if (step_aborted(err)) return;
    using Lay = ReinitLayout<T, NIT, FIX>;
    constexpr int RP = Row<T>::RP;
    extern __shared__ __align__(128) unsigned char smem_dyn[];
    unsigned char* const mk0 = smem_dyn + 2 * Lay::stage;
    float* s_p2 = reinterpret_cast<float*>(mk0 + 2 * Lay::masks);
    float* s_dist = reinterpret_cast<float*>(mk0 + 2 * Lay::masks + Lay::p2);
    auto stage_of = [&](int b) { return reinterpret_cast<T*>(smem_dyn + b * Lay::stage); };
    auto masks_of = [&](int b) { return reinterpret_cast<uint64_t*>(mk0 + b * Lay::masks); };
    __shared__ unsigned short s_list1[NIT == 2 ? kBox : 1];
    __shared__ unsigned short s_list2[kLeafVoxels];
    __shared__ int s_nbr[3][32];   // neighbour rows of the previous, current and next leaf
    __shared__ int s_n1, s_n2;
    __shared__ unsigned s_bx[32];  // the box voxels of D, one bit per flat index
    __shared__ short s_roff[kF * kF];  // stage offset of box row (bx, by) at bz = 0
    __shared__ __align__(16) unsigned s_M2[2][16];  // new mask words (this leaf, the previous one)
    __shared__ int s_pslot[2];
    __shared__ int4 s_po[2];

    const int count = *A.count;
    const int Gs = gridDim.x;
    int li = blockIdx.x;
    if (li >= count) return;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;

    for (int r = threadIdx.x; r < kF * kF; r += kNT)
        s_roff[r] = (short)(((r / kF - 1 + kH) * kE + (r % kF - 1 + kH)) * RP + Row<T>::Z0 - 1);
    int slot = A.list[li];
    int4 o = A.origin[slot];
    if (warp == 0) s_nbr[0][lane] = (lane < kNbr) ? A.nbr[(size_t)slot * kNbr + lane] : -1;
    __syncthreads();
    issue_stage<T>(s_nbr[0], src, A.dmask, stage_of(0), masks_of(0), threadIdx.x, kNT);
    // leaves ahead: the next one's list slot and neighbour row, and the slot
    // of the one after (its neighbour row is loaded one iteration before it
    // is needed, so no global load sits in front of a barrier)
    int slot_n = (li + Gs < count) ? A.list[li + Gs] : -1;
    int nb_next = (warp == 0 && lane < kNbr && slot_n >= 0) ? A.nbr[(size_t)slot_n * kNbr + lane] : -1;
    int slot_nn = (li + 2 * Gs < count) ? A.list[li + 2 * Gs] : -1;
    float hw = params[o.w].hw;

    unsigned it = 0;
    for (;; ++it) {
        const int b = it & 1;
        const int nx = (int)((it + 1u) % 3u), pv = (int)((it + 2u) % 3u);  // next and previous rows
        int4 o_n = make_int4(0, 0, 0, -1);
        if (slot_n >= 0) o_n = A.origin[slot_n];
        const int slot_nnn = (li + 3 * Gs < count) ? A.list[li + 3 * Gs] : -1;
        const int nb_after = (warp == 0 && lane < kNbr && slot_nn >= 0) ? A.nbr[(size_t)slot_nn * kNbr + lane] : -1;
        if (warp == 0) s_nbr[nx][lane] = nb_next;
        cp_async_wait_all();
        __syncthreads();  // barrier A: this leaf's stage is complete; the previous leaf is done
        const T* stage = stage_of(b);
        const uint64_t* s_m = masks_of(b);
        T* out = dst + (size_t)slot * kLeafVoxels;
        // the leaf's voxels of D for the last iteration (offset x * 64 + y * 8 + z)
        auto leaf_list = [&]() {
            const int q = lane >> 2, cq = lane & 3;
            unsigned bits = (unsigned)(s_m[13 * 8 + q] >> (16 * cq)) & 0xffffu;
            const int c = __popc(bits);
            const int incl = warp_incl_scan(c, lane);
            int pos = incl - c;
            while (bits) {
                const int z = __ffs(bits) - 1;
                bits &= bits - 1u;
                s_list2[pos++] = (unsigned short)(q * 64 + 16 * cq + z);
            }
            if (lane == 31) s_n2 = incl;
        };
        if (warp == 0) {
            // the box voxels of D for iteration 1 (flat index t = (bx * 10 +
            // by) * 10 + bz, ascending); without iteration 1 the leaf list
            if (NIT == 2) {
                unsigned bw = box_word(s_m, lane);
                s_bx[lane] = bw;
                const int c = __popc(bw);
                const int incl = warp_incl_scan(c, lane);
                int pos = incl - c;
                while (bw) {
                    const int z = __ffs(bw) - 1;
                    bw &= bw - 1u;
                    s_list1[pos++] = (unsigned short)(32 * lane + z);
                }
                if (lane == 31) s_n1 = incl;
            } else {
                leaf_list();
            }
        } else {
            // warp 1 builds the leaf list first when warp 0 has the box list
            if (NIT == 2 && warp == 1) leaf_list();
            const int t = threadIdx.x - 32;
            if (slot_n >= 0)
                issue_stage<T>(s_nbr[nx], src, A.dmask, stage_of(b ^ 1), masks_of(b ^ 1), t, kNT - 32);
            write_outside<T>(stage, out, hw, t);
            if (t < 16) s_M2[b][t] = 0u;
            if (warp == kNW - 1) {
                // phase 4 of the previous leaf, whose mask words are complete
                // since barrier A; this warp has the least phase-1 work
                if (lane == 0) {
                    s_pslot[b] = slot;
                    s_po[b] = o;
                }
                if (it > 0)
                    spill_and_propose(s_M2[b ^ 1], s_pslot[b ^ 1], s_po[b ^ 1], s_nbr[pv][lane], lane, A, topo, params,
                                      err);
            }
        }
        __syncthreads();  // barrier B: lists and outside-D results are in place
        if (NIT == 2) {
            // iteration 1 on the box voxels of D, consecutive voxels on consecutive lanes
            const int n1 = s_n1;
            for (int i = threadIdx.x; i < n1; i += kNT) {
                const int t = s_list1[i];
                const int r = t / kF;
                const T* c1 = stage + s_roff[r] + (t - r * kF);
                const float p = to_f(c1[0]);
                if (FIX) {
                    const Nb6 n = load_nb6<T, kE * RP, RP>(c1, p, hw);
                    const float d = cut_distance(p, n);
                    s_dist[t] = d;
                    s_p2[t] = (d == d) ? cut_relax(p, p, d) : godunov_update(p, n, p * rsqrtf(p * p + 1.0f));
                } else {
                    s_p2[t] = godunov_update_raw(p, load_nb6_raw<T, kE * RP, RP>(c1), p * rsqrtf(p * p + 1.0f), hw);
                }
            }
            __syncthreads();  // barrier C: phi2 complete on the box
        }
        {
            // the last iteration (or none) on the leaf's voxels of D, trim, stores
            const int n2 = s_n2;
            for (int i = threadIdx.x; i < n2; i += kNT) {
                const int off = s_list2[i];
                const int x = off >> 6, y = (off >> 3) & 7, z = off & 7;
                const T* c1 = at(stage, x, y, z);
                const float p1 = to_f(c1[0]);
                float v;
                if (NIT == 0) {
                    v = p1;
                } else if (NIT == 1) {
                    if (FIX) {
                        const Nb6 n = load_nb6<T, kE * RP, RP>(c1, p1, hw);
                        const float d = cut_distance(p1, n);
                        v = (d == d) ? cut_relax(p1, p1, d) : godunov_update(p1, n, p1 * rsqrtf(p1 * p1 + 1.0f));
                    } else {
                        v = godunov_update_raw(p1, load_nb6_raw<T, kE * RP, RP>(c1), p1 * rsqrtf(p1 * p1 + 1.0f), hw);
                    }
                } else {
                    const int t10 = ((x + 1) * kF + (y + 1)) * kF + (z + 1);
                    const float p2 = s_p2[t10];  // the leaf's voxels of D are box voxels of D
                    const float d = FIX ? s_dist[t10] : __int_as_float(0x7fc00000);
                    if (d == d) {
                        v = cut_relax(p2, p1, d);
                    } else {
                        // a neighbour's phi2 is iteration 1's result on the box voxels
                        // of D and phi1 (the stage) elsewhere
                        auto nb = [&](int dt, int ds) {
                            const int u = t10 + dt;
                            return ((s_bx[u >> 5] >> (u & 31)) & 1u) ? s_p2[u] : to_f(c1[ds]);
                        };
                        const Nb6 n{nb(-kF * kF, -kE * RP), nb(kF * kF, kE * RP), nb(-kF, -RP),
                                    nb(kF, RP),             nb(-1, -1),           nb(1, 1)};
                        v = godunov_update_raw(p2, n, p1 * rsqrtf(p1 * p1 + 1.0f), hw);
                    }
                }
                const bool on = fabsf(v) < hw;
                if (!on) v = copysignf(hw, v);
                out[off] = from_f<T>(v);
                if (on) atomicOr(&s_M2[b][off >> 5], 1u << (off & 31));
            }
        }
        if (slot_n < 0) break;
        li += Gs;
        slot = slot_n;
        if (o_n.w != o.w) hw = params[o_n.w].hw;
        o = o_n;
        slot_n = slot_nn;
        slot_nn = slot_nnn;
        nb_next = nb_after;
    }
    __syncthreads();  // the last leaf's mask words are complete
    if (warp == kNW - 1) spill_and_propose(s_M2[it & 1u], slot, o, s_nbr[it % 3u][lane], lane, A, topo, params, err);
}

#define VLR_REINIT_ARGS(T) MLeafArrays, const T*, T*, const MGridParams*, MTopo, unsigned*
#define VLR_INST_REINIT(T)                                            \
    template __global__ void k_m_reinit<T, 0, 0>(VLR_REINIT_ARGS(T)); \
    template __global__ void k_m_reinit<T, 1, 0>(VLR_REINIT_ARGS(T)); \
    template __global__ void k_m_reinit<T, 2, 0>(VLR_REINIT_ARGS(T)); \
    template __global__ void k_m_reinit<T, 0, 1>(VLR_REINIT_ARGS(T)); \
    template __global__ void k_m_reinit<T, 1, 1>(VLR_REINIT_ARGS(T)); \
    template __global__ void k_m_reinit<T, 2, 1>(VLR_REINIT_ARGS(T));
VLR_INST_REINIT(float)
VLR_INST_REINIT(__half)

size_t reinit_smem_bytes(int precision_f16, int nit, int fix) {
#define VLR_RS(T)                                                                                 \
    (nit == 0 ? (fix ? ReinitLayout<T, 0, 1>::bytes : ReinitLayout<T, 0, 0>::bytes)              \
              : nit == 1 ? (fix ? ReinitLayout<T, 1, 1>::bytes : ReinitLayout<T, 1, 0>::bytes)   \
                         : (fix ? ReinitLayout<T, 2, 1>::bytes : ReinitLayout<T, 2, 0>::bytes))
    return precision_f16 ? VLR_RS(__half) : VLR_RS(float);
#undef VLR_RS
}

}  // namespace vlr
