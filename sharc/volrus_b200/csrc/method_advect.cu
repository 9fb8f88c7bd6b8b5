// The advect kernel of the METHOD step: 26-neighbourhood dilation D of the
// activity mask, then the semi-Lagrangian backtrace (Euler / RK2 midpoint /
// SSP-RK3) of every voxel of D and a trilinear sample of the previous values.
//
// One CTA of 128 threads works on one 8^3 leaf at a time and strides over the
// ordered leaf list (persistent).  Per leaf:
//
//   stage      the (8+2H)^3 halo tile arrives in shared memory by
//              asynchronous copies (cp.async) issued one leaf ahead into the
//              other of two stage buffers, row-packed: tile row (x, y),
//              x, y in [-H, 8+H), holds the upper half-row of the leaf below
//              in z, the leaf's own row and the lower half-row of the leaf
//              above, z in [-4, 12) contiguous; the pieces of absent leaves
//              are set to NaN when the copies are issued; the 27 neighbour
//              masks arrive the same way.  The tile is sampled where it lands
//              (no copy into a second tile).
//   phase 1    (after the stage barrier) warp 0 builds D from the 27 masks
//              with 64-bit plane operations (z- and y-dilation inside a
//              plane word, x-dilation across planes) and compacts it into a
//              voxel list; warps 1-3 issue the next leaf's copies, one tile
//              row per thread, and write every voxel's outside-D result
//              copysign(hw, previous value) to global memory, coalesced.
//   phase 2    (after the second barrier) every thread backtraces voxels of
//              the list and stores the trilinear sample over the outside-D
//              value written in phase 1; a corner that falls in an absent
//              leaf (NaN) takes the missing-leaf rule, copysign(hw, the
//              leaf's own value at the clamped position).
//
// Two CTA barriers per leaf; the stage buffer of leaf i is refilled for leaf
// i + 2 only after leaf i + 1's stage barrier, when every read of it is done.
// Every leaf is computed by one CTA with the same arithmetic whatever the
// grid size, and the kernel's side effects on the per-step re-tracking state
// are clears, so relaunching it on the same inputs (the launch autotuner
// does) leaves the step's result unchanged.
//
// The same file holds k_m_feet, the per-voxel displacement of the frozen-band
// adjoint, which shares the backtrace arithmetic (method_velocity.cuh).
#include "method_kernels.hpp"
#include "method_velocity.cuh"

namespace vlr {
namespace {

constexpr int kNT = kAdvectThreads;

// Staged row of value type T: RP values, z = 0 at element Z0.  f16 rows hold
// [4 unused | 4 below | 8 own | 4 above | 4 unused] (48 bytes), f32 rows
// [4 below | 8 own | 4 above] (64 bytes), so that every piece starts on the
// 16- (own row) or 8-byte (half row) boundary its asynchronous copy needs.
template <typename T>
struct Row {
    static constexpr int RP = sizeof(T) == 2 ? 24 : 16;
    static constexpr int Z0 = sizeof(T) == 2 ? 8 : 4;
};

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

// Stage geometry for halo H: E x E tile rows (x, y), each with three pieces
// from the leaves below / at / above the row in z.
template <int H>
struct Geo {
    static constexpr int E = 8 + 2 * H;
    static constexpr int NROW = E * E;
    static_assert(H >= 1 && H <= 4, "the half-rows hold up to 4 values");
};

// One piece of a stage row: 8 values (full: the own z range) or 4 (a half
// row of a z neighbour) of leaf slot sl starting at value `off`, by asynchronous
// copy; NaN when the leaf is absent (the sampler resolves it with the
// missing-leaf rule).
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

// Copies of one leaf's stage rows into `stage` and of its 27 masks into s_m
// (masks of absent neighbours are zeroed) by a group of ns threads, this
// thread being number t of the group: one tile row (x, y) at a time, its
// three pieces from the z-lower, own and z-upper leaves of that column.
template <typename T, int H>
__device__ __forceinline__ void issue_stage(const int* s_nb, const T* __restrict__ vals,
                                            const uint64_t* __restrict__ masks, T* stage, uint64_t* s_m, int t,
                                            int ns) {
    constexpr int E = Geo<H>::E, RP = Row<T>::RP, Z0 = Row<T>::Z0;
    for (int r = t; r < Geo<H>::NROW; r += ns) {
        const int rx = r / E;
        const int x = rx - H, y = r - rx * E - H;
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

// Four copies of a 16-bit pattern in a 64-bit word.
__device__ __forceinline__ uint64_t rep4(uint64_t h) { return h | (h << 16) | (h << 32) | (h << 48); }
constexpr uint64_t kSign4 = 0x8000800080008000ull;  // sign bits of four f16 values
constexpr unsigned kSign = 0x80000000u;             // sign bit of an f32

// Every voxel's outside-D result, copysign(hw, previous value), written to
// the leaf's output row by row (coalesced); the voxels of D are overwritten
// in phase 2.
template <typename T, int H>
__device__ __forceinline__ void write_outside(const T* stage, T* __restrict__ out, float hw, int t) {
    constexpr int E = Geo<H>::E, RP = Row<T>::RP, Z0 = Row<T>::Z0;
    if (t >= 64) return;
    const int x = t >> 3, y = t & 7;
    const T* crow = stage + ((x + H) * E + (y + H)) * RP + Z0;
    if constexpr (sizeof(T) == 2) {
        const uint64_t hw4 = rep4(__half_as_ushort(__float2half_rn(hw)) & 0x7fffu);
        const uint64_t* c = reinterpret_cast<const uint64_t*>(crow);
        const uint64_t a = hw4 | (c[0] & kSign4), b = hw4 | (c[1] & kSign4);
        *reinterpret_cast<uint4*>(out + t * 8) =
            make_uint4((unsigned)a, (unsigned)(a >> 32), (unsigned)b, (unsigned)(b >> 32));
    } else {
        const unsigned hb = __float_as_uint(hw) & 0x7fffffffu;
        const uint4* c = reinterpret_cast<const uint4*>(crow);
        uint4* o = reinterpret_cast<uint4*>(out + t * 8);
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            const uint4 v = c[h];
            o[h] = make_uint4(hb | (v.x & kSign), hb | (v.y & kSign), hb | (v.z & kSign), hb | (v.w & kSign));
        }
    }
}

// 26-neighbourhood dilation of the activity, restricted to the leaf, from the
// 27 neighbour masks (word w of mask d = x-plane w, bit y*8 + z), by one warp:
// lane j < 30 takes tile plane X = j/3 - 1 and leaf row a_y = j % 3, dilates
// that plane word of the 3 leaves along z in place (borrowing the z = 7 / z = 0
// bits of the leaves below / above), the a_y = 1 lanes then dilate along y
// (borrowing the neighbours' y = 7 / y = 0 rows) and along x across planes.
// Returns the dilated word of plane X on the lanes with a_y = 1 and X in
// [0, 8), zero elsewhere; *xw receives X (-1 if none).
__device__ __forceinline__ uint64_t dilate_leaf(const uint64_t* s_m, int lane, int* xw) {
    constexpr uint64_t Z0 = 0x0101010101010101ull, Z7 = 0x8080808080808080ull;
    const int X = lane / 3 - 1, ay = lane - 3 * (lane / 3);
    uint64_t zc = 0;
    if (lane < 30) {
        const int ax = nb_axis(X), w = X & 7;
        const uint64_t* m = s_m + (ax * 9 + ay * 3) * 8 + w;
        const uint64_t lo = m[0], c = m[8], hi = m[16];
        zc = c | ((c << 1) & ~Z0) | ((c >> 1) & ~Z7) | ((lo & Z7) >> 7) | ((hi & Z0) << 7);
    }
    const uint64_t zl = __shfl_up_sync(0xffffffffu, zc, 1), zu = __shfl_down_sync(0xffffffffu, zc, 1);
    const uint64_t yd = zc | (zc << 8) | (zc >> 8) | (zl >> 56) | (zu << 56);
    const uint64_t pm = __shfl_up_sync(0xffffffffu, yd, 3), pp = __shfl_down_sync(0xffffffffu, yd, 3);
    const bool own = lane < 30 && ay == 1 && X >= 0 && X < 8;
    *xw = own ? X : -1;
    return own ? (pm | yd | pp) : 0ull;
}

// Velocity state of the leaf's grid, for the voxel loop.
struct LeafVel {
    VelConst V;
    float ct1, ct2, ct3;  // vortex time factors cos(pi t / T) at t1, t1 - dt/2, t1 - dt
    int series;
};

// Backtrace and trilinear sample of the listed voxels; results stored over
// the outside-D values.
template <typename T, int H, int VK, int OC, int SER>
__device__ __forceinline__ void advect_list(const LeafVel& L, const float2 (*s_tab)[3][8],
                                            const unsigned short* s_list, int nD, const T* stage, T* __restrict__ out,
                                            float dt, int integrator, float hwT, unsigned& bad) {
    constexpr int E = Geo<H>::E, RP = Row<T>::RP, Z0 = Row<T>::Z0;
    for (int i = threadIdx.x; i < nD; i += kNT) {
        const int off = s_list[i];
        const int x = off >> 6, y = (off >> 3) & 7, z = off & 7;
        const float3 f = backtrace<VK, OC, SER>(L.V, s_tab, x, y, z, dt, integrator, L.ct1, L.ct2, L.ct3);
        const float px = (float)(x + H) + f.x, py = (float)(y + H) + f.y, pz = (float)(z + H) + f.z;
        const float bxf = floorf(px), byf = floorf(py), bzf = floorf(pz);
        float wx = px - bxf, wy = py - byf, wz = pz - bzf;
        int ii = (int)bxf, jj = (int)byf, kk = (int)bzf;
        if ((unsigned)ii > (unsigned)(E - 2) || (unsigned)jj > (unsigned)(E - 2) || (unsigned)kk > (unsigned)(E - 2) ||
            !(px == px) || !(py == py) || !(pz == pz)) {
            bad = 1u;
            ii = min(max(ii, 0), E - 2);
            jj = min(max(jj, 0), E - 2);
            kk = min(max(kk, 0), E - 2);
            wx = fminf(fmaxf(wx, 0.f), 1.f);
            wy = fminf(fmaxf(wy, 0.f), 1.f);
            wz = fminf(fmaxf(wz, 0.f), 1.f);
        }
        // tile (ii, jj, kk) = row (ii, jj), element kk - H + Z0
        const T* q = stage + (ii * E + jj) * RP + (Z0 - H) + kk;
        float c000 = to_f(q[0]), c001 = to_f(q[1]), c010 = to_f(q[RP]), c011 = to_f(q[RP + 1]);
        float c100 = to_f(q[E * RP]), c101 = to_f(q[E * RP + 1]), c110 = to_f(q[E * RP + RP]),
              c111 = to_f(q[E * RP + RP + 1]);
        const float sum = ((c000 + c001) + (c010 + c011)) + ((c100 + c101) + (c110 + c111));
        if (sum != sum) {
            // a corner in an absent leaf (NaN): the missing-leaf rule,
            // copysign(hw, the leaf's own value at the clamped position)
            auto own = [&](int ti, int tj, int tk) {
                const int cx = min(max(ti - H, 0), 7), cy = min(max(tj - H, 0), 7), cz = min(max(tk - H, 0), 7);
                return copysignf(hwT, to_f(stage[((cx + H) * E + (cy + H)) * RP + Z0 + cz]));
            };
            if (c000 != c000) c000 = own(ii, jj, kk);
            if (c001 != c001) c001 = own(ii, jj, kk + 1);
            if (c010 != c010) c010 = own(ii, jj + 1, kk);
            if (c011 != c011) c011 = own(ii, jj + 1, kk + 1);
            if (c100 != c100) c100 = own(ii + 1, jj, kk);
            if (c101 != c101) c101 = own(ii + 1, jj, kk + 1);
            if (c110 != c110) c110 = own(ii + 1, jj + 1, kk);
            if (c111 != c111) c111 = own(ii + 1, jj + 1, kk + 1);
        }
        const float c00 = c000 * (1.f - wx) + c100 * wx, c01 = c001 * (1.f - wx) + c101 * wx;
        const float c10 = c010 * (1.f - wx) + c110 * wx, c11 = c011 * (1.f - wx) + c111 * wx;
        const float c0 = c00 * (1.f - wy) + c10 * wy, c1 = c01 * (1.f - wy) + c11 * wy;
        out[off] = from_f<T>(c0 * (1.f - wz) + c1 * wz);
    }
}

template <typename T, int H, int VK>
__device__ __forceinline__ void advect_dispatch(const LeafVel& L, const float2 (*s_tab)[3][8],
                                                const unsigned short* s_list, int nD, const T* stage,
                                                T* __restrict__ out, float dt, int integrator, float hwT,
                                                unsigned& bad) {
    const bool oc3 = L.V.octaves == 3;
    if (L.series == kSeriesMicro) {
        if (oc3) advect_list<T, H, VK, 3, kSeriesMicro>(L, s_tab, s_list, nD, stage, out, dt, integrator, hwT, bad);
        else advect_list<T, H, VK, 0, kSeriesMicro>(L, s_tab, s_list, nD, stage, out, dt, integrator, hwT, bad);
    } else if (L.series == kSeriesTiny) {
        if (oc3) advect_list<T, H, VK, 3, kSeriesTiny>(L, s_tab, s_list, nD, stage, out, dt, integrator, hwT, bad);
        else advect_list<T, H, VK, 0, kSeriesTiny>(L, s_tab, s_list, nD, stage, out, dt, integrator, hwT, bad);
    } else {
        if (oc3) advect_list<T, H, VK, 3, kSeriesFull>(L, s_tab, s_list, nD, stage, out, dt, integrator, hwT, bad);
        else advect_list<T, H, VK, 0, kSeriesFull>(L, s_tab, s_list, nD, stage, out, dt, integrator, hwT, bad);
    }
}

__device__ __forceinline__ void load_params(const MGridParams* __restrict__ params, int gid, MGridParams* s_P) {
    const int* src = (const int*)(params + gid);
    int* dst = (int*)s_P;
    for (int i = threadIdx.x; i < (int)(sizeof(MGridParams) / 4); i += blockDim.x) dst[i] = src[i];
}

}  // namespace

template <typename T, int H>
struct AdvectLayout {
    static constexpr size_t stage = (size_t)Geo<H>::NROW * Row<T>::RP * sizeof(T);  // one stage buffer
    static constexpr size_t masks = (size_t)kNbr * 64;
    static constexpr size_t bytes = 2 * stage + 2 * masks;
    static_assert(stage % 16 == 0, "16-byte aligned buffers");
};

template <typename T, int H, int VK>
__global__ void __launch_bounds__(kNT, 8) k_m_advect(MLeafArrays A, const T* __restrict__ src, T* __restrict__ dst,
                                                     const MGridParams* __restrict__ params,
                                                     const float2* __restrict__ tab, MStepParams sp, MTopo topo,
                                                     unsigned* __restrict__ err) {
    dep_wait();
    dep_launch();
    if (step_aborted(err)) return;
    // clear this step's re-tracking state (keep flags, proposal table, leaf hash)
    for (int i = blockIdx.x * kNT + threadIdx.x; i < max(topo.cap, topo.hcap); i += gridDim.x * kNT) {
        if (i < topo.cap) topo.keep[i] = 0;
        if (i < topo.hcap) {
            topo.pkey[i] = kEmptyKey;
            topo.pval[i] = INT_MAX;
            topo.hkey[i] = kEmptyKey;
            topo.hval[i] = -1;
        }
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        topo.scalars[4] = 0;  // new count (set by the last scan chunk)
        topo.scalars[5] = 0;  // dropped count (read by the last step's k_t_nbr)
        topo.scalars[7] = 0;  // scan chunk ticket
    }
    using G = Geo<H>;
    using Lay = AdvectLayout<T, H>;
    constexpr int NTAB = kMaxOctaves * 3 * 8;
    static_assert(NTAB <= kNT, "one table entry per thread");
    extern __shared__ __align__(128) unsigned char smem_dyn[];
    // buffer b: stage at smem_dyn + b * Lay::stage, masks at mk0 + b * Lay::masks
    unsigned char* const mk0 = smem_dyn + 2 * Lay::stage;
    auto stage_of = [&](int b) { return reinterpret_cast<T*>(smem_dyn + b * Lay::stage); };
    auto masks_of = [&](int b) { return reinterpret_cast<uint64_t*>(mk0 + b * Lay::masks); };
    __shared__ unsigned short s_list[kLeafVoxels];
    __shared__ int s_nbr[2][32];
    __shared__ int s_nD;
    __shared__ __align__(16) MGridParams s_P;
    __shared__ float2 s_tab[kMaxOctaves][3][8];

    const int count = *A.count;
    const int Gs = gridDim.x;
    int li = blockIdx.x;
    if (li >= count) return;
    const int step = *A.step;
    const float t1 = sp.t0 + (float)(step + 1) * sp.dt;
    const float dt = sp.dt;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    unsigned bad = 0;

    // prologue: the first leaf's stage
    int slot = A.list[li];
    int4 o = A.origin[slot];
    if (warp == 0) s_nbr[0][lane] = (lane < kNbr) ? A.nbr[(size_t)slot * kNbr + lane] : -1;
    __syncthreads();
    issue_stage<T, H>(s_nbr[0], src, A.mask, stage_of(0), masks_of(0), threadIdx.x, kNT);
    // leaves ahead: the next one's list slot and neighbour row, and the slot
    // of the one after (its neighbour row is loaded one iteration before it
    // is needed, so no global load sits in front of a barrier)
    int slot_n = (li + Gs < count) ? A.list[li + Gs] : -1;
    int nb_next = (warp == 0 && lane < kNbr && slot_n >= 0) ? A.nbr[(size_t)slot_n * kNbr + lane] : -1;
    int slot_nn = (li + 2 * Gs < count) ? A.list[li + 2 * Gs] : -1;

    int cur_gid = -1;
    LeafVel L{};
    float hw = 0.f;
    for (unsigned it = 0;; ++it) {
        const int b = it & 1;
        // loads for the leaves ahead (consumed one iteration later)
        int4 o_n = make_int4(0, 0, 0, -1);
        if (slot_n >= 0) o_n = A.origin[slot_n];
        const int slot_nnn = (li + 3 * Gs < count) ? A.list[li + 3 * Gs] : -1;
        const int nb_after = (warp == 0 && lane < kNbr && slot_nn >= 0) ? A.nbr[(size_t)slot_nn * kNbr + lane] : -1;
        if (o.w != cur_gid) {
            __syncthreads();
            load_params(params, o.w, &s_P);
            __syncthreads();
            cur_gid = o.w;
            L.V = vel_const(s_P);
            L.series = s_P.series;
            hw = s_P.hw;
            if (L.V.kind == MVEL_VORTEX) {
                L.ct1 = cosf(s_P.pi_over_T * t1);
                L.ct2 = cosf(s_P.pi_over_T * (t1 - 0.5f * dt));
                L.ct3 = cosf(s_P.pi_over_T * (t1 - dt));
            } else {
                L.ct1 = L.ct2 = L.ct3 = 1.f;
            }
        }
        // this leaf's sin/cos table entries, stored in phase 1
        float2 tv = make_float2(0.f, 0.f);
        bool tvalid = false;
        if (threadIdx.x < NTAB) {
            const int q = threadIdx.x;
            const int f = q / 24, a = (q / 8) % 3, l = q % 8;
            if (L.V.kind != MVEL_CONSTANT && (L.V.kind == MVEL_CURL ? f < L.V.octaves : f == 0)) {
                int oc = (a == 0 ? o.x : (a == 1 ? o.y : o.z)) + l - s_P.tab_lo[a];
                if (oc < 0 || oc >= s_P.tab_len[a]) {
                    bad = 1u;
                    oc = min(max(oc, 0), s_P.tab_len[a] - 1);
                }
                tv = __ldg(&tab[s_P.tab_off[f][a] + oc]);
                tvalid = true;
            }
        }
        if (warp == 0) s_nbr[b ^ 1][lane] = nb_next;
        // barrier A: this leaf's stage and masks are in shared memory, and
        // every thread is done with the previous leaf
        cp_async_wait_all();
        __syncthreads();
        T* stage = stage_of(b);
        T* out = dst + (size_t)slot * kLeafVoxels;
        if (warp == 0) {
            // D: dilation, dilated mask out, compaction into the voxel list
            int X;
            const uint64_t dw = dilate_leaf(masks_of(b), lane, &X);
            if (X >= 0) A.dmask[(size_t)slot * 8 + X] = dw;
            // lane l compacts bits [16c, 16c+16) of word q, q = l >> 2, c = l & 3
            const int q = lane >> 2, c = lane & 3;
            const uint64_t wq = __shfl_sync(0xffffffffu, dw, 3 * (q + 1) + 1);
            unsigned bits = (unsigned)(wq >> (16 * c)) & 0xffffu;
            const int cnt = __popc(bits);
            int incl = cnt;
#pragma unroll
            for (int d = 1; d < 32; d <<= 1) {
                const int y = __shfl_up_sync(0xffffffffu, incl, d);
                if (lane >= d) incl += y;
            }
            int pos = incl - cnt;
            const int base = q * 64 + 16 * c;
            while (bits) {
                const int bi = __ffs(bits) - 1;
                bits &= bits - 1u;
                s_list[pos++] = (unsigned short)(base + bi);
            }
            if (lane == 31) s_nD = incl;
        } else {
            const int t = threadIdx.x - 32;
            if (slot_n >= 0)
                issue_stage<T, H>(s_nbr[b ^ 1], src, A.mask, stage_of(b ^ 1), masks_of(b ^ 1), t, kNT - 32);
            write_outside<T, H>(stage, out, hw, t);
        }
        if (tvalid) (&s_tab[0][0][0])[threadIdx.x] = tv;
        __syncthreads();  // barrier B: list, tables and filled tile are ready
        advect_dispatch<T, H, VK>(L, s_tab, s_list, s_nD, stage, out, dt, sp.integrator, to_f(from_f<T>(hw)), bad);
        if (slot_n < 0) break;
        li += Gs;
        slot = slot_n;
        o = o_n;
        slot_n = slot_nn;
        slot_nn = slot_nnn;
        nb_next = nb_after;
    }
    if (bad) atomicOr(err, kErrReach);
}

// Backtrace displacement of every voxel of n leaves (origins as a level set
// holds them: x, y, z, grid id) over one step of a time-independent velocity
// (constant or curl noise), with k_m_advect's arithmetic (same tables, series
// and integrator): written to disp[bidx[leaf * 512 + voxel]] for voxels with
// bidx >= 0; the largest component magnitude is folded into *maxabs (float
// bits of a non-negative value, atomicMax).  Used by the frozen-band adjoint
// of a level set.
template <int VK>
__global__ void __launch_bounds__(128) k_m_feet(const int4* __restrict__ origin, int n, const int* __restrict__ bidx,
                                               const MGridParams* __restrict__ params, const float2* __restrict__ tab,
                                               float dt, int integrator, float3* __restrict__ disp,
                                               unsigned* __restrict__ maxabs, unsigned* __restrict__ err) {
    constexpr int NTAB = kMaxOctaves * 3 * 8;
    static_assert(NTAB <= 128, "one table entry per thread");
    __shared__ __align__(16) MGridParams s_P;
    __shared__ float2 s_tab[kMaxOctaves][3][8];
    unsigned bad = 0;
    float m = 0.f;
    int cur = -1;
    for (int li = blockIdx.x; li < n; li += gridDim.x) {
        const int4 o = origin[li];
        __syncthreads();  // the previous leaf's table reads are done
        if (o.w != cur) {
            load_params(params, o.w, &s_P);
            __syncthreads();
            cur = o.w;
        }
        const VelConst V = vel_const(s_P);
        if (threadIdx.x < NTAB) {
            const int q = threadIdx.x;
            const int f = q / 24, a = (q / 8) % 3, l = q % 8;
            if (V.kind != MVEL_CONSTANT && (V.kind == MVEL_CURL ? f < V.octaves : f == 0)) {
                int oc = (a == 0 ? o.x : (a == 1 ? o.y : o.z)) + l - s_P.tab_lo[a];
                if (oc < 0 || oc >= s_P.tab_len[a]) {
                    bad = 1u;
                    oc = min(max(oc, 0), s_P.tab_len[a] - 1);
                }
                (&s_tab[0][0][0])[q] = __ldg(&tab[s_P.tab_off[f][a] + oc]);
            }
        }
        __syncthreads();
        const int series = s_P.series;
        for (int off = threadIdx.x; off < kLeafVoxels; off += 128) {
            const int b = bidx[(size_t)li * kLeafVoxels + off];
            if (b < 0) continue;
            const int x = off >> 6, y = (off >> 3) & 7, z = off & 7;
            // the advect kernel's instance of the backtrace for this grid
            const float3 f = backtrace_any<VK>(V, series, s_tab, x, y, z, dt, integrator, 1.f, 1.f, 1.f);
            disp[b] = f;
            const float fm = fmaxf(fabsf(f.x), fmaxf(fabsf(f.y), fabsf(f.z)));
            if (!(fm == fm)) bad = 1u;
            else m = fmaxf(m, fm);
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
    if ((threadIdx.x & 31) == 0) atomicMax(maxabs, __float_as_uint(m));
    if (bad) atomicOr(err, kErrReach);
}

template __global__ void k_m_feet<MVEL_CONSTANT>(const int4*, int, const int*, const MGridParams*, const float2*, float,
                                                 int, float3*, unsigned*, unsigned*);
template __global__ void k_m_feet<MVEL_CURL>(const int4*, int, const int*, const MGridParams*, const float2*, float,
                                             int, float3*, unsigned*, unsigned*);

#define VLR_ADVECT_ARGS(T) MLeafArrays, const T*, T*, const MGridParams*, const float2*, MStepParams, MTopo, unsigned*
#define VLR_INST_ADVECT(T, H)                                                      \
    template __global__ void k_m_advect<T, H, -1>(VLR_ADVECT_ARGS(T));            \
    template __global__ void k_m_advect<T, H, MVEL_CONSTANT>(VLR_ADVECT_ARGS(T)); \
    template __global__ void k_m_advect<T, H, MVEL_VORTEX>(VLR_ADVECT_ARGS(T));   \
    template __global__ void k_m_advect<T, H, MVEL_CURL>(VLR_ADVECT_ARGS(T));
VLR_INST_ADVECT(float, 2)
VLR_INST_ADVECT(float, 3)
VLR_INST_ADVECT(__half, 2)
VLR_INST_ADVECT(__half, 3)

size_t advect_smem_bytes(int precision_f16, int halo) {
    if (precision_f16) return halo == 2 ? AdvectLayout<__half, 2>::bytes : AdvectLayout<__half, 3>::bytes;
    return halo == 2 ? AdvectLayout<float, 2>::bytes : AdvectLayout<float, 3>::bytes;
}

}  // namespace vlr
