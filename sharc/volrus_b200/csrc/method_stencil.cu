// The two stencil kernels of the METHOD step.  One CTA (NT = 128 or 256
// threads, chosen by the launch autotuner) works on one 8^3 leaf at a time and
// strides over the ordered leaf list (persistent).
//
//   k_m_advect   26-neighbourhood dilation D of the activity mask, then the
//                semi-Lagrangian backtrace (Euler / RK2 midpoint / SSP-RK3) of
//                every voxel of D and trilinear sampling from a (8+2H)^3 halo
//                tile of the previous values in shared memory
//   k_m_reinit   NIT (0..2) Jacobi iterations of Godunov-upwind
//                reinitialisation fused in one pass (the first iteration runs
//                on the 10^3 box around the leaf so that the second needs no
//                exchange), trim to |phi| < hw, new mask, spill mask
//
// Staging: the halo tile's rows (8 middle values plus the z-halo pieces of the
// leaves below and above, per (x, y) row) and the masks of the 27-leaf
// neighbourhood arrive in shared memory by asynchronous copies (cp.async, all
// threads, one commit group per leaf) issued one leaf ahead: while the CTA
// computes leaf i, the copies of leaf i+1 are in flight.  The list entry,
// origin and neighbour row of the leaves ahead are loaded into registers one
// or two iterations before they are used, so a leaf costs no dependent global
// round trip.  The float tile is then built from shared memory.
//
// A second staging mode (ST = 1) brings the same pieces by TMA: one tensor
// copy per present neighbour leaf (a box of whole z-rows, or of f32 z-halves)
// completing on an mbarrier, issued by lane 0 of each warp in turn.  It moves
// the same bytes and gives bit-identical results; the launch autotuner times
// both modes.  On B200 the per-copy cost of up to 27 small boxes per leaf
// (about 216 per SM per leaf round at 8 CTAs) leaves it 25-35% slower than
// the cp.async rows, which every thread issues in parallel, so cp.async is
// the mode the autotuner keeps on the measured workloads.
//
// Both kernels are latency- and issue-bound (a leaf moves 2-4 KB but runs a few
// thousand instructions in phases separated by CTA barriers), so a leaf passes
// as few barriers as its data flow allows (advect 3, reinit 4), results leave
// from registers straight to global memory (each warp's stores fall in one
// leaf), and 128-thread CTAs keep eight leaves in flight per SM.  The first
// reinitialisation iteration compacts its voxels per warp (ballot + scan), so
// it needs no CTA barrier of its own.
//
// Launch-shape independence: every leaf is computed by one CTA with the same
// arithmetic whatever NT and the grid size are, and the kernels' side effects
// on shared per-step state are idempotent (flags set to 1, atomicMin of
// proposals, clears), so the autotuner may launch a kernel several times on
// the same inputs within a step and the step's result is unchanged.
#include "method_kernels.hpp"

namespace vlr {

__device__ __forceinline__ int nb_axis(int c) { return (c < 0) ? 0 : (c > 7 ? 2 : 1); }

// ------------------------------------------------------------ async staging

__device__ __forceinline__ uint32_t smem_addr(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

// Asynchronous global -> shared copy of 16 bytes (both addresses 16-byte aligned).
__device__ __forceinline__ void cp_async16(void* dst, const void* src) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(smem_addr(dst)), "l"(src) : "memory");
}

__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }

__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }

// Row-packed halo staging of an (8+2H)^2 x (8+2H) tile: tile row (x, y)
// (local leaf coordinates in [-H, 8+H)) holds the whole z-rows (8 values) of
// the leaves below, at and above it in z, so element 8 + z is voxel z of the
// row for z in [-8, 16).  Whole 16-byte rows keep the copies coalesced; only
// the tile's rows cross from L2, not whole neighbour leaves.
template <typename T, int H>
struct RowStage {
    static constexpr int E = 8 + 2 * H;
    static constexpr int RP = 24;  // elements per staged row
    static constexpr size_t bytes = (size_t)E * E * RP * sizeof(T);
};

// Copy descriptors of the staged pieces: piece p = (row r, z-piece k) of the
// row-packed stage, k = 0 / 1 / 2 for the leaves below / at / above in z.
// They depend only on the piece, so each CTA builds the table once:
//   bits 0-4   neighbour index d of the leaf that holds the piece
//   bits 5-13  element offset of the copied 16 bytes within that leaf
//   bits 14-26 element offset of the destination within the stage
//   bit 27     a second 16-byte copy follows (f32 rows of the centre z-leaf)
// For f32 a z-halo piece copies only the 16-byte half that holds the H <= 4
// values the tile uses (k = 0: z in [8-H, 8), upper half; k = 2: z in [0, H)).
template <typename T, int H>
struct StageDesc {
    static constexpr int E = 8 + 2 * H;
    static constexpr int NP = E * E * 3;
};

template <typename T, int H, int NT>
__device__ __forceinline__ void build_stage_desc(unsigned* s_desc) {
    using R = RowStage<T, H>;
    constexpr int E = R::E, RP = R::RP;
    constexpr int HALF = 16 / (int)sizeof(T);  // elements in 16 bytes
    static_assert(E * E * RP < (1 << 13), "stage offset fits 13 bits");
    for (int p = threadIdx.x; p < StageDesc<T, H>::NP; p += NT) {
        const int r = p / 3, k = p - 3 * r;
        const int rx = r / E;
        const int x = rx - H, y = r - rx * E - H;
        const unsigned d = (unsigned)(nb_axis(x) * 9 + nb_axis(y) * 3 + k);
        unsigned goff = (unsigned)(((x & 7) << 6) | ((y & 7) << 3));
        unsigned soff = (unsigned)(r * RP + 8 * k);
        unsigned two = 0;
        if constexpr (sizeof(T) == 4) {
            if (k == 0) {
                goff += HALF;
                soff += HALF;
            } else if (k == 1) {
                two = 1;
            }
        }
        s_desc[p] = d | (goff << 5) | (soff << 14) | (two << 27);
    }
}

// All threads: start the asynchronous copies of one leaf's tile rows and of
// the 64-byte masks of its 27 neighbours (masks of absent neighbours are
// zeroed; rows of absent leaves are left for the tile build to fill).  `s_nb`
// holds the 27 neighbour slots.  Called after a CTA barrier that ended every
// read of the previous stage; stage_ready() completes it.
template <typename T, int H, int NT>
__device__ __forceinline__ void stage_async(const unsigned* s_desc, const int* s_nb, const T* __restrict__ vals,
                                            const uint64_t* __restrict__ masks, T* s_rows, uint64_t* s_m) {
    constexpr int HALF = 16 / (int)sizeof(T);
    for (int p = threadIdx.x; p < StageDesc<T, H>::NP; p += NT) {
        const unsigned dsc = s_desc[p];
        const int sl = s_nb[dsc & 31u];
        if (sl >= 0) {
            const T* src = vals + (size_t)sl * kLeafVoxels + ((dsc >> 5) & 511u);
            T* d = s_rows + ((dsc >> 14) & 8191u);
            cp_async16(d, src);
            if (sizeof(T) == 4 && (dsc >> 27)) cp_async16(d + HALF, src + HALF);
        }
    }
    if (threadIdx.x < kNbr * 4) {
        const int d = threadIdx.x >> 2, q = threadIdx.x & 3;
        const int sl = s_nb[d];
        if (sl >= 0) cp_async16(s_m + d * 8 + 2 * q, masks + (size_t)sl * 8 + 2 * q);
        else *reinterpret_cast<uint4*>(s_m + d * 8 + 2 * q) = make_uint4(0u, 0u, 0u, 0u);
    }
    cp_async_commit();
}

// All threads: wait for this thread's copies, then a CTA barrier.
__device__ __forceinline__ void stage_ready() {
    cp_async_wait_all();
    __syncthreads();
}

// --------------------------------------------------------- TMA staging (ST = 1)
//
// The tile pieces held by neighbour leaf d = ax * 9 + ay * 3 + az arrive as
// ONE tensor copy of the box of that leaf which the tile covers:
//   x: [8-H, 8) for the leaf below, [0, 8) at, [0, H) above the centre leaf
//   y: the same
//   z: the whole row (f16: 8 values = 16 bytes); f32 z-neighbours copy only
//      the 16-byte half that holds the H <= 4 values the tile uses
// Each box lands dense (z fastest, then y, then x) at a 128-byte aligned
// offset of the stage.  A box of whole z-rows is contiguous over (y, z) in the
// pool, so it is copied through a map whose innermost dimension merges y and
// z: its rows are ey * 8 values wide (up to 128 bytes for f16) rather than
// one 16-byte z-row each, which keeps the number of rows the tensor unit
// walks per leaf low.  The row-offset table (built once per CTA in s_desc,
// 16-bit entries biased by kRowBias) gives, for tile row (x, y) and z-piece
// k, the element offset p_k such that stage[p_k + z] is voxel z of that row
// in the leaf below / at / above (k = 0 / 1 / 2); 16-bit entries keep the
// CTA within the shared memory that 8 resident CTAs per SM leave it.  Up to
// 27 copies per leaf complete on one mbarrier whose expected byte count is
// the sum of the issued boxes; the 27 masks still arrive by cp.async.
template <typename T, int H>
struct BoxStage {
    static constexpr int E = 8 + 2 * H;
    static constexpr int ext(int a) { return a == 1 ? 8 : H; }
    static constexpr int lo(int a) { return a == 0 ? 8 - H : 0; }
    static constexpr int ez(int az) { return (sizeof(T) == 4 && az != 1) ? 4 : 8; }
    static constexpr int z0(int az) { return (sizeof(T) == 4 && az == 0) ? 4 : 0; }
    static constexpr int box_bytes(int d) { return ez(d % 3) * ext((d / 3) % 3) * ext(d / 9) * (int)sizeof(T); }
    static constexpr int off(int d) {
        int s = 0;
        for (int i = 0; i < d; ++i) s += (box_bytes(i) + 127) & ~127;
        return s;
    }
    // tensor map of box d (see StageMaps)
    static constexpr int map_of(int d) {
        return ((d / 9) == 1 ? 2 : 0) | (((d / 3) % 3) == 1 ? 1 : 0) | ((sizeof(T) == 4 && d % 3 != 1) ? 4 : 0);
    }
    static constexpr size_t bytes = (size_t)off(kNbr);
    static_assert(H >= 1 && H <= 4, "the f32 z-halves hold up to 4 values");
};

constexpr int kRowBias = 8;  // f32 k = 0 pieces start up to 4 elements before their box

template <typename T, int H, int NT>
__device__ __forceinline__ void build_row_offsets(unsigned short* s_off) {
    using B = BoxStage<T, H>;
    constexpr int E = B::E;
    for (int p = threadIdx.x; p < E * E * 3; p += NT) {
        const int r = p / 3, k = p - 3 * r;
        const int rx = r / E;
        const int x = rx - H, y = r - rx * E - H;
        const int ax = nb_axis(x), ay = nb_axis(y);
        const int d = ax * 9 + ay * 3 + k;
        const int xl = (x & 7) - B::lo(ax), yl = (y & 7) - B::lo(ay);
        const int start = B::off(d) / (int)sizeof(T) + (xl * B::ext(ay) + yl) * B::ez(k);
        s_off[p] = (unsigned short)(start - B::z0(k) + kRowBias);
    }
    static_assert(B::bytes / sizeof(T) + kRowBias < 65536, "row offsets fit 16 bits");
}

// Copy descriptor of box d: x = stage offset (bytes), y = c0 | c1 << 8 |
// c2 << 16 | map << 24, z = bytes.  Maps 0-3 take coordinates (yz0 = 8 * y0,
// x0, slot), maps 4-7 (z0, y0, x0, slot); the slot is the neighbour's, added
// at issue.  Kept as 16 bytes so the issue loop reads it with one load and no
// unpacking: the loop is on the critical path of its warp.
template <typename T, int H>
__device__ __forceinline__ uint4 tma_piece(int d) {
    using B = BoxStage<T, H>;
    const int ax = d / 9, ay = (d / 3) % 3, az = d % 3;
    const int m = B::map_of(d);
    const unsigned co = (m < 4) ? ((unsigned)(8 * B::lo(ay)) | ((unsigned)B::lo(ax) << 8))
                                : ((unsigned)B::z0(az) | ((unsigned)B::lo(ay) << 8) | ((unsigned)B::lo(ax) << 16));
    return make_uint4((unsigned)B::off(d), co | ((unsigned)m << 24), (unsigned)B::box_bytes(d), 0u);
}

__device__ __forceinline__ void mbar_init(uint32_t bar, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void mbar_expect_tx_only(uint32_t bar, unsigned bytes) {
    asm volatile("mbarrier.expect_tx.relaxed.cta.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}

__device__ __forceinline__ void mbar_arrive(uint32_t bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(bar) : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint32_t bar, unsigned parity) {
    unsigned ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(bar), "r"(parity)
        : "memory");
    return ok != 0u;
}

// 3-D tiled tensor copy global -> shared (coordinates yz, x, slot), completing
// on the mbarrier at `bar`.
__device__ __forceinline__ void tma_load_3d(uint32_t dst, const CUtensorMap* map, int c0, int c1, int c2,
                                            uint32_t bar) {
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, "
        "%4}], [%5];" ::"r"(dst),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(c0), "r"(c1), "r"(c2), "r"(bar)
        : "memory");
}

// 4-D tiled tensor copy global -> shared (coordinates z, y, x, slot), completing
// on the mbarrier at `bar`.
__device__ __forceinline__ void tma_load_4d(uint32_t dst, const CUtensorMap* map, int c0, int c1, int c2, int c3,
                                            uint32_t bar) {
    asm volatile(
        "cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, "
        "%5}], [%6];" ::"r"(dst),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(bar)
        : "memory");
}

// All threads (same place as stage_async): lane 0 of warp w walks the
// neighbours d = w, w + NW, ... and, for each present one, raises the
// mbarrier's expected bytes by its box and issues its tensor copy, then
// arrives; the mbarrier expects one arrival per warp, so the phase cannot
// complete before every expectation is posted.  The masks follow by cp.async.
// One issuing lane per warp keeps the issue out of the register budget of the
// stencil arithmetic (held at the 64-register cap) and splits the serial issue
// chain NW ways.
template <int NT>
__device__ __forceinline__ void stage_tma(const uint4* s_tma, const int* s_nb, const StageMaps& maps,
                                          uint32_t stage, uint32_t bar, const uint64_t* __restrict__ masks,
                                          uint64_t* s_m) {
    if ((threadIdx.x & 31) == 0) {
#pragma unroll 1
        for (int d = threadIdx.x >> 5; d < kNbr; d += NT / 32) {
            const int sl = s_nb[d];
            if (sl >= 0) {
                const uint4 pc = s_tma[d];
                const unsigned m = pc.y >> 24;
                mbar_expect_tx_only(bar, pc.z);
                if (m < 4u)
                    tma_load_3d(stage + pc.x, &maps.m[m], (int)(pc.y & 255u), (int)((pc.y >> 8) & 255u), sl, bar);
                else
                    tma_load_4d(stage + pc.x, &maps.m[m], (int)(pc.y & 255u), (int)((pc.y >> 8) & 255u),
                                (int)((pc.y >> 16) & 255u), sl, bar);
            }
        }
        mbar_arrive(bar);
    }
    if (threadIdx.x < kNbr * 4) {
        const int d = threadIdx.x >> 2, q = threadIdx.x & 3;
        const int sl = s_nb[d];
        if (sl >= 0) cp_async16(s_m + d * 8 + 2 * q, masks + (size_t)sl * 8 + 2 * q);
        else *reinterpret_cast<uint4*>(s_m + d * 8 + 2 * q) = make_uint4(0u, 0u, 0u, 0u);
    }
    cp_async_commit();
}

// Bounded wait of the tensor copies (about a second at most): every thread
// polls the phase, then a CTA barrier that also agrees on the outcome.
// Returns false on every thread if any thread gave up.  The stage of the
// it-th leaf a CTA processes completes phase it of the mbarrier, so the
// parity waited for is it & 1.
constexpr int kStageSpin = 1 << 20;
__device__ __forceinline__ bool stage_ready_tma(uint32_t bar, unsigned parity, long long limit) {
    cp_async_wait_all();
    bool ok = false;
    for (long long i = 0; i < limit; ++i)
        if (mbar_try_wait(bar, parity)) {
            ok = true;
            break;
        }
    return __syncthreads_or(ok ? 0 : 1) == 0;
}

// Shared setup of the stage for mode ST: copy descriptors (ST 0) or row
// offsets, per-neighbour copy descriptors and the mbarrier (ST 1).  Callers
// follow it with a CTA barrier.
template <typename T, int H, int NT, int ST>
__device__ __forceinline__ void stage_setup(unsigned* s_desc, uint4* s_tma, uint64_t* s_bar,
                                            const StageMaps& maps) {
    if constexpr (ST == 0) {
        build_stage_desc<T, H, NT>(s_desc);
    } else {
        // bring the tensor maps' descriptors on chip before the first copy
        if (threadIdx.x < (sizeof(T) == 2 ? 4 : 8))
            asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(&maps.m[threadIdx.x]))
                         : "memory");
        build_row_offsets<T, H, NT>(reinterpret_cast<unsigned short*>(s_desc));
        if (threadIdx.x < kNbr) s_tma[threadIdx.x] = tma_piece<T, H>(threadIdx.x);
        if (threadIdx.x == 0) mbar_init(smem_addr(s_bar), NT / 32);
    }
}

template <typename T, int H, int NT, int ST>
__device__ __forceinline__ void stage_issue(const unsigned* s_desc, const uint4* s_tma, uint64_t* s_bar,
                                            const int* s_nb, const T* __restrict__ vals, const StageMaps& maps,
                                            const uint64_t* __restrict__ masks, T* s_rows, uint64_t* s_m) {
    if constexpr (ST == 0) stage_async<T, H, NT>(s_desc, s_nb, vals, masks, s_rows, s_m);
    else stage_tma<NT>(s_tma, s_nb, maps, smem_addr(s_rows), smem_addr(s_bar), masks, s_m);
}

// Returns false (on every thread) if the tensor copies did not arrive in time.
template <int ST>
__device__ __forceinline__ bool stage_wait(uint64_t* s_bar, unsigned parity, long long limit) {
    if constexpr (ST == 0) {
        stage_ready();
        return true;
    } else {
        return stage_ready_tma(smem_addr(s_bar), parity, limit);
    }
}

// Start of the stage in dynamic shared memory: the tensor copies want 128-byte
// aligned destinations, so mode 1 rounds the base up (its size reserves 128
// bytes for this).
template <int ST>
__device__ __forceinline__ unsigned char* stage_base(unsigned char* smem) {
    if constexpr (ST == 0) return smem;
    else return smem + ((128u - (smem_addr(smem) & 127u)) & 127u);
}

// Copy one grid's parameters into shared memory (all threads call; caller syncs).
__device__ __forceinline__ void load_params(const MGridParams* __restrict__ params, int gid, MGridParams* s_P) {
    const int* src = (const int*)(params + gid);
    int* dst = (int*)s_P;
    for (int i = threadIdx.x; i < (int)(sizeof(MGridParams) / 4); i += blockDim.x) dst[i] = src[i];
}

template <typename T>
__device__ __forceinline__ void lds_row8(const T* p, float* out) {
    if constexpr (sizeof(T) == 2) {
        uint4 u = *reinterpret_cast<const uint4*>(p);
        const __half2* h = reinterpret_cast<const __half2*>(&u);
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            float2 f = __half22float2(h[i]);
            out[2 * i] = f.x;
            out[2 * i + 1] = f.y;
        }
    } else {
        float4 a = *reinterpret_cast<const float4*>(p);
        float4 b = *reinterpret_cast<const float4*>(p + 4);
        out[0] = a.x; out[1] = a.y; out[2] = a.z; out[3] = a.w;
        out[4] = b.x; out[5] = b.y; out[6] = b.z; out[7] = b.w;
    }
}

// Build tile row (x, y) (local leaf coordinates, z over [-H, 8 + H)) from the
// stage: row-packed (ST 0) or boxes located by the row-offset table s_desc
// (ST 1).  Absent leaves: kNaN ? NaN : copysign(hw, centre value at the
// clamped position).
template <typename T, int H, bool kNaN, int ST>
__device__ __forceinline__ void build_row(const T* s_rows, const unsigned* s_desc, const int* s_nbr, int x, int y,
                                          float hw, float* row) {
    using R = RowStage<T, H>;
    constexpr int E = R::E, RP = R::RP;
    const int base = nb_axis(x) * 9 + nb_axis(y) * 3;
    const int r = (x + H) * E + (y + H);
    const int rc = (min(max(x, 0), 7) + H) * E + (min(max(y, 0), 7) + H);
    const T *p0, *p1, *p2, *c;  // z-pieces of the rows below / at / above; centre leaf row
    if constexpr (ST == 0) {
        p0 = s_rows + r * RP;
        p1 = p0 + 8;
        p2 = p0 + 16;
        c = s_rows + rc * RP + 8;
    } else {
        const unsigned short* so = reinterpret_cast<const unsigned short*>(s_desc);
        p0 = s_rows + ((int)so[3 * r] - kRowBias);
        p1 = s_rows + ((int)so[3 * r + 1] - kRowBias);
        p2 = s_rows + ((int)so[3 * r + 2] - kRowBias);
        c = s_rows + ((int)so[3 * rc + 1] - kRowBias);
    }
    const float nan = __int_as_float(0x7fc00000);
    float mid[8];
    if (s_nbr[base + 1] >= 0) {
        lds_row8<T>(p1, mid);
    } else if (!kNaN) {
        lds_row8<T>(c, mid);
#pragma unroll
        for (int i = 0; i < 8; ++i) mid[i] = copysignf(hw, mid[i]);
    } else {
#pragma unroll
        for (int i = 0; i < 8; ++i) mid[i] = nan;
    }
#pragma unroll
    for (int i = 0; i < 8; ++i) row[H + i] = mid[i];
    if (s_nbr[base] >= 0) {
#pragma unroll
        for (int i = 0; i < H; ++i) row[i] = to_f(p0[8 - H + i]);
    } else {
        const float f = kNaN ? nan : copysignf(hw, to_f(c[0]));
#pragma unroll
        for (int i = 0; i < H; ++i) row[i] = f;
    }
    if (s_nbr[base + 2] >= 0) {
#pragma unroll
        for (int i = 0; i < H; ++i) row[H + 8 + i] = to_f(p2[i]);
    } else {
        const float f = kNaN ? nan : copysignf(hw, to_f(c[7]));
#pragma unroll
        for (int i = 0; i < H; ++i) row[H + 8 + i] = f;
    }
}

template <int E>
__device__ __forceinline__ void store_row(float* dst, const float* row) {
    if constexpr (E % 4 == 0) {
#pragma unroll
        for (int i = 0; i < E / 4; ++i)
            reinterpret_cast<float4*>(dst)[i] = make_float4(row[4 * i], row[4 * i + 1], row[4 * i + 2], row[4 * i + 3]);
    } else {
#pragma unroll
        for (int i = 0; i < E / 2; ++i) reinterpret_cast<float2*>(dst)[i] = make_float2(row[2 * i], row[2 * i + 1]);
    }
}

// ------------------------------------------------------------- velocity

// Per-grid velocity constants held in registers for a leaf.
struct VelConst {
    int kind;
    int octaves;
    int doubling;                 // curl: octave o's table angle per voxel is 2^o times octave 0's
    float c[3];
    float scale;                  // vortex: vel_scale
    float dphi[kMaxOctaves];
    float ak[kMaxOctaves];
    float e[kMaxOctaves][3];
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
        V.ak[o] = P.ak[o];
#pragma unroll
        for (int a = 0; a < 3; ++a) V.e[o][a] = P.e[o][a];
    }
    return V;
}

template <bool FULL>
__device__ __forceinline__ void series_sincos(float d, float& sd, float& cd) {
    if (FULL) small_sincos(d, sd, cd);
    else tiny_sincos(d, sd, cd);
}

// (sin, cos) of (table angle - rotation angle) from the table pair and the
// rotation's sine and cosine.
__device__ __forceinline__ float2 rot(float2 t, float sd, float cd) {
    return make_float2(t.x * cd + t.y * sd, t.y * cd - t.x * sd);
}

template <bool FULL>
__device__ __forceinline__ float2 rotate(float2 t, float d) {
    float sd, cd;
    series_sincos<FULL>(d, sd, cd);
    return rot(t, sd, cd);
}

// Curl-noise octave o's contribution grad f_o x e_o, from its rotated
// (sin, cos) pairs per axis.
__device__ __forceinline__ void curl_octave(const VelConst& V, int o, float2 X, float2 Y, float2 Z, float3& u) {
    // grad f_o = a (cos x sin y sin z, sin x cos y sin z, sin x sin y cos z); v += grad f_o x e_o
    const float a = V.ak[o];
    const float syz = Y.x * Z.x, sxa = a * X.x;
    const float gx = a * X.y * syz, gy = sxa * Y.y * Z.x, gz = sxa * Y.x * Z.y;
    u.x += gy * V.e[o][2] - gz * V.e[o][1];
    u.y += gz * V.e[o][0] - gx * V.e[o][2];
    u.z += gx * V.e[o][1] - gy * V.e[o][0];
}

// Velocity (voxels per unit time) at local voxel (lx, ly, lz) + offset, from
// the leaf's staged sin/cos tables.  kOff = false: no offset (voxel centre).
template <int VK, bool kOff, bool FULL>
__device__ __forceinline__ float3 leaf_velocity(const VelConst& V, const float2 (*tab)[3][8], int lx, int ly, int lz,
                                                float ox, float oy, float oz, float ct) {
    const int kind = (VK >= 0) ? VK : V.kind;
    if (kind == MVEL_CONSTANT) return make_float3(V.c[0], V.c[1], V.c[2]);
    if (kind == MVEL_VORTEX) {
        float2 X = tab[0][0][lx], Y = tab[0][1][ly], Z = tab[0][2][lz];
        if (kOff) {
            X = rotate<FULL>(X, V.dphi[0] * ox);
            Y = rotate<FULL>(Y, V.dphi[0] * oy);
            Z = rotate<FULL>(Z, V.dphi[0] * oz);
        }
        // u = 2 sin^2(pi x) sin(2 pi y) sin(2 pi z), v = -sin(2 pi x) sin^2(pi y) sin(2 pi z),
        // w = -sin(2 pi x) sin(2 pi y) sin^2(pi z), times cos(pi t / T), world units / voxel size
        float k = V.scale * ct;
        float sycy = Y.x * Y.y, szcz = Z.x * Z.y, sxcx = X.x * X.y;
        return make_float3(8.0f * k * X.x * X.x * sycy * szcz, -4.0f * k * sxcx * Y.x * Y.x * szcz,
                           -4.0f * k * sxcx * sycy * Z.x * Z.x);
    }
    float3 u = make_float3(0.f, 0.f, 0.f);
    if (kOff && V.doubling) {
        // octave o rotates by 2^o times octave 0's angle: one series per axis,
        // then the double-angle formulas sin 2a = 2 sin a cos a, cos 2a = 1 - 2 sin^2 a
        float sx, cx, sy, cy, sz, cz;
        series_sincos<FULL>(V.dphi[0] * ox, sx, cx);
        series_sincos<FULL>(V.dphi[0] * oy, sy, cy);
        series_sincos<FULL>(V.dphi[0] * oz, sz, cz);
#pragma unroll
        for (int o = 0; o < kMaxOctaves; ++o) {
            if (o < V.octaves) {
                curl_octave(V, o, rot(tab[o][0][lx], sx, cx), rot(tab[o][1][ly], sy, cy), rot(tab[o][2][lz], sz, cz),
                            u);
                float t = sx + sx;
                sx = t * cx;
                cx = 1.0f - t * (t * 0.5f);
                t = sy + sy;
                sy = t * cy;
                cy = 1.0f - t * (t * 0.5f);
                t = sz + sz;
                sz = t * cz;
                cz = 1.0f - t * (t * 0.5f);
            }
        }
        return u;
    }
#pragma unroll
    for (int o = 0; o < kMaxOctaves; ++o) {
        if (o < V.octaves) {
            float2 X = tab[o][0][lx], Y = tab[o][1][ly], Z = tab[o][2][lz];
            if (kOff) {
                X = rotate<FULL>(X, V.dphi[o] * ox);
                Y = rotate<FULL>(Y, V.dphi[o] * oy);
                Z = rotate<FULL>(Z, V.dphi[o] * oz);
            }
            curl_octave(V, o, X, Y, Z, u);
        }
    }
    return u;
}

// Backtrace displacement (voxels) of local voxel (x, y, z) over one step:
// Euler (integrator 1), RK2 midpoint (2) or SSP-RK3 (3), velocities from the
// leaf's staged sin/cos tables at the stage times' cosine factors.
template <int VK, bool FULL>
__device__ __forceinline__ float3 backtrace(const VelConst& V, const float2 (*s_tab)[3][8], int x, int y, int z,
                                            float dt, int integrator, float ct1, float ct2, float ct3) {
    float fx, fy, fz;
    const float3 k1 = leaf_velocity<VK, false, FULL>(V, s_tab, x, y, z, 0.f, 0.f, 0.f, ct1);
    if (integrator == 1) {
        fx = -dt * k1.x;
        fy = -dt * k1.y;
        fz = -dt * k1.z;
    } else if (integrator == 2) {
        const float3 k2 = leaf_velocity<VK, true, FULL>(V, s_tab, x, y, z, -0.5f * dt * k1.x, -0.5f * dt * k1.y,
                                                        -0.5f * dt * k1.z, ct2);
        fx = -dt * k2.x;
        fy = -dt * k2.y;
        fz = -dt * k2.z;
    } else {
        const float h = -dt;
        const float ax = h * k1.x, ay = h * k1.y, az = h * k1.z;
        const float3 k2 = leaf_velocity<VK, true, FULL>(V, s_tab, x, y, z, ax, ay, az, ct3);
        const float bx = 0.25f * (ax + h * k2.x), by = 0.25f * (ay + h * k2.y), bz = 0.25f * (az + h * k2.z);
        const float3 k3 = leaf_velocity<VK, true, FULL>(V, s_tab, x, y, z, bx, by, bz, ct2);
        fx = (2.0f / 3.0f) * (bx + h * k3.x);
        fy = (2.0f / 3.0f) * (by + h * k3.y);
        fz = (2.0f / 3.0f) * (bz + h * k3.z);
    }
    return make_float3(fx, fy, fz);
}

// Backtrace and trilinear sample of the compacted voxels of D; each result is
// stored straight to the leaf's values in global memory.
template <typename T, int VK, bool FULL, int H, int NT>
__device__ __forceinline__ void advect_voxels(const VelConst& V, const float2 (*s_tab)[3][8], const unsigned short* s_list,
                                              int nD, const float* s_tile, T* __restrict__ out, float dt,
                                              int integrator, float ct1, float ct2, float ct3, unsigned& bad) {
    constexpr int E = 8 + 2 * H;
    for (int i = threadIdx.x; i < nD; i += NT) {
        const int off = s_list[i];
        const int x = off >> 6, y = (off >> 3) & 7, z = off & 7;
        const float3 f = backtrace<VK, FULL>(V, s_tab, x, y, z, dt, integrator, ct1, ct2, ct3);
        const float fx = f.x, fy = f.y, fz = f.z;
        const float px = (float)(x + H) + fx, py = (float)(y + H) + fy, pz = (float)(z + H) + fz;
        const float bxf = floorf(px), byf = floorf(py), bzf = floorf(pz);
        float wx = px - bxf, wy = py - byf, wz = pz - bzf;
        int ii = (int)bxf, jj = (int)byf, kk = (int)bzf;
        if (ii < 0 || jj < 0 || kk < 0 || ii > E - 2 || jj > E - 2 || kk > E - 2 || !(px == px) || !(py == py) ||
            !(pz == pz)) {
            bad = 1u;
            ii = min(max(ii, 0), E - 2);
            jj = min(max(jj, 0), E - 2);
            kk = min(max(kk, 0), E - 2);
            wx = fminf(fmaxf(wx, 0.f), 1.f);
            wy = fminf(fmaxf(wy, 0.f), 1.f);
            wz = fminf(fmaxf(wz, 0.f), 1.f);
        }
        const float* q = &s_tile[(ii * E + jj) * E + kk];
        const float c000 = q[0], c001 = q[1], c010 = q[E], c011 = q[E + 1];
        const float c100 = q[E * E], c101 = q[E * E + 1], c110 = q[E * E + E], c111 = q[E * E + E + 1];
        const float c00 = c000 * (1.f - wx) + c100 * wx, c01 = c001 * (1.f - wx) + c101 * wx;
        const float c10 = c010 * (1.f - wx) + c110 * wx, c11 = c011 * (1.f - wx) + c111 * wx;
        const float c0 = c00 * (1.f - wy) + c10 * wy, c1 = c01 * (1.f - wy) + c11 * wy;
        out[off] = from_f<T>(c0 * (1.f - wz) + c1 * wz);
    }
}

// Dynamic shared memory of the advect kernel (stage, masks, float tile; mode 1
// reserves 128 bytes to align the stage).
template <typename T, int H, int ST>
struct AdvectSmem {
    static constexpr int E = 8 + 2 * H;
    static constexpr size_t raw = ST ? BoxStage<T, H>::bytes : RowStage<T, H>::bytes;
    static constexpr size_t masks = (size_t)kNbr * 64;
    static constexpr size_t tile = (size_t)E * E * E * 4;
    static constexpr size_t bytes = raw + masks + tile + (ST ? 128 : 0);
};

// --------------------------------------------------------------- advect

template <typename T, int H, int VK, int NT, int ST>
__global__ void __launch_bounds__(NT, 1024 / NT) k_m_advect(MLeafArrays A, const T* __restrict__ src,
                                                           T* __restrict__ dst, const MGridParams* __restrict__ params,
                                                           const float2* __restrict__ tab, MStepParams sp, MTopo topo,
                                                           unsigned* __restrict__ err,
                                                           const __grid_constant__ StageMaps maps) {
    static_assert(NT == 128 || NT == 256, "128 or 256 threads per CTA");
    dep_wait();
    dep_launch();
    if (step_aborted(err)) return;
    // clear this step's re-tracking state (keep flags, proposal table, leaf hash)
    for (int i = blockIdx.x * NT + threadIdx.x; i < max(topo.cap, topo.hcap); i += gridDim.x * NT) {
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
        topo.scalars[7] = 0;  // scan chunk ticket
    }
    using L = AdvectSmem<T, H, ST>;
    constexpr int E = L::E;
    constexpr int NROW = E * E;
    constexpr int NTAB = kMaxOctaves * 3 * 8;
    static_assert(NTAB <= NT, "one table entry per thread");
    extern __shared__ __align__(128) unsigned char smem_dyn[];
    unsigned char* smem = stage_base<ST>(smem_dyn);
    T* s_raw = reinterpret_cast<T*>(smem);
    uint64_t* s_m = reinterpret_cast<uint64_t*>(smem + L::raw);
    float* s_tile = reinterpret_cast<float*>(smem + L::raw + L::masks);
    __shared__ __align__(16) uint64_t s_D[8];
    __shared__ int s_nbr[2][32];
    __shared__ unsigned short s_list[kLeafVoxels];
    __shared__ __align__(16) MGridParams s_P;
    __shared__ float2 s_tab[kMaxOctaves][3][8];
    __shared__ __align__(16) unsigned s_desc[ST ? (StageDesc<T, H>::NP + 1) / 2 : StageDesc<T, H>::NP];
    __shared__ uint4 s_tma[ST ? kNbr : 1];
    __shared__ uint64_t s_bar;

    const int count = *A.count;
    const int G = gridDim.x;
    int li = blockIdx.x;
    if (li >= count) return;
    const long long stage_limit = wait_limit(err, kStageSpin);
    const int step = *A.step;
    const float t1 = sp.t0 + (float)(step + 1) * sp.dt;
    const float dt = sp.dt;
    const int lane = threadIdx.x & 31;
    const bool w0 = threadIdx.x < 32;
    unsigned bad = 0;

    // prologue: first leaf staged, next leaf's list entry in flight
    int slot = A.list[li];
    int4 o = A.origin[slot];
    stage_setup<T, H, NT, ST>(s_desc, s_tma, &s_bar, maps);
    if (w0) s_nbr[0][lane] = (lane < kNbr) ? A.nbr[(size_t)slot * kNbr + lane] : -1;
    __syncthreads();
    stage_issue<T, H, NT, ST>(s_desc, s_tma, &s_bar, s_nbr[0], src, maps, A.mask, s_raw, s_m);
    int slot_n = (li + G < count) ? A.list[li + G] : -1;

    int cur_gid = -1;
    VelConst V{};
    float ct1 = 1.f, ct2 = 1.f, ct3 = 1.f;  // vortex time factors cos(pi t / T) at t1, t1 - dt/2, t1 - dt
    float hw = 0.f;
    int fullser = 0;
    for (unsigned it = 0;; ++it) {
        const int cur = it & 1;
        // loads for the leaves ahead (consumed one iteration later)
        int4 o_n = make_int4(0, 0, 0, -1);
        if (slot_n >= 0) o_n = A.origin[slot_n];
        const int nb_n = (w0 && lane < kNbr && slot_n >= 0) ? A.nbr[(size_t)slot_n * kNbr + lane] : -1;
        const int slot_nn = (li + 2 * G < count) ? A.list[li + 2 * G] : -1;
        if (o.w != cur_gid) {
            __syncthreads();
            load_params(params, o.w, &s_P);
            __syncthreads();
            cur_gid = o.w;
            V = vel_const(s_P);
            hw = s_P.hw;
            fullser = s_P.full_series;
            if (V.kind == MVEL_VORTEX) {
                ct1 = cosf(s_P.pi_over_T * t1);
                ct2 = cosf(s_P.pi_over_T * (t1 - 0.5f * dt));
                ct3 = cosf(s_P.pi_over_T * (t1 - dt));
            }
        }
        // this leaf's sin/cos table entries, stored after the tile is built
        float2 tv = make_float2(0.f, 0.f);
        bool tvalid = false;
        if (threadIdx.x < NTAB) {
            const int q = threadIdx.x;
            const int f = q / 24, a = (q / 8) % 3, l = q % 8;
            if (V.kind != MVEL_CONSTANT && (V.kind == MVEL_CURL ? f < V.octaves : f == 0)) {
                int oc = (a == 0 ? o.x : (a == 1 ? o.y : o.z)) + l - s_P.tab_lo[a];
                if (oc < 0 || oc >= s_P.tab_len[a]) {
                    bad = 1u;
                    oc = min(max(oc, 0), s_P.tab_len[a] - 1);
                }
                tv = __ldg(&tab[s_P.tab_off[f][a] + oc]);
                tvalid = true;
            }
        }
        // barrier 1: this leaf's rows and masks are in shared memory
        if (!stage_wait<ST>(&s_bar, (unsigned)cur, stage_limit)) {
            if (threadIdx.x == 0) atomicOr(err, kErrTimeout);
            return;
        }
        const int* nbr = s_nbr[cur];
        for (int t = threadIdx.x; t < NROW + 64; t += NT) {
            if (t < NROW) {
                float row[E];
                build_row<T, H, false, ST>(s_raw, s_desc, nbr, t / E - H, t % E - H, hw, row);
                store_row<E>(s_tile + t * E, row);
            } else {
                // dilation: one thread per z-row, 10-bit rows z = -1..8
                const int r = t - NROW;
                const int x = r >> 3, y = r & 7;
                unsigned acc = 0;
                const unsigned char* m = (const unsigned char*)s_m;
#pragma unroll
                for (int dx = -1; dx <= 1; ++dx)
#pragma unroll
                    for (int dy = -1; dy <= 1; ++dy) {
                        const int xx = x + dx, yy = y + dy;
                        const int base = nb_axis(xx) * 9 + nb_axis(yy) * 3;
                        const int bi = ((xx & 7) << 3) | (yy & 7);
                        acc |= ((unsigned)m[base * 64 + bi] >> 7) | ((unsigned)m[(base + 1) * 64 + bi] << 1) |
                               (((unsigned)m[(base + 2) * 64 + bi] & 1u) << 9);
                    }
                ((unsigned char*)s_D)[r] = (unsigned char)(((acc | (acc << 1) | (acc >> 1)) >> 1) & 0xffu);
            }
        }
        if (w0) s_nbr[cur ^ 1][lane] = nb_n;
        __syncthreads();  // barrier 2: tile and D are built; the staging buffers are free
        if (slot_n >= 0)
            stage_issue<T, H, NT, ST>(s_desc, s_tma, &s_bar, s_nbr[cur ^ 1], src, maps, A.mask, s_raw, s_m);
        if (tvalid) (&s_tab[0][0][0])[threadIdx.x] = tv;
        // compact D; voxels outside D keep the sign of their previous value and
        // are stored here
        T* out = dst + (size_t)slot * kLeafVoxels;
        int nD, pre_w[8 / (NT / 32)];
        {
            // prefix of the popcounts of the 8 words of D (x planes) over lanes 0..7
            const int c = (lane < 8) ? __popcll(s_D[lane]) : 0;
            int incl = c;
#pragma unroll
            for (int d = 1; d < 8; d <<= 1) {
                const int y = __shfl_up_sync(0xffffffffu, incl, d);
                if (lane >= d) incl += y;
            }
            nD = __shfl_sync(0xffffffffu, incl, 7);
#pragma unroll
            for (int j = 0; j < 8 / (NT / 32); ++j) {
                const int q = (threadIdx.x >> 5) + (NT / 32) * j;
                pre_w[j] = __shfl_sync(0xffffffffu, incl - c, q);
            }
        }
#pragma unroll
        for (int j = 0; j < 8 / (NT / 32); ++j) {
            // warp w compacts words w, w + NW, ...: lane l handles bits l and l + 32
            const int q = (threadIdx.x >> 5) + (NT / 32) * j;
            const uint64_t word = s_D[q];
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                const int bit = lane + 32 * h;
                const int off = q * 64 + bit;
                if ((word >> bit) & 1ull) {
                    s_list[pre_w[j] + __popcll(word & ((1ull << bit) - 1ull))] = (unsigned short)off;
                } else {
                    const int y = (off >> 3) & 7, z = off & 7;
                    out[off] = from_f<T>(copysignf(hw, s_tile[((q + H) * E + (y + H)) * E + (z + H)]));
                }
            }
        }
        __syncthreads();  // barrier 3: list and velocity tables are ready
        if (fullser)
            advect_voxels<T, VK, true, H, NT>(V, s_tab, s_list, nD, s_tile, out, dt, sp.integrator, ct1, ct2, ct3,
                                              bad);
        else
            advect_voxels<T, VK, false, H, NT>(V, s_tab, s_list, nD, s_tile, out, dt, sp.integrator, ct1, ct2, ct3,
                                               bad);
        if (threadIdx.x < 8) A.dmask[(size_t)slot * 8 + threadIdx.x] = s_D[threadIdx.x];
        if (slot_n < 0) break;
        li += G;
        slot = slot_n;
        o = o_n;
        slot_n = slot_nn;
    }
    if (bad) atomicOr(err, kErrReach);
}

// -------------------------------------------------------------- reinit

// Godunov upwind |grad phi| for the sign of s.  Per axis the upwind one-sided
// differences are u = max(sg (p - phi_-), 0) and w = max(sg (p - phi_+), 0),
// sg = +-1 the sign of s (exact), and the axis term is max(u, w)^2, which
// equals max(u^2, w^2) bit for bit (u, w >= 0 and rounding is monotone): the
// same value as the sign-split form max(max(a-, 0)^2, min(a+, 0)^2) for s >=
// 0 and its mirror for s < 0, without the sign branch.
__device__ __forceinline__ float godunov_g(float p, float xm, float xp, float ym, float yp, float zm, float zp, float s) {
    const float sg = (s >= 0.f) ? 1.f : -1.f;
    const float mx = fmaxf(fmaxf(sg * (p - xm), 0.f), fmaxf(sg * (p - xp), 0.f));
    const float my = fmaxf(fmaxf(sg * (p - ym), 0.f), fmaxf(sg * (p - yp), 0.f));
    const float mz = fmaxf(fmaxf(sg * (p - zm), 0.f), fmaxf(sg * (p - zp), 0.f));
    // squares rounded before the sums, as in the sign-split form (no contraction)
    float g2 = __fmul_rn(mx, mx) + __fmul_rn(my, my);
    g2 += __fmul_rn(mz, mz);
    return sqrtf(g2);
}

// NaN marks a voxel of an unallocated leaf; a 6-neighbour stencil reads it as
// copysign(hw, phi(centre)).
__device__ __forceinline__ float nbv(float v, float centre, float hw) { return (v != v) ? copysignf(hw, centre) : v; }

// The 6 neighbours of a tile voxel (row pitch S), missing-leaf NaNs resolved
// against the centre value p.
struct Nb6 {
    float xm, xp, ym, yp, zm, zp;
};

template <int S>
__device__ __forceinline__ Nb6 load_nb6(const float* c, float p, float hw) {
    return Nb6{nbv(c[-S * S], p, hw), nbv(c[S * S], p, hw), nbv(c[-S], p, hw),
               nbv(c[S], p, hw),      nbv(c[-1], p, hw),    nbv(c[1], p, hw)};
}

__device__ __forceinline__ float godunov_update(float p, const Nb6& n, float s) {
    const float G = godunov_g(p, n.xm, n.xp, n.ym, n.yp, n.zm, n.zp, s);
    return p - 0.5f * s * (G - 1.0f);
}

template <int S>
__device__ __forceinline__ float reinit_update(const float* c, float p, float s, float hw) {
    return godunov_update(p, load_nb6<S>(c, p, hw), s);
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


template <typename T, int ST>
struct ReinitSmem {
    static constexpr size_t raw = ST ? BoxStage<T, 2>::bytes : RowStage<T, 2>::bytes;
    static constexpr size_t masks = (size_t)kNbr * 64;
    static constexpr size_t p1 = 12 * 12 * 12 * 4;  // phi1 tile: leaf + 2-voxel ring
    static constexpr size_t p2 = 10 * 10 * 10 * 4;  // phi2 tile: leaf + 1-voxel ring
    static constexpr size_t bytes = raw + masks + p1 + p2 + (ST ? 128 : 0);
};

template <typename T, int NIT, int NT, int ST>
__global__ void __launch_bounds__(NT, 1024 / NT) k_m_reinit(MLeafArrays A, const T* __restrict__ src,
                                                           T* __restrict__ dst, const MGridParams* __restrict__ params,
                                                           MTopo topo, int mode, unsigned* __restrict__ err,
                                                           const __grid_constant__ StageMaps maps) {
    static_assert(NT == 128 || NT == 256, "128 or 256 threads per CTA");
    dep_wait();
    dep_launch();
    if (step_aborted(err)) return;
    constexpr int E = 12;  // phi1 tile: leaf + 2-voxel ring
    constexpr int F = 10;  // phi2 tile and D rows: leaf + 1-voxel ring
    constexpr int NW = NT / 32;
    constexpr int VPT = kLeafVoxels / NT;
    constexpr int RPW = (F * F + NW - 1) / NW;  // D rows per warp (rows r = lane * NW + warp)
    static_assert(32 * NW >= F * F, "one D row per lane");
    using L = ReinitSmem<T, ST>;
    extern __shared__ __align__(128) unsigned char smem_dyn[];
    unsigned char* smem = stage_base<ST>(smem_dyn);
    T* s_raw = reinterpret_cast<T*>(smem);
    uint64_t* s_dm = reinterpret_cast<uint64_t*>(smem + L::raw);
    float* s_p1 = reinterpret_cast<float*>(smem + L::raw + L::masks);
    float* s_p2 = reinterpret_cast<float*>(smem + L::raw + L::masks + L::p1);
    __shared__ unsigned short s_D[F * F];
    __shared__ unsigned short s_list[NW][RPW * F];
    __shared__ int s_nbr[2][32];
    __shared__ __align__(16) unsigned s_M[16];
    __shared__ __align__(16) unsigned s_desc[ST ? (StageDesc<T, 2>::NP + 1) / 2 : StageDesc<T, 2>::NP];
    __shared__ uint4 s_tma[ST ? kNbr : 1];
    __shared__ uint64_t s_bar;
    __shared__ float s_dist[NIT == 2 ? F * F * F : 1];  // cut-voxel distances of the 10^3 box (NaN: not cut)

    const int count = *A.count;
    const int G = gridDim.x;
    int li = blockIdx.x;
    if (li >= count) return;
    const long long stage_limit = wait_limit(err, kStageSpin);
    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    const bool fix = (mode == 1);
    const bool w0 = threadIdx.x < 32;

    int slot = A.list[li];
    int4 o = A.origin[slot];
    stage_setup<T, 2, NT, ST>(s_desc, s_tma, &s_bar, maps);
    if (w0) s_nbr[0][lane] = (lane < kNbr) ? A.nbr[(size_t)slot * kNbr + lane] : -1;
    __syncthreads();
    stage_issue<T, 2, NT, ST>(s_desc, s_tma, &s_bar, s_nbr[0], src, maps, A.dmask, s_raw, s_dm);
    int slot_n = (li + G < count) ? A.list[li + G] : -1;
    float hw = params[o.w].hw;

    for (unsigned it = 0;; ++it) {
        const int cur = it & 1;
        int4 o_n = make_int4(0, 0, 0, -1);
        if (slot_n >= 0) o_n = A.origin[slot_n];
        const int nb_n = (w0 && lane < kNbr && slot_n >= 0) ? A.nbr[(size_t)slot_n * kNbr + lane] : -1;
        const int slot_nn = (li + 2 * G < count) ? A.list[li + 2 * G] : -1;
        if (!stage_wait<ST>(&s_bar, (unsigned)cur, stage_limit)) {  // barrier 1
            if (threadIdx.x == 0) atomicOr(err, kErrTimeout);
            return;
        }
        const int* nbr = s_nbr[cur];
        for (int t = threadIdx.x; t < E * E + F * F; t += NT) {
            if (t < E * E) {
                float row[E];
                const int x = t / E - 2, y = t % E - 2;
                build_row<T, 2, true, ST>(s_raw, s_desc, nbr, x, y, hw, row);
                store_row<E>(s_p1 + t * E, row);
                if (NIT == 2 && x >= -1 && x <= 8 && y >= -1 && y <= 8) {
                    // phi2 starts as phi1 on the 10^3 box; iteration 1 overwrites the voxels of D
                    float* d2 = s_p2 + ((x + 1) * F + (y + 1)) * F;
#pragma unroll
                    for (int i = 0; i < F; ++i) d2[i] = row[i + 1];
                }
            } else {
                const int r = t - E * E;
                const int x = r / F - 1, y = r % F - 1;
                const int base = nb_axis(x) * 9 + nb_axis(y) * 3;
                const int bi = ((x & 7) << 3) | (y & 7);
                const unsigned char* m = (const unsigned char*)s_dm;
                const unsigned row = ((unsigned)m[base * 64 + bi] >> 7) | ((unsigned)m[(base + 1) * 64 + bi] << 1) |
                                     (((unsigned)m[(base + 2) * 64 + bi] & 1u) << 9);
                s_D[r] = (unsigned short)row;
            }
        }
        if (w0) s_nbr[cur ^ 1][lane] = nb_n;
        __syncthreads();  // barrier 2: tiles and D rows built; staging buffers free
        if (slot_n >= 0)
            stage_issue<T, 2, NT, ST>(s_desc, s_tma, &s_bar, s_nbr[cur ^ 1], src, maps, A.dmask, s_raw, s_dm);
        if (NIT == 2) {
            // iteration 1 on the voxels of D in the 10^3 box that iteration 2
            // reads (the leaf and the 6 face slabs of its ring; the ring's
            // edges and corners are never read), compacted per warp: lane l of
            // warp w owns D row r = l * NW + w
            const int r = lane * NW + warp;
            const int rx = r / F, ry = r - rx * F;
            const int edges = (rx == 0 || rx == F - 1) + (ry == 0 || ry == F - 1);
            const unsigned keep = edges == 0 ? 0x3FFu : (edges == 1 ? 0x1FEu : 0u);
            unsigned row = (r < F * F) ? (s_D[r] & keep) : 0u;
            const int c = __popc(row);
            int incl = c;
#pragma unroll
            for (int off = 1; off < 32; off <<= 1) {
                const int y = __shfl_up_sync(0xffffffffu, incl, off);
                if (lane >= off) incl += y;
            }
            const int nW = __shfl_sync(0xffffffffu, incl, 31);
            int pos = incl - c;
            unsigned short* wl = s_list[warp];
            while (row) {
                const int z = __ffs(row) - 1;
                row &= row - 1u;
                wl[pos++] = (unsigned short)(r * F + z);
            }
            __syncwarp();
            for (int i = lane; i < nW; i += 32) {
                const int t = wl[i];
                const int xr = t / (F * F), yr = (t / F) % F, zr = t % F;
                const float* c1 = &s_p1[((xr + 1) * E + (yr + 1)) * E + (zr + 1)];
                const float p = c1[0];
                const Nb6 n = load_nb6<E>(c1, p, hw);
                const float d = fix ? cut_distance(p, n) : __int_as_float(0x7fc00000);
                s_dist[t] = d;
                s_p2[t] = (d == d) ? cut_relax(p, p, d) : godunov_update(p, n, p * rsqrtf(p * p + 1.0f));
            }
            __syncthreads();  // barrier 3: phi2 complete on the 10^3 box
        }
        T* out = dst + (size_t)slot * kLeafVoxels;
        bool any = false;
#pragma unroll
        for (int r = 0; r < VPT; ++r) {
            const int off = threadIdx.x + NT * r;
            const int x = off >> 6, y = (off >> 3) & 7, z = off & 7;
            const bool inD = (s_D[(x + 1) * F + (y + 1)] >> (z + 1)) & 1u;
            const float* c1 = &s_p1[((x + 2) * E + (y + 2)) * E + (z + 2)];
            const float p1 = c1[0];
            float v;
            if (NIT == 0) {
                v = p1;
            } else if (NIT == 1) {
                v = p1;
                if (inD) {
                    const Nb6 n = load_nb6<E>(c1, p1, hw);
                    const float d = fix ? cut_distance(p1, n) : __int_as_float(0x7fc00000);
                    v = (d == d) ? cut_relax(p1, p1, d) : godunov_update(p1, n, p1 * rsqrtf(p1 * p1 + 1.0f));
                }
            } else {
                const int t10 = ((x + 1) * F + (y + 1)) * F + (z + 1);
                const float* c2 = &s_p2[t10];
                const float p2 = c2[0];
                v = p2;
                if (inD) {
                    const float d = fix ? s_dist[t10] : __int_as_float(0x7fc00000);
                    v = (d == d) ? cut_relax(p2, p1, d) : reinit_update<F>(c2, p2, p1 * rsqrtf(p1 * p1 + 1.0f), hw);
                }
            }
            const bool on = inD && fabsf(v) < hw;
            if (!on) v = copysignf(hw, v);
            out[off] = from_f<T>(v);
            const unsigned b = __ballot_sync(0xffffffffu, on);
            if (lane == 0) s_M[off >> 5] = b;
            any |= on;
        }
        __syncthreads();  // barrier 4: the new mask words are in shared memory
        if (threadIdx.x < 16) reinterpret_cast<unsigned*>(A.mask + (size_t)slot * 8)[threadIdx.x] = s_M[threadIdx.x];
        if (threadIdx.x >= 32 && threadIdx.x < 64) {
            // spill mask from 64-bit (x*8+y) plane masks of z = 0, z = 7 and any z
            const unsigned char* B = (const unsigned char*)s_M;
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
            const unsigned bits = __ballot_sync(0xffffffffu, spl && nbr[lane] < 0);
            if (lane == 0) {
                A.spill[slot] = bits;
                A.nonempty[slot] = (za != 0ull) ? 1 : 0;
                if (za != 0ull) topo.keep[slot] = 1;
            }
            // re-tracking proposals: an existing neighbour touched by the spill
            // survives; a missing one is proposed, keeping the proposer whose
            // direction seen from the new leaf comes first (atomicMin).
            if (spl) {
                const int n = nbr[lane];
                if (n >= 0) {
                    topo.keep[n] = 1;
                } else {
                    const int dx = lane / 9 - 1, dy = (lane / 3) % 3 - 1, dz = lane % 3 - 1;
                    const MGridParams& P = params[o.w];
                    const uint64_t key = mkey((long long)(o.x >> 3) + dx, (long long)(o.y >> 3) + dy,
                                              (long long)(o.z >> 3) + dz, o.w, P.base, topo.key_bits);
                    bool done = false;
                    if (key != kEmptyKey) {
                        uint32_t m = (uint32_t)topo.hcap - 1u, p = (uint32_t)mix64(key) & m;
                        for (int probe = 0; probe < topo.hcap; ++probe) {
                            const unsigned long long prev = atomicCAS((unsigned long long*)&topo.pkey[p],
                                                                      (unsigned long long)kEmptyKey,
                                                                      (unsigned long long)key);
                            if (prev == kEmptyKey || prev == key) {
                                atomicMin(&topo.pval[p], kNbr - 1 - lane);
                                done = true;
                                break;
                            }
                            p = (p + 1u) & m;
                        }
                    }
                    if (!done) atomicOr(err, key == kEmptyKey ? kErrExtent : kErrHashFull);
                }
            }
        }
        (void)any;
        if (slot_n < 0) break;
        li += G;
        slot = slot_n;
        if (o_n.w != o.w) hw = params[o_n.w].hw;
        o = o_n;
        slot_n = slot_nn;
    }
}

// --------------------------------------------------------------- feet

// Backtrace displacement of every voxel of n leaves (origins as a level set
// holds them: x, y, z, grid id) over one step of a time-independent velocity
// (constant or curl noise), with k_m_advect's arithmetic (same tables, series
// rotations and integrator): written to disp[bidx[leaf * 512 + voxel]] for
// voxels with bidx >= 0; the largest component magnitude is folded into
// *maxabs (float bits of a non-negative value, atomicMax).  Used by the
// frozen-band adjoint of a level set.
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
        const bool full = s_P.full_series != 0;
        for (int off = threadIdx.x; off < kLeafVoxels; off += 128) {
            const int b = bidx[(size_t)li * kLeafVoxels + off];
            if (b < 0) continue;
            const int x = off >> 6, y = (off >> 3) & 7, z = off & 7;
            const float3 f = full ? backtrace<VK, true>(V, s_tab, x, y, z, dt, integrator, 1.f, 1.f, 1.f)
                                  : backtrace<VK, false>(V, s_tab, x, y, z, dt, integrator, 1.f, 1.f, 1.f);
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

#define VLR_ADVECT_ARGS(T)                                                                       \
    MLeafArrays, const T*, T*, const MGridParams*, const float2*, MStepParams, MTopo, unsigned*, \
        const __grid_constant__ StageMaps
#define VLR_INST_ADVECT_ST(T, H, NT, ST)                                                  \
    template __global__ void k_m_advect<T, H, -1, NT, ST>(VLR_ADVECT_ARGS(T));            \
    template __global__ void k_m_advect<T, H, MVEL_CONSTANT, NT, ST>(VLR_ADVECT_ARGS(T)); \
    template __global__ void k_m_advect<T, H, MVEL_VORTEX, NT, ST>(VLR_ADVECT_ARGS(T));   \
    template __global__ void k_m_advect<T, H, MVEL_CURL, NT, ST>(VLR_ADVECT_ARGS(T));
#define VLR_INST_ADVECT(T, H)                                                                          \
    VLR_INST_ADVECT_ST(T, H, 128, 0) VLR_INST_ADVECT_ST(T, H, 256, 0) VLR_INST_ADVECT_ST(T, H, 128, 1) \
        VLR_INST_ADVECT_ST(T, H, 256, 1)
#define VLR_REINIT_ARGS(T) \
    MLeafArrays, const T*, T*, const MGridParams*, MTopo, int, unsigned*, const __grid_constant__ StageMaps
#define VLR_INST_REINIT_ST(T, NT, ST)                                      \
    template __global__ void k_m_reinit<T, 0, NT, ST>(VLR_REINIT_ARGS(T)); \
    template __global__ void k_m_reinit<T, 1, NT, ST>(VLR_REINIT_ARGS(T)); \
    template __global__ void k_m_reinit<T, 2, NT, ST>(VLR_REINIT_ARGS(T));
#define VLR_INST_REINIT(T) \
    VLR_INST_REINIT_ST(T, 128, 0) VLR_INST_REINIT_ST(T, 256, 0) VLR_INST_REINIT_ST(T, 128, 1) VLR_INST_REINIT_ST(T, 256, 1)
VLR_INST_ADVECT(float, 2)
VLR_INST_ADVECT(float, 3)
VLR_INST_ADVECT(__half, 2)
VLR_INST_ADVECT(__half, 3)
VLR_INST_REINIT(float)
VLR_INST_REINIT(__half)

size_t advect_smem_bytes(int precision_f16, int halo, int stage) {
    if (stage) {
        if (precision_f16) return halo == 2 ? AdvectSmem<__half, 2, 1>::bytes : AdvectSmem<__half, 3, 1>::bytes;
        return halo == 2 ? AdvectSmem<float, 2, 1>::bytes : AdvectSmem<float, 3, 1>::bytes;
    }
    if (precision_f16) return halo == 2 ? AdvectSmem<__half, 2, 0>::bytes : AdvectSmem<__half, 3, 0>::bytes;
    return halo == 2 ? AdvectSmem<float, 2, 0>::bytes : AdvectSmem<float, 3, 0>::bytes;
}

size_t reinit_smem_bytes(int precision_f16, int stage) {
    if (stage) return precision_f16 ? ReinitSmem<__half, 1>::bytes : ReinitSmem<float, 1>::bytes;
    return precision_f16 ? ReinitSmem<__half, 0>::bytes : ReinitSmem<float, 0>::bytes;
}

}  // namespace vlr
