// The two stencil kernels of the METHOD step.  One CTA (256 threads) works on
// one 8^3 leaf at a time and strides over the ordered leaf list (persistent).
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
// Instruction economy (both kernels are issue-bound at small leaf counts):
// the halo is staged one z-row per thread with 16-byte vector loads, grid
// parameters and the leaf's 8 sin/cos table entries per axis are copied to
// shared memory once per leaf, dilated voxels are compacted into a list so
// warps only run backtraces, and results leave through shared memory in
// 16-byte stores.
#include "method_kernels.hpp"

namespace vlr {

constexpr int kT = 256;

__device__ __forceinline__ int nb_axis(int c) { return (c < 0) ? 0 : (c > 7 ? 2 : 1); }

// Copy one grid's parameters into shared memory (all threads call; caller syncs).
__device__ __forceinline__ void load_params(const MGridParams* __restrict__ params, int gid, MGridParams* s_P) {
    const int* src = (const int*)(params + gid);
    int* dst = (int*)s_P;
    for (int i = threadIdx.x; i < (int)(sizeof(MGridParams) / 4); i += blockDim.x) dst[i] = src[i];
}

// Stage one z-row (E values) of the halo tile.  Row (sx, sy) of the tile maps
// to local (x, y) = (sx - H, sy - H); z runs over [-H, 8 + H).  Missing
// neighbour leaves are filled by `fill(zc)` given the clamped z of the centre
// leaf row.
template <typename T, int H>
__device__ __forceinline__ void load_row8(const T* __restrict__ p, float* out) {
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

// Fill `row` (E floats) for tile row (x, y) in local leaf coordinates.
// missing_mode 0: copysign(hw, centre value at clamped position); 1: NaN.
template <typename T, int H, int MISSING>
__device__ __forceinline__ void stage_row(const T* __restrict__ vals, const int* s_nbr, const T* __restrict__ centre,
                                          int x, int y, float hw, float* row) {
    constexpr int E = 8 + 2 * H;
    const int base = nb_axis(x) * 9 + nb_axis(y) * 3;
    const int rowoff = ((x & 7) << 6) | ((y & 7) << 3);
    const int crow = (min(max(x, 0), 7) << 6) | (min(max(y, 0), 7) << 3);
    const int s0 = s_nbr[base], s1 = s_nbr[base + 1], s2 = s_nbr[base + 2];
    float mid[8];
    if (s1 >= 0) {
        load_row8<T, H>(vals + (size_t)s1 * kLeafVoxels + rowoff, mid);
    } else if (MISSING == 0) {
        load_row8<T, H>(centre + crow, mid);
#pragma unroll
        for (int i = 0; i < 8; ++i) mid[i] = copysignf(hw, mid[i]);
    } else {
#pragma unroll
        for (int i = 0; i < 8; ++i) mid[i] = __int_as_float(0x7fc00000);
    }
#pragma unroll
    for (int i = 0; i < 8; ++i) row[H + i] = mid[i];
#pragma unroll
    for (int i = 0; i < H; ++i) {
        float lo, hi;
        if (s0 >= 0) lo = to_f(vals[(size_t)s0 * kLeafVoxels + rowoff + 8 - H + i]);
        else lo = (MISSING == 0) ? copysignf(hw, to_f(centre[crow])) : __int_as_float(0x7fc00000);
        if (s2 >= 0) hi = to_f(vals[(size_t)s2 * kLeafVoxels + rowoff + i]);
        else hi = (MISSING == 0) ? copysignf(hw, to_f(centre[crow + 7])) : __int_as_float(0x7fc00000);
        row[i] = lo;
        row[H + 8 + i] = hi;
    }
}

template <typename T>
__device__ __forceinline__ void store_leaf(T* __restrict__ dst, const float* s_out) {
    if constexpr (sizeof(T) == 2) {
        if (threadIdx.x < 64) {
            const float4* q = reinterpret_cast<const float4*>(s_out + 8 * threadIdx.x);
            float4 a = q[0], b = q[1];
            __half2 h[4] = {__floats2half2_rn(a.x, a.y), __floats2half2_rn(a.z, a.w), __floats2half2_rn(b.x, b.y),
                            __floats2half2_rn(b.z, b.w)};
            *reinterpret_cast<uint4*>(dst + 8 * threadIdx.x) = *reinterpret_cast<uint4*>(h);
        }
    } else {
        if (threadIdx.x < 128)
            reinterpret_cast<float4*>(dst)[threadIdx.x] = reinterpret_cast<const float4*>(s_out)[threadIdx.x];
    }
}

__device__ __forceinline__ float2 rotate(float2 t, float d, int full) {
    float sd, cd;
    if (full) small_sincos(d, sd, cd);
    else tiny_sincos(d, sd, cd);
    return make_float2(t.x * cd + t.y * sd, t.y * cd - t.x * sd);
}

// Velocity (voxels per unit time) at local voxel (lx, ly, lz) + offset, from
// the leaf's staged tables.  kOff = false: no offset (voxel centre).
template <bool kOff>
__device__ __forceinline__ float3 leaf_velocity(const MGridParams& P, const float2 (*tab)[3][8], int lx, int ly, int lz,
                                                float ox, float oy, float oz, float ct) {
    if (P.vel_kind == MVEL_CONSTANT) return make_float3(P.c[0], P.c[1], P.c[2]);
    if (P.vel_kind == MVEL_VORTEX) {
        float2 X = tab[0][0][lx], Y = tab[0][1][ly], Z = tab[0][2][lz];
        if (kOff) {
            X = rotate(X, P.dphi[0] * ox, P.full_series);
            Y = rotate(Y, P.dphi[0] * oy, P.full_series);
            Z = rotate(Z, P.dphi[0] * oz, P.full_series);
        }
        float k = P.vel_scale * ct;
        float sycy = Y.x * Y.y, szcz = Z.x * Z.y, sxcx = X.x * X.y;
        return make_float3(8.0f * k * X.x * X.x * sycy * szcz, -4.0f * k * sxcx * Y.x * Y.x * szcz,
                           -4.0f * k * sxcx * sycy * Z.x * Z.x);
    }
    float3 u = make_float3(0.f, 0.f, 0.f);
    for (int o = 0; o < P.octaves; ++o) {
        float2 X = tab[o][0][lx], Y = tab[o][1][ly], Z = tab[o][2][lz];
        if (kOff) {
            X = rotate(X, P.dphi[o] * ox, P.full_series);
            Y = rotate(Y, P.dphi[o] * oy, P.full_series);
            Z = rotate(Z, P.dphi[o] * oz, P.full_series);
        }
        float a = P.ak[o];
        float gx = a * X.y * Y.x * Z.x, gy = a * X.x * Y.y * Z.x, gz = a * X.x * Y.x * Z.y;
        u.x += gy * P.e[o][2] - gz * P.e[o][1];
        u.y += gz * P.e[o][0] - gx * P.e[o][2];
        u.z += gx * P.e[o][1] - gy * P.e[o][0];
    }
    return u;
}

// --------------------------------------------------------------- advect

template <typename T, int H>
__global__ void __launch_bounds__(kT, 4) k_m_advect(MLeafArrays A, const T* __restrict__ src, T* __restrict__ dst,
                                                const MGridParams* __restrict__ params, const float2* __restrict__ tab,
                                                MStepParams sp, MTopo topo, unsigned* __restrict__ err) {
    // clear this step's re-tracking state (keep flags, proposal table, leaf hash)
    for (int i = blockIdx.x * kT + threadIdx.x; i < max(topo.cap, topo.hcap); i += gridDim.x * kT) {
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
    constexpr int E = 8 + 2 * H;
    constexpr int NROW = E * E;
    constexpr int NTAB = kMaxOctaves * 3 * 8;
    __shared__ __align__(16) float s_tile[E * E * E];
    __shared__ __align__(16) float s_out[kLeafVoxels];
    __shared__ __align__(16) uint64_t s_m[kNbr * 8];
    __shared__ __align__(16) uint64_t s_D[8];
    __shared__ int s_nbr[kNbr];
    __shared__ unsigned short s_list[kLeafVoxels];
    __shared__ __align__(16) MGridParams s_P;
    __shared__ float2 s_tab[kMaxOctaves][3][8];
    const int count = *A.count;
    const int step = *A.step;
    const float t1 = sp.t0 + (float)(step + 1) * sp.dt;
    const float dt = sp.dt;
    unsigned bad = 0;
    int cur_gid = -1;
    float ct1 = 1.f, ct2 = 1.f, ct3 = 1.f;  // vortex time factors cos(pi t / T) at t1, t1 - dt/2, t1 - dt
    for (int li = blockIdx.x; li < count; li += gridDim.x) {
        const int slot = A.list[li];
        const int4 o = A.origin[slot];
        if (o.w != cur_gid) {
            load_params(params, o.w, &s_P);
            cur_gid = o.w;
            const MGridParams& G = params[o.w];
            if (G.vel_kind == MVEL_VORTEX) {
                ct1 = cosf(G.pi_over_T * t1);
                ct2 = cosf(G.pi_over_T * (t1 - 0.5f * dt));
                ct3 = cosf(G.pi_over_T * (t1 - dt));
            }
        }
        if (threadIdx.x < kNbr * 8) {
            int d = threadIdx.x >> 3;
            int s = A.nbr[slot * kNbr + d];
            if ((threadIdx.x & 7) == 0) s_nbr[d] = s;
            s_m[threadIdx.x] = (s < 0) ? 0ull : A.mask[(size_t)s * 8 + (threadIdx.x & 7)];
        }
        __syncthreads();
        const float hw = s_P.hw;
        const T* centre = src + (size_t)slot * kLeafVoxels;
        for (int t = threadIdx.x; t < NROW + NTAB + 64; t += kT) {
            if (t < NROW) {
                float row[E];
                stage_row<T, H, 0>(src, s_nbr, centre, t / E - H, t % E - H, hw, row);
                float* dstrow = s_tile + t * E;
#pragma unroll
                for (int i = 0; i < E; ++i) dstrow[i] = row[i];
            } else if (t < NROW + NTAB) {
                int q = t - NROW;
                int f = q / 24, a = (q / 8) % 3, l = q % 8;
                if (s_P.vel_kind != MVEL_CONSTANT && (s_P.vel_kind == MVEL_CURL ? f < s_P.octaves : f == 0)) {
                    int oc = (a == 0 ? o.x : (a == 1 ? o.y : o.z)) + l - s_P.tab_lo[a];
                    if (oc < 0 || oc >= s_P.tab_len[a]) {
                        bad = 1u;
                        oc = min(max(oc, 0), s_P.tab_len[a] - 1);
                    }
                    s_tab[f][a][l] = __ldg(&tab[s_P.tab_off[f][a] + oc]);
                }
            } else {
                // dilation: one thread per z-row, 10-bit rows z = -1..8
                int r = t - NROW - NTAB;
                int x = r >> 3, y = r & 7;
                unsigned acc = 0;
#pragma unroll
                for (int dx = -1; dx <= 1; ++dx)
#pragma unroll
                    for (int dy = -1; dy <= 1; ++dy) {
                        int xx = x + dx, yy = y + dy;
                        int base = nb_axis(xx) * 9 + nb_axis(yy) * 3;
                        int bi = ((xx & 7) << 3) | (yy & 7);
                        const unsigned char* m = (const unsigned char*)s_m;
                        acc |= ((unsigned)m[base * 64 + bi] >> 7) | ((unsigned)m[(base + 1) * 64 + bi] << 1) |
                               (((unsigned)m[(base + 2) * 64 + bi] & 1u) << 9);
                    }
                ((unsigned char*)s_D)[r] = (unsigned char)(((acc | (acc << 1) | (acc >> 1)) >> 1) & 0xffu);
            }
        }
        __syncthreads();
        // compact D; voxels outside D keep the sign of their previous value
        int nD = 0, pre = 0;
        const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
#pragma unroll
        for (int q = 0; q < 8; ++q) {
            int c = __popcll(s_D[q]);
            if (q < w) pre += c;
            nD += c;
        }
        {
            const uint64_t word = s_D[w];
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                const int bit = lane + 32 * h;
                const int off = w * 64 + bit;
                const int x = off >> 6, y = (off >> 3) & 7, z = off & 7;
                if ((word >> bit) & 1ull)
                    s_list[pre + __popcll(word & ((1ull << bit) - 1ull))] = (unsigned short)off;
                else
                    s_out[off] = copysignf(hw, s_tile[((x + H) * E + (y + H)) * E + (z + H)]);
            }
        }
        __syncthreads();
        for (int i = threadIdx.x; i < nD; i += kT) {
            const int off = s_list[i];
            const int x = off >> 6, y = (off >> 3) & 7, z = off & 7;
            float fx, fy, fz;
            float3 k1 = leaf_velocity<false>(s_P, s_tab, x, y, z, 0.f, 0.f, 0.f, ct1);
            if (sp.integrator == 1) {
                fx = -dt * k1.x;
                fy = -dt * k1.y;
                fz = -dt * k1.z;
            } else if (sp.integrator == 2) {
                float3 k2 = leaf_velocity<true>(s_P, s_tab, x, y, z, -0.5f * dt * k1.x, -0.5f * dt * k1.y,
                                                -0.5f * dt * k1.z, ct2);
                fx = -dt * k2.x;
                fy = -dt * k2.y;
                fz = -dt * k2.z;
            } else {
                const float h = -dt;
                float ax = h * k1.x, ay = h * k1.y, az = h * k1.z;
                float3 k2 = leaf_velocity<true>(s_P, s_tab, x, y, z, ax, ay, az, ct3);
                float bx = 0.25f * (ax + h * k2.x), by = 0.25f * (ay + h * k2.y), bz = 0.25f * (az + h * k2.z);
                float3 k3 = leaf_velocity<true>(s_P, s_tab, x, y, z, bx, by, bz, ct2);
                fx = (2.0f / 3.0f) * (bx + h * k3.x);
                fy = (2.0f / 3.0f) * (by + h * k3.y);
                fz = (2.0f / 3.0f) * (bz + h * k3.z);
            }
            float px = (float)(x + H) + fx, py = (float)(y + H) + fy, pz = (float)(z + H) + fz;
            float bxf = floorf(px), byf = floorf(py), bzf = floorf(pz);
            float wx = px - bxf, wy = py - byf, wz = pz - bzf;
            int ii = (int)bxf, jj = (int)byf, kk = (int)bzf;
            if (ii < 0 || jj < 0 || kk < 0 || ii > E - 2 || jj > E - 2 || kk > E - 2 || !(px == px) ||
                !(py == py) || !(pz == pz)) {
                bad = 1u;
                ii = min(max(ii, 0), E - 2);
                jj = min(max(jj, 0), E - 2);
                kk = min(max(kk, 0), E - 2);
                wx = fminf(fmaxf(wx, 0.f), 1.f);
                wy = fminf(fmaxf(wy, 0.f), 1.f);
                wz = fminf(fmaxf(wz, 0.f), 1.f);
            }
            const float* q = &s_tile[(ii * E + jj) * E + kk];
            float c000 = q[0], c001 = q[1], c010 = q[E], c011 = q[E + 1];
            float c100 = q[E * E], c101 = q[E * E + 1], c110 = q[E * E + E], c111 = q[E * E + E + 1];
            float c00 = c000 * (1.f - wx) + c100 * wx, c01 = c001 * (1.f - wx) + c101 * wx;
            float c10 = c010 * (1.f - wx) + c110 * wx, c11 = c011 * (1.f - wx) + c111 * wx;
            float c0 = c00 * (1.f - wy) + c10 * wy, c1 = c01 * (1.f - wy) + c11 * wy;
            s_out[off] = c0 * (1.f - wz) + c1 * wz;
        }
        __syncthreads();
        store_leaf<T>(dst + (size_t)slot * kLeafVoxels, s_out);
        if (threadIdx.x < 8) A.dmask[(size_t)slot * 8 + threadIdx.x] = s_D[threadIdx.x];
        __syncthreads();
    }
    if (bad) atomicOr(err, kErrReach);
}

// -------------------------------------------------------------- reinit

__device__ __forceinline__ float godunov_g(float p, float xm, float xp, float ym, float yp, float zm, float zp, float s) {
    float am0 = p - xm, am1 = p - ym, am2 = p - zm;
    float ap0 = xp - p, ap1 = yp - p, ap2 = zp - p;
    float u0, u1, u2, w0, w1, w2;
    if (s >= 0.f) {
        u0 = fmaxf(am0, 0.f); u1 = fmaxf(am1, 0.f); u2 = fmaxf(am2, 0.f);
        w0 = fminf(ap0, 0.f); w1 = fminf(ap1, 0.f); w2 = fminf(ap2, 0.f);
    } else {
        u0 = fminf(am0, 0.f); u1 = fminf(am1, 0.f); u2 = fminf(am2, 0.f);
        w0 = fmaxf(ap0, 0.f); w1 = fmaxf(ap1, 0.f); w2 = fmaxf(ap2, 0.f);
    }
    float g2 = fmaxf(u0 * u0, w0 * w0) + fmaxf(u1 * u1, w1 * w1);
    g2 += fmaxf(u2 * u2, w2 * w2);
    return sqrtf(g2);
}

// NaN marks a voxel of an unallocated leaf; a 6-neighbour stencil reads it as
// copysign(hw, phi(centre)).
__device__ __forceinline__ float nbv(float v, float centre, float hw) { return (v != v) ? copysignf(hw, centre) : v; }

template <int S>
__device__ __forceinline__ float reinit_update(const float* c, float p, float s, float hw) {
    float G = godunov_g(p, nbv(c[-S * S], p, hw), nbv(c[S * S], p, hw), nbv(c[-S], p, hw), nbv(c[S], p, hw),
                        nbv(c[-1], p, hw), nbv(c[1], p, hw), s);
    return p - 0.5f * s * (G - 1.0f);
}

template <typename T, int NIT>
__global__ void __launch_bounds__(kT) k_m_reinit(MLeafArrays A, const T* __restrict__ src, T* __restrict__ dst,
                                                const MGridParams* __restrict__ params, MTopo topo,
                                                unsigned* __restrict__ err) {
    constexpr int E = 12;  // phi1 tile: leaf + 2-voxel ring
    constexpr int F = 10;  // phi2 tile and D rows: leaf + 1-voxel ring
    __shared__ __align__(16) float s_p1[E * E * E];
    __shared__ __align__(16) float s_p2[F * F * F];
    __shared__ __align__(16) float s_out[kLeafVoxels];
    __shared__ __align__(16) uint64_t s_dm[kNbr * 8];
    __shared__ unsigned short s_D[F * F];
    __shared__ int s_nbr[kNbr];
    __shared__ __align__(16) unsigned s_M[16];
    const int count = *A.count;
    for (int li = blockIdx.x; li < count; li += gridDim.x) {
        const int slot = A.list[li];
        const int4 o = A.origin[slot];
        const float hw = params[o.w].hw;
        if (threadIdx.x < kNbr * 8) {
            int d = threadIdx.x >> 3;
            int s = A.nbr[slot * kNbr + d];
            if ((threadIdx.x & 7) == 0) s_nbr[d] = s;
            s_dm[threadIdx.x] = (s < 0) ? 0ull : A.dmask[(size_t)s * 8 + (threadIdx.x & 7)];
        }
        __syncthreads();
        for (int t = threadIdx.x; t < E * E + F * F; t += kT) {
            if (t < E * E) {
                float row[E];
                stage_row<T, 2, 1>(src, s_nbr, nullptr, t / E - 2, t % E - 2, hw, row);
                float4* d4 = reinterpret_cast<float4*>(s_p1 + t * E);
                d4[0] = make_float4(row[0], row[1], row[2], row[3]);
                d4[1] = make_float4(row[4], row[5], row[6], row[7]);
                d4[2] = make_float4(row[8], row[9], row[10], row[11]);
            } else {
                int r = t - E * E;
                int x = r / F - 1, y = r % F - 1;
                int base = nb_axis(x) * 9 + nb_axis(y) * 3;
                int bi = ((x & 7) << 3) | (y & 7);
                const unsigned char* m = (const unsigned char*)s_dm;
                s_D[r] = (unsigned short)(((unsigned)m[base * 64 + bi] >> 7) | ((unsigned)m[(base + 1) * 64 + bi] << 1) |
                                          (((unsigned)m[(base + 2) * 64 + bi] & 1u) << 9));
            }
        }
        __syncthreads();
        if (NIT == 2) {
            for (int t = threadIdx.x; t < F * F * F; t += kT) {
                int xr = t / (F * F), yr = (t / F) % F, zr = t % F;
                const float* c = &s_p1[((xr + 1) * E + (yr + 1)) * E + (zr + 1)];
                float p = c[0];
                float q = p;
                if ((s_D[xr * F + yr] >> zr) & 1u) q = reinit_update<E>(c, p, p * rsqrtf(p * p + 1.0f), hw);
                s_p2[t] = q;
            }
            __syncthreads();
        }
        bool any = false;
#pragma unroll
        for (int r = 0; r < 2; ++r) {
            const int off = threadIdx.x + kT * r;
            const int x = off >> 6, y = (off >> 3) & 7, z = off & 7;
            const bool inD = (s_D[(x + 1) * F + (y + 1)] >> (z + 1)) & 1u;
            const float* c1 = &s_p1[((x + 2) * E + (y + 2)) * E + (z + 2)];
            const float p1 = c1[0];
            float v;
            if (NIT == 0) {
                v = p1;
            } else if (NIT == 1) {
                v = inD ? reinit_update<E>(c1, p1, p1 * rsqrtf(p1 * p1 + 1.0f), hw) : p1;
            } else {
                const float* c2 = &s_p2[((x + 1) * F + (y + 1)) * F + (z + 1)];
                float p2 = c2[0];
                v = inD ? reinit_update<F>(c2, p2, p1 * rsqrtf(p1 * p1 + 1.0f), hw) : p2;
            }
            const bool on = inD && fabsf(v) < hw;
            if (!on) v = copysignf(hw, v);
            s_out[off] = v;
            unsigned b = __ballot_sync(0xffffffffu, on);
            if ((threadIdx.x & 31) == 0) s_M[off >> 5] = b;
            any |= on;
        }
        __syncthreads();
        store_leaf<T>(dst + (size_t)slot * kLeafVoxels, s_out);
        if (threadIdx.x < 16) reinterpret_cast<unsigned*>(A.mask + (size_t)slot * 8)[threadIdx.x] = s_M[threadIdx.x];
        if (threadIdx.x < 32) {
            // spill mask from 64-bit (x*8+y) plane masks of z = 0, z = 7 and any z
            const int lane = threadIdx.x;
            const unsigned char* B = (const unsigned char*)s_M;
            unsigned b0 = B[lane], b1 = B[lane + 32];
            uint64_t z0 = (uint64_t)__ballot_sync(0xffffffffu, b0 & 1u) | ((uint64_t)__ballot_sync(0xffffffffu, b1 & 1u) << 32);
            uint64_t z7 = (uint64_t)__ballot_sync(0xffffffffu, b0 & 0x80u) | ((uint64_t)__ballot_sync(0xffffffffu, b1 & 0x80u) << 32);
            uint64_t za = (uint64_t)__ballot_sync(0xffffffffu, b0 != 0u) | ((uint64_t)__ballot_sync(0xffffffffu, b1 != 0u) << 32);
            bool spl = false;
            if (lane < kNbr && lane != 13) {
                int dx = lane / 9 - 1, dy = (lane / 3) % 3 - 1, dz = lane % 3 - 1;
                uint64_t plane = dz < 0 ? z0 : (dz > 0 ? z7 : za);
                uint64_t xs = dx < 0 ? 0xFFull : (dx > 0 ? (0xFFull << 56) : ~0ull);
                uint64_t ys = dy < 0 ? 0x0101010101010101ull : (dy > 0 ? 0x8080808080808080ull : ~0ull);
                spl = (plane & xs & ys) != 0ull;
            }
            unsigned bits = __ballot_sync(0xffffffffu, spl);
            if (lane == 0) {
                A.spill[slot] = bits;
                A.nonempty[slot] = (za != 0ull) ? 1 : 0;
                if (za != 0ull) topo.keep[slot] = 1;
            }
            // re-tracking proposals: an existing neighbour touched by the spill
            // survives; a missing one is proposed, keeping the proposer whose
            // direction seen from the new leaf comes first (atomicMin).
            if (spl) {
                const int n = s_nbr[lane];
                if (n >= 0) {
                    topo.keep[n] = 1;
                } else {
                    int dx = lane / 9 - 1, dy = (lane / 3) % 3 - 1, dz = lane % 3 - 1;
                    const MGridParams& P = params[o.w];
                    uint64_t key = mkey((long long)(o.x >> 3) + dx, (long long)(o.y >> 3) + dy,
                                        (long long)(o.z >> 3) + dz, o.w, P.base, topo.key_bits);
                    bool done = false;
                    if (key != kEmptyKey) {
                        uint32_t m = (uint32_t)topo.hcap - 1u, p = (uint32_t)mix64(key) & m;
                        for (int probe = 0; probe < topo.hcap; ++probe) {
                            unsigned long long prev = atomicCAS((unsigned long long*)&topo.pkey[p],
                                                                (unsigned long long)kEmptyKey, (unsigned long long)key);
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
        __syncthreads();
    }
}

#define VLR_INST_STENCIL(T)                                                                                      \
    template __global__ void k_m_advect<T, 2>(MLeafArrays, const T*, T*, const MGridParams*, const float2*,        \
                                              MStepParams, MTopo, unsigned*);                                    \
    template __global__ void k_m_advect<T, 3>(MLeafArrays, const T*, T*, const MGridParams*, const float2*,        \
                                              MStepParams, MTopo, unsigned*);                                    \
    template __global__ void k_m_reinit<T, 0>(MLeafArrays, const T*, T*, const MGridParams*, MTopo, unsigned*);    \
    template __global__ void k_m_reinit<T, 1>(MLeafArrays, const T*, T*, const MGridParams*, MTopo, unsigned*);    \
    template __global__ void k_m_reinit<T, 2>(MLeafArrays, const T*, T*, const MGridParams*, MTopo, unsigned*);
VLR_INST_STENCIL(float)
VLR_INST_STENCIL(__half)

}  // namespace vlr
