// Level sets made of unions of spheres, one or many grids per leaf pool
// (vlr_ls_create_spheres), and per-grid download (vlr_ls_download_grid).
//
// Candidate leaves are found on the host per sphere (leaves whose 10^3 box,
// the leaf plus a one-voxel ring, meets the sphere's band), each with the
// list of spheres whose band-expanded ball meets the box; a box that lies
// deeper than the half width inside one sphere is skipped.  On the device
// phi = min over the leaf's spheres of |p - c| - r (f64, as the oracle), which
// equals the union's SDF wherever |phi| < hw and has its sign elsewhere; a
// leaf is kept when its 10^3 box holds a band voxel (the leaf is touched by
// dilate26 of the band).
#include <algorithm>
#include <array>
#include <cmath>
#include <cstring>
#include <numeric>
#include <unordered_map>
#include <vector>

#include "method_state.hpp"

namespace vlr {

template <typename T>
__global__ void __launch_bounds__(256) k_m_spheres(const int4* __restrict__ cand, int n_cand,
                                                  const int* __restrict__ off, const int* __restrict__ sidx,
                                                  const double4* __restrict__ spheres, double hwd, int4* origin,
                                                  uint64_t* mask, T* vals, int* touched) {
    __shared__ int s_touch;
    for (int c = blockIdx.x; c < n_cand; c += gridDim.x) {
        const int4 L = cand[c];
        const int b = off[c], e = off[c + 1];
        if (threadIdx.x == 0) s_touch = 0;
        __syncthreads();
        auto phi_at = [&](int x, int y, int z) -> double {
            double best = 1e300;
            for (int q = b; q < e; ++q) {
                double4 S = spheres[sidx[q]];
                double dx = __dsub_rn((double)x, S.x), dy = __dsub_rn((double)y, S.y), dz = __dsub_rn((double)z, S.z);
                double d = __dsqrt_rn(__dadd_rn(__dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy)), __dmul_rn(dz, dz)));
                best = fmin(best, __dsub_rn(d, S.w));
            }
            return best;
        };
        bool any = false;
        for (int t = threadIdx.x; t < 1000; t += 256) {
            int x = L.x + t / 100 - 1, y = L.y + (t / 10) % 10 - 1, z = L.z + t % 10 - 1;
            if (fabs(phi_at(x, y, z)) < hwd) any = true;
        }
        if (any) s_touch = 1;
        __syncthreads();
        for (int r = 0; r < 2; ++r) {
            int o = threadIdx.x + 256 * r;
            double p = phi_at(L.x + (o >> 6), L.y + ((o >> 3) & 7), L.z + (o & 7));
            bool on = fabs(p) < hwd;
            float v = on ? (float)p : copysignf((float)hwd, (float)p);
            vals[(size_t)c * kLeafVoxels + o] = from_f<T>(v);
            unsigned bal = __ballot_sync(0xffffffffu, on);
            if ((threadIdx.x & 31) == 0) ((unsigned*)(mask + (size_t)c * 8))[o >> 5] = bal;
        }
        if (threadIdx.x == 0) {
            origin[c] = L;
            touched[c] = s_touch;
        }
        __syncthreads();
    }
}

template <typename T>
__global__ void k_m_pick(const int* flags, const int* pos, int n, const int4* o_in, const uint64_t* m_in,
                         const T* v_in, int4* o_out, uint64_t* m_out, T* v_out) {
    for (int i = blockIdx.x; i < n; i += gridDim.x) {
        if (!flags[i]) continue;
        int j = pos[i];
        if (threadIdx.x == 0) o_out[j] = o_in[i];
        if (threadIdx.x < 8) m_out[(size_t)j * 8 + threadIdx.x] = m_in[(size_t)i * 8 + threadIdx.x];
        for (int t = threadIdx.x; t < kLeafVoxels; t += blockDim.x)
            v_out[(size_t)j * kLeafVoxels + t] = v_in[(size_t)i * kLeafVoxels + t];
    }
}

namespace {

struct LeafKey {
    int32_t x, y, z;
    bool operator==(const LeafKey& o) const { return x == o.x && y == o.y && z == o.z; }
};
struct LeafKeyHash {
    size_t operator()(const LeafKey& k) const {
        return (size_t)mix64(((uint64_t)(uint32_t)k.x << 42) ^ ((uint64_t)(uint32_t)k.y << 21) ^ (uint32_t)k.z);
    }
};

// Distance from point c to the box [lo, hi] (nearest and farthest).
inline void box_dist(const double c[3], const double lo[3], const double hi[3], double& dmin, double& dmax) {
    double a = 0.0, b = 0.0;
    for (int k = 0; k < 3; ++k) {
        double n = std::max(0.0, std::max(lo[k] - c[k], c[k] - hi[k]));
        double f = std::max(std::fabs(c[k] - lo[k]), std::fabs(c[k] - hi[k]));
        a += n * n;
        b += f * f;
    }
    dmin = std::sqrt(a);
    dmax = std::sqrt(b);
}

}  // namespace

int create_spheres_impl(vlr_ctx* ctx, vlr_level_set* ls, const vlr_method_desc* m, const vlr_batch_grid* grids,
                        int n_grids) {
    const double hw = (double)m->half_width;
    ls->key_bits = (n_grids == 1) ? 21 : 18;
    if (n_grids > 1 && n_grids > (1 << (63 - 3 * 18)))
        return set_error(ctx, VLR_ERR_INVALID, "at most 512 grids per batch");
    std::vector<double4> spheres;
    std::vector<int4> cand;          // candidate leaf origins (+ grid id)
    std::vector<int> off(1, 0), sidx;
    std::vector<const vlr_velocity_desc*> vels(n_grids);
    std::vector<std::array<int32_t, 3>> blo(n_grids), bhi(n_grids);
    for (int g = 0; g < n_grids; ++g) {
        const vlr_batch_grid& G = grids[g];
        vels[g] = &G.velocity;
        if (G.n_spheres < 1 || !G.spheres) return set_error(ctx, VLR_ERR_INVALID, "grid without spheres");
        const int s0 = (int)spheres.size();
        double lo[3] = {1e300, 1e300, 1e300}, hi[3] = {-1e300, -1e300, -1e300};
        for (int i = 0; i < G.n_spheres; ++i) {
            const vlr_sphere& S = G.spheres[i];
            if (!(S.radius > 0.0)) return set_error(ctx, VLR_ERR_INVALID, "sphere radius must be positive");
            spheres.push_back(make_double4(S.center[0], S.center[1], S.center[2], S.radius));
            for (int a = 0; a < 3; ++a) {
                lo[a] = std::min(lo[a], S.center[a] - S.radius);
                hi[a] = std::max(hi[a], S.center[a] + S.radius);
            }
        }
        for (int a = 0; a < 3; ++a) {
            blo[g][a] = (int32_t)std::floor(lo[a] - hw - 2.0);
            bhi[g][a] = (int32_t)std::ceil(hi[a] + hw + 2.0);
            if (((long long)bhi[g][a] - blo[g][a]) >> 3 >= (1ll << (ls->key_bits - 1)) - 4)
                return set_error(ctx, VLR_ERR_EXTENT, "grid spans too many voxels along an axis for its batch");
        }
        // candidate leaves: the 10^3 box meets some sphere's band.  Each
        // sphere visits the boxes of its own bounding range once and records
        // (box, sphere) pairs; a box lying deeper than hw inside any sphere is
        // interior and skipped.  Candidates keep the order in which a band
        // first reaches them, and each lists its spheres in ascending index
        // (the spheres whose band-expanded ball meets the box).
        std::unordered_map<LeafKey, int, LeafKeyHash> kid;   // box -> index in keys
        std::vector<LeafKey> keys;
        std::vector<int> disc;                               // discovery rank per key, -1 if none
        std::vector<char> inner;                             // key lies inside some sphere
        std::vector<std::pair<int, int>> pairs;              // (key index, sphere), sphere-major
        int n_disc = 0;
        auto key_index = [&](const LeafKey& k) {
            auto it = kid.emplace(k, (int)keys.size());
            if (it.second) {
                keys.push_back(k);
                disc.push_back(-1);
                inner.push_back(0);
            }
            return it.first->second;
        };
        for (int i = 0; i < G.n_spheres; ++i) {
            const vlr_sphere& S = G.spheres[i];
            int32_t l0[3], l1[3];
            for (int a = 0; a < 3; ++a) {
                l0[a] = ((int32_t)std::floor(S.center[a] - S.radius - hw - 2.0)) >> 3;
                l1[a] = ((int32_t)std::ceil(S.center[a] + S.radius + hw + 2.0)) >> 3;
            }
            for (int32_t x = l0[0]; x <= l1[0]; ++x)
                for (int32_t y = l0[1]; y <= l1[1]; ++y)
                    for (int32_t z = l0[2]; z <= l1[2]; ++z) {
                        double bl[3] = {8.0 * x - 1, 8.0 * y - 1, 8.0 * z - 1}, bh[3] = {8.0 * x + 8, 8.0 * y + 8, 8.0 * z + 8};
                        double dmin, dmax;
                        box_dist(S.center, bl, bh, dmin, dmax);
                        if (dmax < S.radius - hw) {
                            inner[key_index(LeafKey{x, y, z})] = 1;
                        } else if (dmin < S.radius + hw) {
                            const int j = key_index(LeafKey{x, y, z});
                            pairs.emplace_back(j, s0 + i);
                            if (dmax > S.radius - hw && disc[j] < 0) disc[j] = n_disc++;
                        }
                    }
        }
        // pairs grouped by key (stable: spheres stay ascending within a key)
        std::vector<int> start(keys.size() + 1, 0);
        for (const auto& pr : pairs) ++start[pr.first + 1];
        for (size_t j = 0; j < keys.size(); ++j) start[j + 1] += start[j];
        std::vector<int> by_key(pairs.size());
        {
            std::vector<int> fill(start.begin(), start.end() - 1);
            for (const auto& pr : pairs) by_key[fill[pr.first]++] = pr.second;
        }
        std::vector<int> order_of(n_disc, -1);
        for (size_t j = 0; j < keys.size(); ++j)
            if (disc[j] >= 0) order_of[disc[j]] = (int)j;
        for (int r = 0; r < n_disc; ++r) {
            const int j = order_of[r];
            if (inner[j]) continue;
            const LeafKey& k = keys[j];
            sidx.insert(sidx.end(), by_key.begin() + start[j], by_key.begin() + start[j + 1]);
            cand.push_back(make_int4(8 * k.x, 8 * k.y, 8 * k.z, g));
            off.push_back((int)sidx.size());
        }
    }
    int rc = ls_setup_grids(ctx, ls, m, vels.data(), reinterpret_cast<const int32_t(*)[3]>(blo.data()),
                            reinterpret_cast<const int32_t(*)[3]>(bhi.data()), n_grids);
    if (rc) return rc;
    const long long n_cand = (long long)cand.size();
    if (n_cand == 0) return set_error(ctx, VLR_ERR_INVALID, "no band leaves");
    if (n_cand > (1ll << 28)) return set_error(ctx, VLR_ERR_CAPACITY, "too many candidate leaves");
    size_t vb = (ls->precision == VLR_PREC_F16) ? 2 : 4;
    int4 *d_cand = nullptr, *o_tmp = nullptr;
    int *d_off = nullptr, *d_sidx = nullptr, *touched = nullptr, *pos = nullptr;
    double4* d_sph = nullptr;
    uint64_t* m_tmp = nullptr;
    void* v_tmp = nullptr;
    DeviceTemps temps;  // freed on every return
    VLR_CUDA(ctx, cudaMalloc(&d_cand, sizeof(int4) * n_cand));
    temps.track(d_cand);
    VLR_CUDA(ctx, cudaMalloc(&d_off, sizeof(int) * (n_cand + 1)));
    temps.track(d_off);
    VLR_CUDA(ctx, cudaMalloc(&d_sidx, sizeof(int) * std::max<size_t>(sidx.size(), 1)));
    temps.track(d_sidx);
    VLR_CUDA(ctx, cudaMalloc(&d_sph, sizeof(double4) * spheres.size()));
    temps.track(d_sph);
    VLR_CUDA(ctx, cudaMalloc(&o_tmp, sizeof(int4) * n_cand));
    temps.track(o_tmp);
    VLR_CUDA(ctx, cudaMalloc(&m_tmp, 64ull * n_cand));
    temps.track(m_tmp);
    VLR_CUDA(ctx, cudaMalloc(&v_tmp, vb * kLeafVoxels * n_cand));
    temps.track(v_tmp);
    VLR_CUDA(ctx, cudaMalloc(&touched, sizeof(int) * (n_cand + 1)));
    temps.track(touched);
    VLR_CUDA(ctx, cudaMalloc(&pos, sizeof(int) * (n_cand + 1)));
    temps.track(pos);
    VLR_CUDA(ctx, cudaMemcpyAsync(d_cand, cand.data(), sizeof(int4) * n_cand, cudaMemcpyHostToDevice, ctx->stream));
    VLR_CUDA(ctx, cudaMemcpyAsync(d_off, off.data(), sizeof(int) * (n_cand + 1), cudaMemcpyHostToDevice, ctx->stream));
    if (!sidx.empty())
        VLR_CUDA(ctx, cudaMemcpyAsync(d_sidx, sidx.data(), sizeof(int) * sidx.size(), cudaMemcpyHostToDevice,
                                      ctx->stream));
    VLR_CUDA(ctx, cudaMemcpyAsync(d_sph, spheres.data(), sizeof(double4) * spheres.size(), cudaMemcpyHostToDevice,
                                  ctx->stream));
    int blocks = (int)std::min<long long>(n_cand, (long long)ctx->sm_count * 16);
    if (ls->precision == VLR_PREC_F16)
        k_m_spheres<__half><<<blocks, 256, 0, ctx->stream>>>(d_cand, (int)n_cand, d_off, d_sidx, d_sph, hw, o_tmp,
                                                             m_tmp, (__half*)v_tmp, touched);
    else
        k_m_spheres<float><<<blocks, 256, 0, ctx->stream>>>(d_cand, (int)n_cand, d_off, d_sidx, d_sph, hw, o_tmp,
                                                            m_tmp, (float*)v_tmp, touched);
    VLR_CUDA(ctx, cudaGetLastError());
    rc = scan_exclusive(ctx, touched, pos, (int)n_cand, pos + n_cand);
    if (rc) return rc;
    int n = 0;
    rc = read_int(ctx, pos + n_cand, &n);
    if (rc) return rc;
    int cap = m->capacity ? (int)std::min<size_t>(m->capacity, (size_t)1 << 30) : (int)std::min<long long>(2ll * n + 4096, 1ll << 30);
    if (cap < n) return set_error(ctx, VLR_ERR_CAPACITY, "capacity below the initial leaf count");
    rc = ls_alloc(ctx, ls, cap);
    if (rc) return rc;
    if (ls->precision == VLR_PREC_F16)
        k_m_pick<__half><<<blocks, 256, 0, ctx->stream>>>(touched, pos, (int)n_cand, o_tmp, m_tmp,
                                                          (const __half*)v_tmp, ls->origin, ls->mask,
                                                          (__half*)ls->vals[0]);
    else
        k_m_pick<float><<<blocks, 256, 0, ctx->stream>>>(touched, pos, (int)n_cand, o_tmp, m_tmp, (const float*)v_tmp,
                                                         ls->origin, ls->mask, (float*)ls->vals[0]);
    VLR_CUDA(ctx, cudaGetLastError());
    VLR_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    return ls_init_lists(ctx, ls, n, true);
}

}  // namespace vlr

using namespace vlr;

extern "C" {

int vlr_ls_create_spheres(vlr_ctx* ctx, const vlr_method_desc* m, const vlr_batch_grid* grids, int n_grids,
                          vlr_level_set** out) {
    if (!ctx || !m || !grids || !out || n_grids < 1) return set_error(ctx, VLR_ERR_INVALID, "null argument");
    *out = nullptr;
    vlr_level_set* ls = new vlr_level_set();
    ls->ctx = ctx;
    ls->precision = m->precision == VLR_PREC_F16 ? VLR_PREC_F16 : VLR_PREC_F32;
    int rc = create_spheres_impl(ctx, ls, m, grids, n_grids);
    if (rc) {
        vlr_ls_destroy(ls);
        return rc;
    }
    *out = ls;
    return VLR_OK;
}

}  // extern "C"
