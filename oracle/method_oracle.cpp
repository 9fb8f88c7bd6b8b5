// ORACLE — test infrastructure only.  FP64 restatement of the narrow-band
// method step (see method_oracle.hpp for the definition), plus C entry
// points for ctypes.
#include "method_oracle.hpp"

#include <algorithm>
#include <atomic>
#include <thread>

namespace vlr_method {

namespace {

template <class F>
void parallel_for(int n, int nthreads, F&& f) {
    if (nthreads <= 1 || n < 64) {
        for (int i = 0; i < n; ++i) f(i);
        return;
    }
    std::atomic<int> next{0};
    std::vector<std::thread> th;
    for (int t = 0; t < nthreads; ++t)
        th.emplace_back([&]() {
            for (;;) {
                int i = next.fetch_add(16);
                if (i >= n) break;
                for (int j = i; j < std::min(n, i + 16); ++j) f(j);
            }
        });
    for (auto& t : th) t.join();
}

const int kDir[27][3] = {{-1, -1, -1}, {-1, -1, 0}, {-1, -1, 1}, {-1, 0, -1}, {-1, 0, 0}, {-1, 0, 1}, {-1, 1, -1},
                         {-1, 1, 0},   {-1, 1, 1},  {0, -1, -1}, {0, -1, 0},  {0, -1, 1}, {0, 0, -1},  {0, 0, 0},
                         {0, 0, 1},    {0, 1, -1},  {0, 1, 0},   {0, 1, 1},   {1, -1, -1}, {1, -1, 0}, {1, -1, 1},
                         {1, 0, -1},   {1, 0, 0},   {1, 0, 1},   {1, 1, -1},  {1, 1, 0},  {1, 1, 1}};

// Does leaf L have an active voxel within Chebyshev distance 1 of the leaf
// box at leaf offset d (dx, dy, dz) from L?
bool spills(const Leaf& L, const int* d) {
    for (int off = 0; off < 512; ++off) {
        if (!L.on(off)) continue;
        int x = off >> 6, y = (off >> 3) & 7, z = off & 7;
        int c[3] = {x, y, z};
        bool ok = true;
        for (int a = 0; a < 3 && ok; ++a) {
            if (d[a] == -1) ok = (c[a] == 0);
            else if (d[a] == 1) ok = (c[a] == 7);
        }
        if (ok) return true;
    }
    return false;
}

}  // namespace

bool step(Grid& g, const Velocity& v, int integrator, int reinit_iters, double t, double dt, int nthreads,
          int reinit_mode) {
    const int n = (int)g.leaves.size();
    const double hw = g.hw;
    std::vector<std::vector<char>> Dm(n, std::vector<char>(512));
    parallel_for(n, nthreads, [&](int i) {
        bool D[512];
        dilated(g, i, D);
        for (int q = 0; q < 512; ++q) Dm[i][q] = D[q];
    });
    // 2. advect
    std::vector<Leaf> L1 = g.leaves;
    std::atomic<bool> reach_ok{true};
    parallel_for(n, nthreads, [&](int i) {
        const Leaf& C = g.leaves[i];
        for (int off = 0; off < 512; ++off) {
            if (!Dm[i][off]) {
                L1[i].phi[off] = std::copysign(hw, C.phi[off]);
                continue;
            }
            double x[3] = {(double)(C.o[0] + (off >> 6)), (double)(C.o[1] + ((off >> 3) & 7)),
                           (double)(C.o[2] + (off & 7))};
            double f[3];
            foot(v, integrator, x, t, dt, f);
            for (int a = 0; a < 3; ++a) {
                double b = std::floor(f[a]) - C.o[a];
                if (b < -8 || b + 1 > 15) reach_ok = false;
            }
            L1[i].phi[off] = trilinear(g, g.leaves, i, f);
        }
    });
    // 3. reinit (Jacobi), S0 from the advected field.  Mode 1 (subcell fix):
    //    voxels whose 6-neighbourhood in the advected field crosses zero relax
    //    toward the distance estimated from that field instead of taking the
    //    Godunov update, so reinitialisation does not move the interface.
    std::vector<std::vector<double>> dist;
    if (reinit_iters > 0 && reinit_mode == 1) {
        dist.assign(n, std::vector<double>(512, kNoCut));
        parallel_for(n, nthreads, [&](int i) {
            for (int off = 0; off < 512; ++off)
                if (Dm[i][off]) dist[i][off] = cut_distance(g, L1, i, off);
        });
    }
    std::vector<Leaf> cur = L1, nxt = L1;
    for (int it = 0; it < reinit_iters; ++it) {
        parallel_for(n, nthreads, [&](int i) {
            for (int off = 0; off < 512; ++off) {
                double p = cur[i].phi[off];
                if (!Dm[i][off]) {
                    nxt[i].phi[off] = p;
                    continue;
                }
                double p1 = L1[i].phi[off];
                if (reinit_mode == 1 && dist[i][off] != kNoCut) {
                    nxt[i].phi[off] = p - 0.5 * (std::copysign(std::fabs(p), p1) - dist[i][off]);
                    continue;
                }
                double s = p1 / std::sqrt(p1 * p1 + 1.0);
                double G = godunov(g, cur, i, off, s);
                nxt[i].phi[off] = p - 0.5 * s * (G - 1.0);
            }
        });
        std::swap(cur, nxt);
    }
    // 4. trim
    for (int i = 0; i < n; ++i) {
        std::memset(cur[i].m, 0, sizeof(cur[i].m));
        for (int off = 0; off < 512; ++off) {
            double p = cur[i].phi[off];
            if (Dm[i][off] && std::fabs(p) < hw) cur[i].m[off >> 6] |= 1ull << (off & 63);
            else cur[i].phi[off] = std::copysign(hw, p);
        }
    }
    g.leaves.swap(cur);
    // 5. re-track
    std::vector<char> keep(n, 0);
    std::unordered_map<Key, int, KeyHash> newleaf;  // key -> owner leaf index
    std::vector<Key> new_order;
    for (int i = 0; i < n; ++i) {
        const Leaf& L = g.leaves[i];
        bool any = false;
        for (int w = 0; w < 8; ++w) any |= L.m[w] != 0;
        if (any) keep[i] = 1;
    }
    for (int i = 0; i < n; ++i) {
        const Leaf& L = g.leaves[i];
        int lx = L.o[0] >> 3, ly = L.o[1] >> 3, lz = L.o[2] >> 3;
        for (int d = 0; d < 27; ++d) {
            if (d == 13) continue;
            if (!spills(L, kDir[d])) continue;
            int s = g.find(lx + kDir[d][0], ly + kDir[d][1], lz + kDir[d][2]);
            if (s >= 0) {
                keep[s] = 1;
            } else {
                Key k{lx + kDir[d][0], ly + kDir[d][1], lz + kDir[d][2]};
                if (!newleaf.count(k)) {
                    newleaf[k] = -1;
                    new_order.push_back(k);
                }
            }
        }
    }
    // owners: first existing neighbour (direction order seen from the new leaf) that spills into it
    std::vector<Leaf> out;
    out.reserve(n + new_order.size());
    for (int i = 0; i < n; ++i)
        if (keep[i]) out.push_back(g.leaves[i]);
    for (const Key& k : new_order) {
        int owner = -1;
        for (int d = 0; d < 27 && owner < 0; ++d) {
            if (d == 13) continue;
            int s = g.find(k.x + kDir[d][0], k.y + kDir[d][1], k.z + kDir[d][2]);
            if (s < 0) continue;
            int back[3] = {-kDir[d][0], -kDir[d][1], -kDir[d][2]};
            if (spills(g.leaves[s], back)) owner = s;
        }
        Leaf N;
        N.o[0] = k.x * 8;
        N.o[1] = k.y * 8;
        N.o[2] = k.z * 8;
        std::memset(N.m, 0, sizeof(N.m));
        const Leaf& C = g.leaves[owner];
        for (int off = 0; off < 512; ++off) {
            int px = N.o[0] + (off >> 6), py = N.o[1] + ((off >> 3) & 7), pz = N.o[2] + (off & 7);
            int cx = std::min(7, std::max(0, px - C.o[0]));
            int cy = std::min(7, std::max(0, py - C.o[1]));
            int cz = std::min(7, std::max(0, pz - C.o[2]));
            N.phi[off] = std::copysign(hw, C.phi[(cx << 6) | (cy << 3) | cz]);
        }
        out.push_back(N);
    }
    g.leaves.swap(out);
    g.reindex();
    return reach_ok;
}

Grid sphere(double radius, const double center[3], double vs, const double w0[3], double hw,
            const int32_t*, const int32_t*) {
    Grid g;
    g.hw = hw;
    int32_t lo[3], hi[3];
    for (int a = 0; a < 3; ++a) {
        double c = (center[a] - w0[a]) / vs, r = radius / vs;
        lo[a] = (int32_t)std::floor(c - r - hw - 2.0);
        hi[a] = (int32_t)std::ceil(c + r + hw + 2.0);
    }
    auto phi_at = [&](int32_t x, int32_t y, int32_t z) {
        double dx = w0[0] + vs * x - center[0], dy = w0[1] + vs * y - center[1], dz = w0[2] + vs * z - center[2];
        return (std::sqrt(dx * dx + dy * dy + dz * dz) - radius) / vs;
    };
    for (int32_t lx = lo[0] >> 3; lx <= hi[0] >> 3; ++lx)
        for (int32_t ly = lo[1] >> 3; ly <= hi[1] >> 3; ++ly)
            for (int32_t lz = lo[2] >> 3; lz <= hi[2] >> 3; ++lz) {
                // keep the leaf iff its 10^3 box (one-voxel ring) holds a band voxel
                bool touched = false;
                for (int x = -1; x <= 8 && !touched; ++x)
                    for (int y = -1; y <= 8 && !touched; ++y)
                        for (int z = -1; z <= 8 && !touched; ++z)
                            if (std::fabs(phi_at(lx * 8 + x, ly * 8 + y, lz * 8 + z)) < hw) touched = true;
                if (!touched) continue;
                Leaf L;
                L.o[0] = lx * 8;
                L.o[1] = ly * 8;
                L.o[2] = lz * 8;
                std::memset(L.m, 0, sizeof(L.m));
                for (int off = 0; off < 512; ++off) {
                    double p = phi_at(L.o[0] + (off >> 6), L.o[1] + ((off >> 3) & 7), L.o[2] + (off & 7));
                    if (std::fabs(p) < hw) {
                        L.phi[off] = p;
                        L.m[off >> 6] |= 1ull << (off & 63);
                    } else {
                        L.phi[off] = std::copysign(hw, p);
                    }
                }
                g.leaves.push_back(L);
            }
    g.reindex();
    return g;
}

// Union of spheres in index units (voxel size 1): phi = min_i |p - c_i| - r_i
// over ALL spheres; leaves kept when their 10^3 box holds a band voxel.
Grid spheres_union(const double* sph, int n, double hw) {
    Grid g;
    g.hw = hw;
    auto phi_at = [&](int32_t x, int32_t y, int32_t z) {
        double best = 1e300;
        for (int i = 0; i < n; ++i) {
            double dx = (double)x - sph[4 * i], dy = (double)y - sph[4 * i + 1], dz = (double)z - sph[4 * i + 2];
            best = std::min(best, std::sqrt(dx * dx + dy * dy + dz * dz) - sph[4 * i + 3]);
        }
        return best;
    };
    std::unordered_map<Key, int, KeyHash> cand;
    std::vector<Key> order;
    for (int i = 0; i < n; ++i) {
        int32_t l0[3], l1[3];
        for (int a = 0; a < 3; ++a) {
            l0[a] = ((int32_t)std::floor(sph[4 * i + a] - sph[4 * i + 3] - hw - 2.0)) >> 3;
            l1[a] = ((int32_t)std::ceil(sph[4 * i + a] + sph[4 * i + 3] + hw + 2.0)) >> 3;
        }
        for (int32_t x = l0[0]; x <= l1[0]; ++x)
            for (int32_t y = l0[1]; y <= l1[1]; ++y)
                for (int32_t z = l0[2]; z <= l1[2]; ++z)
                    if (cand.emplace(Key{x, y, z}, 1).second) order.push_back(Key{x, y, z});
    }
    for (const Key& k : order) {
        bool touched = false;
        for (int x = -1; x <= 8 && !touched; ++x)
            for (int y = -1; y <= 8 && !touched; ++y)
                for (int z = -1; z <= 8 && !touched; ++z)
                    if (std::fabs(phi_at(8 * k.x + x, 8 * k.y + y, 8 * k.z + z)) < hw) touched = true;
        if (!touched) continue;
        Leaf L;
        L.o[0] = 8 * k.x;
        L.o[1] = 8 * k.y;
        L.o[2] = 8 * k.z;
        std::memset(L.m, 0, sizeof(L.m));
        for (int off = 0; off < 512; ++off) {
            double p = phi_at(L.o[0] + (off >> 6), L.o[1] + ((off >> 3) & 7), L.o[2] + (off & 7));
            if (std::fabs(p) < hw) {
                L.phi[off] = p;
                L.m[off >> 6] |= 1ull << (off & 63);
            } else {
                L.phi[off] = std::copysign(hw, p);
            }
        }
        g.leaves.push_back(L);
    }
    g.reindex();
    return g;
}

double volume(const Grid& g, const double ref[3]) {
    const double pi = 3.14159265358979323846, eps = 1.5;
    double total = 0.0;
    for (size_t i = 0; i < g.leaves.size(); ++i) {
        const Leaf& L = g.leaves[i];
        for (int off = 0; off < 512; ++off) {
            if (!L.on(off)) continue;
            double p = L.phi[off];
            if (std::fabs(p) >= eps) continue;
            int x = L.o[0] + (off >> 6), y = L.o[1] + ((off >> 3) & 7), z = L.o[2] + (off & 7);
            double gx = 0.5 * (g.read(g.leaves, (int)i, x + 1, y, z) - g.read(g.leaves, (int)i, x - 1, y, z));
            double gy = 0.5 * (g.read(g.leaves, (int)i, x, y + 1, z) - g.read(g.leaves, (int)i, x, y - 1, z));
            double gz = 0.5 * (g.read(g.leaves, (int)i, x, y, z + 1) - g.read(g.leaves, (int)i, x, y, z - 1));
            double delta = (1.0 + std::cos(pi * p / eps)) / (2.0 * eps);
            total += delta * ((x - ref[0]) * gx + (y - ref[1]) * gy + (z - ref[2]) * gz);
        }
    }
    return total / 3.0;
}

}  // namespace vlr_method

// ------------------------------------------------------------------ C API
using namespace vlr_method;

extern "C" {

void* vm_sphere(double radius, const double* center, double vs, const double* w0, double hw) {
    return new Grid(sphere(radius, center, vs, w0, hw, nullptr, nullptr));
}

void vm_free(void* g) { delete (Grid*)g; }

// spheres: n x (cx, cy, cz, r) in index units
void* vm_spheres(const double* spheres, int n, double hw) { return new Grid(spheres_union(spheres, n, hw)); }

size_t vm_leaf_count(void* g) { return ((Grid*)g)->leaves.size(); }

// Export sorted by origin (x, y, z): origins i32[n][3], masks u64[n][8], phi f64[n][512].
void vm_export(void* gp, int32_t* origins, uint64_t* masks, double* phi) {
    Grid* g = (Grid*)gp;
    std::vector<int> order(g->leaves.size());
    for (size_t i = 0; i < order.size(); ++i) order[i] = (int)i;
    std::sort(order.begin(), order.end(), [&](int a, int b) {
        const int32_t* A = g->leaves[a].o;
        const int32_t* B = g->leaves[b].o;
        if (A[0] != B[0]) return A[0] < B[0];
        if (A[1] != B[1]) return A[1] < B[1];
        return A[2] < B[2];
    });
    for (size_t i = 0; i < order.size(); ++i) {
        const Leaf& L = g->leaves[order[i]];
        std::memcpy(origins + 3 * i, L.o, 12);
        std::memcpy(masks + 8 * i, L.m, 64);
        std::memcpy(phi + 512 * i, L.phi, 512 * sizeof(double));
    }
}

void* vm_import(const int32_t* origins, const uint64_t* masks, const double* phi, size_t n, double hw) {
    Grid* g = new Grid();
    g->hw = hw;
    g->leaves.resize(n);
    for (size_t i = 0; i < n; ++i) {
        std::memcpy(g->leaves[i].o, origins + 3 * i, 12);
        std::memcpy(g->leaves[i].m, masks + 8 * i, 64);
        std::memcpy(g->leaves[i].phi, phi + 512 * i, 512 * sizeof(double));
    }
    g->reindex();
    return g;
}

// vel: kind, then parameters packed as doubles:
//   constant: c[3]
//   vortex:   vs, w0[3], period
//   curl:     octaves, then per octave: A, k, ph[3], e[3]
static Velocity unpack_vel(int kind, const double* p) {
    Velocity v;
    v.kind = kind;
    if (kind == VEL_CONSTANT) {
        for (int a = 0; a < 3; ++a) v.c[a] = p[a];
    } else if (kind == VEL_VORTEX) {
        v.vs = p[0];
        for (int a = 0; a < 3; ++a) v.w0[a] = p[1 + a];
        v.period = p[4];
    } else {
        v.octaves = (int)p[0];
        for (int o = 0; o < v.octaves && o < 4; ++o) {
            const double* q = p + 1 + 8 * o;
            v.A[o] = q[0];
            v.k[o] = q[1];
            for (int a = 0; a < 3; ++a) {
                v.ph[o][a] = q[2 + a];
                v.e[o][a] = q[5 + a];
            }
        }
    }
    return v;
}

int vm_step(void* g, int vel_kind, const double* vel_params, int integrator, int reinit_iters, int reinit_mode,
            double t, double dt,
            int nthreads) {
    Velocity v = unpack_vel(vel_kind, vel_params);
    return step(*(Grid*)g, v, integrator, reinit_iters, t, dt, nthreads, reinit_mode) ? 1 : 0;
}

void vm_velocity(int vel_kind, const double* vel_params, const double* p, double t, double* u) {
    Velocity v = unpack_vel(vel_kind, vel_params);
    velocity(v, p, t, u);
}

double vm_volume(void* g, const double* ref) { return volume(*(Grid*)g, ref); }

}  // extern "C"
