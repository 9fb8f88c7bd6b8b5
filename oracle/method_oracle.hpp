// ORACLE — test infrastructure only. Never linked into the product library.
//
// FP64 CPU restatement of the narrow-band level-set METHOD step that the GPU
// library runs (semi-Lagrangian RK backtrace with analytic velocity,
// Godunov-upwind reinitialisation, dilation-based re-tracking, FP64 volume).
// None of this exists in the Sharc.Volrus crate: parity with the reference is
// unpinned for this part; the oracle is written from the mathematics and
// defines the method that the GPU kernels must reproduce (to rounding).
//
// State of a grid: allocated 8^3 leaves (ZYX order as src/math/coord.rs:74-82),
// values phi in VOXEL units, activity masks.  Invariants between steps:
//   * every voxel of dilate26(active) lies in an allocated leaf;
//   * inactive voxels of allocated leaves hold +-hw (sign-aware background).
// Reading a voxel of an unallocated leaf from a computation centred on leaf C
// gives copysign(hw, phi_C[clamp(p - origin_C, 0, 7)]).
//
// Step t -> t + dt (velocity u in index units per unit time):
//  1. D = dilate26(active)                      (26-neighbourhood, one voxel)
//  2. advect: x in D  -> phi1(x) = trilinear(phi0)(foot(x))
//             x not in D -> copysign(hw, phi0(x))
//     foot: Euler x - dt u(x, t1); RK2 midpoint; SSP-RK3 (Shu-Osher), t1 = t + dt
//  3. reinit (N iterations, Jacobi, dtau = 0.5): S0 = phi1/sqrt(phi1^2 + 1);
//     phi <- phi - dtau S0 (G(phi) - 1) on D, G = Godunov |grad phi|; in mode
//     1 cut voxels (a 6-neighbour of opposite sign in phi1) instead relax
//     toward the distance d = phi1 / |grad phi1|:
//     phi <- phi - dtau (sign(phi1) |phi| - d)   (cut_distance below)
//  4. trim: active = D and |phi| < hw; others become copysign(hw, phi)
//  5. re-track: keep leaves touched by dilate26(active); allocate missing ones,
//     filled from the first proposing neighbour (fixed direction order) by the
//     clamped-sign rule above; drop the rest.
#pragma once
#include <cmath>
#include <cstdint>
#include <cstring>
#include <unordered_map>
#include <vector>

namespace vlr_method {

enum VelKind { VEL_CONSTANT = 0, VEL_VORTEX = 1, VEL_CURL = 2 };

struct Velocity {
    int kind = VEL_CONSTANT;
    double c[3] = {0, 0, 0};      // constant, index units per unit time
    // vortex (world coordinates of the unit cube): world = w0 + vs * p
    double vs = 1.0, w0[3] = {0, 0, 0}, period = 1.0;
    // curl noise: v = sum_o grad f_o x e_o,
    // f_o(p) = A_o prod_a sin(k_o p_a + ph_{o,a})   (index units)
    int octaves = 0;
    double A[4] = {0, 0, 0, 0}, k[4] = {0, 0, 0, 0}, ph[4][3] = {}, e[4][3] = {};
};

// velocity in index units per unit time at index position p, time t
inline void velocity(const Velocity& v, const double p[3], double t, double u[3]) {
    if (v.kind == VEL_CONSTANT) {
        u[0] = v.c[0];
        u[1] = v.c[1];
        u[2] = v.c[2];
    } else if (v.kind == VEL_VORTEX) {
        const double pi = 3.14159265358979323846;
        double x = v.w0[0] + v.vs * p[0], y = v.w0[1] + v.vs * p[1], z = v.w0[2] + v.vs * p[2];
        double sx = std::sin(pi * x), cx = std::cos(pi * x);
        double sy = std::sin(pi * y), cy = std::cos(pi * y);
        double sz = std::sin(pi * z), cz = std::cos(pi * z);
        double ct = std::cos(pi * t / v.period);
        // u = 2 sin^2(pi x) sin(2 pi y) sin(2 pi z) cos(pi t / T), etc. (world units) / vs
        u[0] = 8.0 * sx * sx * sy * cy * sz * cz * ct / v.vs;
        u[1] = -4.0 * sx * cx * sy * sy * sz * cz * ct / v.vs;
        u[2] = -4.0 * sx * cx * sy * cy * sz * sz * ct / v.vs;
    } else {
        u[0] = u[1] = u[2] = 0.0;
        for (int o = 0; o < v.octaves; ++o) {
            double s[3], c[3];
            for (int a = 0; a < 3; ++a) {
                s[a] = std::sin(v.k[o] * p[a] + v.ph[o][a]);
                c[a] = std::cos(v.k[o] * p[a] + v.ph[o][a]);
            }
            double ak = v.A[o] * v.k[o];
            double g[3] = {ak * c[0] * s[1] * s[2], ak * s[0] * c[1] * s[2], ak * s[0] * s[1] * c[2]};
            const double* e = v.e[o];
            u[0] += g[1] * e[2] - g[2] * e[1];
            u[1] += g[2] * e[0] - g[0] * e[2];
            u[2] += g[0] * e[1] - g[1] * e[0];
        }
    }
}

struct Key {
    int32_t x, y, z;  // leaf origin / 8
    bool operator==(const Key& o) const { return x == o.x && y == o.y && z == o.z; }
};
struct KeyHash {
    size_t operator()(const Key& k) const {
        uint64_t h = (uint64_t)(uint32_t)k.x * 0x9E3779B97F4A7C15ull;
        h ^= (uint64_t)(uint32_t)k.y * 0xC2B2AE3D27D4EB4Full + (h << 6) + (h >> 2);
        h ^= (uint64_t)(uint32_t)k.z * 0x165667B19E3779F9ull + (h << 6) + (h >> 2);
        return (size_t)h;
    }
};

struct Leaf {
    int32_t o[3];
    double phi[512];
    uint64_t m[8];
    bool on(int off) const { return (m[off >> 6] >> (off & 63)) & 1ull; }
};

inline int floordiv8(int32_t v) { return v >> 3; }

struct Grid {
    double hw = 3.0;
    std::vector<Leaf> leaves;
    std::unordered_map<Key, int, KeyHash> index;

    void reindex() {
        index.clear();
        index.reserve(leaves.size() * 2);
        for (size_t i = 0; i < leaves.size(); ++i)
            index[Key{leaves[i].o[0] >> 3, leaves[i].o[1] >> 3, leaves[i].o[2] >> 3}] = (int)i;
    }
    int find(int32_t lx, int32_t ly, int32_t lz) const {
        auto it = index.find(Key{lx, ly, lz});
        return it == index.end() ? -1 : it->second;
    }
    // phi at absolute voxel p read from a computation centred on leaf c
    double read(const std::vector<Leaf>& L, int c, int32_t px, int32_t py, int32_t pz) const {
        int s = find(px >> 3, py >> 3, pz >> 3);
        if (s >= 0) return L[s].phi[((px & 7) << 6) | ((py & 7) << 3) | (pz & 7)];
        const Leaf& C = L[c];
        int cx = std::min(7, std::max(0, px - C.o[0]));
        int cy = std::min(7, std::max(0, py - C.o[1]));
        int cz = std::min(7, std::max(0, pz - C.o[2]));
        return std::copysign(hw, C.phi[(cx << 6) | (cy << 3) | cz]);
    }
    bool active_at(int32_t px, int32_t py, int32_t pz) const {
        int s = find(px >> 3, py >> 3, pz >> 3);
        if (s < 0) return false;
        return leaves[s].on(((px & 7) << 6) | ((py & 7) << 3) | (pz & 7));
    }
};

// D = dilate26(active) restricted to leaf i, as a 512-entry bool array.
inline void dilated(const Grid& g, int i, bool D[512]) {
    const Leaf& L = g.leaves[i];
    for (int off = 0; off < 512; ++off) {
        int x = L.o[0] + (off >> 6), y = L.o[1] + ((off >> 3) & 7), z = L.o[2] + (off & 7);
        bool d = false;
        for (int dx = -1; dx <= 1 && !d; ++dx)
            for (int dy = -1; dy <= 1 && !d; ++dy)
                for (int dz = -1; dz <= 1 && !d; ++dz)
                    if (g.active_at(x + dx, y + dy, z + dz)) d = true;
        D[off] = d;
    }
}

inline double trilinear(const Grid& g, const std::vector<Leaf>& L, int c, const double p[3]) {
    double bx = std::floor(p[0]), by = std::floor(p[1]), bz = std::floor(p[2]);
    double fx = p[0] - bx, fy = p[1] - by, fz = p[2] - bz;
    int32_t i = (int32_t)bx, j = (int32_t)by, k = (int32_t)bz;
    double c000 = g.read(L, c, i, j, k), c100 = g.read(L, c, i + 1, j, k);
    double c010 = g.read(L, c, i, j + 1, k), c110 = g.read(L, c, i + 1, j + 1, k);
    double c001 = g.read(L, c, i, j, k + 1), c101 = g.read(L, c, i + 1, j, k + 1);
    double c011 = g.read(L, c, i, j + 1, k + 1), c111 = g.read(L, c, i + 1, j + 1, k + 1);
    double c00 = c000 * (1 - fx) + c100 * fx, c01 = c001 * (1 - fx) + c101 * fx;
    double c10 = c010 * (1 - fx) + c110 * fx, c11 = c011 * (1 - fx) + c111 * fx;
    double c0 = c00 * (1 - fy) + c10 * fy, c1 = c01 * (1 - fy) + c11 * fy;
    return c0 * (1 - fz) + c1 * fz;
}

// Backtrace of voxel x over [t, t + dt] (integrate dX/ds = u backwards from t1).
inline void foot(const Velocity& v, int integrator, const double x[3], double t, double dt, double out[3]) {
    double t1 = t + dt, u[3];
    if (integrator == 1) {
        velocity(v, x, t1, u);
        for (int a = 0; a < 3; ++a) out[a] = x[a] - dt * u[a];
    } else if (integrator == 2) {
        velocity(v, x, t1, u);
        double mid[3];
        for (int a = 0; a < 3; ++a) mid[a] = x[a] - 0.5 * dt * u[a];
        velocity(v, mid, t1 - 0.5 * dt, u);
        for (int a = 0; a < 3; ++a) out[a] = x[a] - dt * u[a];
    } else {
        // SSP-RK3 with step h = -dt from s0 = t1:
        // X1 = X0 + h u(X0, s0); X2 = 3/4 X0 + 1/4 (X1 + h u(X1, s0 + h));
        // X3 = 1/3 X0 + 2/3 (X2 + h u(X2, s0 + h/2))
        double h = -dt, X1[3], X2[3];
        velocity(v, x, t1, u);
        for (int a = 0; a < 3; ++a) X1[a] = x[a] + h * u[a];
        velocity(v, X1, t1 + h, u);
        for (int a = 0; a < 3; ++a) X2[a] = 0.75 * x[a] + 0.25 * (X1[a] + h * u[a]);
        velocity(v, X2, t1 + 0.5 * h, u);
        for (int a = 0; a < 3; ++a) out[a] = x[a] / 3.0 + (2.0 / 3.0) * (X2[a] + h * u[a]);
    }
}

// Godunov |grad phi| at voxel off of leaf c, upwinded by the sign s.
inline double godunov(const Grid& g, const std::vector<Leaf>& L, int c, int off, double s) {
    const Leaf& C = L[c];
    int x = C.o[0] + (off >> 6), y = C.o[1] + ((off >> 3) & 7), z = C.o[2] + (off & 7);
    double p0 = C.phi[off];
    double nb[6] = {g.read(L, c, x - 1, y, z), g.read(L, c, x + 1, y, z), g.read(L, c, x, y - 1, z),
                    g.read(L, c, x, y + 1, z), g.read(L, c, x, y, z - 1), g.read(L, c, x, y, z + 1)};
    double g2 = 0.0;
    for (int a = 0; a < 3; ++a) {
        double am = p0 - nb[2 * a];      // backward difference
        double ap = nb[2 * a + 1] - p0;  // forward difference
        double q;
        if (s >= 0.0) {
            double u = std::max(am, 0.0), w = std::min(ap, 0.0);
            q = std::max(u * u, w * w);
        } else {
            double u = std::min(am, 0.0), w = std::max(ap, 0.0);
            q = std::max(u * u, w * w);
        }
        g2 += q;
    }
    return std::sqrt(g2);
}

// Subcell fix of the reinitialisation (Russo & Smereka, J. Comput. Phys. 163,
// 2000): a voxel whose 6-neighbourhood in phi0 (the field before
// reinitialisation) changes sign is a cut voxel; its distance to the interface
// is estimated as phi0 / |grad phi0| with, per axis, the largest of the
// central and the two one-sided differences (at least 1e-6), and the
// iteration relaxes it toward that distance,
//   phi <- phi - 1/2 (sign(phi0) |phi| - d),
// instead of taking the Godunov update.  Returns kNoCut for other voxels.
constexpr double kNoCut = 1e300;
inline double cut_distance(const Grid& g, const std::vector<Leaf>& L0, int c, int off) {
    const Leaf& C = L0[c];
    int x = C.o[0] + (off >> 6), y = C.o[1] + ((off >> 3) & 7), z = C.o[2] + (off & 7);
    double p = C.phi[off];
    double nb[6] = {g.read(L0, c, x - 1, y, z), g.read(L0, c, x + 1, y, z), g.read(L0, c, x, y - 1, z),
                    g.read(L0, c, x, y + 1, z), g.read(L0, c, x, y, z - 1), g.read(L0, c, x, y, z + 1)};
    bool cut = false;
    for (int k = 0; k < 6; ++k) cut |= (p * nb[k] < 0.0);
    if (!cut) return kNoCut;
    double d2 = 0.0;
    for (int a = 0; a < 3; ++a) {
        double m = std::max(std::max(std::fabs(nb[2 * a + 1] - nb[2 * a]) * 0.5, std::fabs(nb[2 * a + 1] - p)),
                            std::max(std::fabs(p - nb[2 * a]), 1e-6));
        d2 += m * m;
    }
    return p / std::sqrt(d2);
}

// One method step; returns false if a foot left the 27-leaf neighbourhood.
// reinit_mode 0: plain Godunov; 1: Godunov with the subcell fix at cut voxels.
bool step(Grid& g, const Velocity& v, int integrator, int reinit_iters, double t, double dt, int nthreads,
          int reinit_mode = 0);

// Initial state from the sphere SDF (index units): phi = (|p*vs + w0 - c| - r)/vs.
Grid sphere(double radius, const double center[3], double vs, const double w0[3], double hw,
            const int32_t box_lo[3], const int32_t box_hi[3]);

// Union of spheres (index units, voxel size 1): phi = min_i |p - c_i| - r_i.
Grid spheres_union(const double* sph, int n, double hw);

// Enclosed volume in index units^3 by the smeared-delta surface integral
// V = (1/3) sum_active delta_eps(phi) (p - ref) . grad phi, eps = 1.5 voxels.
double volume(const Grid& g, const double ref[3]);

}  // namespace vlr_method
