// ORACLE — test infrastructure only.  FP64 restatement of the frozen-band
// differentiable advection (vlr_adj_* in the library): forward steps
//   phi_{k+1}(x) = trilinear(phi_k)(x - dt cos(pi t_{k+1}/T) u(x)),
// u = trilinear upsample of a staggered field, and the exact adjoint
//   lambda_k(c) = sum_x lambda_{k+1}(x) w_c(p_k(x)),
//   dL/du(x) = sum_k lambda_{k+1}(x) (-dt c_k) grad trilinear(phi_k)(p_k(x)),
//   dL/dV = upsample^T dL/du,
// accumulated serially in double.  Not in the reference crate (parity with the
// reference is unpinned for this part); checked against FP64 central
// differences in tests/test_adjoint.py.
#include <array>
#include <cmath>
#include <cstring>
#include <vector>

#include "method_oracle.hpp"

using namespace vlr_method;

namespace {

struct Problem {
    Grid g;                       // leaves of phi_0 (double), hw
    std::vector<int> bleaf, boff;  // band voxel -> leaf, offset
    std::vector<double> V;
    int n = 0;
    double H = 1.0, dt = 0.0, T = 1.0, t0 = 0.0;
    int K = 0;
    bool disp = false;  // ub holds fixed displacements, step factor 1 (level-set adjoint)
    std::vector<std::array<double, 3>> ub;
    std::vector<std::vector<Leaf>> states;  // phi_0 .. phi_{K-1} of the last forward run
};

double stag_at(const Problem& P, int a, int i, int j, int k) {
    int n = P.n;
    i = std::min(std::max(i, 0), n - 1);
    j = std::min(std::max(j, 0), n - 1);
    k = std::min(std::max(k, 0), n - 1);
    return P.V[(size_t)a * n * n * n + ((size_t)i * n + j) * n + k];
}

// trilinear upsample weights of component a at voxel point p: 8 (index, weight)
void stag_weights(const Problem& P, int a, const double p[3], int idx[8][3], double w[8]) {
    double g[3] = {p[0] / P.H, p[1] / P.H, p[2] / P.H};
    for (int q = 0; q < 3; ++q)
        if (q != a) g[q] -= 0.5;
    int i0[3];
    double f[3];
    for (int q = 0; q < 3; ++q) {
        double fl = std::floor(g[q]);
        i0[q] = (int)fl;
        f[q] = g[q] - fl;
    }
    for (int q = 0; q < 8; ++q) {
        int di = q >> 2, dj = (q >> 1) & 1, dk = q & 1;
        idx[q][0] = i0[0] + di;
        idx[q][1] = i0[1] + dj;
        idx[q][2] = i0[2] + dk;
        w[q] = (di ? f[0] : 1 - f[0]) * (dj ? f[1] : 1 - f[1]) * (dk ? f[2] : 1 - f[2]);
    }
}

void upsample(Problem& P) {
    P.ub.resize(P.bleaf.size());
    for (size_t b = 0; b < P.bleaf.size(); ++b) {
        const Leaf& L = P.g.leaves[P.bleaf[b]];
        int off = P.boff[b];
        double p[3] = {(double)(L.o[0] + (off >> 6)), (double)(L.o[1] + ((off >> 3) & 7)), (double)(L.o[2] + (off & 7))};
        for (int a = 0; a < 3; ++a) {
            int idx[8][3];
            double w[8];
            stag_weights(P, a, p, idx, w);
            double s = 0.0;
            for (int q = 0; q < 8; ++q) s += w[q] * stag_at(P, a, idx[q][0], idx[q][1], idx[q][2]);
            P.ub[b][a] = s;
        }
    }
}

double step_factor(const Problem& P, int k) {
    if (P.disp) return 1.0;
    const double pi = 3.14159265358979323846;
    return -P.dt * std::cos(pi * (P.t0 + (k + 1) * P.dt) / P.T);
}

}  // namespace

extern "C" {

void* va_create(const int32_t* origins, const uint64_t* masks, const double* phi, size_t n_leaves, double hw,
                const double* V, int n, double H, double dt, double T, double t0, int K) {
    Problem* P = new Problem();
    P->g.hw = hw;
    P->g.leaves.resize(n_leaves);
    for (size_t i = 0; i < n_leaves; ++i) {
        Leaf& L = P->g.leaves[i];
        std::memcpy(L.o, origins + 3 * i, 12);
        std::memcpy(L.m, masks + 8 * i, 64);
        std::memcpy(L.phi, phi + 512 * i, 512 * sizeof(double));
        for (int off = 0; off < 512; ++off)
            if (L.on(off)) {
                P->bleaf.push_back((int)i);
                P->boff.push_back(off);
            }
    }
    P->g.reindex();
    P->n = n;
    P->H = H;
    P->V.assign(V, V + 3ull * n * n * n);
    P->dt = dt;
    P->T = T;
    P->t0 = t0;
    P->K = K;
    upsample(*P);
    return P;
}

// Displacement form (vlr_adj_create_level_set): phi_{k+1}(x) = trilinear(phi_k)(x + d(x))
// with d given per band voxel (band order: leaf order, then ZYX).
void* va_create_disp(const int32_t* origins, const uint64_t* masks, const double* phi, size_t n_leaves, double hw,
                     const double* disp, int K) {
    Problem* P = new Problem();
    P->g.hw = hw;
    P->g.leaves.resize(n_leaves);
    for (size_t i = 0; i < n_leaves; ++i) {
        Leaf& L = P->g.leaves[i];
        std::memcpy(L.o, origins + 3 * i, 12);
        std::memcpy(L.m, masks + 8 * i, 64);
        std::memcpy(L.phi, phi + 512 * i, 512 * sizeof(double));
        for (int off = 0; off < 512; ++off)
            if (L.on(off)) {
                P->bleaf.push_back((int)i);
                P->boff.push_back(off);
            }
    }
    P->g.reindex();
    P->n = 0;
    P->K = K;
    P->disp = true;
    P->ub.resize(P->bleaf.size());
    for (size_t b = 0; b < P->bleaf.size(); ++b)
        for (int a = 0; a < 3; ++a) P->ub[b][a] = disp[3 * b + a];
    return P;
}

void va_free(void* p) { delete (Problem*)p; }
int va_nband(void* p) { return (int)((Problem*)p)->bleaf.size(); }

void va_forward(void* pp, const double* phi0_band, const double* V, double* phik_band) {
    Problem& P = *(Problem*)pp;
    if (V) {
        std::memcpy(P.V.data(), V, sizeof(double) * P.V.size());
        upsample(P);
    }
    std::vector<Leaf> cur = P.g.leaves;
    if (phi0_band)
        for (size_t b = 0; b < P.bleaf.size(); ++b) cur[P.bleaf[b]].phi[P.boff[b]] = phi0_band[b];
    P.states.clear();
    for (int k = 0; k < P.K; ++k) {
        P.states.push_back(cur);
        std::vector<Leaf> nxt = cur;
        double s = step_factor(P, k);
        for (size_t b = 0; b < P.bleaf.size(); ++b) {
            int li = P.bleaf[b], off = P.boff[b];
            const Leaf& L = cur[li];
            double p[3] = {L.o[0] + (off >> 6) + s * P.ub[b][0], L.o[1] + ((off >> 3) & 7) + s * P.ub[b][1],
                           L.o[2] + (off & 7) + s * P.ub[b][2]};
            nxt[li].phi[off] = trilinear(P.g, cur, li, p);
        }
        cur.swap(nxt);
    }
    for (size_t b = 0; b < P.bleaf.size(); ++b) phik_band[b] = cur[P.bleaf[b]].phi[P.boff[b]];
}

void va_backward(void* pp, const double* lamK, double* grad_phi0, double* grad_V) {
    Problem& P = *(Problem*)pp;
    const size_t nb = P.bleaf.size();
    // band index of each (leaf, offset)
    std::vector<int> bidx(P.g.leaves.size() * 512, -1);
    for (size_t b = 0; b < nb; ++b) bidx[(size_t)P.bleaf[b] * 512 + P.boff[b]] = (int)b;
    std::vector<double> lam(lamK, lamK + nb), G(3 * nb, 0.0);
    for (int k = P.K - 1; k >= 0; --k) {
        const std::vector<Leaf>& phik = P.states[k];
        std::vector<double> nl(nb, 0.0);
        double s = step_factor(P, k);
        for (size_t b = 0; b < nb; ++b) {
            int li = P.bleaf[b], off = P.boff[b];
            const Leaf& L = phik[li];
            double p[3] = {L.o[0] + (off >> 6) + s * P.ub[b][0], L.o[1] + ((off >> 3) & 7) + s * P.ub[b][1],
                           L.o[2] + (off & 7) + s * P.ub[b][2]};
            int base[3];
            double f[3];
            for (int a = 0; a < 3; ++a) {
                double fl = std::floor(p[a]);
                base[a] = (int)fl;
                f[a] = p[a] - fl;
            }
            double c[8];
            for (int q = 0; q < 8; ++q) {
                int di = q >> 2, dj = (q >> 1) & 1, dk = q & 1;
                int x = base[0] + di, y = base[1] + dj, z = base[2] + dk;
                double w = (di ? f[0] : 1 - f[0]) * (dj ? f[1] : 1 - f[1]) * (dk ? f[2] : 1 - f[2]);
                c[q] = P.g.read(phik, li, x, y, z);
                int sl = P.g.find(x >> 3, y >> 3, z >> 3);
                if (sl >= 0) {
                    int bb = bidx[(size_t)sl * 512 + (((x & 7) << 6) | ((y & 7) << 3) | (z & 7))];
                    if (bb >= 0) nl[bb] += lam[b] * w;
                }
            }
            double wx[2] = {1 - f[0], f[0]}, wy[2] = {1 - f[1], f[1]}, wz[2] = {1 - f[2], f[2]};
            double gx = wy[0] * wz[0] * (c[4] - c[0]) + wy[1] * wz[0] * (c[6] - c[2]) + wy[0] * wz[1] * (c[5] - c[1]) +
                        wy[1] * wz[1] * (c[7] - c[3]);
            double gy = wx[0] * wz[0] * (c[2] - c[0]) + wx[1] * wz[0] * (c[6] - c[4]) + wx[0] * wz[1] * (c[3] - c[1]) +
                        wx[1] * wz[1] * (c[7] - c[5]);
            double gz = wx[0] * wy[0] * (c[1] - c[0]) + wx[1] * wy[0] * (c[5] - c[4]) + wx[0] * wy[1] * (c[3] - c[2]) +
                        wx[1] * wy[1] * (c[7] - c[6]);
            G[3 * b] += lam[b] * s * gx;
            G[3 * b + 1] += lam[b] * s * gy;
            G[3 * b + 2] += lam[b] * s * gz;
        }
        lam.swap(nl);
    }
    std::memcpy(grad_phi0, lam.data(), sizeof(double) * nb);
    if (P.disp || !grad_V) return;
    std::fill(grad_V, grad_V + P.V.size(), 0.0);
    for (size_t b = 0; b < nb; ++b) {
        const Leaf& L = P.g.leaves[P.bleaf[b]];
        int off = P.boff[b];
        double p[3] = {(double)(L.o[0] + (off >> 6)), (double)(L.o[1] + ((off >> 3) & 7)), (double)(L.o[2] + (off & 7))};
        for (int a = 0; a < 3; ++a) {
            int idx[8][3];
            double w[8];
            stag_weights(P, a, p, idx, w);
            for (int q = 0; q < 8; ++q) {
                int n = P.n;
                int i = std::min(std::max(idx[q][0], 0), n - 1), j = std::min(std::max(idx[q][1], 0), n - 1),
                    kk = std::min(std::max(idx[q][2], 0), n - 1);
                grad_V[(size_t)a * n * n * n + ((size_t)i * n + j) * n + kk] += G[3 * b + a] * w[q];
            }
        }
    }
}

}  // extern "C"
