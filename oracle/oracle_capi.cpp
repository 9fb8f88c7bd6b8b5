// ORACLE — test infrastructure only (loaded by tests/, smoke() and the CPU
// baseline leg of bench.py through ctypes).  Plain-C entry points over the
// restatement in ref_tree.hpp.  Grids cross the boundary as flat leaf arrays
// (origin i32[3], mask u64[8], values f32[512]) sorted lexicographically by
// origin, the order NanoGrid::from_grid uses (src/nano/layout.rs:81-106).
#include "ref_tree.hpp"

#include <algorithm>
#include <array>
#include <chrono>
#include <cmath>

using namespace vlr_oracle;

namespace {
std::vector<const Leaf*> sorted_leaves(const Grid& g) {
    std::vector<const Leaf*> v;
    g.for_each_leaf([&](const Leaf& l) { v.push_back(&l); });
    std::sort(v.begin(), v.end(), [](const Leaf* a, const Leaf* b) {
        if (a->origin.x != b->origin.x) return a->origin.x < b->origin.x;
        if (a->origin.y != b->origin.y) return a->origin.y < b->origin.y;
        return a->origin.z < b->origin.z;
    });
    return v;
}
}  // namespace

extern "C" {

void* vo_grid_new(float bg, double vs, const double* t_origin, const double* mat12, double affine_vs) {
    Grid* g = new Grid();
    g->background = bg;
    g->voxel_size = vs;
    for (int i = 0; i < 3; ++i) g->t_origin[i] = t_origin ? t_origin[i] : 0.0;
    if (mat12) {
        for (int r = 0; r < 3; ++r)
            for (int c = 0; c < 4; ++c) g->mat[r][c] = mat12[r * 4 + c];
    } else {
        std::memset(g->mat, 0, sizeof(g->mat));
        g->mat[0][0] = g->mat[1][1] = g->mat[2][2] = vs;
    }
    g->affine_voxel_size = affine_vs;
    return g;
}

void vo_grid_free(void* g) { delete (Grid*)g; }

void vo_grid_put_leaves(void* gp, const int32_t* origins, const uint64_t* masks, const float* values, size_t n) {
    Grid* g = (Grid*)gp;
    for (size_t i = 0; i < n; ++i)
        g->put_leaf(Coord{origins[3 * i], origins[3 * i + 1], origins[3 * i + 2]}, masks + 8 * i, values + 512 * i);
}

size_t vo_grid_leaf_count(void* g) { return ((Grid*)g)->leaf_count(); }
uint64_t vo_grid_active_count(void* g) { return ((Grid*)g)->active_voxel_count(); }

void vo_grid_export(void* gp, int32_t* origins, uint64_t* masks, float* values) {
    auto v = sorted_leaves(*(Grid*)gp);
    for (size_t i = 0; i < v.size(); ++i) {
        origins[3 * i] = v[i]->origin.x;
        origins[3 * i + 1] = v[i]->origin.y;
        origins[3 * i + 2] = v[i]->origin.z;
        std::memcpy(masks + 8 * i, v[i]->active, 64);
        std::memcpy(values + 512 * i, v[i]->values, 2048);
    }
}

void vo_grid_meta(void* gp, float* bg, double* vs, double* t_origin, double* mat12, double* affine_vs) {
    Grid* g = (Grid*)gp;
    *bg = g->background;
    *vs = g->voxel_size;
    for (int i = 0; i < 3; ++i) t_origin[i] = g->t_origin[i];
    for (int r = 0; r < 3; ++r)
        for (int c = 0; c < 4; ++c) mat12[r * 4 + c] = g->mat[r][c];
    *affine_vs = g->affine_voxel_size;
}

float vo_get(void* g, int32_t x, int32_t y, int32_t z) { return ((Grid*)g)->get(Coord{x, y, z}); }
int vo_is_active(void* g, int32_t x, int32_t y, int32_t z) { return ((Grid*)g)->is_active(Coord{x, y, z}); }
void vo_set(void* g, int32_t x, int32_t y, int32_t z, float v) { ((Grid*)g)->set(Coord{x, y, z}, v); }
void vo_deactivate(void* g, int32_t x, int32_t y, int32_t z) { ((Grid*)g)->deactivate(Coord{x, y, z}); }

void* vo_make_level_set_sphere(double radius, const double* center, double vs, double hw) {
    return new Grid(make_level_set_sphere(radius, center, vs, hw));
}

void vo_sample_trilinear(void* g, const double* world, size_t n, float* out) {
    for (size_t i = 0; i < n; ++i) out[i] = sample_trilinear(*(Grid*)g, world + 3 * i);
}

// advect_particles / advect_particles_euler (src/tools/advection.rs:58-110):
// the position update only, f64, in the reference's evaluation order.
void vo_advect_particles(void* vx, void* vy, void* vz, double* pos, size_t n, double dt, int rk4) {
    const Grid &gx = *(Grid*)vx, &gy = *(Grid*)vy, &gz = *(Grid*)vz;
    auto sample = [&](const double p[3], double v[3]) {
        v[0] = (double)sample_trilinear(gx, p);
        v[1] = (double)sample_trilinear(gy, p);
        v[2] = (double)sample_trilinear(gz, p);
    };
    for (size_t i = 0; i < n; ++i) {
        double* p = pos + 3 * i;
        double v[3];
        if (!rk4) {
            sample(p, v);
            for (int a = 0; a < 3; ++a) p[a] += dt * v[a];
            continue;
        }
        double k1[3], k2[3], k3[3], k4[3], q[3];
        sample(p, v);
        for (int a = 0; a < 3; ++a) k1[a] = dt * v[a];
        for (int a = 0; a < 3; ++a) q[a] = p[a] + k1[a] * 0.5;
        sample(q, v);
        for (int a = 0; a < 3; ++a) k2[a] = dt * v[a];
        for (int a = 0; a < 3; ++a) q[a] = p[a] + k2[a] * 0.5;
        sample(q, v);
        for (int a = 0; a < 3; ++a) k3[a] = dt * v[a];
        for (int a = 0; a < 3; ++a) q[a] = p[a] + k3[a];
        sample(q, v);
        for (int a = 0; a < 3; ++a) k4[a] = dt * v[a];
        for (int a = 0; a < 3; ++a) p[a] = p[a] + (k1[a] + 2.0 * k2[a] + 2.0 * k3[a] + k4[a]) / 6.0;
    }
}

// PointDataGrid::rebin (src/points/point_grid.rs:258-266) after a position
// update: each particle goes to the leaf of AffineMap::world_to_index(pos)
// (src/grid.rs:259-277: rows of the inverse map applied left to right in f64,
// f64::round half away from zero, saturating `as i32`) aligned to 8
// (Coord::aligned(3), src/math/coord.rs:63-70).  The crate drains its leaves
// in HashMap order; with leaves drained in ascending (x, y, z) order and
// particles given in that binned order, the re-inserted grid is a stable
// sort of the particles by their new leaf.  Writes the permutation (new
// position -> input index) and returns the leaf count; leaf origins (3 ints)
// and the first particle of each leaf (n_leaves + 1 entries) go to `origins`
// and `start` when non-null.
static int32_t rust_round_to_i32(double f) {
    const double r = std::round(f);  // half away from zero, like f64::round
    if (r != r) return 0;
    if (r >= 2147483647.0) return 2147483647;
    if (r <= -2147483648.0) return (-2147483647 - 1);
    return (int32_t)r;
}

size_t vo_rebin_points(const double* pos, size_t n, const double* inv, uint32_t* perm, int32_t* origins,
                       uint32_t* start) {
    std::vector<std::array<int32_t, 3>> leaf(n);
    for (size_t i = 0; i < n; ++i) {
        const double* p = pos + 3 * i;
        for (int a = 0; a < 3; ++a) {
            const double* r = inv + 4 * a;
            const double f = r[0] * p[0] + r[1] * p[1] + r[2] * p[2] + r[3];
            leaf[i][a] = rust_round_to_i32(f) & ~7;
        }
    }
    std::vector<uint32_t> idx(n);
    for (size_t i = 0; i < n; ++i) idx[i] = (uint32_t)i;
    std::stable_sort(idx.begin(), idx.end(), [&](uint32_t a, uint32_t b) { return leaf[a] < leaf[b]; });
    size_t nl = 0;
    for (size_t j = 0; j < n; ++j) {
        if (perm) perm[j] = idx[j];
        if (j == 0 || leaf[idx[j]] != leaf[idx[j - 1]]) {
            if (origins)
                for (int a = 0; a < 3; ++a) origins[3 * nl + a] = leaf[idx[j]][a];
            if (start) start[nl] = (uint32_t)j;
            ++nl;
        }
    }
    if (start) start[nl] = (uint32_t)n;
    return nl;
}

void* vo_advect_level_set(void* g, void* vx, void* vy, void* vz, double dt) {
    return new Grid(advect_level_set(*(Grid*)g, *(Grid*)vx, *(Grid*)vy, *(Grid*)vz, dt));
}

// Returns the crossing count; writes up to `cap` coordinates sorted (x, y, z).
size_t vo_find_zero_crossings(void* g, int32_t* out, size_t cap) {
    auto v = find_zero_crossings(*(Grid*)g);
    std::sort(v.begin(), v.end(), [](const Coord& a, const Coord& b) {
        if (a.x != b.x) return a.x < b.x;
        if (a.y != b.y) return a.y < b.y;
        return a.z < b.z;
    });
    for (size_t i = 0; i < v.size() && i < cap; ++i) {
        out[3 * i] = v[i].x;
        out[3 * i + 1] = v[i].y;
        out[3 * i + 2] = v[i].z;
    }
    return v.size();
}

void vo_trim_narrow_band(void* g, float hw) { trim_narrow_band(*(Grid*)g, hw); }
void vo_rebuild_narrow_band(void* g, float hw, int brute) { rebuild_narrow_band(*(Grid*)g, hw, brute != 0); }
void vo_dilate(void* g, unsigned iterations) { dilate(*(Grid*)g, iterations); }
void vo_extend_velocity(void* sdf, void* vx, void* vy, void* vz, float hw) {
    extend_velocity(*(Grid*)sdf, *(Grid*)vx, *(Grid*)vy, *(Grid*)vz, hw);
}
void vo_remove_empty_leaves(void* g) { ((Grid*)g)->remove_empty_leaves(); }
void vo_flood_fill_sign(void* g) { flood_fill_sign(*(Grid*)g); }

// volume_to_mesh: returns the vertex count and sets *n_tris; copies up to the
// given capacities (vertices as x, y, z doubles; triangles as 3 indices).
size_t vo_volume_to_mesh(void* g, float iso, const int8_t* tri, double* verts, size_t cap_v, uint32_t* tris,
                         size_t cap_t, size_t* n_tris) {
    std::vector<double> v;
    std::vector<uint32_t> t;
    volume_to_mesh(*(Grid*)g, iso, tri, v, t);
    const size_t nv = v.size() / 3, nt = t.size() / 3;
    if (verts) std::copy(v.begin(), v.begin() + 3 * std::min(nv, cap_v), verts);
    if (tris) std::copy(t.begin(), t.begin() + 3 * std::min(nt, cap_t), tris);
    *n_tris = nt;
    return nv;
}

// One step of the reference pipeline, timed on this thread: advect_level_set
// followed by rebuild_narrow_band (brute-force loop, as the crate runs it)
// restricted to the first `rebuild_sample` active voxels when non-zero (the
// O(N x M) loop is extrapolated linearly from that sample).  Returns seconds
// for advect and for the sampled rebuild; the advected grid replaces *g.
void vo_time_ref_step(void** gp, void* vx, void* vy, void* vz, double dt, float hw,
                      size_t rebuild_sample, double* t_advect, double* t_rebuild, size_t* n_rebuilt,
                      double* t_cross, size_t* n_cross) {
    using clk = std::chrono::steady_clock;
    Grid* g = (Grid*)*gp;
    auto t0 = clk::now();
    Grid* a = new Grid(advect_level_set(*g, *(Grid*)vx, *(Grid*)vy, *(Grid*)vz, dt));
    auto t1 = clk::now();
    // Rebuild: crossings on the full grid, distance loop over the sample.
    float vs = (float)a->voxel_size;
    float band = hw * vs;
    auto cross = find_zero_crossings(*a);
    auto t1c = clk::now();
    std::vector<std::pair<Coord, float>> active;
    a->for_each_active([&](Coord c, float v) { active.push_back({c, v}); });
    size_t n = active.size();
    if (rebuild_sample && rebuild_sample < n) n = rebuild_sample;
    volatile float sink = 0.0f;
    for (size_t i = 0; i < n && !cross.empty(); ++i) {
        Coord c = active[i].first;
        float old = active[i].second;
        float sign = old >= 0.0f ? 1.0f : -1.0f;
        float md = std::numeric_limits<float>::max();
        for (auto& x : cross) {
            float dx = (float)(c.x - x.x), dy = (float)(c.y - x.y), dz = (float)(c.z - x.z);
            md = std::min(md, std::sqrt(dx * dx + dy * dy + dz * dz));
        }
        float nv = sign * md * vs;
        if (std::fabs(nv) < band) a->set(c, nv);
        else a->deactivate(c);
        sink = sink + nv;
    }
    a->remove_empty_leaves();
    auto t2 = clk::now();
    *t_advect = std::chrono::duration<double>(t1 - t0).count();
    *t_rebuild = std::chrono::duration<double>(t2 - t1).count();
    *n_rebuilt = n;
    if (t_cross) *t_cross = std::chrono::duration<double>(t1c - t1).count();
    if (n_cross) *n_cross = cross.size();
    delete g;
    *gp = a;
}

}  // extern "C"
