// ORACLE — test infrastructure only. Never linked into the product library.
//
// CPU restatement of the Sharc.Volrus sparse tree and of the narrow-band
// level-set tools on the advection path.  It keeps the reference's data
// structure (hash root -> 16^3 internal node -> boxed 8^3 leaf, one hashed
// lookup per `get`), its operation order and its types (f64 positions, f32
// fractions and blends, f32 sqrt), so that it serves both as the parity
// checker for the CUDA path and as the single-threaded "reference-structured"
// CPU baseline.  Build with -ffp-contract=off: Rust never fuses a*b+c.
//
// Parity pinning: the reference crate cannot be compiled here (no Rust
// toolchain), so this restatement is pinned by porting the crate's own
// inline known-answer tests (see tests/test_oracle_kats.py).
//
// Not restated: active/inactive *tiles* inside internal nodes (created only
// by `prune`, which is not on the advection path).  Every slot is either a
// leaf or the background.
#pragma once
#include <cmath>
#include <cstdint>
#include <cstring>
#include <memory>
#include <unordered_map>
#include <vector>
#include <algorithm>
#include <limits>

namespace vlr_oracle {

struct Coord {
    int32_t x, y, z;
    bool operator==(const Coord& o) const { return x == o.x && y == o.y && z == o.z; }
};

// src/math/coord.rs:63-70  (mask !(2^L-1), two's complement floor for negatives)
inline Coord aligned(Coord c, int log2dim) {
    int32_t m = ~((int32_t(1) << log2dim) - 1);
    return Coord{c.x & m, c.y & m, c.z & m};
}
// src/math/coord.rs:74-82  (ZYX order: x<<2L | y<<L | z)
inline int offset_in_tile(Coord c, int log2dim) {
    int32_t m = (1 << log2dim) - 1;
    return ((c.x & m) << (2 * log2dim)) | ((c.y & m) << log2dim) | (c.z & m);
}

struct CoordHash {
    size_t operator()(const Coord& c) const {
        uint64_t h = (uint64_t)(uint32_t)c.x * 0x9E3779B97F4A7C15ull;
        h ^= (uint64_t)(uint32_t)c.y * 0xC2B2AE3D27D4EB4Full + (h << 6) + (h >> 2);
        h ^= (uint64_t)(uint32_t)c.z * 0x165667B19E3779F9ull + (h << 6) + (h >> 2);
        return (size_t)h;
    }
};

// Rust `f64 as i32`: saturating, NaN -> 0.
inline int32_t sat_i32(double v) {
    if (std::isnan(v)) return 0;
    if (v <= -2147483648.0) return INT32_MIN;
    if (v >= 2147483647.0) return INT32_MAX;
    return (int32_t)v;
}

// src/tree/leaf.rs:18-35 — dense 512 values (ZYX) + 512-bit mask, created
// filled with the background.
struct Leaf {
    Coord origin;
    float values[512];
    uint64_t active[8];
    Leaf(Coord o, float bg) : origin(aligned(o, 3)) {
        for (int i = 0; i < 512; ++i) values[i] = bg;
        std::memset(active, 0, sizeof(active));
    }
    bool is_empty() const {
        for (int w = 0; w < 8; ++w) if (active[w]) return false;
        return true;
    }
    bool is_on(int off) const { return (active[off >> 6] >> (off & 63)) & 1ull; }
};

// src/tree/internal.rs:39-52 — 16^3 slots, each a boxed leaf or background.
struct Internal {
    Coord origin;
    std::vector<std::unique_ptr<Leaf>> children;  // 4096 slots
    float background;
    Internal(Coord o, float bg) : origin(aligned(o, 7)), children(4096), background(bg) {}
    // src/tree/internal.rs:88-95
    int child_index(Coord c) const {
        int lx = (c.x - origin.x) >> 3, ly = (c.y - origin.y) >> 3, lz = (c.z - origin.z) >> 3;
        return (lx << 8) | (ly << 4) | lz;
    }
};

// src/tree/root.rs:16-19 plus the Grid<f32> facade of src/grid.rs:349-362.
struct Grid {
    std::unordered_map<Coord, std::unique_ptr<Internal>, CoordHash> tiles;
    float background = 0.0f;
    // VoxelTransform (src/grid.rs:62-67): used by sample_trilinear.
    double voxel_size = 1.0;
    double t_origin[3] = {0, 0, 0};
    // AffineMap forward rows (src/grid.rs:131-138): used by advect_level_set.
    double mat[3][4] = {{1, 0, 0, 0}, {0, 1, 0, 0}, {0, 0, 1, 0}};
    double affine_voxel_size = 1.0;

    // Grid::new (src/grid.rs:366-375): uniform scale, no translation.
    static Grid make(float bg, double vs) {
        Grid g;
        g.background = bg;
        g.set_uniform(vs);
        return g;
    }
    void set_uniform(double vs) {
        voxel_size = vs;
        t_origin[0] = t_origin[1] = t_origin[2] = 0.0;
        std::memset(mat, 0, sizeof(mat));
        mat[0][0] = mat[1][1] = mat[2][2] = vs;
        affine_voxel_size = vs;
    }

    // src/tree/root.rs:55-61, internal.rs:118-124, leaf.rs:45-48
    float get(Coord c) const {
        auto it = tiles.find(aligned(c, 7));
        if (it == tiles.end()) return background;
        const Internal& n = *it->second;
        const Leaf* l = n.children[n.child_index(c)].get();
        if (!l) return n.background;
        return l->values[offset_in_tile(c, 3)];
    }
    // src/tree/root.rs:75-80
    bool is_active(Coord c) const {
        auto it = tiles.find(aligned(c, 7));
        if (it == tiles.end()) return false;
        const Internal& n = *it->second;
        const Leaf* l = n.children[n.child_index(c)].get();
        if (!l) return false;
        return l->is_on(offset_in_tile(c, 3));
    }
    // src/tree/root.rs:64-72, internal.rs:127-143, leaf.rs:52-56
    void set(Coord c, float v) {
        Coord key = aligned(c, 7);
        auto it = tiles.find(key);
        if (it == tiles.end())
            it = tiles.emplace(key, std::make_unique<Internal>(key, background)).first;
        Internal& n = *it->second;
        auto& slot = n.children[n.child_index(c)];
        if (!slot) slot = std::make_unique<Leaf>(aligned(c, 3), n.background);
        int off = offset_in_tile(c, 3);
        slot->values[off] = v;
        slot->active[off >> 6] |= 1ull << (off & 63);
    }
    // src/tree/root.rs:142-147, internal.rs:156-166, leaf.rs:60-64
    void deactivate(Coord c) {
        auto it = tiles.find(aligned(c, 7));
        if (it == tiles.end()) return;
        Internal& n = *it->second;
        Leaf* l = n.children[n.child_index(c)].get();
        if (!l) return;
        int off = offset_in_tile(c, 3);
        l->values[off] = n.background;
        l->active[off >> 6] &= ~(1ull << (off & 63));
    }
    // src/tree/root.rs:161-165, internal.rs:231-247
    void remove_empty_leaves() {
        for (auto& kv : tiles)
            for (auto& ch : kv.second->children)
                if (ch && ch->is_empty()) ch.reset();
    }
    // leaf iteration: tiles in ascending (x, y, z) of origin (the crate's
    // HashMap order is unspecified; dilate's values depend on it and the GPU
    // uses this order), then children in index order (x*256 + y*16 + z,
    // src/tree/internal.rs:88-95)
    template <class F> void for_each_leaf(F&& f) const {
        std::vector<const std::pair<const Coord, std::unique_ptr<Internal>>*> kv;
        for (auto& t : tiles) kv.push_back(&t);
        std::sort(kv.begin(), kv.end(), [](auto* a, auto* b) {
            if (a->first.x != b->first.x) return a->first.x < b->first.x;
            if (a->first.y != b->first.y) return a->first.y < b->first.y;
            return a->first.z < b->first.z;
        });
        for (auto* t : kv)
            for (auto& ch : t->second->children)
                if (ch) f(*ch);
    }
    template <class F> void for_each_leaf_mut(F&& f) {
        for (auto& kv : tiles)
            for (auto& ch : kv.second->children)
                if (ch) f(*ch);
    }
    // src/tree/leaf.rs:145-165 (trailing-zeros bit walk, off = x*64+y*8+z)
    template <class F> void for_each_active(F&& f) const {
        for_each_leaf([&](const Leaf& l) {
            for (int w = 0; w < 8; ++w) {
                uint64_t word = l.active[w];
                while (word) {
                    int bit = __builtin_ctzll(word);
                    word &= word - 1;
                    int off = w * 64 + bit;
                    Coord c{l.origin.x + (off >> 6), l.origin.y + ((off >> 3) & 7), l.origin.z + (off & 7)};
                    f(c, l.values[off]);
                }
            }
        });
    }
    size_t leaf_count() const {
        size_t n = 0;
        for_each_leaf([&](const Leaf&) { ++n; });
        return n;
    }
    uint64_t active_voxel_count() const {
        uint64_t n = 0;
        for_each_leaf([&](const Leaf& l) {
            for (int w = 0; w < 8; ++w) n += __builtin_popcountll(l.active[w]);
        });
        return n;
    }
    // Insert a whole leaf (flat import, NanoGrid-style).
    void put_leaf(Coord origin, const uint64_t* mask, const float* vals) {
        Coord key = aligned(origin, 7);
        auto it = tiles.find(key);
        if (it == tiles.end())
            it = tiles.emplace(key, std::make_unique<Internal>(key, background)).first;
        Internal& n = *it->second;
        auto& slot = n.children[n.child_index(origin)];
        slot = std::make_unique<Leaf>(aligned(origin, 3), n.background);
        std::memcpy(slot->values, vals, sizeof(float) * 512);
        std::memcpy(slot->active, mask, sizeof(uint64_t) * 8);
    }
};

// VoxelTransform::world_to_index_f64 (src/grid.rs:114-121)
inline void world_to_index(const Grid& g, const double w[3], double idx[3]) {
    double inv = 1.0 / g.voxel_size;
    idx[0] = (w[0] - g.t_origin[0]) * inv;
    idx[1] = (w[1] - g.t_origin[1]) * inv;
    idx[2] = (w[2] - g.t_origin[2]) * inv;
}

// AffineMap::index_to_world (src/grid.rs:248-257), left-to-right sums.
inline void index_to_world(const Grid& g, Coord c, double w[3]) {
    double x = c.x, y = c.y, z = c.z;
    for (int r = 0; r < 3; ++r)
        w[r] = g.mat[r][0] * x + g.mat[r][1] * y + g.mat[r][2] * z + g.mat[r][3];
}

// sample_trilinear (src/tools/interpolation.rs:11-48)
inline float sample_trilinear(const Grid& g, const double wpos[3]) {
    double idx[3];
    world_to_index(g, wpos, idx);
    double ix = std::floor(idx[0]), iy = std::floor(idx[1]), iz = std::floor(idx[2]);
    float fx = (float)(idx[0] - ix), fy = (float)(idx[1] - iy), fz = (float)(idx[2] - iz);
    int32_t i = sat_i32(ix), j = sat_i32(iy), k = sat_i32(iz);
    // Rust i32 addition in release builds wraps; mirror with unsigned arithmetic.
    auto add1 = [](int32_t a) { return (int32_t)((uint32_t)a + 1u); };
    float c000 = g.get({i, j, k});
    float c100 = g.get({add1(i), j, k});
    float c010 = g.get({i, add1(j), k});
    float c110 = g.get({add1(i), add1(j), k});
    float c001 = g.get({i, j, add1(k)});
    float c101 = g.get({add1(i), j, add1(k)});
    float c011 = g.get({i, add1(j), add1(k)});
    float c111 = g.get({add1(i), add1(j), add1(k)});
    float c00 = c000 * (1.0f - fx) + c100 * fx;
    float c01 = c001 * (1.0f - fx) + c101 * fx;
    float c10 = c010 * (1.0f - fx) + c110 * fx;
    float c11 = c011 * (1.0f - fx) + c111 * fx;
    float c0 = c00 * (1.0f - fy) + c10 * fy;
    float c1 = c01 * (1.0f - fy) + c11 * fy;
    return c0 * (1.0f - fz) + c1 * fz;
}

// advect_level_set (src/tools/advection.rs:32-56).  The output keeps the
// input's affine and background; Grid::with_affine resets the legacy
// transform to uniform(affine.voxel_size) with no translation (src/grid.rs:378-388).
inline Grid advect_level_set(const Grid& g, const Grid& vx, const Grid& vy, const Grid& vz, double dt) {
    Grid out;
    out.background = g.background;
    std::memcpy(out.mat, g.mat, sizeof(out.mat));
    out.affine_voxel_size = g.affine_voxel_size;
    out.voxel_size = g.affine_voxel_size;
    out.t_origin[0] = out.t_origin[1] = out.t_origin[2] = 0.0;
    g.for_each_active([&](Coord c, float) {
        double w[3];
        index_to_world(g, c, w);
        double v[3] = {(double)sample_trilinear(vx, w), (double)sample_trilinear(vy, w),
                       (double)sample_trilinear(vz, w)};
        double xp[3] = {w[0] - dt * v[0], w[1] - dt * v[1], w[2] - dt * v[2]};
        out.set(c, sample_trilinear(g, xp));
    });
    return out;
}

static const Coord kNbr6[6] = {{1, 0, 0}, {-1, 0, 0}, {0, 1, 0}, {0, -1, 0}, {0, 0, 1}, {0, 0, -1}};

// find_zero_crossings (src/tools/level_set_track.rs:14-47)
inline std::vector<Coord> find_zero_crossings(const Grid& g) {
    std::vector<Coord> out;
    g.for_each_active([&](Coord c, float val) {
        if (val == 0.0f) { out.push_back(c); return; }
        for (auto& o : kNbr6) {
            Coord nb{c.x + o.x, c.y + o.y, c.z + o.z};
            if (!g.is_active(nb)) continue;
            float nv = g.get(nb);
            if (val * nv < 0.0f) { out.push_back(c); break; }
        }
    });
    return out;
}

// trim_narrow_band (src/tools/level_set_track.rs:53-68)
inline void trim_narrow_band(Grid& g, float half_width) {
    float vs = (float)g.voxel_size;
    float thr = half_width * vs;
    std::vector<Coord> off;
    g.for_each_active([&](Coord c, float v) { if (std::fabs(v) >= thr) off.push_back(c); });
    for (auto& c : off) g.deactivate(c);
    g.remove_empty_leaves();
}

// rebuild_narrow_band (src/tools/level_set_track.rs:80-114).  `brute`
// follows the reference loop literally (O(N_active x N_cross)); otherwise the
// nearest crossing is searched in a cube window, which gives identical values
// for every voxel kept (a voxel is kept only when min_dist*vs < hw*vs, and a
// crossing outside a cube of half-size R >= ceil(hw)-1 lies at distance
// >= R+1 >= hw, whose product with vs rounds to >= band).
inline void rebuild_narrow_band(Grid& g, float half_width, bool brute) {
    float vs = (float)g.voxel_size;
    float band = half_width * vs;
    std::vector<Coord> cross = find_zero_crossings(g);
    if (cross.empty()) return;
    std::vector<std::pair<Coord, float>> active;
    g.for_each_active([&](Coord c, float v) { active.push_back({c, v}); });

    bool use_window = !brute && std::isfinite(half_width) && half_width <= 64.0f && vs > 0.0f;
    std::unordered_map<Coord, char, CoordHash> cset;
    int R = 0;
    if (use_window) {
        cset.reserve(cross.size() * 2);
        for (auto& c : cross) cset[c] = 1;
        R = std::max(0, (int)std::ceil(half_width) - 1);
    }
    for (auto& cv : active) {
        Coord c = cv.first;
        float old = cv.second;
        float sign = old >= 0.0f ? 1.0f : -1.0f;
        float min_dist = std::numeric_limits<float>::max();
        if (!use_window) {
            for (auto& x : cross) {
                float dx = (float)(int32_t)((uint32_t)c.x - (uint32_t)x.x);
                float dy = (float)(int32_t)((uint32_t)c.y - (uint32_t)x.y);
                float dz = (float)(int32_t)((uint32_t)c.z - (uint32_t)x.z);
                float d = std::sqrt(dx * dx + dy * dy + dz * dz);
                min_dist = std::min(min_dist, d);
            }
        } else {
            int64_t best = -1;
            for (int dx = -R; dx <= R; ++dx)
                for (int dy = -R; dy <= R; ++dy)
                    for (int dz = -R; dz <= R; ++dz) {
                        int64_t d2 = (int64_t)dx * dx + (int64_t)dy * dy + (int64_t)dz * dz;
                        if (best >= 0 && d2 >= best) continue;
                        if (cset.count(Coord{c.x + dx, c.y + dy, c.z + dz})) best = d2;
                    }
            if (best >= 0) {
                float fd = (float)best;  // exact below 2^24
                min_dist = std::sqrt(fd);
            }
        }
        float nv = sign * min_dist * vs;
        if (std::fabs(nv) < band) g.set(c, nv);
        else g.deactivate(c);
    }
    g.remove_empty_leaves();
}

// extend_velocity (src/tools/level_set_track.rs:115-160): band voxels copy
// the velocity of their nearest interface voxel (first minimum in iteration
// order, as min_by_key returns it) and become active in each velocity grid.
inline void extend_velocity(const Grid& sdf, Grid& vx, Grid& vy, Grid& vz, float half_width) {
    const float vs = (float)sdf.voxel_size;
    const float band = half_width * vs;
    std::vector<Coord> iface, bandv;
    sdf.for_each_active([&](Coord c, float v) {
        if (std::fabs(v) < vs) iface.push_back(c);
    });
    if (iface.empty()) return;
    sdf.for_each_active([&](Coord c, float v) {
        const float a = std::fabs(v);
        if (a >= vs && a < band) bandv.push_back(c);
    });
    auto dist_sq = [](const Coord& a, const Coord& b) {
        const int64_t dx = (int64_t)(a.x - b.x), dy = (int64_t)(a.y - b.y), dz = (int64_t)(a.z - b.z);
        return dx * dx + dy * dy + dz * dz;
    };
    for (const Coord& c : bandv) {
        size_t best = 0;
        int64_t bd = dist_sq(c, iface[0]);
        for (size_t k = 1; k < iface.size(); ++k) {
            const int64_t d = dist_sq(c, iface[k]);
            if (d < bd) {
                bd = d;
                best = k;
            }
        }
        const Coord& s = iface[best];
        vx.set(c, vx.get(s));
        vy.set(c, vy.get(s));
        vz.set(c, vz.get(s));
    }
}

// dilate (src/tools/morphology.rs:20-35): snapshot, then activate inactive
// 6-neighbours with the current voxel's value.  First writer wins, so the
// values depend on iteration order; only the topology is order independent.
inline void dilate(Grid& g, unsigned iterations) {
    for (unsigned it = 0; it < iterations; ++it) {
        std::vector<std::pair<Coord, float>> active;
        g.for_each_active([&](Coord c, float v) { active.push_back({c, v}); });
        for (auto& cv : active)
            for (auto& o : kNbr6) {
                Coord nb{cv.first.x + o.x, cv.first.y + o.y, cv.first.z + o.z};
                if (!g.is_active(nb)) g.set(nb, cv.second);
            }
    }
}

// make_level_set_sphere (src/tools/sphere.rs:17-59)
inline Grid make_level_set_sphere(double radius, const double center[3], double voxel_size, double half_width) {
    double band = half_width * voxel_size;
    float bg = (float)band;
    Grid g = Grid::make(bg, voxel_size);
    double extent = radius + band;
    double inv = 1.0 / voxel_size;
    int32_t imin = sat_i32(std::floor((center[0] - extent) * inv));
    int32_t jmin = sat_i32(std::floor((center[1] - extent) * inv));
    int32_t kmin = sat_i32(std::floor((center[2] - extent) * inv));
    int32_t imax = sat_i32(std::ceil((center[0] + extent) * inv));
    int32_t jmax = sat_i32(std::ceil((center[1] + extent) * inv));
    int32_t kmax = sat_i32(std::ceil((center[2] + extent) * inv));
    for (int64_t i = imin; i <= imax; ++i) {
        double wx = (double)i * voxel_size - center[0];
        for (int64_t j = jmin; j <= jmax; ++j) {
            double wy = (double)j * voxel_size - center[1];
            for (int64_t k = kmin; k <= kmax; ++k) {
                double wz = (double)k * voxel_size - center[2];
                double dist = std::sqrt(wx * wx + wy * wy + wz * wz);
                float sdf = (float)(dist - radius);
                if (std::fabs(sdf) < bg) g.set(Coord{(int32_t)i, (int32_t)j, (int32_t)k}, sdf);
            }
        }
    }
    return g;
}


// flood_fill_sign (src/tools/flood_fill.rs:18-107): per leaf with an active
// voxel, the leaf's majority sign (negative only if strictly more active
// values are < 0); each inactive voxel then takes -bg if strictly more of its
// active 6-neighbours inside the leaf are < 0 than not, +bg if not, and the
// leaf majority if it has no active neighbour in the leaf.  Reads a snapshot
// of the leaf, so the result does not depend on the voxel order.
inline void flood_fill_sign(Grid& g) {
    const float bg = g.background;
    g.for_each_leaf_mut([&](Leaf& l) {
        int neg = 0, pos = 0;
        for (int off = 0; off < 512; ++off)
            if (l.is_on(off)) {
                if (l.values[off] < 0.0f) ++neg;
                else ++pos;
            }
        if (neg == 0 && pos == 0) return;
        const float global = neg > pos ? -bg : bg;
        float snap[512];
        std::memcpy(snap, l.values, sizeof(snap));
        for (int off = 0; off < 512; ++off) {
            if (l.is_on(off)) continue;
            const int lx = off >> 6, ly = (off >> 3) & 7, lz = off & 7;
            int ln = 0, lp = 0;
            for (const auto& d : kNbr6) {
                const int nx = lx + d.x, ny = ly + d.y, nz = lz + d.z;
                if (nx < 0 || nx > 7 || ny < 0 || ny > 7 || nz < 0 || nz > 7) continue;
                const int no = (nx << 6) | (ny << 3) | nz;
                if (!l.is_on(no)) continue;
                if (snap[no] < 0.0f) ++ln;
                else ++lp;
            }
            l.values[off] = (ln + lp > 0) ? (ln > lp ? -bg : bg) : global;
        }
    });
}

// volume_to_mesh (src/tools/volume_to_mesh.rs:46-201): cells of the leaf
// tiles and their 6 face neighbours, tiles in ascending (x, y, z), cells in
// x-major order within a tile; corners read with Grid::get; an edge vertex is
// created the first time a cell with that edge flagged is processed (the
// HashMap edge cache keyed by the sorted corner pair), interpolated from the
// creating cell's first endpoint toward its second in f32 t, f64 position.
// `tri` holds the triangle table (16 entries per case, -1 terminated); the
// edge table is the classification rule (edge flagged iff its corners differ).
struct CoordPairHash {
    size_t operator()(const std::pair<Coord, Coord>& p) const {
        CoordHash h;
        return h(p.first) * 31u ^ h(p.second);
    }
};

inline bool coord_less(const Coord& a, const Coord& b) {
    if (a.x != b.x) return a.x < b.x;
    if (a.y != b.y) return a.y < b.y;
    return a.z < b.z;
}

inline void volume_to_mesh(const Grid& g, float iso, const int8_t* tri, std::vector<double>& verts,
                           std::vector<uint32_t>& tris) {
    static const int kCorner[8][3] = {{0, 0, 0}, {1, 0, 0}, {1, 1, 0}, {0, 1, 0},
                                      {0, 0, 1}, {1, 0, 1}, {1, 1, 1}, {0, 1, 1}};
    static const int kEdge[12][2] = {{0, 1}, {1, 2}, {2, 3}, {3, 0}, {4, 5}, {5, 6},
                                     {6, 7}, {7, 4}, {0, 4}, {1, 5}, {2, 6}, {3, 7}};
    verts.clear();
    tris.clear();
    std::vector<Coord> cells;
    g.for_each_leaf([&](const Leaf& l) {
        const Coord o = l.origin;
        cells.push_back(o);
        cells.push_back({o.x - 8, o.y, o.z});
        cells.push_back({o.x + 8, o.y, o.z});
        cells.push_back({o.x, o.y - 8, o.z});
        cells.push_back({o.x, o.y + 8, o.z});
        cells.push_back({o.x, o.y, o.z - 8});
        cells.push_back({o.x, o.y, o.z + 8});
    });
    std::sort(cells.begin(), cells.end(), coord_less);
    cells.erase(std::unique(cells.begin(), cells.end()), cells.end());
    const double vs = g.voxel_size;
    std::unordered_map<std::pair<Coord, Coord>, uint32_t, CoordPairHash> cache;
    for (const Coord& o : cells)
        for (int lx = 0; lx < 8; ++lx)
            for (int ly = 0; ly < 8; ++ly)
                for (int lz = 0; lz < 8; ++lz) {
                    Coord c[8];
                    float v[8];
                    int ci = 0;
                    for (int i = 0; i < 8; ++i) {
                        c[i] = {o.x + lx + kCorner[i][0], o.y + ly + kCorner[i][1], o.z + lz + kCorner[i][2]};
                        v[i] = g.get(c[i]);
                        if (v[i] < iso) ci |= 1 << i;
                    }
                    uint32_t ev[12] = {0};
                    bool any = false;
                    for (int e = 0; e < 12; ++e) {
                        const int a = kEdge[e][0], b = kEdge[e][1];
                        if (((ci >> a) & 1) == ((ci >> b) & 1)) continue;
                        any = true;
                        std::pair<Coord, Coord> key =
                            coord_less(c[a], c[b]) ? std::make_pair(c[a], c[b]) : std::make_pair(c[b], c[a]);
                        auto it = cache.find(key);
                        if (it != cache.end()) {
                            ev[e] = it->second;
                            continue;
                        }
                        const float d = v[b] - v[a];
                        const double t = (std::fabs(d) > 1e-10f) ? (double)((iso - v[a]) / d) : 0.5;
                        const double pa[3] = {(double)c[a].x * vs, (double)c[a].y * vs, (double)c[a].z * vs};
                        const double pb[3] = {(double)c[b].x * vs, (double)c[b].y * vs, (double)c[b].z * vs};
                        const uint32_t idx = (uint32_t)(verts.size() / 3);
                        for (int k = 0; k < 3; ++k) verts.push_back(pa[k] + t * (pb[k] - pa[k]));
                        cache.emplace(key, idx);
                        ev[e] = idx;
                    }
                    if (!any) continue;
                    const int8_t* row = tri + 16 * ci;
                    for (int t = 0; t < 15 && row[t] != -1; t += 3)
                        for (int k = 0; k < 3; ++k) tris.push_back(ev[row[t + k]]);
                }
}

}  // namespace vlr_oracle
