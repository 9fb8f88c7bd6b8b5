// Shared device-side definitions for the narrow-band level-set library.
//
// Device layout of a grid ("leaf pool"), modelled on the reference's flat
// NanoGrid (src/nano/layout.rs:41-52) but split into structure-of-arrays and
// extended with a 27-neighbour table and a hash index:
//   origin[slot]        int4 {x, y, z, grid id}; x,y,z are leaf origins (multiples of 8)
//   mask[slot*8 + w]    u64 activity words; bit off = x*64 + y*8 + z  (src/math/coord.rs:74-82)
//   values[slot*512+off] f32 (world units) or f16 (voxel units, narrow-band method)
//   nbr[slot*27 + d]    slot of the leaf at leaf offset d = (dx+1)*9+(dy+1)*3+(dz+1), or -1
//   hash                open addressing, key = packed leaf coordinate relative to a per-grid base
#pragma once
#include <cstdint>
#include <cuda_runtime.h>
#include <cuda_fp16.h>

namespace vlr {

constexpr int kLeafVoxels = 512;
constexpr int kNbr = 27;
constexpr uint64_t kEmptyKey = 0xFFFFFFFFFFFFFFFFull;
constexpr int kKeyBits = 21;              // leaf coordinate bits per axis in a hash key
constexpr long long kKeyHalf = 1ll << 20; // base = centre - kKeyHalf

// Device-side error bits (OR-ed into a context error word).
enum : unsigned {
    kErrHashFull = 1u << 0,    // a probe sequence exhausted the table
    kErrCapacity = 1u << 1,    // leaf pool capacity exceeded
    kErrReach = 1u << 2,       // a backtrace left the staged neighbourhood
    kErrExtent = 1u << 3,      // a leaf coordinate left the hashable range
    kErrTimeout = 1u << 4,     // a bounded device wait gave up
    kErrInput = 1u << 5,       // device-resident input failed a check (leaf origin not a multiple of 8)
};

__host__ __device__ inline uint64_t mix64(uint64_t k) {
    k ^= k >> 33;
    k *= 0xff51afd7ed558ccdull;
    k ^= k >> 33;
    k *= 0xc4ceb9fe1a85ec53ull;
    k ^= k >> 33;
    return k;
}

// Pack a leaf coordinate (origin >> 3) relative to `base`; returns kEmptyKey
// when it lies outside the 2^21-leaf window (such a leaf cannot exist).
__host__ __device__ inline uint64_t pack_key(long long lx, long long ly, long long lz, const long long* base) {
    long long rx = lx - base[0], ry = ly - base[1], rz = lz - base[2];
    const long long lim = 1ll << kKeyBits;
    if (rx < 0 || ry < 0 || rz < 0 || rx >= lim || ry >= lim || rz >= lim) return kEmptyKey;
    return (uint64_t)rx | ((uint64_t)ry << 21) | ((uint64_t)rz << 42);
}

struct HashView {
    const uint64_t* key;
    const int* val;
    int cap;  // power of two
    long long base[3];
};

__device__ inline int hash_find(const HashView& h, uint64_t key) {
    if (key == kEmptyKey) return -1;
    uint32_t m = (uint32_t)h.cap - 1u;
    uint32_t p = (uint32_t)mix64(key) & m;
    for (int probe = 0; probe < h.cap; ++probe) {
        uint64_t k = h.key[p];
        if (k == key) return h.val[p];
        if (k == kEmptyKey) return -1;
        p = (p + 1u) & m;
    }
    return -1;
}

__device__ inline int hash_find_leaf(const HashView& h, long long lx, long long ly, long long lz) {
    return hash_find(h, pack_key(lx, ly, lz, h.base));
}

// Read-only view of a world-unit f32 grid (the reference-semantics path).
struct GridView {
    const int4* origin;
    const uint64_t* mask;
    const float* values;
    const int* nbr;
    HashView hash;
    int n;
    float background;
    double inv_vs;        // 1.0 / VoxelTransform::voxel_size (computed on the host)
    double t_origin[3];   // VoxelTransform::origin
    double mat[12];       // AffineMap forward rows (index -> world)
};

__device__ inline bool mask_bit(const uint64_t* m, int off) { return (m[off >> 6] >> (off & 63)) & 1ull; }

__device__ inline int voxel_off(int x, int y, int z) { return ((x & 7) << 6) | ((y & 7) << 3) | (z & 7); }

// Leaf lookup with an optional hint leaf: offsets within +-1 of the hint use
// the neighbour table, anything else goes through the hash.
__device__ inline int find_leaf_hint(const GridView& g, int hint, int hlx, int hly, int hlz, int lx, int ly, int lz) {
    if (hint >= 0) {
        int dx = lx - hlx, dy = ly - hly, dz = lz - hlz;
        if (dx >= -1 && dx <= 1 && dy >= -1 && dy <= 1 && dz >= -1 && dz <= 1)
            return g.nbr[hint * kNbr + (dx + 1) * 9 + (dy + 1) * 3 + (dz + 1)];
    }
    return hash_find_leaf(g.hash, lx, ly, lz);
}

__device__ inline uint32_t wrap_inc(int32_t a) { return (uint32_t)a + 1u; }

// sample_trilinear (src/tools/interpolation.rs:11-48) with the reference's
// exact operation order: f64 world->index, f64 floor, f32 fractions, eight
// reads, f32 blend x then y then z.  All products and sums are explicitly
// rounded (no contraction), so results match the CPU bit for bit.
__device__ inline float sample_trilinear_ref(const GridView& g, double wx, double wy, double wz, int hint = -1,
                                             int hlx = 0, int hly = 0, int hlz = 0) {
    double ix_ = __dmul_rn(__dsub_rn(wx, g.t_origin[0]), g.inv_vs);
    double iy_ = __dmul_rn(__dsub_rn(wy, g.t_origin[1]), g.inv_vs);
    double iz_ = __dmul_rn(__dsub_rn(wz, g.t_origin[2]), g.inv_vs);
    double fx0 = floor(ix_), fy0 = floor(iy_), fz0 = floor(iz_);
    float fx = __double2float_rn(__dsub_rn(ix_, fx0));
    float fy = __double2float_rn(__dsub_rn(iy_, fy0));
    float fz = __double2float_rn(__dsub_rn(iz_, fz0));
    int32_t i = __double2int_rz(fx0), j = __double2int_rz(fy0), k = __double2int_rz(fz0);
    int32_t i1 = (int32_t)wrap_inc(i), j1 = (int32_t)wrap_inc(j), k1 = (int32_t)wrap_inc(k);
    int lx0 = i >> 3, lx1 = i1 >> 3, ly0 = j >> 3, ly1 = j1 >> 3, lz0 = k >> 3, lz1 = k1 >> 3;
    int s000 = find_leaf_hint(g, hint, hlx, hly, hlz, lx0, ly0, lz0);
    int s100 = (lx1 == lx0) ? s000 : find_leaf_hint(g, hint, hlx, hly, hlz, lx1, ly0, lz0);
    int s010 = (ly1 == ly0) ? s000 : find_leaf_hint(g, hint, hlx, hly, hlz, lx0, ly1, lz0);
    int s110 = (ly1 == ly0) ? s100 : ((lx1 == lx0) ? s010 : find_leaf_hint(g, hint, hlx, hly, hlz, lx1, ly1, lz0));
    int s001 = (lz1 == lz0) ? s000 : find_leaf_hint(g, hint, hlx, hly, hlz, lx0, ly0, lz1);
    int s101 = (lz1 == lz0) ? s100 : ((lx1 == lx0) ? s001 : find_leaf_hint(g, hint, hlx, hly, hlz, lx1, ly0, lz1));
    int s011 = (lz1 == lz0) ? s010 : ((ly1 == ly0) ? s001 : find_leaf_hint(g, hint, hlx, hly, hlz, lx0, ly1, lz1));
    int s111 = (lz1 == lz0) ? s110
                            : ((ly1 == ly0) ? s101 : ((lx1 == lx0) ? s011 : find_leaf_hint(g, hint, hlx, hly, hlz, lx1, ly1, lz1)));
    const float bg = g.background;
    auto rd = [&](int s, int x, int y, int z) -> float {
        return s < 0 ? bg : g.values[(size_t)s * kLeafVoxels + voxel_off(x, y, z)];
    };
    float c000 = rd(s000, i, j, k), c100 = rd(s100, i1, j, k);
    float c010 = rd(s010, i, j1, k), c110 = rd(s110, i1, j1, k);
    float c001 = rd(s001, i, j, k1), c101 = rd(s101, i1, j, k1);
    float c011 = rd(s011, i, j1, k1), c111 = rd(s111, i1, j1, k1);
    float ox = __fsub_rn(1.0f, fx), oy = __fsub_rn(1.0f, fy), oz = __fsub_rn(1.0f, fz);
    float c00 = __fadd_rn(__fmul_rn(c000, ox), __fmul_rn(c100, fx));
    float c01 = __fadd_rn(__fmul_rn(c001, ox), __fmul_rn(c101, fx));
    float c10 = __fadd_rn(__fmul_rn(c010, ox), __fmul_rn(c110, fx));
    float c11 = __fadd_rn(__fmul_rn(c011, ox), __fmul_rn(c111, fx));
    float c0 = __fadd_rn(__fmul_rn(c00, oy), __fmul_rn(c10, fy));
    float c1 = __fadd_rn(__fmul_rn(c01, oy), __fmul_rn(c11, fy));
    return __fadd_rn(__fmul_rn(c0, oz), __fmul_rn(c1, fz));
}

// AffineMap::index_to_world (src/grid.rs:248-257): ((m0*x + m1*y) + m2*z) + m3.
__device__ inline void index_to_world_ref(const double* m, int x, int y, int z, double w[3]) {
    double dx = (double)x, dy = (double)y, dz = (double)z;
#pragma unroll
    for (int r = 0; r < 3; ++r)
        w[r] = __dadd_rn(__dadd_rn(__dadd_rn(__dmul_rn(m[r * 4], dx), __dmul_rn(m[r * 4 + 1], dy)),
                                   __dmul_rn(m[r * 4 + 2], dz)),
                         m[r * 4 + 3]);
}

}  // namespace vlr
