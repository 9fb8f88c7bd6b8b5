// The reference's serialised grid formats on the device upload and download
// paths (vlr_grid_from_vol / vlr_grid_to_vol, vlr_grid_from_nano /
// vlr_grid_to_nano):
//
//   .vol (src/io/vol_format.rs:1-160), little-endian:
//     header (32 B): magic "VOLR", u32 version = 1, u32 grid class (0 unknown,
//       1 level set, 2 fog volume), f64 voxel size, f32 background, u32 leaf
//       count, 4 reserved bytes;
//     per leaf (2,124 B): i32 origin[3], u64 mask[8], f32 values[512] (ZYX),
//       leaves in the writer's tree order.
//   NanoGrid (src/nano/layout.rs:13-286), the repr(C) image of NanoHeader
//     (320 B: magic "NANO" @0, u32 version = 1 @4, u32 class @8, f64 voxel
//     size @16, f32 background @24, u32 leaf count @28, i32 active bbox min
//     @32 and max @44, f64 forward 4x4 @56, f64 inverse 4x4 @184, pad) and
//     NanoLeaf (2,128 B: i32 origin[3], i32 pad, u64 mask[8] @16, f32
//     values[512] @80), leaves strictly sorted by (x, y, z) of origin.
//
// Reading validates as the reference does (magic, version, class, size, leaf
// order) and moves the leaf block to the device in one copy; a kernel
// scatters the records into the pool's structure-of-arrays layout in (x, y, z)
// order of origin.  Writing packs the pool into records on the device and
// brings them back in one copy.  The host side assumes a little-endian CPU,
// as the formats are little-endian.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <numeric>
#include <vector>

#include "ref_ops.hpp"

using namespace vlr;

namespace {

constexpr size_t kVolHeader = 32, kVolLeaf = 12 + 64 + 2048;
constexpr size_t kNanoHeader = 320, kNanoLeaf = 2128;
// NanoHeader field offsets
constexpr size_t kNhVersion = 4, kNhClass = 8, kNhVoxel = 16, kNhBackground = 24, kNhCount = 28, kNhBboxMin = 32,
                 kNhBboxMax = 44, kNhMat = 56, kNhInv = 184;

template <class T>
T rd(const unsigned char* p) {
    T v;
    std::memcpy(&v, p, sizeof(T));
    return v;
}
template <class T>
void wr(unsigned char* p, T v) {
    std::memcpy(p, &v, sizeof(T));
}

// One warp per leaf: record src[i] -> pool slot i.  Records are 4-byte
// aligned (the .vol stride is 2,124 B), so every access is a 4-byte word;
// lanes stride through the 512 values so a warp reads 128 contiguous bytes at
// a time.  drop_inactive: inactive voxels take the background and the mask is
// kept (NanoGrid::to_grid inserts only active voxels into a fresh grid).
__global__ void k_unpack_records(const unsigned char* __restrict__ rec, size_t stride, int o_off, int m_off,
                                 int v_off, const int* __restrict__ src, int n, int drop_inactive, float bg,
                                 int4* __restrict__ origin, uint64_t* __restrict__ mask, float* __restrict__ values) {
    const int lane = threadIdx.x & 31;
    for (long long i = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < n;
         i += ((long long)gridDim.x * blockDim.x) >> 5) {
        const unsigned char* r = rec + (size_t)src[i] * stride;
        const unsigned* ro = reinterpret_cast<const unsigned*>(r + o_off);
        const unsigned* rm = reinterpret_cast<const unsigned*>(r + m_off);
        const unsigned* rv = reinterpret_cast<const unsigned*>(r + v_off);
        const unsigned mw = rm[lane & 15];
        const unsigned mlo = __shfl_sync(0xffffffffu, mw, (lane & 7) * 2);
        const unsigned mhi = __shfl_sync(0xffffffffu, mw, (lane & 7) * 2 + 1);
        if (lane < 8) mask[(size_t)i * 8 + lane] = ((uint64_t)mhi << 32) | mlo;
        if (lane == 0) {
            // a record's leaf is the one holding its origin voxel: align down to 8
            origin[i] = make_int4((int)ro[0] & ~7, (int)ro[1] & ~7, (int)ro[2] & ~7, 0);
        }
        float* out = values + (size_t)i * kLeafVoxels;
#pragma unroll 4
        for (int k = lane; k < kLeafVoxels; k += 32) {
            float v = __uint_as_float(rv[k]);
            if (drop_inactive) {
                // word k >> 6 of the mask: 32-bit half (k >> 5) & 1 of it, from lane (k >> 5)
                const unsigned half = __shfl_sync(0xffffffffu, mw, k >> 5);
                if (!((half >> (k & 31)) & 1u)) v = bg;
            }
            out[k] = v;
        }
    }
}

// Pool slot i -> record i (the inverse of k_unpack_records; pad_off >= 0
// zeroes a 4-byte pad word).
__global__ void k_pack_records(const int4* __restrict__ origin, const uint64_t* __restrict__ mask,
                               const float* __restrict__ values, int n, unsigned char* __restrict__ rec, size_t stride,
                               int o_off, int m_off, int v_off, int pad_off) {
    const int lane = threadIdx.x & 31;
    for (long long i = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < n;
         i += ((long long)gridDim.x * blockDim.x) >> 5) {
        unsigned char* r = rec + (size_t)i * stride;
        unsigned* ro = reinterpret_cast<unsigned*>(r + o_off);
        unsigned* rm = reinterpret_cast<unsigned*>(r + m_off);
        unsigned* rv = reinterpret_cast<unsigned*>(r + v_off);
        if (lane < 16) {
            const uint64_t w = mask[(size_t)i * 8 + (lane >> 1)];
            rm[lane] = (lane & 1) ? (unsigned)(w >> 32) : (unsigned)w;
        }
        if (lane == 0) {
            const int4 o = origin[i];
            ro[0] = (unsigned)o.x;
            ro[1] = (unsigned)o.y;
            ro[2] = (unsigned)o.z;
            if (pad_off >= 0) *reinterpret_cast<unsigned*>(r + pad_off) = 0u;
        }
        const float* in = values + (size_t)i * kLeafVoxels;
#pragma unroll 4
        for (int k = lane; k < kLeafVoxels; k += 32) rv[k] = __float_as_uint(in[k]);
    }
}

int warp_blocks(vlr_ctx* ctx, long long n) {
    return (int)std::max<long long>(1, std::min<long long>((n * 32 + 255) / 256, (long long)ctx->sm_count * 16));
}

bool origin_less(const int32_t* a, const int32_t* b) {
    if (a[0] != b[0]) return a[0] < b[0];
    if (a[1] != b[1]) return a[1] < b[1];
    return a[2] < b[2];
}

// Build a grid from `n` records of `bytes` (host) at `stride`.  `order[i]` is
// the record of the i-th leaf in (x, y, z) order and `origins` its aligned
// origin (3 per leaf).
int grid_from_records(vlr_ctx* ctx, vlr_grid* g, const unsigned char* block, size_t n_records, size_t stride,
                      int o_off, int m_off, int v_off, const std::vector<int>& order,
                      const std::vector<int32_t>& origins, bool drop_inactive) {
    const size_t n = order.size();
    int rc = choose_base(ctx, origins.data(), n, g->base);
    if (rc) return rc;
    rc = grid_alloc(ctx, g, (int)std::max<size_t>(n, 1));
    if (rc) return rc;
    g->n = (int)n;
    if (n) {
        const size_t bytes = n_records * stride;
        void* scratch = nullptr;
        rc = ctx_scratch(ctx, bytes + sizeof(int) * n + 256, &scratch);
        if (rc) return rc;
        unsigned char* d_rec = static_cast<unsigned char*>(scratch);
        int* d_src = reinterpret_cast<int*>(d_rec + ((bytes + 255) & ~size_t(255)));
        VLR_CUDA(ctx, cudaMemcpyAsync(d_rec, block, bytes, cudaMemcpyHostToDevice, ctx->stream));
        VLR_CUDA(ctx, cudaMemcpyAsync(d_src, order.data(), sizeof(int) * n, cudaMemcpyHostToDevice, ctx->stream));
        k_unpack_records<<<warp_blocks(ctx, (long long)n), 256, 0, ctx->stream>>>(
            d_rec, stride, o_off, m_off, v_off, d_src, (int)n, drop_inactive ? 1 : 0, g->background, g->origin,
            g->mask, (float*)g->values);
        VLR_CUDA(ctx, cudaGetLastError());
        VLR_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    }
    return grid_index(ctx, g);
}

// Pack a grid's leaves (pool order = (x, y, z) order of origin) into records
// written to host memory at `out`.
int grid_to_records(vlr_ctx* ctx, const vlr_grid* g, unsigned char* out, size_t stride, int o_off, int m_off,
                    int v_off, int pad_off) {
    const size_t n = (size_t)g->n;
    if (!n) return VLR_OK;
    void* scratch = nullptr;
    int rc = ctx_scratch(ctx, n * stride, &scratch);
    if (rc) return rc;
    unsigned char* d_rec = static_cast<unsigned char*>(scratch);
    k_pack_records<<<warp_blocks(ctx, (long long)n), 256, 0, ctx->stream>>>(
        g->origin, g->mask, (const float*)g->values, (int)n, d_rec, stride, o_off, m_off, v_off, pad_off);
    VLR_CUDA(ctx, cudaGetLastError());
    return d2h_copy(ctx, out, d_rec, n * stride);
}

vlr_transform uniform_transform(double vs) {
    vlr_transform t{};
    t.voxel_size = vs;
    t.affine[0] = t.affine[5] = t.affine[10] = vs;
    t.affine_voxel_size = vs;
    return t;
}

}  // namespace

extern "C" {

int vlr_grid_from_vol(vlr_ctx* ctx, const void* bytes, size_t n_bytes, vlr_grid** out, int* grid_class) {
    if (!ctx || !out || (!bytes && n_bytes)) return set_error(ctx, VLR_ERR_INVALID, "null argument");
    *out = nullptr;
    const unsigned char* b = static_cast<const unsigned char*>(bytes);
    // read_vol (src/io/vol_format.rs:85-150)
    if (n_bytes < kVolHeader) return set_error(ctx, VLR_ERR_FORMAT, ".vol: truncated header");
    if (std::memcmp(b, "VOLR", 4) != 0) return set_error(ctx, VLR_ERR_FORMAT, "not a .vol file (bad magic)");
    const uint32_t version = rd<uint32_t>(b + 4);
    if (version != 1) return set_error(ctx, VLR_ERR_FORMAT, "unsupported .vol version: " + std::to_string(version));
    const uint32_t cls = rd<uint32_t>(b + 8);
    if (cls > 2) return set_error(ctx, VLR_ERR_FORMAT, "unknown grid class: " + std::to_string(cls));
    const double vs = rd<double>(b + 12);
    const float bg = rd<float>(b + 20);
    const size_t count = rd<uint32_t>(b + 24);
    if ((n_bytes - kVolHeader) / kVolLeaf < count) return set_error(ctx, VLR_ERR_FORMAT, ".vol: truncated leaf data");
    if (count > (size_t)(1 << 30)) return set_error(ctx, VLR_ERR_CAPACITY, "too many leaves");
    const unsigned char* block = b + kVolHeader;
    // a later record of the same leaf overwrites an earlier one (bulk write of
    // values and mask after grid.set(origin)): keep the last record per leaf
    std::vector<int32_t> o(3 * count);
    for (size_t i = 0; i < count; ++i)
        for (int a = 0; a < 3; ++a) o[3 * i + a] = rd<int32_t>(block + i * kVolLeaf + 4 * a) & ~7;
    std::vector<int> idx(count);
    std::iota(idx.begin(), idx.end(), 0);
    std::stable_sort(idx.begin(), idx.end(), [&](int x, int y) { return origin_less(&o[3 * x], &o[3 * y]); });
    std::vector<int> order;
    std::vector<int32_t> origins;
    for (size_t k = 0; k < count; ++k) {
        const bool last = (k + 1 == count) || origin_less(&o[3 * idx[k]], &o[3 * idx[k + 1]]);
        if (!last) continue;
        order.push_back(idx[k]);
        origins.insert(origins.end(), &o[3 * idx[k]], &o[3 * idx[k]] + 3);
    }
    vlr_grid* g = new vlr_grid();
    g->ctx = ctx;
    g->kind = VLR_KIND_F32_WORLD;
    g->background = bg;
    g->xf = uniform_transform(vs);  // Grid::new(background, voxel_size)
    g->grid_class = (int)cls;
    int rc = grid_from_records(ctx, g, block, count, kVolLeaf, 0, 12, 76, order, origins, false);
    if (rc) {
        vlr_grid_destroy(g);
        return rc;
    }
    if (grid_class) *grid_class = (int)cls;
    *out = g;
    return VLR_OK;
}

int vlr_grid_to_vol(vlr_ctx* ctx, const vlr_grid* g, int grid_class, void* out, size_t cap, size_t* n_bytes) {
    if (!ctx || !g || !n_bytes) return set_error(ctx, VLR_ERR_INVALID, "null argument");
    if (g->kind != VLR_KIND_F32_WORLD) return set_error(ctx, VLR_ERR_INVALID, "grid is not a world-unit f32 grid");
    const int cls = grid_class < 0 ? g->grid_class : grid_class;
    if (cls > 2) return set_error(ctx, VLR_ERR_INVALID, "grid class must be 0, 1 or 2 (or -1: the grid's own)");
    const size_t need = kVolHeader + (size_t)g->n * kVolLeaf;
    *n_bytes = need;
    if (!out) return VLR_OK;
    if (cap < need) return set_error(ctx, VLR_ERR_CAPACITY, "output buffer too small");
    // write_vol (src/io/vol_format.rs:53-83)
    unsigned char* b = static_cast<unsigned char*>(out);
    std::memcpy(b, "VOLR", 4);
    wr<uint32_t>(b + 4, 1u);
    wr<uint32_t>(b + 8, (uint32_t)cls);
    wr<double>(b + 12, g->xf.voxel_size);
    wr<float>(b + 20, g->background);
    wr<uint32_t>(b + 24, (uint32_t)g->n);
    wr<uint32_t>(b + 28, 0u);
    return grid_to_records(ctx, g, b + kVolHeader, kVolLeaf, 0, 12, 76, -1);
}

int vlr_grid_from_nano(vlr_ctx* ctx, const void* bytes, size_t n_bytes, vlr_grid** out, int* grid_class) {
    if (!ctx || !out || (!bytes && n_bytes)) return set_error(ctx, VLR_ERR_INVALID, "null argument");
    *out = nullptr;
    const unsigned char* b = static_cast<const unsigned char*>(bytes);
    // NanoGrid::from_bytes (src/nano/layout.rs:208-252)
    if (n_bytes < kNanoHeader) return set_error(ctx, VLR_ERR_FORMAT, "Buffer too small for NanoHeader");
    if (std::memcmp(b, "NANO", 4) != 0) return set_error(ctx, VLR_ERR_FORMAT, "Invalid magic");
    const uint32_t version = rd<uint32_t>(b + kNhVersion);
    if (version != 1) return set_error(ctx, VLR_ERR_FORMAT, "Unsupported version: " + std::to_string(version));
    const size_t count = rd<uint32_t>(b + kNhCount);
    if ((n_bytes - kNanoHeader) / kNanoLeaf < count) return set_error(ctx, VLR_ERR_FORMAT, "Buffer too small");
    if (count > (size_t)(1 << 30)) return set_error(ctx, VLR_ERR_CAPACITY, "too many leaves");
    const unsigned char* block = b + kNanoHeader;
    std::vector<int32_t> o(3 * count);
    for (size_t i = 0; i < count; ++i)
        for (int a = 0; a < 3; ++a) o[3 * i + a] = rd<int32_t>(block + i * kNanoLeaf + 4 * a);
    for (size_t i = 1; i < count; ++i)
        if (!origin_less(&o[3 * (i - 1)], &o[3 * i])) return set_error(ctx, VLR_ERR_FORMAT, "Leaves not sorted");
    for (size_t i = 0; i < 3 * count; ++i)
        if (o[i] & 7) return set_error(ctx, VLR_ERR_FORMAT, "NanoGrid leaf origin not a multiple of 8");
    // NanoGrid::to_grid (src/nano/layout.rs:255-286): a fresh grid holding the
    // active voxels only, so leaves without active voxels are not created and
    // inactive voxels read the background
    std::vector<int> order;
    std::vector<int32_t> origins;
    for (size_t i = 0; i < count; ++i) {
        bool any = false;
        for (int w = 0; w < 8 && !any; ++w) any = rd<uint64_t>(block + i * kNanoLeaf + 16 + 8 * w) != 0;
        if (!any) continue;
        order.push_back((int)i);
        origins.insert(origins.end(), &o[3 * i], &o[3 * i] + 3);
    }
    const uint32_t cls = rd<uint32_t>(b + kNhClass);
    vlr_grid* g = new vlr_grid();
    g->ctx = ctx;
    g->kind = VLR_KIND_F32_WORLD;
    g->background = rd<float>(b + kNhBackground);
    // Grid::with_affine (src/grid.rs:378-388): uniform transform at the map's voxel size
    const double vs = rd<double>(b + kNhVoxel);
    g->xf = uniform_transform(vs);
    for (int r = 0; r < 3; ++r)
        for (int c = 0; c < 4; ++c) {
            g->xf.affine[4 * r + c] = rd<double>(b + kNhMat + 8 * (4 * r + c));
            g->affine_inv[4 * r + c] = rd<double>(b + kNhInv + 8 * (4 * r + c));
        }
    g->has_inv = 1;
    g->grid_class = cls <= 2 ? (int)cls : 0;  // u32_to_grid_class: anything else is Unknown
    int rc = grid_from_records(ctx, g, block, count, kNanoLeaf, 0, 16, 80, order, origins, true);
    if (rc) {
        vlr_grid_destroy(g);
        return rc;
    }
    if (grid_class) *grid_class = g->grid_class;
    *out = g;
    return VLR_OK;
}

int vlr_grid_to_nano(vlr_ctx* ctx, const vlr_grid* g, int grid_class, const double* affine_inv, void* out,
                     size_t cap, size_t* n_bytes) {
    if (!ctx || !g || !n_bytes) return set_error(ctx, VLR_ERR_INVALID, "null argument");
    if (g->kind != VLR_KIND_F32_WORLD) return set_error(ctx, VLR_ERR_INVALID, "grid is not a world-unit f32 grid");
    const int cls = grid_class < 0 ? g->grid_class : grid_class;
    if (cls > 2) return set_error(ctx, VLR_ERR_INVALID, "grid class must be 0, 1 or 2 (or -1: the grid's own)");
    const size_t n = (size_t)g->n;
    const size_t need = kNanoHeader + n * kNanoLeaf;
    *n_bytes = need;
    if (!out) return VLR_OK;
    if (cap < need) return set_error(ctx, VLR_ERR_CAPACITY, "output buffer too small");
    // NanoGrid::from_grid (src/nano/layout.rs:89-170)
    unsigned char* b = static_cast<unsigned char*>(out);
    std::memset(b, 0, kNanoHeader);
    int rc = grid_to_records(ctx, g, b + kNanoHeader, kNanoLeaf, 0, 16, 80, 12);
    if (rc) return rc;
    // active bounding box, (0, 0, 0) for a grid without active voxels
    int32_t lo[3] = {INT32_MAX, INT32_MAX, INT32_MAX}, hi[3] = {INT32_MIN, INT32_MIN, INT32_MIN};
    // per leaf from its mask words (offset x * 64 + y * 8 + z): word x is the
    // x-plane, the bytes of the words' OR are the y-rows, the OR of those
    // bytes the z-columns
    for (size_t i = 0; i < n; ++i) {
        const unsigned char* r = b + kNanoHeader + i * kNanoLeaf;
        uint64_t any = 0;
        int x0 = 8, x1 = -1;
        for (int x = 0; x < 8; ++x) {
            const uint64_t w = rd<uint64_t>(r + 16 + 8 * x);
            if (!w) continue;
            any |= w;
            x0 = std::min(x0, x);
            x1 = x;
        }
        if (!any) continue;
        int y0 = 8, y1 = -1;
        unsigned zb = 0;
        for (int y = 0; y < 8; ++y) {
            const unsigned row = (unsigned)(any >> (8 * y)) & 0xFFu;
            if (!row) continue;
            zb |= row;
            y0 = std::min(y0, y);
            y1 = y;
        }
        const int z0 = __builtin_ctz(zb), z1 = 31 - __builtin_clz(zb);
        const int32_t o[3] = {rd<int32_t>(r), rd<int32_t>(r + 4), rd<int32_t>(r + 8)};
        const int l3[3] = {x0, y0, z0}, h3[3] = {x1, y1, z1};
        for (int a = 0; a < 3; ++a) {
            lo[a] = std::min(lo[a], o[a] + l3[a]);
            hi[a] = std::max(hi[a], o[a] + h3[a]);
        }
    }
    if (lo[0] == INT32_MAX)
        for (int a = 0; a < 3; ++a) lo[a] = hi[a] = 0;
    std::memcpy(b, "NANO", 4);
    wr<uint32_t>(b + kNhVersion, 1u);
    wr<uint32_t>(b + kNhClass, (uint32_t)cls);
    wr<double>(b + kNhVoxel, g->xf.affine_voxel_size);
    wr<float>(b + kNhBackground, g->background);
    wr<uint32_t>(b + kNhCount, (uint32_t)n);
    for (int a = 0; a < 3; ++a) {
        wr<int32_t>(b + kNhBboxMin + 4 * a, lo[a]);
        wr<int32_t>(b + kNhBboxMax + 4 * a, hi[a]);
    }
    // forward and inverse matrices: rows 0-2 from the grid, row 3 = (0, 0, 0, 1);
    // the inverse is the caller's, else the one the grid was read with, else
    // that of a uniform scale (1 / voxel size on the diagonal, as
    // AffineMap::from_uniform_scale stores it)
    double inv[12] = {0};
    if (affine_inv) std::memcpy(inv, affine_inv, sizeof(inv));
    else if (g->has_inv) std::memcpy(inv, g->affine_inv, sizeof(inv));
    else {
        const double is = 1.0 / g->xf.affine_voxel_size;
        inv[0] = inv[5] = inv[10] = is;
    }
    for (int r = 0; r < 4; ++r)
        for (int c = 0; c < 4; ++c) {
            const double m = r < 3 ? g->xf.affine[4 * r + c] : (c == 3 ? 1.0 : 0.0);
            const double v = r < 3 ? inv[4 * r + c] : (c == 3 ? 1.0 : 0.0);
            wr<double>(b + kNhMat + 8 * (4 * r + c), m);
            wr<double>(b + kNhInv + 8 * (4 * r + c), v);
        }
    return VLR_OK;
}

}  // extern "C"
