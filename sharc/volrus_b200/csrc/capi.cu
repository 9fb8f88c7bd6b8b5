// C ABI entry points (include/volrus_b200.h).  Thin: argument checks, host
// staging of flat leaf arrays, and calls into the kernels' host wrappers.
#include <algorithm>
#include <cstring>
#include <numeric>
#include <string>
#include <vector>

#include "ref_ops.hpp"

using namespace vlr;

namespace {

bool lex_less(const int32_t* a, const int32_t* b) {
    if (a[0] != b[0]) return a[0] < b[0];
    if (a[1] != b[1]) return a[1] < b[1];
    return a[2] < b[2];
}

// Upload n leaves (any order) as a world-unit f32 grid, stored in (x, y, z) order.
int upload_leaves(vlr_ctx* ctx, vlr_grid* g, const int32_t* origins, const uint64_t* masks, const float* values,
                  size_t n) {
    if (n > (size_t)(1 << 30)) return set_error(ctx, VLR_ERR_CAPACITY, "too many leaves");
    for (size_t i = 0; i < 3 * n; ++i)
        if (origins[i] & 7) return set_error(ctx, VLR_ERR_INVALID, "leaf origin not a multiple of 8");
    std::vector<size_t> order(n);
    std::iota(order.begin(), order.end(), 0);
    std::sort(order.begin(), order.end(),
              [&](size_t a, size_t b) { return lex_less(origins + 3 * a, origins + 3 * b); });
    for (size_t i = 1; i < n; ++i)
        if (!lex_less(origins + 3 * order[i - 1], origins + 3 * order[i]))
            return set_error(ctx, VLR_ERR_INVALID, "duplicate leaf origin");
    int rc = choose_base(ctx, origins, n, g->base);
    if (rc) return rc;
    rc = grid_alloc(ctx, g, (int)std::max<size_t>(n, 1));
    if (rc) return rc;
    g->n = (int)n;
    if (n) {
        std::vector<int4> o(n);
        std::vector<uint64_t> m(8 * n);
        std::vector<float> v(512 * n);
        for (size_t i = 0; i < n; ++i) {
            size_t s = order[i];
            o[i] = make_int4(origins[3 * s], origins[3 * s + 1], origins[3 * s + 2], 0);
            std::memcpy(&m[8 * i], masks + 8 * s, 64);
            std::memcpy(&v[512 * i], values + 512 * s, 2048);
        }
        VLR_CUDA(ctx, cudaMemcpyAsync(g->origin, o.data(), sizeof(int4) * n, cudaMemcpyHostToDevice, ctx->stream));
        VLR_CUDA(ctx, cudaMemcpyAsync(g->mask, m.data(), 64 * n, cudaMemcpyHostToDevice, ctx->stream));
        VLR_CUDA(ctx, cudaMemcpyAsync(g->values, v.data(), 2048 * n, cudaMemcpyHostToDevice, ctx->stream));
        VLR_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    }
    return grid_index(ctx, g);
}

int download_leaves(vlr_ctx* ctx, const vlr_grid* g, int32_t* origins, uint64_t* masks, float* values) {
    size_t n = (size_t)g->n;
    if (!n) return VLR_OK;
    std::vector<int4> o(n);
    VLR_CUDA(ctx, cudaMemcpyAsync(o.data(), g->origin, sizeof(int4) * n, cudaMemcpyDeviceToHost, ctx->stream));
    std::vector<uint64_t> m(8 * n);
    std::vector<float> v(512 * n);
    VLR_CUDA(ctx, cudaMemcpyAsync(m.data(), g->mask, 64 * n, cudaMemcpyDeviceToHost, ctx->stream));
    VLR_CUDA(ctx, cudaMemcpyAsync(v.data(), g->values, 2048 * n, cudaMemcpyDeviceToHost, ctx->stream));
    VLR_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    std::vector<size_t> order(n);
    std::iota(order.begin(), order.end(), 0);
    auto key = [&](size_t i) { return o[i]; };
    std::sort(order.begin(), order.end(), [&](size_t a, size_t b) {
        int4 A = key(a), B = key(b);
        if (A.x != B.x) return A.x < B.x;
        if (A.y != B.y) return A.y < B.y;
        return A.z < B.z;
    });
    for (size_t i = 0; i < n; ++i) {
        size_t s = order[i];
        origins[3 * i] = o[s].x;
        origins[3 * i + 1] = o[s].y;
        origins[3 * i + 2] = o[s].z;
        std::memcpy(masks + 8 * i, &m[8 * s], 64);
        std::memcpy(values + 512 * i, &v[512 * s], 2048);
    }
    return VLR_OK;
}

uint64_t count_active_host(vlr_ctx* ctx, const vlr_grid* g, int* rc) {
    *rc = VLR_OK;
    if (!g->n) return 0;
    std::vector<uint64_t> m(8 * (size_t)g->n);
    cudaError_t e = cudaMemcpyAsync(m.data(), g->mask, 64 * (size_t)g->n, cudaMemcpyDeviceToHost, ctx->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    if (e != cudaSuccess) {
        *rc = check_cuda(ctx, e, "count active");
        return 0;
    }
    uint64_t c = 0;
    for (uint64_t w : m) c += (uint64_t)__builtin_popcountll(w);
    return c;
}

vlr_grid* new_grid(vlr_ctx* ctx) {
    vlr_grid* g = new vlr_grid();
    g->ctx = ctx;
    return g;
}

}  // namespace

extern "C" {

int vlr_ctx_create(int device, vlr_ctx** out) {
    if (!out) return VLR_ERR_INVALID;
    *out = nullptr;
    vlr_ctx* c = new vlr_ctx();
    c->device = device;
    cudaError_t e = cudaSetDevice(device);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking);
    if (e == cudaSuccess) {
        // a private pool for the library's stream-ordered temporaries, keeping
        // freed memory for reuse (the device's default pool hands it back to
        // the driver at every synchronisation, so each call would allocate anew)
        cudaMemPoolProps props = {};
        props.allocType = cudaMemAllocationTypePinned;
        props.location.type = cudaMemLocationTypeDevice;
        props.location.id = device;
        e = cudaMemPoolCreate(&c->pool, &props);
        if (e == cudaSuccess) {
            uint64_t keep = UINT64_MAX;
            e = cudaMemPoolSetAttribute(c->pool, cudaMemPoolAttrReleaseThreshold, &keep);
        }
    }
    if (e == cudaSuccess) e = cudaMalloc(&c->d_errword, sizeof(unsigned) * 4);
    if (e == cudaSuccess) e = cudaMemset(c->d_errword, 0, sizeof(unsigned) * 4);
    if (e == cudaSuccess) e = cudaMallocHost(&c->pinned, 4096);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&c->sm_count, cudaDevAttrMultiProcessorCount, device);
    if (e != cudaSuccess) {
        delete c;
        return VLR_ERR_CUDA;
    }
    *out = c;
    return VLR_OK;
}

void vlr_ctx_destroy(vlr_ctx* ctx) {
    if (!ctx) return;
    vlr::DeviceGuard guard(ctx->device);  // the caller's current device is restored on return
    if (ctx->stream) cudaStreamSynchronize(ctx->stream);
    cudaFree(ctx->scratch);
    cudaFree(ctx->d_errword);
    cudaFreeHost(ctx->pinned);
    if (ctx->stage) cudaFreeHost(ctx->stage);
    for (auto& e : ctx->stage_ev)
        if (e) cudaEventDestroy(e);
    if (ctx->stream) cudaStreamDestroy(ctx->stream);
    if (ctx->pool) cudaMemPoolDestroy(ctx->pool);
    delete ctx;
}

const char* vlr_last_error(const vlr_ctx* ctx) { return ctx ? ctx->last_error.c_str() : "null context"; }

// Words 2 and 3 of the device error word hold the test-stall flag and the
// wait bound; kernels read them when they start.
int vlr_ctx_set_wait_limit(vlr_ctx* ctx, uint32_t polls) {
    if (!ctx) return VLR_ERR_INVALID;
    unsigned* h = (unsigned*)ctx->pinned + 48;  // a slot no other read-back uses
    *h = polls;
    VLR_CUDA(ctx, cudaMemcpyAsync(ctx->d_errword + 3, h, sizeof(unsigned), cudaMemcpyHostToDevice, ctx->stream));
    VLR_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    return VLR_OK;
}

int vlr_ctx_test_stall(vlr_ctx* ctx, int on) {
    if (!ctx) return VLR_ERR_INVALID;
    unsigned* h = (unsigned*)ctx->pinned + 49;
    *h = on ? 1u : 0u;
    VLR_CUDA(ctx, cudaMemcpyAsync(ctx->d_errword + 2, h, sizeof(unsigned), cudaMemcpyHostToDevice, ctx->stream));
    VLR_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    return VLR_OK;
}

int vlr_ctx_synchronize(vlr_ctx* ctx) {
    if (!ctx) return VLR_ERR_INVALID;
    VLR_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    return VLR_OK;
}

int vlr_ctx_stream(vlr_ctx* ctx, void** stream) {
    if (!ctx || !stream) return set_error(ctx, VLR_ERR_INVALID, "null argument");
    *stream = (void*)ctx->stream;
    return VLR_OK;
}

int vlr_host_alloc(vlr_ctx* ctx, size_t bytes, void** out) {
    if (!ctx || !out) return set_error(ctx, VLR_ERR_INVALID, "null argument");
    *out = nullptr;
    if (!bytes) return VLR_OK;
    vlr::DeviceGuard guard(ctx->device);
    const cudaError_t e = cudaMallocHost(out, bytes);
    if (e != cudaSuccess) {
        *out = nullptr;
        cudaGetLastError();
        return set_error(ctx, VLR_ERR_NOMEM, "page-locked host allocation failed");
    }
    return VLR_OK;
}

int vlr_host_free(vlr_ctx* ctx, void* p) {
    if (!ctx) return VLR_ERR_INVALID;
    if (!p) return VLR_OK;
    vlr::DeviceGuard guard(ctx->device);
    const cudaError_t e = cudaFreeHost(p);
    return e == cudaSuccess ? VLR_OK : vlr::check_cuda(ctx, e, "cudaFreeHost");
}

int vlr_ctx_profile(vlr_ctx* ctx, int enable) {
    if (!ctx) return VLR_ERR_INVALID;
    int rc = timer_collect(ctx);
    if (rc) return rc;
    ctx->timer.enabled = enable != 0;
    if (enable) ctx->timer.totals.clear();
    return VLR_OK;
}

int vlr_ctx_profile_read(vlr_ctx* ctx, const char* kernel, double* total_ms, long long* launches) {
    if (!ctx || !kernel || !total_ms || !launches) return set_error(ctx, VLR_ERR_INVALID, "null argument");
    int rc = timer_collect(ctx);
    if (rc) return rc;
    *total_ms = 0.0;
    *launches = 0;
    for (auto& kv : ctx->timer.totals)
        if (kv.first == kernel) {
            *total_ms = kv.second.first;
            *launches = kv.second.second;
        }
    return VLR_OK;
}

int vlr_grid_create(vlr_ctx* ctx, const vlr_transform* xf, float background, const int32_t* origins,
                    const uint64_t* masks, const float* values, size_t n_leaves, vlr_grid** out) {
    if (!ctx || !xf || !out) return set_error(ctx, VLR_ERR_INVALID, "null argument");
    if (n_leaves && (!origins || !masks || !values)) return set_error(ctx, VLR_ERR_INVALID, "null leaf arrays");
    *out = nullptr;
    vlr_grid* g = new_grid(ctx);
    g->kind = VLR_KIND_F32_WORLD;
    g->background = background;
    g->xf = *xf;
    int rc = upload_leaves(ctx, g, origins, masks, values, n_leaves);
    if (rc) {
        vlr_grid_destroy(g);
        return rc;
    }
    *out = g;
    return VLR_OK;
}

__global__ void k_origins_to_int4(const int32_t* o3, size_t n, int4* origin) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
        origin[i] = make_int4(o3[3 * i], o3[3 * i + 1], o3[3 * i + 2], 0);
}

int vlr_grid_create_device(vlr_ctx* ctx, const vlr_transform* xf, float background, const int32_t* d_origins,
                           const uint64_t* d_masks, const float* d_values, size_t n_leaves, vlr_grid** out) {
    if (!ctx || !xf || !out) return set_error(ctx, VLR_ERR_INVALID, "null argument");
    if (n_leaves && (!d_origins || !d_masks || !d_values)) return set_error(ctx, VLR_ERR_INVALID, "null leaf arrays");
    if (n_leaves > (size_t)(1 << 30)) return set_error(ctx, VLR_ERR_CAPACITY, "too many leaves");
    *out = nullptr;
    // the origins come to the host (12 bytes a leaf) for the order check and
    // the hash-key base; masks and values stay on the device
    std::vector<int32_t> o(3 * n_leaves);
    if (n_leaves) {
        VLR_CUDA(ctx, cudaMemcpyAsync(o.data(), d_origins, 12 * n_leaves, cudaMemcpyDeviceToHost, ctx->stream));
        VLR_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    }
    for (size_t i = 0; i < 3 * n_leaves; ++i)
        if (o[i] & 7) return set_error(ctx, VLR_ERR_INVALID, "leaf origin not a multiple of 8");
    for (size_t i = 1; i < n_leaves; ++i)
        if (!lex_less(&o[3 * (i - 1)], &o[3 * i]))
            return set_error(ctx, VLR_ERR_INVALID, "device leaves not sorted by (x, y, z) or origin repeated");
    vlr_grid* g = new_grid(ctx);
    g->kind = VLR_KIND_F32_WORLD;
    g->background = background;
    g->xf = *xf;
    int rc = choose_base(ctx, o.data(), n_leaves, g->base);
    if (!rc) rc = grid_alloc(ctx, g, (int)std::max<size_t>(n_leaves, 1));
    if (!rc && n_leaves) {
        g->n = (int)n_leaves;
        k_origins_to_int4<<<ctx->sm_count * 4, 256, 0, ctx->stream>>>(d_origins, n_leaves, g->origin);
        cudaError_t e = cudaGetLastError();
        if (e == cudaSuccess) e = cudaMemcpyAsync(g->mask, d_masks, 64 * n_leaves, cudaMemcpyDeviceToDevice, ctx->stream);
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(g->values, d_values, 2048 * n_leaves, cudaMemcpyDeviceToDevice, ctx->stream);
        if (e != cudaSuccess) rc = check_cuda(ctx, e, "vlr_grid_create_device");
    }
    if (!rc) rc = grid_index(ctx, g);
    if (rc) {
        vlr_grid_destroy(g);
        return rc;
    }
    *out = g;
    return VLR_OK;
}

int vlr_grid_info(vlr_ctx* ctx, const vlr_grid* g, size_t* n_leaves, uint64_t* n_active, float* background,
                  vlr_transform* xf) {
    if (!ctx || !g) return set_error(ctx, VLR_ERR_INVALID, "null argument");
    if (n_leaves) *n_leaves = (size_t)g->n;
    if (background) *background = g->background;
    if (xf) *xf = g->xf;
    if (n_active) {
        int rc;
        *n_active = count_active_host(ctx, g, &rc);
        if (rc) return rc;
    }
    return VLR_OK;
}

int vlr_grid_download(vlr_ctx* ctx, const vlr_grid* g, int32_t* origins, uint64_t* masks, float* values,
                      size_t cap_leaves) {
    if (!ctx || !g) return set_error(ctx, VLR_ERR_INVALID, "null argument");
    if (g->kind != VLR_KIND_F32_WORLD) return set_error(ctx, VLR_ERR_INVALID, "grid is not a world-unit f32 grid");
    if (cap_leaves < (size_t)g->n) return set_error(ctx, VLR_ERR_CAPACITY, "output buffers too small");
    if (g->n && (!origins || !masks || !values)) return set_error(ctx, VLR_ERR_INVALID, "null output arrays");
    return download_leaves(ctx, g, origins, masks, values);
}

void vlr_grid_destroy(vlr_grid* g) {
    if (!g) return;
    if (g->ctx) cudaStreamSynchronize(g->ctx->stream);
    grid_free_arrays(g);
    delete g;
}

int vlr_make_level_set_sphere(vlr_ctx* ctx, double radius, const double center[3], double voxel_size,
                              double half_width, vlr_grid** out) {
    if (!ctx || !center || !out) return set_error(ctx, VLR_ERR_INVALID, "null argument");
    *out = nullptr;
    vlr_grid* g = new_grid(ctx);
    int rc = make_sphere(ctx, radius, center, voxel_size, half_width, g);
    if (rc) {
        vlr_grid_destroy(g);
        return rc;
    }
    *out = g;
    return VLR_OK;
}

int vlr_sample_trilinear(vlr_ctx* ctx, const vlr_grid* g, const double* world_xyz, size_t n, float* out) {
    if (!ctx || !g || (n && (!world_xyz || !out))) return set_error(ctx, VLR_ERR_INVALID, "null argument");
    if (g->kind != VLR_KIND_F32_WORLD) return set_error(ctx, VLR_ERR_INVALID, "grid is not a world-unit f32 grid");
    return sample_points(ctx, g, world_xyz, n, out);
}

int vlr_advect_level_set(vlr_ctx* ctx, const vlr_grid* g, const vlr_grid* vx, const vlr_grid* vy,
                         const vlr_grid* vz, double dt, vlr_grid** out) {
    if (!ctx || !g || !vx || !vy || !vz || !out) return set_error(ctx, VLR_ERR_INVALID, "null argument");
    for (const vlr_grid* q : {g, vx, vy, vz})
        if (q->kind != VLR_KIND_F32_WORLD) return set_error(ctx, VLR_ERR_INVALID, "grid is not a world-unit f32 grid");
    *out = nullptr;
    vlr_grid* o = new_grid(ctx);
    int rc = advect_ref(ctx, g, vx, vy, vz, dt, o);
    if (rc) {
        vlr_grid_destroy(o);
        return rc;
    }
    *out = o;
    return VLR_OK;
}

int vlr_find_zero_crossings(vlr_ctx* ctx, const vlr_grid* g, int32_t* coords, size_t cap, size_t* count) {
    if (!ctx || !g || !count) return set_error(ctx, VLR_ERR_INVALID, "null argument");
    if (g->kind != VLR_KIND_F32_WORLD) return set_error(ctx, VLR_ERR_INVALID, "grid is not a world-unit f32 grid");
    bool sorted = false;
    int rc = find_zero_crossings(ctx, g, coords, cap, count, &sorted);
    if (rc) return rc;
    if (coords && cap && !sorted) {  // keys over 63 bits: sort on the host
        size_t m = std::min(cap, *count);
        std::vector<size_t> order(m);
        std::iota(order.begin(), order.end(), 0);
        std::vector<int32_t> tmp(coords, coords + 3 * m);
        std::sort(order.begin(), order.end(),
                  [&](size_t a, size_t b) { return lex_less(&tmp[3 * a], &tmp[3 * b]); });
        for (size_t i = 0; i < m; ++i) std::memcpy(coords + 3 * i, &tmp[3 * order[i]], 12);
    }
    return VLR_OK;
}

int vlr_trim_narrow_band(vlr_ctx* ctx, vlr_grid* g, float half_width) {
    if (!ctx || !g) return set_error(ctx, VLR_ERR_INVALID, "null argument");
    if (g->kind != VLR_KIND_F32_WORLD) return set_error(ctx, VLR_ERR_INVALID, "grid is not a world-unit f32 grid");
    return trim_narrow_band(ctx, g, half_width);
}

int vlr_rebuild_narrow_band(vlr_ctx* ctx, vlr_grid* g, float half_width) {
    if (!ctx || !g) return set_error(ctx, VLR_ERR_INVALID, "null argument");
    if (g->kind != VLR_KIND_F32_WORLD) return set_error(ctx, VLR_ERR_INVALID, "grid is not a world-unit f32 grid");
    return rebuild_narrow_band(ctx, g, half_width);
}

int vlr_advect_rebuild_host(vlr_ctx* ctx, const vlr_transform* xf, float background, const int32_t* origins,
                            const uint64_t* masks, const float* values, size_t n_leaves, const float velocity[3],
                            double dt, float half_width, int32_t* out_origins, uint64_t* out_masks,
                            float* out_values, size_t cap_leaves, size_t* out_n) {
    if (!ctx || !xf || !velocity || !out_n) return set_error(ctx, VLR_ERR_INVALID, "null argument");
    *out_n = 0;
    vlr_grid* g = nullptr;
    int rc = vlr_grid_create(ctx, xf, background, origins, masks, values, n_leaves, &g);
    if (rc) return rc;
    vlr_grid* vel[3] = {nullptr, nullptr, nullptr};
    vlr_transform vxf;
    std::memset(&vxf, 0, sizeof(vxf));
    vxf.voxel_size = xf->voxel_size;
    vxf.affine[0] = vxf.affine[5] = vxf.affine[10] = xf->voxel_size;
    vxf.affine_voxel_size = xf->voxel_size;
    for (int a = 0; a < 3 && !rc; ++a) rc = vlr_grid_create(ctx, &vxf, velocity[a], nullptr, nullptr, nullptr, 0, &vel[a]);
    vlr_grid* o = nullptr;
    if (!rc) rc = vlr_advect_level_set(ctx, g, vel[0], vel[1], vel[2], dt, &o);
    if (!rc) rc = vlr_rebuild_narrow_band(ctx, o, half_width);
    if (!rc) {
        *out_n = (size_t)o->n;
        if ((size_t)o->n > cap_leaves) rc = set_error(ctx, VLR_ERR_CAPACITY, "output buffers too small");
        else rc = download_leaves(ctx, o, out_origins, out_masks, out_values);
    }
    vlr_grid_destroy(o);
    for (auto* v : vel) vlr_grid_destroy(v);
    vlr_grid_destroy(g);
    return rc;
}

}  // extern "C"
