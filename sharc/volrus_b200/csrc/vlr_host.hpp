// Host-side context and grid handles behind the C ABI (include/volrus_b200.h).
#pragma once
#include <cstdint>
#include <string>
#include <vector>
#include <cuda_runtime.h>

#include "vlr_common.cuh"
#include "../../../include/volrus_b200.h"

// Optional per-kernel timing with CUDA events on the context stream (enabled
// by vlr_ctx_profile); durations are accumulated per kernel name.
struct vlr_kernel_timer {
    bool enabled = false;
    struct Pending {
        const char* name;
        cudaEvent_t a, b;
    };
    std::vector<Pending> pending;
    std::vector<cudaEvent_t> free_events;
    std::vector<std::pair<std::string, std::pair<double, long long>>> totals;  // name -> (ms, launches)
};

struct vlr_ctx {
    int device = 0;
    int sm_count = 148;
    cudaStream_t stream = nullptr;
    cudaMemPool_t pool = nullptr;       // stream-ordered temporaries; freed memory stays with the pool
    unsigned* d_errword = nullptr;      // device error bits (vlr::kErr*)
    std::string last_error;
    // Scratch reused across calls on this context (grown on demand).
    void* scratch = nullptr;
    size_t scratch_bytes = 0;
    void* pinned = nullptr;             // small pinned host buffer for scalar read-backs
    void* stage = nullptr;              // pinned double buffer for large copies into pageable memory
    cudaEvent_t stage_ev[2] = {nullptr, nullptr};
    vlr_kernel_timer timer;
};

// Value storage kinds.
enum vlr_value_kind : int {
    VLR_KIND_F32_WORLD = 0,   // f32 values in world units: reference semantics
    VLR_KIND_F32_VOXEL = 1,   // f32 values in voxel units: narrow-band method, plain FP32
    VLR_KIND_F16_VOXEL = 2,   // f16 values in voxel units: narrow-band method, FP16 leaves
};

struct vlr_grid {
    vlr_ctx* ctx = nullptr;
    int n = 0;          // live leaves (slots 0..n-1 in list order)
    int cap = 0;        // allocated slots
    int kind = VLR_KIND_F32_WORLD;
    float background = 0.0f;
    vlr_transform xf{};
    long long base[3] = {0, 0, 0};
    void* block = nullptr;  // one stream-ordered allocation (ctx->pool) holding the arrays below
    int4* origin = nullptr;
    uint64_t* mask = nullptr;
    void* values = nullptr;
    int* nbr = nullptr;
    uint64_t* hkey = nullptr;
    int* hval = nullptr;
    int hcap = 0;
    // metadata carried for the serialised formats (src/io/vol_format.rs, src/nano/layout.rs)
    int grid_class = 0;          // 0 unknown, 1 level set, 2 fog volume
    int has_inv = 0;             // affine_inv holds the inverse map the grid was read with
    double affine_inv[12] = {0}; // rows 0..2 of the inverse 4x4 (world -> index)
};

namespace vlr {

// Makes `device` current for a scope and restores the calling thread's
// previous current device on exit (also on early returns), so a one-time
// per-device set-up does not change which device the caller works on.
struct DeviceGuard {
    int prev = -1;
    int dev = -1;
    cudaError_t status = cudaSuccess;
    explicit DeviceGuard(int device) : dev(device) {
        status = cudaGetDevice(&prev);
        if (status == cudaSuccess && prev != dev) status = cudaSetDevice(dev);
    }
    ~DeviceGuard() {
        if (prev >= 0 && prev != dev) cudaSetDevice(prev);
    }
    DeviceGuard(const DeviceGuard&) = delete;
    DeviceGuard& operator=(const DeviceGuard&) = delete;
};

// Device temporaries of one host function: each pointer registered with
// track() is freed (cudaFree, which waits for the work using it) when the
// holder goes out of scope, on every return path, so an early error return
// leaks nothing.
struct DeviceTemps {
    std::vector<void*> ptrs;
    template <typename P>
    P* track(P* p) {
        ptrs.push_back((void*)p);
        return p;
    }
    ~DeviceTemps() {
        for (void* p : ptrs)
            if (p) cudaFree(p);
    }
};

// Error helpers: record a message on the context and return a status.
int set_error(vlr_ctx* ctx, int code, const std::string& msg);
int check_cuda(vlr_ctx* ctx, cudaError_t e, const char* what);
#define VLR_CUDA(ctx, call)                                   \
    do {                                                      \
        cudaError_t _e = (call);                              \
        if (_e != cudaSuccess) return vlr::check_cuda(ctx, _e, #call); \
    } while (0)

size_t value_bytes(int kind);

// Allocation of a grid's device arrays for `cap` slots (values of `kind`).
int grid_alloc(vlr_ctx* ctx, vlr_grid* g, int cap);
void grid_free_arrays(vlr_grid* g);
// (Re)build hash table and neighbour table for slots 0..n-1.
int grid_index(vlr_ctx* ctx, vlr_grid* g);
// Choose the hash-key base from the leaf-coordinate bounding box (host origins).
int choose_base(vlr_ctx* ctx, const int32_t* origins, size_t n, long long base[3]);
// Keep slots whose flag is non-zero (order preserved); rebuilds the index.
int grid_compact(vlr_ctx* ctx, vlr_grid* g, const int* d_flags);
// Scratch memory owned by the context (valid until the next call that grows it).
int ctx_scratch(vlr_ctx* ctx, size_t bytes, void** out);
// Exclusive scan of n ints on the context stream; writes total to *d_total (device).
int scan_exclusive(vlr_ctx* ctx, const int* d_in, int* d_out, int n, int* d_total);
// Read the device error word, clear it, and map it to a status.
int consume_device_errors(vlr_ctx* ctx, const char* what);
// Device-to-host copy of `bytes` on the context stream, returning after it.
// Large copies into pageable memory go through a pinned double buffer (the
// DMA of one chunk overlaps the host copy of the previous one), twice the
// driver's own pageable rate here; small or pinned destinations take one copy.
int d2h_copy(vlr_ctx* ctx, void* dst, const void* src, size_t bytes);
int read_int(vlr_ctx* ctx, const int* d_ptr, int* out);

// Kernel timing: bracket a launch with timer_begin/timer_end (no-ops unless
// profiling is enabled); timer_collect folds finished event pairs into totals.
void timer_begin(vlr_ctx* ctx, const char* name);
void timer_end(vlr_ctx* ctx);
int timer_collect(vlr_ctx* ctx);
#define VLR_TIMED(ctx, name, ...)    \
    do {                             \
        vlr::timer_begin(ctx, name); \
        __VA_ARGS__;                 \
        vlr::timer_end(ctx);         \
    } while (0)

}  // namespace vlr
