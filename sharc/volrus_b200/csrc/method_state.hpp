// Host-side state of a method grid (or a batch of grids): slot pool, ordered
// leaf list, hash index, neighbour table, per-grid parameters, velocity
// tables and the captured step graph.
#pragma once
#include <vector>

#include "method_kernels.hpp"
#include "vlr_host.hpp"

// Launch shape of a stencil kernel: threads per CTA, persistent CTAs and the
// staging of its halo tiles.
struct StencilShape {
    int nt = 0;       // threads per CTA (128; 0: not chosen)
    int blocks = 0;   // grid size (CTAs per SM x SMs)
    int stage = 0;    // staging of the halo tile: 0, row pieces by cp.async (the only mode)
};

// Most slabs a host step is cut into (vlr_ls_set_host_slabs).
constexpr int kHostSlabsMax = 16;

// One timed candidate of the launch autotuner.
struct TuneEntry {
    StencilShape shape;
    float ms;
};

struct vlr_level_set {
    vlr_ctx* ctx = nullptr;
    int precision = 0;       // VLR_PREC_F32 / VLR_PREC_F16
    int cap = 0;             // slots
    int n_grids = 1;
    int key_bits = 21;
    int halo = 2;
    int reinit_iters = 2;
    // slot-indexed arrays
    int4* origin = nullptr;
    uint64_t* mask = nullptr;
    uint64_t* dmask = nullptr;
    void* vals[2] = {nullptr, nullptr};  // vals[0] holds the state between steps
    int* nbr = nullptr;
    unsigned* spill = nullptr;
    int* nonempty = nullptr;
    int* keep = nullptr;
    // list (position-indexed)
    int* list = nullptr;
    int* list_new = nullptr;
    int* owned = nullptr;    // cap + 1: slots of leaves dropped this step (recycle list)
    int* pos = nullptr;      // status words of the look-back scan (zeroed at allocation)
    int* newinfo = nullptr;  // cap: per new-list position, owner slot * 32 + direction (-1 survivor)
    int* free_stack = nullptr;
    int* scalars = nullptr;  // [0] count, [1] step, [2] free top, [3] new count
    // hash (key -> slot) and proposal table (key -> min owner direction)
    uint64_t* hkey = nullptr;
    int* hval = nullptr;
    uint64_t* pkey = nullptr;
    int* pval = nullptr;
    int hcap = 0;
    // parameters
    vlr::MGridParams* d_params = nullptr;
    std::vector<vlr::MGridParams> h_params;
    float2* d_tab = nullptr;
    vlr::MStepParams sp{};
    // reductions
    double* d_partial = nullptr;
    double* d_sum = nullptr;
    // staging for uploads and downloads (grown on demand)
    void* staging = nullptr;
    size_t staging_bytes = 0;
    // captured step
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t graph_exec = nullptr;
    int grid_blocks = 0;     // persistent grid size of the index and topology kernels
    int vel_kind = -1;       // velocity kind shared by every grid (MVEL_*), -1 if mixed
    StencilShape adv_shape;  // launch shapes of the stencil kernels
    StencilShape re_shape;
    bool tuned = false;      // shapes chosen (by the autotuner or the caller)
    bool state_lost = false; // a step failed with VLR_ERR_TIMEOUT or VLR_ERR_CAPACITY: the state is undefined
    bool autotune = true;    // choose the shapes on the first step
    // host steps over x-slabs (vlr_ls_step_host): 0 automatic, 1 one pass,
    // k >= 2 at most k slabs; the copy streams and events, made on first use
    int host_slabs = 0;
    cudaStream_t slab_stream[2] = {nullptr, nullptr};  // host -> device, device -> host
    cudaEvent_t slab_ev[2 * kHostSlabsMax + 2] = {};
    std::vector<TuneEntry> tune_log[2];  // candidates timed by the autotuner (advect, reinit)
    int scan_levels = 0;

    vlr::MLeafArrays arrays() const {
        vlr::MLeafArrays A;
        A.list = list;
        A.count = scalars;
        A.step = scalars + 1;
        A.origin = origin;
        A.mask = mask;
        A.dmask = dmask;
        A.nbr = nbr;
        A.spill = spill;
        A.nonempty = nonempty;
        return A;
    }
};

namespace vlr {

int ls_alloc(vlr_ctx* ctx, vlr_level_set* ls, int cap);
void ls_free(vlr_level_set* ls);
// Enqueue one step (no host synchronisation; capturable).
int ls_enqueue_step(vlr_ctx* ctx, vlr_level_set* ls);
// Rebuild hash and neighbour table from the list (enqueued).
int ls_enqueue_index(vlr_ctx* ctx, vlr_level_set* ls);
int ls_enqueue_retrack(vlr_ctx* ctx, vlr_level_set* ls);
// One step whose stencil kernels are launched at every candidate shape (timed,
// synchronising); keeps the fastest shape of each kernel.  The step's result
// is the same as ls_enqueue_step's.
int ls_autotune_step(vlr_ctx* ctx, vlr_level_set* ls);
// Parameters and velocity tables of n grids (bounding boxes in index units).
int ls_setup_grids(vlr_ctx* ctx, vlr_level_set* ls, const vlr_method_desc* m, const vlr_velocity_desc* const* vels,
                   const int32_t (*bb_lo)[3], const int32_t (*bb_hi)[3], int n);
// List = slots 0..n-1, free stack = the rest; rebuilds hash and neighbours (synchronises).
int ls_init_lists(vlr_ctx* ctx, vlr_level_set* ls, int n, bool reset_step);

}  // namespace vlr
