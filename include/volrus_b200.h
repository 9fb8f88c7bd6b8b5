/*
 * volrus_b200.h — C ABI of the B200 narrow-band level-set advection library.
 *
 * This is the drop-in boundary for the Sharc.Volrus advection path.  The
 * reference exposes that path as plain Rust free functions over Grid<f32>
 * (re-exported at src/lib.rs:29-43); each entry point below names the
 * function it replaces.  Grids cross the boundary as flat leaf arrays, the
 * record the reference already uses for its flat layout NanoLeaf
 * (src/nano/layout.rs:41-52) and its .vol format (src/io/vol_format.rs:1-21):
 *   origins  int32[n][3]    leaf origins (multiples of 8), sorted (x, y, z)
 *   masks    uint64[n][8]   activity bits, bit off = x*64 + y*8 + z (ZYX order)
 *   values   float[n][512]  voxel values in ZYX order
 * Device grids are opaque handles owned by a context; every buffer passed in
 * is caller-owned host memory.  All functions return VLR_OK (0) or an error
 * code; vlr_last_error() gives the message.  A context is thread-compatible:
 * one thread at a time, one CUDA stream per context.
 */
#ifndef VOLRUS_B200_H
#define VOLRUS_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum {
    VLR_OK = 0,
    VLR_ERR_INVALID = 1,   /* bad argument (null pointer, duplicate leaf, unaligned origin, ...) */
    VLR_ERR_CUDA = 2,      /* CUDA runtime error */
    VLR_ERR_CAPACITY = 3,  /* leaf pool or hash capacity exceeded (a level-set step that reports it is
                              abandoned and leaves the state undefined, as for VLR_ERR_TIMEOUT) */
    VLR_ERR_EXTENT = 4,    /* grid spans more than 2^24 voxels along an axis */
    VLR_ERR_REACH = 5,     /* a backtrace left the staged neighbourhood (time step too large) */
    VLR_ERR_NOMEM = 6,     /* device allocation failed */
    VLR_ERR_FORMAT = 7,    /* malformed flat-grid buffer */
    VLR_ERR_TIMEOUT = 8,   /* a bounded device-side wait gave up; the operation's outputs (a level set's
                              state included) are undefined: synchronise the context and upload or
                              re-create the level set before stepping it again */
    VLR_ERR_UNSUPPORTED = 9
};

typedef struct vlr_ctx vlr_ctx;
typedef struct vlr_grid vlr_grid;

/* Transform of a grid: the legacy VoxelTransform (voxel_size, origin) that
 * sample_trilinear uses (src/grid.rs:62-121) and the forward rows of the
 * AffineMap that advect_level_set uses for index->world (src/grid.rs:131-257). */
typedef struct vlr_transform {
    double voxel_size;
    double origin[3];
    double affine[12];       /* rows 0..2 of the 4x4 forward matrix, row-major */
    double affine_voxel_size;/* AffineMap::voxel_size() */
} vlr_transform;

/* ---- context ---------------------------------------------------------- */
int vlr_ctx_create(int device, vlr_ctx** out);
void vlr_ctx_destroy(vlr_ctx* ctx);
const char* vlr_last_error(const vlr_ctx* ctx);
int vlr_ctx_synchronize(vlr_ctx* ctx);
/* The context's CUDA stream (cudaStream_t), for callers that order their own
 * work or events with the library's.  No counterpart in the reference. */
int vlr_ctx_stream(vlr_ctx* ctx, void** stream);
/* Page-locked host memory (freed with vlr_host_free): the buffers that let
 * host-resident calls copy at the link's full rate and overlap their copies
 * (vlr_ls_step_host's slab pipeline takes effect only on such buffers), for
 * callers without a CUDA runtime of their own.  No counterpart in the
 * reference. */
int vlr_host_alloc(vlr_ctx* ctx, size_t bytes, void** out);
int vlr_host_free(vlr_ctx* ctx, void* p);
/* Per-kernel timing with CUDA events on the context stream: enable/disable,
 * and read the accumulated milliseconds and launch count of one kernel
 * (reading resets nothing; vlr_ctx_profile(ctx, 1) clears the totals).
 * No counterpart in the reference. */
int vlr_ctx_profile(vlr_ctx* ctx, int enable);
int vlr_ctx_profile_read(vlr_ctx* ctx, const char* kernel, double* total_ms, long long* launches);
/* Bound of every device-side wait of the context's kernels (the look-back
 * scan of a level-set step, the TMA staging barrier), in polls; 0 restores
 * each wait's default (about half a second).  A wait that reaches its bound
 * sets VLR_ERR_TIMEOUT for the operation and the rest of that step is
 * abandoned.  Takes effect for work enqueued afterwards.  No counterpart in
 * the reference (its code is serial). */
int vlr_ctx_set_wait_limit(vlr_ctx* ctx, uint32_t polls);
/* Test hook for the timeout path: while `on` is non-zero, the first chunk of
 * every level-set step's look-back scan withholds its prefix, so the waits
 * of the later chunks run out (VLR_ERR_TIMEOUT once the bound is reached)
 * instead of completing.  Off by default; it makes no GPU fault or hang, only
 * a bounded wait that gives up.  No counterpart in the reference. */
int vlr_ctx_test_stall(vlr_ctx* ctx, int on);

/* ---- grids (reference semantics: f32 values in world units) ------------ */

/* Upload a Grid<f32>: replaces NanoGrid::from_grid + upload (src/nano/layout.rs:89-170).
 * Leaves must have distinct, 8-aligned origins; any order is accepted.
 * Grids hold leaves only: a tree with tiles (made only by RootNode::prune,
 * src/tree/internal.rs:253-299) passes each active tile as a leaf record
 * with all 512 bits set and the tile's value in every voxel, which reads and
 * iterates as the tile does (src/tree/internal.rs:118-124, 319-349). */
int vlr_grid_create(vlr_ctx* ctx, const vlr_transform* xf, float background, const int32_t* origins,
                    const uint64_t* masks, const float* values, size_t n_leaves, vlr_grid** out);
/* Device-resident form of vlr_grid_create, for leaves already in this
 * context's device memory (origins i32[3], masks u64[8], values f32[512]):
 * they must be sorted by (x, y, z) with distinct 8-aligned origins, the order
 * a device grid keeps (VLR_ERR_INVALID otherwise).  Masks and values are
 * copied on the device; only the origins visit the host. */
int vlr_grid_create_device(vlr_ctx* ctx, const vlr_transform* xf, float background, const int32_t* d_origins,
                           const uint64_t* d_masks, const float* d_values, size_t n_leaves, vlr_grid** out);
/* Leaf count, active voxel count, background and transform of a grid. */
int vlr_grid_info(vlr_ctx* ctx, const vlr_grid* g, size_t* n_leaves, uint64_t* n_active, float* background,
                  vlr_transform* xf);
/* Replaces extend_velocity(&Grid<f32>, &mut vx, &mut vy, &mut vz, f32)
 * (src/tools/level_set_track.rs:115-160): band voxels of the SDF copy the
 * velocity of the nearest interface voxel (ties: first in iteration order,
 * 128^3 tiles in ascending origin order) and become active in vx, vy, vz,
 * whose missing leaves are allocated at their backgrounds. */
int vlr_extend_velocity(vlr_ctx* ctx, const vlr_grid* sdf, vlr_grid* vx, vlr_grid* vy, vlr_grid* vz,
                        float half_width);
/* Replaces the position update of advect_particles (RK4, rk4 = 1) and
 * advect_particles_euler (rk4 = 0) (src/tools/advection.rs:58-110): positions
 * (f64, 3 per particle, world units) move in place through VelocityField
 * {vx, vy, vz}; the position update alone (vlr_advect_points below is the
 * whole crate call, re-binning included). */
int vlr_advect_particles(vlr_ctx* ctx, const vlr_grid* vx, const vlr_grid* vy, const vlr_grid* vz, double* positions,
                         size_t n, double dt, int rk4);
/* A particle of the crate's PointDataGrid (Particle, src/points/point_grid.rs:
 * 9-17): world position, velocity attribute, id. */
typedef struct vlr_particle {
    double position[3];
    double velocity[3];
    uint64_t id;
} vlr_particle;
/* Replaces advect_particles(&mut PointDataGrid, &VelocityField, dt) (RK4,
 * rk4 = 1) and advect_particles_euler (rk4 = 0) (src/tools/advection.rs:58-110)
 * including their closing PointDataGrid::rebin (src/points/point_grid.rs:
 * 258-266).  `particles` holds the point grid's particles in binned order
 * (leaves in ascending (x, y, z) origin order, each leaf's particles in its
 * stored order) and is rewritten in place: positions moved, then the
 * particles re-binned into the leaf of AffineMap::world_to_index(position)
 * aligned to 8, leaves again in ascending origin order and each leaf's
 * particles in their drain order (the crate drains leaves in HashMap order;
 * ascending order makes the result deterministic).  world_to_index holds rows
 * 0..2 of the point grid's inverse 4x4 map (AffineMap::inverse).  The
 * re-binned leaves go to leaf_origins (cap_leaves x 3) and leaf_start
 * (cap_leaves + 1 entries: first particle of each leaf, then n); *n_leaves
 * is always set, and VLR_ERR_CAPACITY (particles left unchanged) reports
 * more leaves than cap_leaves (cap_leaves = n always suffices).  At most
 * 2^28 particles per call. */
int vlr_advect_points(vlr_ctx* ctx, const vlr_grid* vx, const vlr_grid* vy, const vlr_grid* vz,
                      const double world_to_index[12], vlr_particle* particles, size_t n, double dt, int rk4,
                      int32_t* leaf_origins, uint32_t* leaf_start, size_t cap_leaves, size_t* n_leaves);
/* Replaces dilate(&mut Grid<f32>, iterations) (src/tools/morphology.rs:20-35):
 * every inactive voxel with an active 6-neighbour becomes active with the
 * value of the neighbour that comes first in the tree's iteration order
 * (128^3 tiles in ascending origin order, then leaves, then voxels in ZYX
 * order); missing leaves are allocated at the background. */
int vlr_dilate(vlr_ctx* ctx, vlr_grid* g, unsigned iterations);
/* Replaces flood_fill_sign(&mut Grid<f32>) (src/tools/flood_fill.rs:18-107):
 * in every leaf with an active voxel, each inactive voxel becomes -background
 * if strictly more of its active 6-neighbours inside the leaf are negative
 * than not, +background if not, and the leaf's majority sign (negative only
 * if strictly more active values are negative) if it has none.  Enqueued on
 * the context stream. */
int vlr_flood_fill_sign(vlr_ctx* ctx, vlr_grid* g);
/* Replaces volume_to_mesh(&Grid<f32>, isovalue) -> Mesh
 * (src/tools/volume_to_mesh.rs:46-201): marching cubes over the cells of every
 * leaf tile and its 6 face neighbours.  Vertices (x, y, z doubles, world
 * units) come in the reference's order and with its values: vertex i is the
 * i-th edge crossing first met in the reference's visit order (tiles in
 * ascending origin, cells x-major), interpolated from that cell's first edge
 * endpoint.  Triangles (3 vertex indices) follow per cell in visit order from
 * the crate's own triangle table (src/tools/volume_to_mesh.rs:246-503, returned
 * by vlr_mc_triangle_table), so both lists equal the crate's.  *n_vertices
 * and *n_triangles are always set; up to cap_vertices vertices and
 * cap_triangles triangles are copied (pass null buffers to count only).  World-unit f32 grids only. */
int vlr_volume_to_mesh(vlr_ctx* ctx, const vlr_grid* g, float isovalue, double* vertices, size_t cap_vertices,
                       uint32_t* triangles, size_t cap_triangles, size_t* n_vertices, size_t* n_triangles);
/* The triangulation table used by vlr_volume_to_mesh: 256 cases (bit i set:
 * corner i below the isovalue) x 16 edge indices, three per triangle, -1
 * padded: the crate's TRI_TABLE (src/tools/volume_to_mesh.rs:246-503).
 * Host-only; the reference keeps it as a private constant. */
int vlr_mc_triangle_table(int8_t* out);

/* ---- serialised formats ------------------------------------------------
 * .vol byte image (src/io/vol_format.rs:1-160) <-> device grid.  Replaces
 * read_vol (:85-150): validates magic, version, grid class and length
 * (VLR_ERR_FORMAT), keeps the last record of a repeated leaf, builds
 * Grid::new(background, voxel_size) semantics (uniform transform); the leaf
 * block crosses to the device in one copy.  *grid_class receives the class. */
int vlr_grid_from_vol(vlr_ctx* ctx, const void* bytes, size_t n_bytes, vlr_grid** out, int* grid_class);
/* Replaces write_vol (src/io/vol_format.rs:53-83); leaves in (x, y, z) order
 * of origin.  grid_class -1 writes the grid's own class.  out = NULL queries
 * *n_bytes only. */
int vlr_grid_to_vol(vlr_ctx* ctx, const vlr_grid* g, int grid_class, void* out, size_t cap, size_t* n_bytes);
/* NanoGrid byte image (src/nano/layout.rs:13-286) <-> device grid.  Replaces
 * NanoGrid::from_bytes (:208-252) + to_grid (:255-286): validates magic,
 * version, length and strictly sorted leaves (VLR_ERR_FORMAT), keeps active
 * voxels only (leaves without active voxels dropped, inactive voxels =
 * background), with_affine transform from the header's forward matrix. */
int vlr_grid_from_nano(vlr_ctx* ctx, const void* bytes, size_t n_bytes, vlr_grid** out, int* grid_class);
/* Replaces NanoGrid::from_grid (:89-170): header with the active bounding
 * box and the forward/inverse matrices, leaves sorted by origin with all 512
 * values.  affine_inv (rows 0..2 of the inverse 4x4) may be NULL: the inverse
 * the grid was read with, else 1 / voxel size on the diagonal. */
int vlr_grid_to_nano(vlr_ctx* ctx, const vlr_grid* g, int grid_class, const double* affine_inv, void* out,
                     size_t cap, size_t* n_bytes);

/* Copy a grid back into caller buffers sized for at least vlr_grid_info's leaf
 * count, sorted (x, y, z) like NanoGrid (src/nano/layout.rs:81-106). */
int vlr_grid_download(vlr_ctx* ctx, const vlr_grid* g, int32_t* origins, uint64_t* masks, float* values,
                      size_t cap_leaves);
void vlr_grid_destroy(vlr_grid* g);

/* make_level_set_sphere (src/tools/sphere.rs:17-59), generated on the device. */
int vlr_make_level_set_sphere(vlr_ctx* ctx, double radius, const double center[3], double voxel_size,
                              double half_width, vlr_grid** out);

/* sample_trilinear (src/tools/interpolation.rs:11-48) at n world positions (host arrays). */
int vlr_sample_trilinear(vlr_ctx* ctx, const vlr_grid* g, const double* world_xyz, size_t n, float* out);

/* advect_level_set (src/tools/advection.rs:32-56): VelocityField{vx, vy, vz}
 * (src/tools/advection.rs:10-24) as three grids.  Writes a new grid. */
int vlr_advect_level_set(vlr_ctx* ctx, const vlr_grid* g, const vlr_grid* vx, const vlr_grid* vy,
                         const vlr_grid* vz, double dt, vlr_grid** out);

/* find_zero_crossings (src/tools/level_set_track.rs:14-47): writes the first
 * cap coordinates (int32[3] each) of the crossing list sorted (x, y, z), and
 * the total count.  A cap of the grid's active voxel count holds them all. */
int vlr_find_zero_crossings(vlr_ctx* ctx, const vlr_grid* g, int32_t* coords, size_t cap, size_t* count);

/* trim_narrow_band (src/tools/level_set_track.rs:53-68), in place. */
int vlr_trim_narrow_band(vlr_ctx* ctx, vlr_grid* g, float half_width);

/* rebuild_narrow_band (src/tools/level_set_track.rs:80-114), in place. */
int vlr_rebuild_narrow_band(vlr_ctx* ctx, vlr_grid* g, float half_width);

/* find_zero_crossings for callers that cannot allocate device memory (code
 * inside a stream capture, real-time loops, hosts whose device memory belongs
 * to another allocator).  No counterpart in the reference: it is an
 * allocation-free variant of vlr_find_zero_crossings.  It enqueues its kernels
 * on the context stream and returns without waiting; results are valid once
 * that stream has been synchronised.  d_coords (int32[cap][3]) and d_count are
 * caller-owned DEVICE buffers; crossings come in the grid's leaf order, ZYX
 * within a leaf (not sorted), *d_count receives the total even when it
 * exceeds cap.  Scratch is a fixed 4.5 MiB device array shared by all calls
 * on a device: grids over 65,536 leaves are rejected (VLR_ERR_CAPACITY); the
 * first call on a device resolves the array's address and should come before
 * any stream capture; calls that overlap on the GPU race on the array. */
int vlr_find_zero_crossings_noalloc(vlr_ctx* ctx, const vlr_grid* g, int32_t* d_coords, size_t cap,
                                    unsigned long long* d_count);

/* Host-buffer convenience: one step of the reference pipeline, advect_level_set
 * then rebuild_narrow_band, from and to flat host arrays.  Upload, kernels and
 * download run on the context stream.  out_* buffers hold cap_leaves leaves;
 * *out_n receives the leaf count (VLR_ERR_CAPACITY if it exceeds cap_leaves). */
int vlr_advect_rebuild_host(vlr_ctx* ctx, const vlr_transform* xf, float background, const int32_t* origins,
                            const uint64_t* masks, const float* values, size_t n_leaves, const float velocity[3],
                            double dt, float half_width, int32_t* out_origins, uint64_t* out_masks,
                            float* out_values, size_t cap_leaves, size_t* out_n);

/* ---- narrow-band method (no counterpart in the reference) --------------
 *
 * The reference's step (advect_level_set + rebuild_narrow_band) never moves
 * the active set, so its band is lost within a few steps of motion.  The
 * method grid below is a full narrow-band level-set step:
 * semi-Lagrangian backtrace (Euler, RK2 midpoint or SSP-RK3) through an
 * analytic velocity, two Godunov-upwind reinitialisation iterations, and
 * dilation-based re-tracking of the band, with values stored in voxel units
 * as f32 or f16 and arithmetic in f32.  A method grid holds one or more
 * independent grids (a batch) in one leaf pool; each step is one CUDA-graph
 * replay. */
typedef struct vlr_level_set vlr_level_set;

enum { VLR_PREC_F32 = 0, VLR_PREC_F16 = 1 };
enum { VLR_VEL_CONSTANT = 0, VLR_VEL_VORTEX = 1, VLR_VEL_CURL = 2 };

/* Analytic velocity of one grid.  Index space is voxels; world = w0 + voxel_size * index. */
typedef struct vlr_velocity_desc {
    int kind;
    double constant[3];            /* CONSTANT: voxels per unit time */
    double voxel_size;             /* VORTEX: deformation field on the unit cube (world units) */
    double w0[3];
    double period;                 /* VORTEX: T in cos(pi t / T) */
    int octaves;                   /* CURL: v = sum_o grad f_o x e_o, voxels per unit time, */
    double amp[4];                 /*   f_o = amp_o prod_a sin(wavenumber_o * p_a + phase_o[a]) */
    double wavenumber[4];
    double phase[4][3];
    double dir[4][3];
    int32_t domain_lo[3];          /* index box in which the field may be sampled; lo > hi: the */
    int32_t domain_hi[3];          /*   unit cube + 16 voxels (VORTEX), initial box +- 256 (others) */
} vlr_velocity_desc;

typedef struct vlr_method_desc {
    int precision;                 /* VLR_PREC_F32 or VLR_PREC_F16 */
    float half_width;              /* band half width, voxels */
    int integrator;                /* 1 Euler, 2 RK2 midpoint, 3 SSP-RK3 */
    int reinit_iters;              /* 0, 1 or 2 Godunov iterations per step */
    double dt;                     /* time step */
    double t0;                     /* time of the initial state */
    size_t capacity;               /* leaf slots; 0 = 2 x initial + 4096 */
    int reinit_mode;               /* 0: plain Godunov (default); 1: Godunov with the
                                      Russo-Smereka subcell fix at cut voxels (keeps
                                      the interface in place, but its sign test makes
                                      long runs sensitive to rounding) */
} vlr_method_desc;

/* Sphere of `radius` (world units) at `center` (world), voxel size vs, world = w0 + vs * index. */
int vlr_ls_create_sphere(vlr_ctx* ctx, const vlr_method_desc* m, const vlr_velocity_desc* vel, double radius,
                         const double center[3], double voxel_size, const double w0[3], vlr_level_set** out);
/* From leaves in voxel units (inactive values must hold +-half_width and every
 * voxel within one voxel of an active one must lie in a given leaf). */
int vlr_ls_create_from_leaves(vlr_ctx* ctx, const vlr_method_desc* m, const vlr_velocity_desc* vel,
                              const int32_t* origins, const uint64_t* masks, const float* phi, size_t n_leaves,
                              vlr_level_set** out);
/* A sphere in index units (voxels) of one grid of a batch. */
typedef struct vlr_sphere {
    double center[3];
    double radius;
} vlr_sphere;

/* One grid of a batch: the union of its spheres (SDF = min over spheres of
 * |p - c| - r, in voxels) and its own velocity. */
typedef struct vlr_batch_grid {
    const vlr_sphere* spheres;
    int n_spheres;
    vlr_velocity_desc velocity;
} vlr_batch_grid;

/* Many independent grids in one leaf pool: every kernel of a step processes
 * all leaves of all grids in one persistent launch.  Voxel size 1, world =
 * index.  n_grids <= 512 when n_grids > 1 (each grid spans < 2^21 voxels per
 * axis); a single grid may span 2^24 voxels per axis. */
int vlr_ls_create_spheres(vlr_ctx* ctx, const vlr_method_desc* m, const vlr_batch_grid* grids, int n_grids,
                          vlr_level_set** out);
/* Leaves of one grid of a batch (sorted (x, y, z)); pass grid = -1 for all
 * leaves (sorted by grid then (x, y, z)) with grid_ids receiving each leaf's grid. */
int vlr_ls_download_grid(vlr_ctx* ctx, const vlr_level_set* ls, int grid, int32_t* grid_ids, int32_t* origins,
                         uint64_t* masks, float* phi, size_t cap_leaves, size_t* n_out);

/* Advance n_steps steps (each one graph replay on the context stream) and
 * wait for them; device-side errors are reported here.  The first step of a
 * level set also chooses the launch shapes of its two stencil kernels (see
 * vlr_ls_set_launch_shape): it launches each kernel at every candidate shape
 * on the same inputs, times them and keeps the fastest, which synchronises
 * the stream; its result is that of an ordinary step. */
int vlr_ls_step(vlr_ctx* ctx, vlr_level_set* ls, int n_steps);
/* Enqueue n_steps steps on the context stream and return without waiting
 * (apart from the first step's launch tuning); vlr_ctx_check() later waits and
 * reports device-side errors. */
int vlr_ls_enqueue(vlr_ctx* ctx, vlr_level_set* ls, int n_steps);
/* Launch shapes of the advect and reinitialisation kernels: threads per CTA
 * (128 only), persistent CTAs (> 0) and the staging of the halo tiles (0 only:
 * cp.async row copies by every thread, double-buffered; other values are
 * rejected with VLR_ERR_INVALID).  Fixing them turns the first-step autotuning
 * off; advect_threads = 0 turns it back on for the next step.  Results never
 * depend on the shape.  No counterpart in the reference (its step is serial
 * Rust). */
int vlr_ls_set_launch_shape(vlr_ctx* ctx, vlr_level_set* ls, int advect_threads, int advect_ctas, int advect_staging,
                            int reinit_threads, int reinit_ctas, int reinit_staging);
/* shape[0..5] = advect threads, CTAs, staging, reinit threads, CTAs, staging
 * (0 before the first step); *n_timed = candidates the autotuner timed, and if
 * `log` is non-null, up to cap_log rows of (kernel 0/1, threads, CTAs,
 * staging, microseconds) for them. */
int vlr_ls_get_launch_shape(vlr_ctx* ctx, const vlr_level_set* ls, int shape[6], int* n_timed, float* log,
                            int cap_log);
int vlr_ctx_check(vlr_ctx* ctx);
int vlr_ls_info(vlr_ctx* ctx, const vlr_level_set* ls, size_t* n_leaves, uint64_t* n_active, double* time);
/* Replace the state of a single-grid level set with host leaves (same layout
 * and invariants as vlr_ls_create_from_leaves), keeping its time, velocity
 * and allocations: the host-resident form of a step is upload, step, download. */
int vlr_ls_upload(vlr_ctx* ctx, vlr_level_set* ls, const int32_t* origins, const uint64_t* masks, const float* phi,
                  size_t n_leaves);
/* Set the step counter of a level set (its time is t0 + step * dt, computed in
 * f32 by the kernels).  A run continued in a new level set (one with a larger
 * capacity, say) and created with the same t0 resumes at the same time, bit for
 * bit, once its counter is set to the old one's.  step >= 0. */
int vlr_ls_set_step(vlr_ctx* ctx, vlr_level_set* ls, int step);
/* The terms of vlr_ls_volume before their sum: one FP64 partial per
 * allocated leaf, in the level set's list order (the order of
 * vlr_ls_download_device, and after an upload the upload's order), into the
 * device buffer d_partials of cap entries; *n_out = leaves.  A grid divided
 * over GPUs sums the partials of the leaves each rank owns. */
int vlr_ls_volume_partials(vlr_ctx* ctx, vlr_level_set* ls, const double ref[3], double* d_partials, size_t cap,
                           size_t* n_out);
/* Device-resident forms of vlr_ls_upload and vlr_ls_download, for callers
 * that keep leaves in device memory on the context's device (the exchange of a
 * grid divided over GPUs).  Records as in vlr_ls_upload: origins i32[3] on the
 * 8-voxel lattice, masks u64[8], values f32[512] in voxel units.  The upload
 * replaces the state and keeps the time; the download writes the allocated
 * leaves in the level set's list order (unsorted) and sets *n_out, failing
 * with VLR_ERR_CAPACITY above cap_leaves.  Both return after their work. */
int vlr_ls_upload_device(vlr_ctx* ctx, vlr_level_set* ls, const int32_t* d_origins, const uint64_t* d_masks,
                         const float* d_phi, size_t n_leaves);
int vlr_ls_download_device(vlr_ctx* ctx, const vlr_level_set* ls, int32_t* d_origins, uint64_t* d_masks,
                           float* d_phi, size_t cap_leaves, size_t* n_out);
/* In-place edits of a single-grid level set's pool, for a grid divided over
 * GPUs whose ranks keep their owned leaves resident.  Values travel in the
 * pool's own type: f16[512] for an FP16 level set, f32[512] otherwise.
 * vlr_ls_gather_device copies the leaves at list positions d_pos[0..n) (or
 * the first n when d_pos is null) into device buffers: origins i32[3], and
 * masks and values where those pointers are non-null; a position outside
 * the list fails with VLR_ERR_INVALID.
 * vlr_ls_edit_device drops the listed leaves whose d_drop byte (one per list
 * position, n_list = the current leaf count) is non-zero, keeps the others in
 * their order, appends n_add leaves (origins on the 8-voxel lattice, masks,
 * values) and rebuilds the index.  No room for them fails with
 * VLR_ERR_CAPACITY before anything changes; an added leaf off the lattice,
 * outside the hashable range or already listed fails with a device error
 * that leaves the state undefined until the next upload.  Both return after
 * their work. */
int vlr_ls_gather_device(vlr_ctx* ctx, const vlr_level_set* ls, const int32_t* d_pos, size_t n,
                         int32_t* d_origins, uint64_t* d_masks, void* d_phi);
int vlr_ls_edit_device(vlr_ctx* ctx, vlr_level_set* ls, const uint8_t* d_drop, size_t n_list,
                       const int32_t* d_origins, const uint64_t* d_masks, const void* d_phi, size_t n_add);
/* The host-resident form of n_steps steps in one call: replace the state with
 * host leaves (as vlr_ls_upload), step, and write the result (as
 * vlr_ls_download) into caller buffers of cap_leaves leaves; *n_out = leaves
 * written.  The copies of the first min(n_leaves, cap_leaves) records start
 * before the leaf count is known, so records past *n_out (up to that bound)
 * may be overwritten; the call then waits once for the count, the device
 * errors and those copies, and copies any records beyond them.
 * One step of a large single-grid state (at least 2^18 leaves by default)
 * whose host leaves are sorted by x and whose six host buffers are pinned
 * runs as a pipeline over slabs of consecutive x instead: each slab steps its
 * leaves with the input leaves within 16 voxels beside it and keeps the
 * outputs in its own x range, which are bit for bit the one-pass step's; its
 * input goes up and its outputs, sorted (x, y, z), go down on copy streams
 * while other slabs step, so the two copy directions overlap.  The result and
 * the level set's state afterwards are those of the one-pass call, and no
 * record past *n_out is written; an error (the output buffers or the pool
 * too small, a device error) leaves the state undefined until the next
 * upload.  vlr_ls_set_host_slabs sets the slab count: 0 automatic (one slab
 * per 2^17 leaves, at most 16), 1 always one pass, k >= 2 at most k slabs
 * (fewer when the leaves have fewer distinct x).  No counterpart in the
 * reference (its step is serial Rust). */
int vlr_ls_set_host_slabs(vlr_ctx* ctx, vlr_level_set* ls, int slabs);
int vlr_ls_step_host(vlr_ctx* ctx, vlr_level_set* ls, const int32_t* origins, const uint64_t* masks, const float* phi,
                     size_t n_leaves, int n_steps, int32_t* out_origins, uint64_t* out_masks, float* out_phi,
                     size_t cap_leaves, size_t* n_out);
/* Allocated leaves (sorted (x, y, z)), masks, values in voxel units as f32. */
int vlr_ls_download(vlr_ctx* ctx, const vlr_level_set* ls, int32_t* origins, uint64_t* masks, float* phi,
                    size_t cap_leaves);
/* Enclosed volume in voxel units^3 (FP64 smeared-delta surface integral
 * V = 1/3 sum delta(phi) (p - ref) . grad phi, eps = 1.5 voxels). */
int vlr_ls_volume(vlr_ctx* ctx, vlr_level_set* ls, const double ref[3], double* volume);
void vlr_ls_destroy(vlr_level_set* ls);

/* ---- differentiable advection (no counterpart in the reference) ---------
 *
 * Frozen-band semi-Lagrangian advection phi_{k+1}(x) = trilinear(phi_k)(x -
 * dt cos(pi t_{k+1} / T) u(x)) over the active voxels of the given leaves
 * (values in voxel units, inactive values +-half_width), with u the trilinear
 * upsample of a staggered field V: 3 components of n^3 cells of `stag_cell`
 * voxels, component a on the faces normal to axis a, index ((i*n)+j)*n+k.
 * forward/backward follow the autograd-Function contract: forward(phi_0, V)
 * -> phi_K, backward(dL/dphi_K) -> (dL/dphi_0, dL/dV).  The backward pass
 * recomputes states from checkpoints taken every `checkpoint_every` steps and
 * scatters trilinear weights by stable radix sort + segmented sum (no float
 * atomics; deterministic).  Band arrays follow vlr_adj_band's order. */
typedef struct vlr_adjoint vlr_adjoint;

int vlr_adj_create(vlr_ctx* ctx, const int32_t* origins, const uint64_t* masks, const float* phi, size_t n_leaves,
                   float half_width, const float* vel, int n_stag, double stag_cell, double dt, double period,
                   double t0, int steps, int checkpoint_every, vlr_adjoint** out);
/* The frozen-band adjoint of a single-grid level set's own step: phi_0 is
 * the level set's current state (band = its active voxels, values in voxel
 * units) and each band voxel moves by the level set's backtrace displacement
 * over one step (its integrator, dt and velocity, computed by the same device
 * code as its advect kernel), so phi_{k+1}(x) = trilinear(phi_k)(x + d(x)).
 * The velocity must be time-independent (constant or curl noise; the vortex
 * is refused with VLR_ERR_UNSUPPORTED); there is no velocity input or
 * gradient (vlr_adj_set_inputs with vel and grad_vel outputs are refused).
 * Everything is built on the device.  No counterpart in the reference. */
int vlr_adj_create_level_set(vlr_ctx* ctx, vlr_level_set* ls, int steps, int checkpoint_every, vlr_adjoint** out);
/* The per-band-voxel displacement d of a level-set adjoint (float[n_band][3],
 * voxels). */
int vlr_adj_displacement(vlr_ctx* ctx, const vlr_adjoint* a, float* out);
/* phi_0 translated by (sx, sy, sz) voxels (each within +-8), read on the band:
 * d_out[b] = phi_0(x_b - s), device buffer of n_band floats, enqueued on the
 * context stream (the target of an L2 loss against a translated copy). */
int vlr_adj_shifted_phi0(vlr_ctx* ctx, const vlr_adjoint* a, int sx, int sy, int sz, float* d_out);
/* The kernel of the backward pass's lambda transpose: 0 (default) the quad
 * gather for bands under 2^20 voxels at a reach of one voxel per step, the
 * windowed gather otherwise; 1 always the windowed gather; 2 always the quad
 * gather (reach 1 only, VLR_ERR_INVALID otherwise).  Both sum each voxel's
 * terms in a fixed order but associate them differently, so a grid divided
 * over ranks pins one kernel to reproduce the undivided sums bit for bit. */
int vlr_adj_set_gather(vlr_ctx* ctx, vlr_adjoint* a, int mode);
/* Band voxel coordinates (int32[n][3]); coords may be null to query n. */
int vlr_adj_band(vlr_ctx* ctx, const vlr_adjoint* a, int32_t* coords, size_t cap, size_t* n);
/* Replace phi_0 on the band and/or the staggered field (either may be null). */
int vlr_adj_set_inputs(vlr_ctx* ctx, vlr_adjoint* a, const float* phi0_band, const float* vel);
int vlr_adj_forward(vlr_ctx* ctx, vlr_adjoint* a, float* phi_k_band);
int vlr_adj_backward(vlr_ctx* ctx, vlr_adjoint* a, const float* grad_phik_band, float* grad_phi0_band,
                     float* grad_vel);
/* Device-resident forms for GPU training loops: the same passes with device
 * buffers (band arrays of n_band floats, grad_vel of 3 n^3), enqueued on the
 * context stream without waiting; vlr_ctx_check() waits and reports
 * device-side errors.  Output pointers may be null to skip that output. */
int vlr_adj_forward_device(vlr_ctx* ctx, vlr_adjoint* a, float* d_phi_k_band);
int vlr_adj_backward_device(vlr_ctx* ctx, vlr_adjoint* a, const float* d_grad_phik_band, float* d_grad_phi0_band,
                            float* d_grad_vel);
void vlr_adj_destroy(vlr_adjoint* a);

#ifdef __cplusplus
}
#endif
#endif /* VOLRUS_B200_H */
