// Host entry points of the reference-semantics kernels (ref_ops.cu).
#pragma once
#include <vector>

#include "vlr_host.hpp"

namespace vlr {

GridView make_view(const vlr_grid* g);
int advect_ref(vlr_ctx* ctx, const vlr_grid* g, const vlr_grid* vx, const vlr_grid* vy, const vlr_grid* vz, double dt,
               vlr_grid* out);
int sample_points(vlr_ctx* ctx, const vlr_grid* g, const double* h_pts, size_t n, float* h_out);
// The crossings in (x, y, z) order when *sorted comes back true (sorted on the
// device); in emission order (leaf by leaf) when it is false or null.
int find_zero_crossings(vlr_ctx* ctx, const vlr_grid* g, int32_t* h_coords, size_t cap, size_t* count,
                        bool* sorted = nullptr);
int trim_narrow_band(vlr_ctx* ctx, vlr_grid* g, float half_width);
int rebuild_narrow_band(vlr_ctx* ctx, vlr_grid* g, float half_width);
int make_sphere(vlr_ctx* ctx, double radius, const double c[3], double vs, double hw, vlr_grid* out);
// Marching-cubes isosurface (mesh.cu): counts always; copies up to the capacities.
int volume_to_mesh(vlr_ctx* ctx, const vlr_grid* g, float iso, double* h_verts, size_t cap_v, uint32_t* h_tris,
                   size_t cap_t, size_t* n_verts, size_t* n_tris);
// The derived marching-cubes triangle table, 256 x 16 entries (-1 padded).
int mc_triangle_table(int8_t* out);
// Add inactive background leaves at `origins` (3 ints each) to a world-unit grid (morphology.cu).
int grid_add_leaves(vlr_ctx* ctx, vlr_grid* g, const std::vector<int32_t>& origins);

}  // namespace vlr
