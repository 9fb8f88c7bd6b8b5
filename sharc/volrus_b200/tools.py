"""GPU implementations of the Sharc.Volrus advection-path tools.

Each function keeps the name, arguments and semantics of the reference tool
it replaces and runs on the B200 through the C ABI:

    advect_level_set(grid, velocity, dt) -> Grid     src/tools/advection.rs:32-56
    VelocityField(vx, vy, vz)                        src/tools/advection.rs:10-24
    sample_trilinear(grid, world_pos) -> float       src/tools/interpolation.rs:11-48
    find_zero_crossings(grid) -> list[Coord]         src/tools/level_set_track.rs:14-47
    trim_narrow_band(grid, half_width)               src/tools/level_set_track.rs:53-68
    rebuild_narrow_band(grid, half_width)            src/tools/level_set_track.rs:80-114
    make_level_set_sphere(r, c, vs, hw) -> Grid      src/tools/sphere.rs:17-59
    dilate(grid, iterations)                         src/tools/morphology.rs:20-35
    extend_velocity(sdf, vx, vy, vz, half_width)     src/tools/level_set_track.rs:115-160
    advect_particles(positions, velocity, dt)        src/tools/advection.rs:58-95 (positions only)
    advect_particles_euler(positions, velocity, dt)  src/tools/advection.rs:97-110 (positions only)

Host ``Grid`` arguments are uploaded, processed and downloaded per call (the
drop-in form); ``DeviceGrid`` arguments stay resident in HBM between calls.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from . import _lib
from ._lib import Context, ptr
from .grid import AffineMap, Grid, GridClass, VoxelTransform


class DeviceGrid:
    """A world-unit f32 grid resident on the GPU (opaque ``vlr_grid*``)."""

    def __init__(self, ctx: Context, handle: C.c_void_p, name: str = "", grid_class=GridClass.UNKNOWN):
        self.ctx = ctx
        self.handle = handle
        self.name = name
        self.grid_class = grid_class

    @classmethod
    def upload(cls, grid: Grid, ctx: Context | None = None) -> "DeviceGrid":
        ctx = ctx or Context.default()
        o, m, v = grid.to_arrays()
        h = C.c_void_p()
        t = grid.c_transform()
        ctx.check(ctx.lib.vlr_grid_create(ctx.handle, C.byref(t), C.c_float(grid.background), ptr(o, C.c_int32),
                                          ptr(m, C.c_uint64), ptr(v, C.c_float), len(o), C.byref(h)),
                  "vlr_grid_create")
        return cls(ctx, h, grid.name, grid.grid_class)

    @classmethod
    def from_device(cls, d_origins: int, d_masks: int, d_values: int, n: int, background: float,
                    voxel_size: float = 1.0, ctx: Context | None = None) -> "DeviceGrid":
        """A grid from n leaves in device memory (pointers: i32[3] origins, u64[8]
        masks, f32[512] world-unit values), sorted by (x, y, z), with the
        transform of a voxel size and zero origin."""
        ctx = ctx or Context.default()
        t = Grid(background, voxel_size).c_transform()
        h = C.c_void_p()
        ctx.check(ctx.lib.vlr_grid_create_device(ctx.handle, C.byref(t), C.c_float(background), C.c_void_p(d_origins),
                                                 C.c_void_p(d_masks), C.c_void_p(d_values), int(n), C.byref(h)),
                  "vlr_grid_create_device")
        return cls(ctx, h)

    def info(self):
        n = C.c_size_t()
        a = C.c_uint64()
        bg = C.c_float()
        t = _lib.vlr_transform()
        self.ctx.check(self.ctx.lib.vlr_grid_info(self.ctx.handle, self.handle, C.byref(n), C.byref(a), C.byref(bg),
                                                  C.byref(t)), "vlr_grid_info")
        return n.value, a.value, bg.value, t

    def leaf_count(self) -> int:
        return self.info()[0]

    def active_voxel_count(self) -> int:
        return self.info()[1]

    def download(self) -> Grid:
        n, _, bg, t = self.info()
        o = np.zeros((n, 3), np.int32)
        m = np.zeros((n, 8), np.uint64)
        v = np.zeros((n, 512), np.float32)
        self.ctx.check(self.ctx.lib.vlr_grid_download(self.ctx.handle, self.handle, ptr(o, C.c_int32),
                                                      ptr(m, C.c_uint64), ptr(v, C.c_float), n),
                       "vlr_grid_download")
        vt = VoxelTransform(t.voxel_size, tuple(t.origin))
        am = AffineMap(np.array(list(t.affine), np.float64).reshape(3, 4), t.affine_voxel_size)
        g = Grid.from_arrays(o, m, v, bg, vt, am)
        g.name = self.name
        g.grid_class = self.grid_class
        return g

    def close(self):
        if self.handle:
            self.ctx.lib.vlr_grid_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


@dataclass
class VelocityField:
    """``VelocityField{vx, vy, vz}`` (src/tools/advection.rs:10-14)."""
    vx: Grid
    vy: Grid
    vz: Grid


def _as_device(g, ctx):
    if isinstance(g, DeviceGrid):
        return g, False
    return DeviceGrid.upload(g, ctx), True


def _replace(host: Grid, new: Grid):
    host._o, host._m, host._v, host._n, host._index = new._o, new._m, new._v, new._n, new._index


def advect_level_set(grid, velocity: VelocityField, dt: float, ctx: Context | None = None):
    """Semi-Lagrangian advection (src/tools/advection.rs:32-56) on the GPU."""
    ctx = ctx or (grid.ctx if isinstance(grid, DeviceGrid) else Context.default())
    g, _ = _as_device(grid, ctx)
    vs = [_as_device(c, ctx)[0] for c in (velocity.vx, velocity.vy, velocity.vz)]
    h = C.c_void_p()
    ctx.check(ctx.lib.vlr_advect_level_set(ctx.handle, g.handle, vs[0].handle, vs[1].handle, vs[2].handle,
                                           C.c_double(dt), C.byref(h)), "vlr_advect_level_set")
    out = DeviceGrid(ctx, h, g.name, g.grid_class)
    if isinstance(grid, DeviceGrid):
        return out
    return out.download()


def sample_trilinear(grid, world_pos, ctx: Context | None = None):
    """``sample_trilinear`` (src/tools/interpolation.rs:11-48).  ``world_pos`` is
    one [x, y, z] or an (n, 3) array; returns a float or an f32 array."""
    ctx = ctx or (grid.ctx if isinstance(grid, DeviceGrid) else Context.default())
    g, _ = _as_device(grid, ctx)
    p = np.ascontiguousarray(world_pos, np.float64)
    single = p.ndim == 1
    p = p.reshape(-1, 3)
    out = np.zeros(len(p), np.float32)
    ctx.check(ctx.lib.vlr_sample_trilinear(ctx.handle, g.handle, ptr(p, C.c_double), len(p), ptr(out, C.c_float)),
              "vlr_sample_trilinear")
    return float(out[0]) if single else out


def find_zero_crossings(grid, ctx: Context | None = None) -> np.ndarray:
    """``find_zero_crossings`` (src/tools/level_set_track.rs:14-47); (n, 3) int32 sorted (x, y, z)."""
    ctx = ctx or (grid.ctx if isinstance(grid, DeviceGrid) else Context.default())
    g, _ = _as_device(grid, ctx)
    cnt = C.c_size_t()
    # a crossing is an active voxel: one call with room for all of them
    cap = g.active_voxel_count()
    out = np.empty((max(cap, 1), 3), np.int32)
    ctx.check(ctx.lib.vlr_find_zero_crossings(ctx.handle, g.handle, ptr(out, C.c_int32), cap, C.byref(cnt)),
              "vlr_find_zero_crossings")
    return out[: cnt.value].copy()


def trim_narrow_band(grid, half_width: float, ctx: Context | None = None):
    """``trim_narrow_band`` (src/tools/level_set_track.rs:53-68), in place."""
    ctx = ctx or (grid.ctx if isinstance(grid, DeviceGrid) else Context.default())
    g, uploaded = _as_device(grid, ctx)
    ctx.check(ctx.lib.vlr_trim_narrow_band(ctx.handle, g.handle, C.c_float(half_width)), "vlr_trim_narrow_band")
    if uploaded:
        _replace(grid, g.download())


def rebuild_narrow_band(grid, half_width: float, ctx: Context | None = None):
    """``rebuild_narrow_band`` (src/tools/level_set_track.rs:80-114), in place."""
    ctx = ctx or (grid.ctx if isinstance(grid, DeviceGrid) else Context.default())
    g, uploaded = _as_device(grid, ctx)
    ctx.check(ctx.lib.vlr_rebuild_narrow_band(ctx.handle, g.handle, C.c_float(half_width)),
              "vlr_rebuild_narrow_band")
    if uploaded:
        _replace(grid, g.download())


def extend_velocity(sdf, vx, vy, vz, half_width: float, ctx: Context | None = None):
    """``extend_velocity`` (src/tools/level_set_track.rs:115-160), in place on
    vx, vy, vz (host ``Grid`` or ``DeviceGrid``)."""
    ctx = ctx or Context.default()
    made = [_as_device(g, ctx) for g in (sdf, vx, vy, vz)]
    try:
        ctx.check(ctx.lib.vlr_extend_velocity(ctx.handle, *(d.handle for d, _ in made), C.c_float(half_width)),
                  "vlr_extend_velocity")
        for (d, created), host in zip(made[1:], (vx, vy, vz)):
            if created:
                _replace(host, d.download())
    finally:
        for d, created in made:
            if created:
                d.close()


def _particles(positions, velocity: VelocityField, dt: float, rk4: bool, ctx):
    ctx = ctx or Context.default()
    p = np.ascontiguousarray(positions, np.float64).reshape(-1, 3).copy()
    made = [_as_device(g, ctx) for g in (velocity.vx, velocity.vy, velocity.vz)]
    try:
        ctx.check(ctx.lib.vlr_advect_particles(ctx.handle, made[0][0].handle, made[1][0].handle, made[2][0].handle,
                                               ptr(p, C.c_double), len(p), float(dt), 1 if rk4 else 0),
                  "vlr_advect_particles")
    finally:
        for d, created in made:
            if created:
                d.close()
    return p


def _advect_points(points, velocity: VelocityField, dt: float, rk4: bool, ctx):
    """advect_particles on a PointDataGrid, in place: RK4 / Euler position
    update and the closing PointDataGrid::rebin, in one C-ABI call."""
    from .points import PARTICLE
    ctx = ctx or Context.default()
    parts = np.ascontiguousarray(points.particles, PARTICLE).copy()
    n = len(parts)
    inv = points.inverse_rows()
    origins = np.zeros((max(n, 1), 3), np.int32)
    start = np.zeros(n + 1, np.uint32)
    nl = C.c_size_t()
    made = [_as_device(g, ctx) for g in (velocity.vx, velocity.vy, velocity.vz)]
    try:
        ctx.check(ctx.lib.vlr_advect_points(ctx.handle, made[0][0].handle, made[1][0].handle, made[2][0].handle,
                                            ptr(inv, C.c_double), parts.ctypes.data_as(C.c_void_p), n, float(dt),
                                            1 if rk4 else 0, ptr(origins, C.c_int32), ptr(start, C.c_uint32),
                                            max(n, 1), C.byref(nl)), "vlr_advect_points")
    finally:
        for d, created in made:
            if created:
                d.close()
    k = nl.value
    points.particles = parts
    points.leaf_origins = origins[:k].copy()
    points.leaf_start = start[:k + 1].copy()
    return points


def advect_particles(points, velocity: VelocityField, dt: float, ctx: Context | None = None):
    """``advect_particles`` (src/tools/advection.rs:58-95): RK4 through the
    velocity field.  Given a :class:`PointDataGrid` it is the crate call,
    position update then ``PointDataGrid::rebin``, in place (the grid is also
    returned); given an (n, 3) array of world positions it returns the new
    positions (the update alone)."""
    from .points import PointDataGrid
    if isinstance(points, PointDataGrid):
        return _advect_points(points, velocity, dt, True, ctx)
    return _particles(points, velocity, dt, True, ctx)


def advect_particles_euler(points, velocity: VelocityField, dt: float, ctx: Context | None = None):
    """``advect_particles_euler`` (src/tools/advection.rs:97-110), like
    :func:`advect_particles` with a forward Euler update."""
    from .points import PointDataGrid
    if isinstance(points, PointDataGrid):
        return _advect_points(points, velocity, dt, False, ctx)
    return _particles(points, velocity, dt, False, ctx)


def dilate(grid, iterations: int, ctx: Context | None = None):
    """``dilate`` (src/tools/morphology.rs:20-35), in place: inactive voxels with
    an active 6-neighbour become active with that neighbour's value (the first
    in tree iteration order, 128^3 tiles taken in ascending origin order)."""
    ctx = ctx or (grid.ctx if isinstance(grid, DeviceGrid) else Context.default())
    d, created = _as_device(grid, ctx)
    ctx.check(ctx.lib.vlr_dilate(ctx.handle, d.handle, int(iterations)), "vlr_dilate")
    if created:
        _replace(grid, d.download())
        d.close()


def flood_fill_sign(grid, ctx: Context | None = None):
    """``flood_fill_sign`` (src/tools/flood_fill.rs:18-107), in place: inactive
    voxels of each leaf take -background or +background from the signs of
    their active 6-neighbours in the leaf (the leaf's majority if none)."""
    ctx = ctx or (grid.ctx if isinstance(grid, DeviceGrid) else Context.default())
    d, created = _as_device(grid, ctx)
    ctx.check(ctx.lib.vlr_flood_fill_sign(ctx.handle, d.handle), "vlr_flood_fill_sign")
    if created:
        _replace(grid, d.download())
        d.close()


class Mesh:
    """``Mesh`` (src/tools/volume_to_mesh.rs:11-40): vertices (n, 3) f64 in
    world units and triangles (m, 3) u32 vertex indices."""

    def __init__(self, vertices: np.ndarray, triangles: np.ndarray):
        self.vertices = vertices
        self.triangles = triangles

    def tri_count(self) -> int:
        return len(self.triangles)

    def vertex_count(self) -> int:
        return len(self.vertices)

    def is_watertight(self) -> bool:
        """Every undirected edge is shared by exactly two triangles."""
        if len(self.triangles) == 0:
            return True
        t = self.triangles.astype(np.int64)
        e = np.concatenate([t[:, [0, 1]], t[:, [1, 2]], t[:, [2, 0]]])
        e.sort(axis=1)
        _, counts = np.unique(e[:, 0] * (1 << 32) + e[:, 1], return_counts=True)
        return bool(np.all(counts == 2))


def volume_to_mesh(grid, isovalue: float = 0.0, ctx: Context | None = None) -> Mesh:
    """``volume_to_mesh`` (src/tools/volume_to_mesh.rs:46-201) on the GPU:
    vertices in the reference's order with its values; triangles from this
    library's triangulation table (``mc_triangle_table``)."""
    ctx = ctx or (grid.ctx if isinstance(grid, DeviceGrid) else Context.default())
    d, created = _as_device(grid, ctx)
    try:
        nv, nt = C.c_size_t(), C.c_size_t()
        ctx.check(ctx.lib.vlr_volume_to_mesh(ctx.handle, d.handle, C.c_float(isovalue), None, 0, None, 0,
                                             C.byref(nv), C.byref(nt)), "vlr_volume_to_mesh")
        v = np.zeros((nv.value, 3), np.float64)
        t = np.zeros((nt.value, 3), np.uint32)
        if nv.value or nt.value:
            ctx.check(ctx.lib.vlr_volume_to_mesh(ctx.handle, d.handle, C.c_float(isovalue),
                                                 v.ctypes.data_as(C.POINTER(C.c_double)), nv.value,
                                                 t.ctypes.data_as(C.POINTER(C.c_uint32)), nt.value,
                                                 C.byref(nv), C.byref(nt)), "vlr_volume_to_mesh")
        return Mesh(v, t)
    finally:
        if created:
            d.close()


def mc_triangle_table() -> np.ndarray:
    """The triangulation table of ``volume_to_mesh``: (256, 16) int8, three
    edge indices per triangle, -1 padded.  Host-only (no GPU needed)."""
    from ._lib import load
    out = np.zeros((256, 16), np.int8)
    rc = load().vlr_mc_triangle_table(out.ctypes.data_as(C.POINTER(C.c_int8)))
    if rc:
        raise RuntimeError(f"vlr_mc_triangle_table failed: {rc}")
    return out


def make_level_set_sphere(radius: float, center, voxel_size: float, half_width: float, ctx: Context | None = None,
                          device: bool = False):
    """``make_level_set_sphere`` (src/tools/sphere.rs:17-59), generated on the GPU."""
    ctx = ctx or Context.default()
    c = np.ascontiguousarray(center, np.float64)
    h = C.c_void_p()
    ctx.check(ctx.lib.vlr_make_level_set_sphere(ctx.handle, C.c_double(radius), ptr(c, C.c_double),
                                                C.c_double(voxel_size), C.c_double(half_width), C.byref(h)),
              "vlr_make_level_set_sphere")
    d = DeviceGrid(ctx, h, "sdf", GridClass.LEVEL_SET)
    return d if device else d.download()


def make_uniform_velocity(voxel_size: float, vel, bbox_min=None, bbox_max=None) -> VelocityField:
    """Constant field as three grids, like the crate's test helper
    ``make_uniform_velocity`` (src/tools/advection.rs:116-134)."""
    comps = []
    for a in range(3):
        g = Grid(float(np.float32(vel[a])), voxel_size)
        for c in (bbox_min, bbox_max):
            if c is not None:
                g.set(c, vel[a])
        comps.append(g)
    return VelocityField(*comps)
