"""ORACLE — test infrastructure only.

ctypes wrapper over ``oracle/lib/libvolrus_oracle.so``, the C++ restatement of
the Sharc.Volrus advection path (``ref_tree.hpp``) and of the narrow-band
method (``method_oracle.hpp``).  Imported only by ``tests/``,
``__graft_entry__.smoke()`` and the CPU-baseline leg of ``bench.py``, always as
the checker or the timed CPU baseline, never as the product path.
"""
from __future__ import annotations

import ctypes as C
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB = HERE / "lib" / "libvolrus_oracle.so"

P = C.c_void_p
dbl_p = C.POINTER(C.c_double)
flt_p = C.POINTER(C.c_float)
i32_p = C.POINTER(C.c_int32)
u64_p = C.POINTER(C.c_uint64)
size_p = C.POINTER(C.c_size_t)

SIGS = {
    "vo_grid_new": (P, [C.c_float, C.c_double, dbl_p, dbl_p, C.c_double]),
    "vo_grid_free": (None, [P]),
    "vo_grid_put_leaves": (None, [P, i32_p, u64_p, flt_p, C.c_size_t]),
    "vo_grid_leaf_count": (C.c_size_t, [P]),
    "vo_grid_active_count": (C.c_uint64, [P]),
    "vo_grid_export": (None, [P, i32_p, u64_p, flt_p]),
    "vo_grid_meta": (None, [P, flt_p, dbl_p, dbl_p, dbl_p, dbl_p]),
    "vo_get": (C.c_float, [P, C.c_int32, C.c_int32, C.c_int32]),
    "vo_is_active": (C.c_int, [P, C.c_int32, C.c_int32, C.c_int32]),
    "vo_set": (None, [P, C.c_int32, C.c_int32, C.c_int32, C.c_float]),
    "vo_deactivate": (None, [P, C.c_int32, C.c_int32, C.c_int32]),
    "vo_make_level_set_sphere": (P, [C.c_double, dbl_p, C.c_double, C.c_double]),
    "vo_sample_trilinear": (None, [P, dbl_p, C.c_size_t, flt_p]),
    "vo_advect_level_set": (P, [P, P, P, P, C.c_double]),
    "vo_find_zero_crossings": (C.c_size_t, [P, i32_p, C.c_size_t]),
    "vo_trim_narrow_band": (None, [P, C.c_float]),
    "vo_rebuild_narrow_band": (None, [P, C.c_float, C.c_int]),
    "vo_dilate": (None, [P, C.c_uint]),
    "vo_advect_particles": (None, [P, P, P, dbl_p, C.c_size_t, C.c_double, C.c_int]),
    "vo_rebin_points": (C.c_size_t, [dbl_p, C.c_size_t, dbl_p, C.POINTER(C.c_uint32), i32_p,
                                     C.POINTER(C.c_uint32)]),
    "vo_extend_velocity": (None, [P, P, P, P, C.c_float]),
    "vo_remove_empty_leaves": (None, [P]),
    "vo_flood_fill_sign": (None, [P]),
    "vo_volume_to_mesh": (C.c_size_t, [P, C.c_float, C.POINTER(C.c_int8), dbl_p, C.c_size_t,
                                       C.POINTER(C.c_uint32), C.c_size_t, size_p]),
    "vo_time_ref_step": (None, [C.POINTER(P), P, P, P, C.c_double, C.c_float, C.c_size_t, dbl_p, dbl_p, size_p,
                                dbl_p, size_p]),
    "vm_sphere": (P, [C.c_double, dbl_p, C.c_double, dbl_p, C.c_double]),
    "vm_free": (None, [P]),
    "vm_spheres": (P, [dbl_p, C.c_int, C.c_double]),
    "va_create": (P, [i32_p, u64_p, dbl_p, C.c_size_t, C.c_double, dbl_p, C.c_int, C.c_double, C.c_double,
                      C.c_double, C.c_double, C.c_int]),
    "va_free": (None, [P]),
    "va_create_disp": (P, [i32_p, u64_p, dbl_p, C.c_size_t, C.c_double, dbl_p, C.c_int]),
    "va_nband": (C.c_int, [P]),
    "va_forward": (None, [P, dbl_p, dbl_p, dbl_p]),
    "va_backward": (None, [P, dbl_p, dbl_p, dbl_p]),
    "vm_leaf_count": (C.c_size_t, [P]),
    "vm_export": (None, [P, i32_p, u64_p, dbl_p]),
    "vm_import": (P, [i32_p, u64_p, dbl_p, C.c_size_t, C.c_double]),
    "vm_step": (C.c_int, [P, C.c_int, dbl_p, C.c_int, C.c_int, C.c_int, C.c_double, C.c_double, C.c_int]),
    "vm_velocity": (None, [C.c_int, dbl_p, dbl_p, C.c_double, dbl_p]),
    "vm_volume": (C.c_double, [P, dbl_p]),
}

_lib = None


def build():
    """Compile the oracle library (make, in this directory)."""
    subprocess.run(["make", "-s", "-C", str(HERE)], check=True)


def load():
    global _lib
    if _lib is None:
        if not LIB.exists():
            build()
        lib = C.CDLL(str(LIB))
        for name, (res, args) in SIGS.items():
            f = getattr(lib, name)
            f.restype = res
            f.argtypes = args
        _lib = lib
    return _lib


def _p(a, t):
    return a.ctypes.data_as(C.POINTER(t))


class OGrid:
    """Handle to an oracle grid (reference data structure, f32 values)."""

    def __init__(self, handle):
        self.lib = load()
        self.h = handle

    @classmethod
    def new(cls, background, voxel_size=1.0, t_origin=(0.0, 0.0, 0.0), affine=None, affine_vs=None):
        lib = load()
        to = np.asarray(t_origin, np.float64)
        if affine is None:
            affine = np.zeros((3, 4))
            affine[0, 0] = affine[1, 1] = affine[2, 2] = voxel_size
        af = np.ascontiguousarray(affine, np.float64).reshape(12)
        h = lib.vo_grid_new(C.c_float(background), voxel_size, _p(to, C.c_double), _p(af, C.c_double),
                            voxel_size if affine_vs is None else affine_vs)
        return cls(h)

    @classmethod
    def from_arrays(cls, origins, masks, values, background, voxel_size=1.0, t_origin=(0.0, 0.0, 0.0), affine=None,
                    affine_vs=None):
        g = cls.new(background, voxel_size, t_origin, affine, affine_vs)
        o = np.ascontiguousarray(origins, np.int32)
        m = np.ascontiguousarray(masks, np.uint64)
        v = np.ascontiguousarray(values, np.float32)
        g.lib.vo_grid_put_leaves(g.h, _p(o, C.c_int32), _p(m, C.c_uint64), _p(v, C.c_float), len(o))
        return g

    @classmethod
    def sphere(cls, radius, center, voxel_size, half_width):
        lib = load()
        c = np.asarray(center, np.float64)
        return cls(lib.vo_make_level_set_sphere(radius, _p(c, C.c_double), voxel_size, half_width))

    def arrays(self):
        n = self.lib.vo_grid_leaf_count(self.h)
        o = np.zeros((n, 3), np.int32)
        m = np.zeros((n, 8), np.uint64)
        v = np.zeros((n, 512), np.float32)
        if n:
            self.lib.vo_grid_export(self.h, _p(o, C.c_int32), _p(m, C.c_uint64), _p(v, C.c_float))
        return o, m, v

    def meta(self):
        bg = C.c_float()
        vs = C.c_double()
        to = np.zeros(3)
        mat = np.zeros(12)
        avs = C.c_double()
        self.lib.vo_grid_meta(self.h, C.byref(bg), C.byref(vs), _p(to, C.c_double), _p(mat, C.c_double),
                              C.byref(avs))
        return bg.value, vs.value, to, mat.reshape(3, 4), avs.value

    def leaf_count(self):
        return self.lib.vo_grid_leaf_count(self.h)

    def active_voxel_count(self):
        return self.lib.vo_grid_active_count(self.h)

    def get(self, c):
        return self.lib.vo_get(self.h, *map(int, c))

    def is_active(self, c):
        return bool(self.lib.vo_is_active(self.h, *map(int, c)))

    def set(self, c, v):
        self.lib.vo_set(self.h, *map(int, c), C.c_float(v))

    def deactivate(self, c):
        self.lib.vo_deactivate(self.h, *map(int, c))

    def sample_trilinear(self, world):
        w = np.ascontiguousarray(world, np.float64).reshape(-1, 3)
        out = np.zeros(len(w), np.float32)
        self.lib.vo_sample_trilinear(self.h, _p(w, C.c_double), len(w), _p(out, C.c_float))
        return out

    def advect(self, vx, vy, vz, dt):
        return OGrid(self.lib.vo_advect_level_set(self.h, vx.h, vy.h, vz.h, dt))

    def zero_crossings(self):
        n = self.lib.vo_find_zero_crossings(self.h, None, 0)
        out = np.zeros((n, 3), np.int32)
        if n:
            self.lib.vo_find_zero_crossings(self.h, _p(out, C.c_int32), n)
        return out

    def trim(self, hw):
        self.lib.vo_trim_narrow_band(self.h, C.c_float(hw))

    def rebuild(self, hw, brute=False):
        self.lib.vo_rebuild_narrow_band(self.h, C.c_float(hw), 1 if brute else 0)

    def dilate(self, iterations=1):
        self.lib.vo_dilate(self.h, iterations)

    def extend_velocity(self, vx, vy, vz, half_width):
        """extend_velocity(self as the SDF, vx, vy, vz, half_width), in place on vx, vy, vz."""
        self.lib.vo_extend_velocity(self.h, vx.h, vy.h, vz.h, half_width)

    def volume_to_mesh(self, isovalue=0.0):
        """(vertices (n, 3) f64, triangles (m, 3) u32) with the triangle table of
        oracle/mc_table.py."""
        from oracle import mc_table
        tab = np.asarray(mc_table.tri_table(), np.int8).reshape(-1)
        lib = load()
        nt = C.c_size_t()
        nv = lib.vo_volume_to_mesh(self.h, isovalue, _p(tab, C.c_int8), None, 0, None, 0, C.byref(nt))
        v = np.zeros((nv, 3), np.float64)
        t = np.zeros((nt.value, 3), np.uint32)
        lib.vo_volume_to_mesh(self.h, isovalue, _p(tab, C.c_int8), _p(v, C.c_double), nv, _p(t, C.c_uint32),
                              nt.value, C.byref(nt))
        return v, t

    def flood_fill_sign(self):
        self.lib.vo_flood_fill_sign(self.h)

    def remove_empty_leaves(self):
        self.lib.vo_remove_empty_leaves(self.h)

    def __del__(self):
        try:
            if self.h:
                self.lib.vo_grid_free(self.h)
                self.h = None
        except Exception:
            pass


def advect_particles(vx, vy, vz, positions, dt, rk4=True):
    """Positions (n, 3) f64 after one advect_particles (RK4) or
    advect_particles_euler step through the grids vx, vy, vz."""
    p = np.ascontiguousarray(positions, np.float64).reshape(-1, 3).copy()
    load().vo_advect_particles(vx.h, vy.h, vz.h, _p(p, C.c_double), len(p), dt, 1 if rk4 else 0)
    return p


def rebin_points(positions, world_to_index_rows):
    """PointDataGrid::rebin (src/points/point_grid.rs:258-266) of particles
    given in binned order, leaves drained in ascending origin order: returns
    (perm, leaf_origins (k, 3), leaf_start (k + 1)) with perm[j] the input index
    of the j-th particle of the re-binned grid."""
    p = np.ascontiguousarray(positions, np.float64).reshape(-1, 3)
    inv = np.ascontiguousarray(world_to_index_rows, np.float64).reshape(12)
    n = len(p)
    perm = np.zeros(max(n, 1), np.uint32)
    org = np.zeros((max(n, 1), 3), np.int32)
    start = np.zeros(n + 1, np.uint32)
    k = load().vo_rebin_points(_p(p, C.c_double), n, _p(inv, C.c_double), _p(perm, C.c_uint32),
                               _p(org, C.c_int32), _p(start, C.c_uint32))
    return perm[:n], org[:k], start[:k + 1]


def uniform_velocity(voxel_size, vel, bbox_min=None, bbox_max=None):
    """Oracle twin of the crate's ``make_uniform_velocity`` test helper (src/tools/advection.rs:116-134)."""
    out = []
    for a in range(3):
        g = OGrid.new(float(np.float32(vel[a])), voxel_size)
        for c in (bbox_min, bbox_max):
            if c is not None:
                g.set(c, vel[a])
        out.append(g)
    return out


# --------------------------------------------------------------------------
# narrow-band method oracle (FP64), method_oracle.hpp

VEL_CONSTANT, VEL_VORTEX, VEL_CURL = 0, 1, 2


def pack_velocity(vel: dict) -> tuple[int, np.ndarray]:
    """Velocity description -> (kind, packed f64 params) shared with the GPU side.

    {"kind": "constant", "c": (ux, uy, uz)}            index units per unit time
    {"kind": "vortex", "vs": vs, "w0": (x, y, z), "period": T}
    {"kind": "curl", "octaves": [(A, k, (ph0, ph1, ph2), (e0, e1, e2)), ...]}
    """
    k = vel["kind"]
    if k == "constant":
        return VEL_CONSTANT, np.array(vel["c"], np.float64)
    if k == "vortex":
        return VEL_VORTEX, np.array([vel["vs"], *vel.get("w0", (0.0, 0.0, 0.0)), vel["period"]], np.float64)
    if k == "curl":
        p = [float(len(vel["octaves"]))]
        for A, kk, ph, e in vel["octaves"]:
            p += [A, kk, *ph, *e]
        return VEL_CURL, np.array(p, np.float64)
    raise ValueError(k)


class MOGrid:
    """FP64 method-oracle grid (values in voxel units)."""

    def __init__(self, handle, hw):
        self.lib = load()
        self.h = handle
        self.hw = hw

    @classmethod
    def sphere(cls, radius, center, voxel_size, half_width, w0=(0.0, 0.0, 0.0)):
        lib = load()
        c = np.asarray(center, np.float64)
        w = np.asarray(w0, np.float64)
        return cls(lib.vm_sphere(radius, _p(c, C.c_double), voxel_size, _p(w, C.c_double), half_width), half_width)

    @classmethod
    def spheres(cls, spheres, half_width):
        """Union of spheres, rows (cx, cy, cz, r) in voxels."""
        lib = load()
        s = np.ascontiguousarray(spheres, np.float64).reshape(-1, 4)
        return cls(lib.vm_spheres(_p(s, C.c_double), len(s), half_width), half_width)

    @classmethod
    def from_arrays(cls, origins, masks, phi, half_width):
        lib = load()
        o = np.ascontiguousarray(origins, np.int32)
        m = np.ascontiguousarray(masks, np.uint64)
        v = np.ascontiguousarray(phi, np.float64)
        return cls(lib.vm_import(_p(o, C.c_int32), _p(m, C.c_uint64), _p(v, C.c_double), len(o), half_width),
                   half_width)

    def arrays(self):
        n = self.lib.vm_leaf_count(self.h)
        o = np.zeros((n, 3), np.int32)
        m = np.zeros((n, 8), np.uint64)
        v = np.zeros((n, 512), np.float64)
        if n:
            self.lib.vm_export(self.h, _p(o, C.c_int32), _p(m, C.c_uint64), _p(v, C.c_double))
        return o, m, v

    def leaf_count(self):
        return self.lib.vm_leaf_count(self.h)

    def step(self, vel: dict, integrator: int, reinit_iters: int, t: float, dt: float, nthreads: int = 8,
             reinit_mode: int = 0) -> bool:
        kind, p = pack_velocity(vel)
        return bool(self.lib.vm_step(self.h, kind, _p(p, C.c_double), integrator, reinit_iters, reinit_mode, t, dt,
                                     nthreads))

    def volume(self, ref=(0.0, 0.0, 0.0)):
        r = np.asarray(ref, np.float64)
        return self.lib.vm_volume(self.h, _p(r, C.c_double))

    def __del__(self):
        try:
            if self.h:
                self.lib.vm_free(self.h)
                self.h = None
        except Exception:
            pass


def velocity_at(vel: dict, p, t):
    kind, prm = pack_velocity(vel)
    pp = np.ascontiguousarray(p, np.float64)
    u = np.zeros(3)
    load().vm_velocity(kind, _p(prm, C.c_double), _p(pp, C.c_double), t, _p(u, C.c_double))
    return u
