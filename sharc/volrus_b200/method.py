"""Narrow-band level-set method grids on the GPU (``vlr_ls_*`` in the C ABI).

The reference's own step (``advect_level_set`` + ``rebuild_narrow_band``,
``src/tools/advection.rs:32-56``, ``src/tools/level_set_track.rs:80-114``)
keeps the active set fixed, so a moving interface leaves its band.
:class:`LevelSet` runs the full narrow-band step instead: semi-Lagrangian
backtrace (Euler / RK2 midpoint / SSP-RK3) through an analytic velocity,
Godunov-upwind reinitialisation, and dilation-based re-tracking of the band,
with leaf values in voxel units stored as f32 or f16.
"""
from __future__ import annotations

import ctypes as C
import math

import numpy as np

from . import _lib
from ._lib import Context, ptr

F32, F16 = 0, 1
CONSTANT, VORTEX, CURL = 0, 1, 2


def velocity_desc(vel: dict) -> _lib.vlr_velocity_desc:
    """Velocity dictionary -> C descriptor.

    {"kind": "constant", "c": (ux, uy, uz)}                      voxels per unit time
    {"kind": "vortex", "vs": vs, "w0": (x, y, z), "period": T}   deformation field on the unit cube
    {"kind": "curl", "octaves": [(A, k, (ph0, ph1, ph2), (e0, e1, e2)), ...]}
    optional "domain": ((lo_x, lo_y, lo_z), (hi_x, hi_y, hi_z)) in voxels
    """
    d = _lib.vlr_velocity_desc()
    k = vel["kind"]
    if k == "constant":
        d.kind = CONSTANT
        for a in range(3):
            d.constant[a] = float(vel["c"][a])
    elif k == "vortex":
        d.kind = VORTEX
        d.voxel_size = float(vel["vs"])
        for a, w in enumerate(vel.get("w0", (0.0, 0.0, 0.0))):
            d.w0[a] = float(w)
        d.period = float(vel["period"])
    elif k == "curl":
        d.kind = CURL
        d.octaves = len(vel["octaves"])
        for o, (A, kk, ph, e) in enumerate(vel["octaves"]):
            d.amp[o] = A
            d.wavenumber[o] = kk
            for a in range(3):
                d.phase[o][a] = ph[a]
                d.dir[o][a] = e[a]
    else:
        raise ValueError(k)
    dom = vel.get("domain")
    for a in range(3):
        d.domain_lo[a] = int(dom[0][a]) if dom else 1
        d.domain_hi[a] = int(dom[1][a]) if dom else 0
    return d


def curl_noise(seed: int, extent: float, amplitude: float = 1.0, octaves: int = 3) -> dict:
    """Divergence-free curl noise from a sinusoidal stream potential.

    psi = sum_o f_o e_o with f_o = A_o prod_a sin(k_o p_a + phase_{o,a}),
    k_o = 2 pi 2^o / extent, seeded phases and unit directions e_o; the curl
    v = sum_o grad f_o x e_o is scaled so that |v_a| <= amplitude voxels per
    unit time (octave weights 1, 1/2, 1/4, normalised)."""
    rng = np.random.default_rng(seed)
    w = np.array([2.0 ** -o for o in range(octaves)])
    w /= w.sum()
    octs = []
    for o in range(octaves):
        k = 2.0 * math.pi * 2 ** o / extent
        e = rng.normal(size=3)
        e /= np.linalg.norm(e)
        ph = rng.uniform(0, 2 * math.pi, 3)
        A = amplitude * w[o] / (2.0 * k)  # |grad f x e|_a <= 2 A k
        octs.append((float(A), float(k), tuple(float(x) for x in ph), tuple(float(x) for x in e)))
    return {"kind": "curl", "octaves": octs}


def random_sphere_grids(n_grids: int, seed: int, extent_log2=(6.0, 10.0), spheres=(1, 64), radius=(4.0, 24.0),
                        amplitude: float = 1.0, octaves: int = 3):
    """Seeded batch of uneven grids: each grid has a cubic extent 2^U(extent_log2)
    voxels (log-uniform), 1-64 spheres with radii U(radius) and centres uniform in
    the extent, and its own curl-noise velocity (amplitude voxels per unit time).
    Returns [(spheres (n, 4), velocity dict, extent)]."""
    out = []
    for g in range(n_grids):
        rng = np.random.default_rng([seed, g])
        extent = float(2.0 ** rng.uniform(*extent_log2))
        ns = int(rng.integers(spheres[0], spheres[1] + 1))
        r = rng.uniform(radius[0], radius[1], ns)
        c = rng.uniform(0.0, extent, (ns, 3))
        vel = curl_noise(int(rng.integers(1 << 30)), extent, amplitude, octaves)
        m = 256  # sampling margin: bands may drift ~amplitude voxels per step
        vel["domain"] = ((-m, -m, -m), (int(extent) + m, int(extent) + m, int(extent) + m))
        out.append((np.column_stack([c, r]), vel, extent))
    return out


def large_sphere_grid(n_spheres: int = 8000, seed: int = 7, extent: float = 8192.0, radius=(6.0, 40.0),
                      amplitude: float = 1.0, octaves: int = 3):
    """One large grid: n seeded random spheres, radii U(radius) voxels, centres
    uniform in an extent^3 index box, with a curl-noise velocity of `amplitude`
    voxels per unit time sampled over the extent plus a 256-voxel margin.
    Returns (spheres (n, 4), velocity dict)."""
    rng = np.random.default_rng(seed)
    sph = np.column_stack([rng.uniform(0.0, extent, (n_spheres, 3)), rng.uniform(*radius, n_spheres)])
    vel = curl_noise(int(rng.integers(1 << 30)), extent, amplitude, octaves)
    m = 256
    vel["domain"] = ((-m, -m, -m), (int(extent) + m, int(extent) + m, int(extent) + m))
    return sph, vel


def spheres_near_box(spheres: np.ndarray, lo, hi, margin: float) -> np.ndarray:
    """Spheres whose narrow band (radius + margin) reaches the box [lo, hi)^3."""
    c, r = spheres[:, :3], spheres[:, 3]
    lo, hi = np.asarray(lo, np.float64), np.asarray(hi, np.float64)
    d = np.maximum(np.maximum(lo - c, c - hi), 0.0)
    return spheres[np.sqrt((d * d).sum(axis=1)) <= r + margin]


def leaves_in_box(origins: np.ndarray, lo, hi) -> np.ndarray:
    """Boolean selector of the leaves whose 8^3 block lies inside [lo, hi)^3."""
    o = np.asarray(origins)
    return np.all((o >= np.asarray(lo)) & (o + 8 <= np.asarray(hi)), axis=1)


class LevelSet:
    """A narrow-band level set (method grid) resident on the GPU."""

    def __init__(self, ctx: Context, handle, half_width: float, precision: int, dt: float, voxel_size: float = 1.0):
        self.ctx = ctx
        self.handle = handle
        self.half_width = half_width
        self.precision = precision
        self.dt = dt
        self.voxel_size = voxel_size

    @staticmethod
    def _method(precision, half_width, integrator, reinit_iters, dt, t0, capacity, reinit_mode=0):
        m = _lib.vlr_method_desc()
        m.precision = precision
        m.half_width = half_width
        m.integrator = integrator
        m.reinit_iters = reinit_iters
        m.dt = dt
        m.t0 = t0
        m.capacity = capacity
        m.reinit_mode = reinit_mode
        return m

    @classmethod
    def sphere(cls, radius, center, voxel_size, velocity: dict, dt: float, half_width: float = 3.0,
               precision: int = F32, integrator: int = 2, reinit_iters: int = 2, t0: float = 0.0, w0=(0.0, 0.0, 0.0),
               capacity: int = 0, reinit_mode: int = 0, ctx: Context | None = None) -> "LevelSet":
        """``reinit_mode`` 0: plain Godunov reinitialisation; 1: Godunov with the
        subcell fix at cut voxels (the interface does not move, but the fix's
        sign test makes long runs sensitive to rounding)."""
        ctx = ctx or Context.default()
        m = cls._method(precision, half_width, integrator, reinit_iters, dt, t0, capacity, reinit_mode)
        v = velocity_desc(velocity)
        c = np.asarray(center, np.float64)
        w = np.asarray(w0, np.float64)
        h = C.c_void_p()
        ctx.check(ctx.lib.vlr_ls_create_sphere(ctx.handle, C.byref(m), C.byref(v), C.c_double(radius),
                                               ptr(c, C.c_double), C.c_double(voxel_size), ptr(w, C.c_double),
                                               C.byref(h)), "vlr_ls_create_sphere")
        return cls(ctx, h, half_width, precision, dt, voxel_size)

    @classmethod
    def spheres(cls, grids, dt: float, half_width: float = 3.0, precision: int = F16, integrator: int = 3,
                reinit_iters: int = 2, t0: float = 0.0, capacity: int = 0, reinit_mode: int = 0,
                ctx: Context | None = None) -> "LevelSet":
        """One or many grids, each a union of spheres with its own velocity.

        ``grids``: list of (spheres, velocity) with spheres an (n, 4) array of
        (cx, cy, cz, r) in voxels (voxel size 1, world = index)."""
        ctx = ctx or Context.default()
        m = cls._method(precision, half_width, integrator, reinit_iters, dt, t0, capacity, reinit_mode)
        n = len(grids)
        arr = (_lib.vlr_batch_grid * n)()
        keep = []
        for g, (sph, vel) in enumerate(grids):
            s = np.ascontiguousarray(sph, np.float64).reshape(-1, 4)
            cs = (_lib.vlr_sphere * len(s))()
            for i, row in enumerate(s):
                cs[i].center[0], cs[i].center[1], cs[i].center[2] = row[0], row[1], row[2]
                cs[i].radius = row[3]
            keep.append(cs)
            arr[g].spheres = cs
            arr[g].n_spheres = len(s)
            arr[g].velocity = velocity_desc(vel)
        h = C.c_void_p()
        ctx.check(ctx.lib.vlr_ls_create_spheres(ctx.handle, C.byref(m), arr, n, C.byref(h)), "vlr_ls_create_spheres")
        ls = cls(ctx, h, half_width, precision, dt)
        ls.n_grids = n
        return ls

    def grid_arrays(self, grid: int):
        """(origins, masks, phi) of one grid of a batch, sorted (x, y, z)."""
        n = self.info()[0]
        o = np.zeros((n, 3), np.int32)
        m = np.zeros((n, 8), np.uint64)
        v = np.zeros((n, 512), np.float32)
        k = C.c_size_t()
        self.ctx.check(self.ctx.lib.vlr_ls_download_grid(self.ctx.handle, self.handle, grid, None, ptr(o, C.c_int32),
                                                         ptr(m, C.c_uint64), ptr(v, C.c_float), n, C.byref(k)),
                       "vlr_ls_download_grid")
        return o[: k.value], m[: k.value], v[: k.value]

    @classmethod
    def from_leaves(cls, origins, masks, phi, velocity: dict, dt: float, half_width: float = 3.0,
                    precision: int = F32, integrator: int = 2, reinit_iters: int = 2, t0: float = 0.0,
                    capacity: int = 0, reinit_mode: int = 0, ctx: Context | None = None) -> "LevelSet":
        ctx = ctx or Context.default()
        m = cls._method(precision, half_width, integrator, reinit_iters, dt, t0, capacity, reinit_mode)
        v = velocity_desc(velocity)
        o = np.ascontiguousarray(origins, np.int32)
        mk = np.ascontiguousarray(masks, np.uint64)
        p = np.ascontiguousarray(phi, np.float32)
        h = C.c_void_p()
        ctx.check(ctx.lib.vlr_ls_create_from_leaves(ctx.handle, C.byref(m), C.byref(v), ptr(o, C.c_int32),
                                                    ptr(mk, C.c_uint64), ptr(p, C.c_float), len(o), C.byref(h)),
                  "vlr_ls_create_from_leaves")
        return cls(ctx, h, half_width, precision, dt)

    def step(self, n: int = 1):
        self.ctx.check(self.ctx.lib.vlr_ls_step(self.ctx.handle, self.handle, n), "vlr_ls_step")

    def enqueue(self, n: int = 1):
        """Enqueue n steps without waiting (check later with ``Context.check_device``)."""
        self.ctx.check(self.ctx.lib.vlr_ls_enqueue(self.ctx.handle, self.handle, n), "vlr_ls_enqueue")

    def set_launch_shape(self, advect=None, reinit=None):
        """Fix the stencil kernels' launch shapes as (threads, CTAs[, staging])
        tuples (threads 128 and staging 0, cp.async row copies, are the only
        kernels built), or pass nothing to let the next step's autotuner choose
        the CTA counts again."""
        if advect is None:
            self.ctx.check(self.ctx.lib.vlr_ls_set_launch_shape(self.ctx.handle, self.handle, 0, 0, 0, 0, 0, 0),
                           "vlr_ls_set_launch_shape")
            return
        a = tuple(advect) + (0,) * (3 - len(advect))
        r = tuple(reinit) + (0,) * (3 - len(reinit))
        self.ctx.check(self.ctx.lib.vlr_ls_set_launch_shape(self.ctx.handle, self.handle, *a, *r),
                       "vlr_ls_set_launch_shape")

    def launch_shape(self):
        """{"advect": (threads, CTAs, staging), "reinit": (threads, CTAs, staging),
        "timed": [(kernel, threads, CTAs, staging, us), ...]}."""
        shape = (C.c_int * 6)()
        n = C.c_int()
        self.ctx.check(self.ctx.lib.vlr_ls_get_launch_shape(self.ctx.handle, self.handle, shape, C.byref(n), None, 0),
                       "vlr_ls_get_launch_shape")
        log = np.zeros((max(n.value, 1), 5), np.float32)
        self.ctx.check(self.ctx.lib.vlr_ls_get_launch_shape(self.ctx.handle, self.handle, shape, C.byref(n),
                                                            ptr(log, C.c_float), len(log)), "vlr_ls_get_launch_shape")
        names = ("k_m_advect", "k_m_reinit")
        timed = [(names[int(r[0])], int(r[1]), int(r[2]), int(r[3]), float(r[4])) for r in log[: n.value]]
        return {"advect": (shape[0], shape[1], shape[2]), "reinit": (shape[3], shape[4], shape[5]), "timed": timed}

    def info(self):
        n = C.c_size_t()
        a = C.c_uint64()
        t = C.c_double()
        self.ctx.check(self.ctx.lib.vlr_ls_info(self.ctx.handle, self.handle, C.byref(n), C.byref(a), C.byref(t)),
                       "vlr_ls_info")
        return n.value, a.value, t.value

    def leaf_count(self) -> int:
        return self.info()[0]

    def active_voxel_count(self) -> int:
        return self.info()[1]

    def arrays(self):
        """(origins, masks, phi) of all allocated leaves, sorted (x, y, z); phi in voxel units."""
        n = self.info()[0]
        o = np.zeros((n, 3), np.int32)
        m = np.zeros((n, 8), np.uint64)
        v = np.zeros((n, 512), np.float32)
        self.ctx.check(self.ctx.lib.vlr_ls_download(self.ctx.handle, self.handle, ptr(o, C.c_int32),
                                                    ptr(m, C.c_uint64), ptr(v, C.c_float), n), "vlr_ls_download")
        return o, m, v

    def step_host(self, origins, masks, phi, n_steps: int = 1, out=None):
        """Host-resident steps in one call: state from host leaves, n steps,
        result into host arrays (``out`` = (origins, masks, phi) buffers to
        reuse, else new ones sized for twice the input).  Returns the result."""
        o = np.ascontiguousarray(origins, np.int32)
        m = np.ascontiguousarray(masks, np.uint64)
        p = np.ascontiguousarray(phi, np.float32)
        if out is None:
            cap = 2 * len(o) + 64
            out = (np.zeros((cap, 3), np.int32), np.zeros((cap, 8), np.uint64), np.zeros((cap, 512), np.float32))
        k = C.c_size_t()
        self.ctx.check(self.ctx.lib.vlr_ls_step_host(self.ctx.handle, self.handle, ptr(o, C.c_int32),
                                                     ptr(m, C.c_uint64), ptr(p, C.c_float), len(o), int(n_steps),
                                                     ptr(out[0], C.c_int32), ptr(out[1], C.c_uint64),
                                                     ptr(out[2], C.c_float), len(out[0]), C.byref(k)),
                       "vlr_ls_step_host")
        return out[0][: k.value], out[1][: k.value], out[2][: k.value]

    def upload(self, origins, masks, phi):
        """Replace the state with host leaves (voxel units), keeping time and allocations."""
        o = np.ascontiguousarray(origins, np.int32)
        m = np.ascontiguousarray(masks, np.uint64)
        p = np.ascontiguousarray(phi, np.float32)
        self.ctx.check(self.ctx.lib.vlr_ls_upload(self.ctx.handle, self.handle, ptr(o, C.c_int32), ptr(m, C.c_uint64),
                                                  ptr(p, C.c_float), len(o)), "vlr_ls_upload")

    def upload_device(self, d_origins: int, d_masks: int, d_phi: int, n: int):
        """Replace the state with n leaves in device memory (pointers: i32[3] origins,
        u64[8] masks, f32[512] values), keeping time and allocations."""
        self.ctx.check(self.ctx.lib.vlr_ls_upload_device(self.ctx.handle, self.handle, C.c_void_p(d_origins),
                                                         C.c_void_p(d_masks), C.c_void_p(d_phi), int(n)),
                       "vlr_ls_upload_device")

    def download_device(self, d_origins: int, d_masks: int, d_phi: int, cap: int) -> int:
        """The allocated leaves, in list order, into device buffers of ``cap``
        records; returns their count."""
        k = C.c_size_t()
        self.ctx.check(self.ctx.lib.vlr_ls_download_device(self.ctx.handle, self.handle, C.c_void_p(d_origins),
                                                           C.c_void_p(d_masks), C.c_void_p(d_phi), int(cap),
                                                           C.byref(k)), "vlr_ls_download_device")
        return k.value

    def gather_device(self, d_pos: int | None, n: int, d_origins: int, d_masks: int | None = None,
                      d_phi: int | None = None):
        """Leaves at list positions ``d_pos[0..n)`` (device i32; None: the first
        n) into device buffers: origins i32[3], and masks u64[8] and values
        (the pool's type, f16 or f32 [512]) where given."""
        self.ctx.check(self.ctx.lib.vlr_ls_gather_device(self.ctx.handle, self.handle, C.c_void_p(d_pos or None),
                                                         int(n), C.c_void_p(d_origins), C.c_void_p(d_masks or None),
                                                         C.c_void_p(d_phi or None)), "vlr_ls_gather_device")

    def edit_device(self, d_drop: int | None, n_list: int, d_origins: int | None = None, d_masks: int | None = None,
                    d_phi: int | None = None, n_add: int = 0):
        """Drop the listed leaves whose ``d_drop`` byte is non-zero (one per list
        position, ``n_list`` = the leaf count), keep the rest in order, append
        ``n_add`` leaves (device origins i32[3], masks u64[8], values in the
        pool's type) and rebuild the index."""
        self.ctx.check(self.ctx.lib.vlr_ls_edit_device(self.ctx.handle, self.handle, C.c_void_p(d_drop or None),
                                                       int(n_list), C.c_void_p(d_origins or None),
                                                       C.c_void_p(d_masks or None), C.c_void_p(d_phi or None),
                                                       int(n_add)), "vlr_ls_edit_device")

    def volume_partials(self, d_partials: int, cap: int, ref=(0.0, 0.0, 0.0)) -> int:
        """One FP64 volume term per allocated leaf, in list order, into a device
        buffer of ``cap`` doubles; returns the leaf count."""
        r = np.asarray(ref, np.float64)
        k = C.c_size_t()
        self.ctx.check(self.ctx.lib.vlr_ls_volume_partials(self.ctx.handle, self.handle, ptr(r, C.c_double),
                                                           C.c_void_p(d_partials), int(cap), C.byref(k)),
                       "vlr_ls_volume_partials")
        return k.value

    def set_host_slabs(self, slabs: int):
        """Slab count of the next host steps (``step_host``): 0 automatic, 1
        always one pass, k >= 2 at most k slabs of consecutive x, whose copies
        to and from the host overlap the other slabs' steps (one step of an
        x-sorted state in pinned buffers only; the result is the one pass's)."""
        self.ctx.check(self.ctx.lib.vlr_ls_set_host_slabs(self.ctx.handle, self.handle, int(slabs)),
                       "vlr_ls_set_host_slabs")

    def set_step(self, step: int):
        """Set the step counter (time = t0 + step * dt): resume a run in a new level set."""
        self.ctx.check(self.ctx.lib.vlr_ls_set_step(self.ctx.handle, self.handle, int(step)), "vlr_ls_set_step")

    def volume(self, ref=(0.0, 0.0, 0.0)) -> float:
        """Enclosed volume in voxel units^3 (FP64 reduction)."""
        r = np.asarray(ref, np.float64)
        out = C.c_double()
        self.ctx.check(self.ctx.lib.vlr_ls_volume(self.ctx.handle, self.handle, ptr(r, C.c_double), C.byref(out)),
                       "vlr_ls_volume")
        return out.value

    def close(self):
        if self.handle:
            self.ctx.lib.vlr_ls_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
