"""Differentiable frozen-band advection with a hand-written adjoint (``vlr_adj_*``).

:class:`AdvectionFunction` follows the autograd-Function contract:
``forward(phi_0, V) -> phi_K`` keeps what the backward pass needs
(checkpoints every C steps), ``backward(dL/dphi_K) -> (dL/dphi_0, dL/dV)``.
``phi`` arrays are band values (active voxels, in :meth:`band` order, voxel
units); ``V`` is a staggered field of shape (3, n, n, n), voxels per unit
time, component a on the cell faces normal to axis a.
"""
from __future__ import annotations

import ctypes as C
import math

import numpy as np

from ._lib import Context, ptr


def staggered_vortex(n: int, cell: float, voxel_size: float) -> np.ndarray:
    """The deformation field at t = 0 on an n^3 staggered grid of `cell`
    voxels (unit cube world = voxel_size * index), in voxels per unit time."""
    i = np.arange(n, dtype=np.float64)
    face = i * cell * voxel_size             # world coordinate of a face
    mid = (i + 0.5) * cell * voxel_size      # world coordinate of a cell centre
    s, pi = np.sin, math.pi

    def field(a, x, y, z):
        if a == 0:
            return 2 * s(pi * x) ** 2 * s(2 * pi * y) * s(2 * pi * z)
        if a == 1:
            return -s(2 * pi * x) * s(pi * y) ** 2 * s(2 * pi * z)
        return -s(2 * pi * x) * s(2 * pi * y) * s(pi * z) ** 2

    V = np.zeros((3, n, n, n), np.float32)
    for a in range(3):
        axes = [mid, mid, mid]
        axes[a] = face
        X, Y, Z = np.meshgrid(*axes, indexing="ij")
        V[a] = (field(a, X, Y, Z) / voxel_size).astype(np.float32)
    return V


class AdvectionFunction:
    """Frozen-band semi-Lagrangian advection phi_0 -> phi_K and its adjoint."""

    def __init__(self, origins, masks, phi, V, cell: float, dt: float, period: float, steps: int,
                 checkpoint_every: int, half_width: float = 3.0, t0: float = 0.0, ctx: Context | None = None):
        self.ctx = ctx or Context.default()
        o = np.ascontiguousarray(origins, np.int32)
        m = np.ascontiguousarray(masks, np.uint64)
        p = np.ascontiguousarray(phi, np.float32)
        V = np.ascontiguousarray(V, np.float32)
        self.n = V.shape[-1]
        h = C.c_void_p()
        self.ctx.check(self.ctx.lib.vlr_adj_create(self.ctx.handle, ptr(o, C.c_int32), ptr(m, C.c_uint64),
                                                   ptr(p, C.c_float), len(o), C.c_float(half_width),
                                                   ptr(V, C.c_float), self.n, cell, dt, period, t0, steps,
                                                   checkpoint_every, C.byref(h)), "vlr_adj_create")
        self.handle = h
        nb = C.c_size_t()
        self.ctx.check(self.ctx.lib.vlr_adj_band(self.ctx.handle, h, None, 0, C.byref(nb)), "vlr_adj_band")
        self.n_band = nb.value

    @classmethod
    def from_level_set(cls, ls, steps: int, checkpoint_every: int):
        """The frozen-band adjoint of a single-grid level set's own step
        (``vlr_adj_create_level_set``): phi_0 is its current state and every
        band voxel moves by its fixed backtrace displacement per step.  There
        is no velocity input, and ``backward`` returns (dL/dphi_0, None)."""
        self = cls.__new__(cls)
        self.ctx = ls.ctx
        self.n = 0
        h = C.c_void_p()
        self.ctx.check(self.ctx.lib.vlr_adj_create_level_set(self.ctx.handle, ls.handle, steps, checkpoint_every,
                                                             C.byref(h)), "vlr_adj_create_level_set")
        self.handle = h
        nb = C.c_size_t()
        self.ctx.check(self.ctx.lib.vlr_adj_band(self.ctx.handle, h, None, 0, C.byref(nb)), "vlr_adj_band")
        self.n_band = nb.value
        return self

    def set_gather(self, mode: int):
        """Pin the backward pass's lambda-transpose kernel (0 automatic, 1
        windowed, 2 quad); the two kernels associate each voxel's sum
        differently, so runs compared bit for bit use the same one."""
        self.ctx.check(self.ctx.lib.vlr_adj_set_gather(self.ctx.handle, self.handle, int(mode)), "vlr_adj_set_gather")

    def shifted_phi0_device(self, shift, out_ptr: int):
        """phi_0 translated by `shift` voxels (each within +-8), read on the band,
        into a device buffer of n_band floats (enqueued, no wait)."""
        self.ctx.check(self.ctx.lib.vlr_adj_shifted_phi0(self.ctx.handle, self.handle, int(shift[0]), int(shift[1]),
                                                         int(shift[2]), out_ptr), "vlr_adj_shifted_phi0")

    def displacement(self) -> np.ndarray:
        """(n_band, 3) backtrace displacement of a level-set adjoint, voxels."""
        d = np.zeros((self.n_band, 3), np.float32)
        self.ctx.check(self.ctx.lib.vlr_adj_displacement(self.ctx.handle, self.handle, ptr(d, C.c_float)),
                       "vlr_adj_displacement")
        return d

    def band(self) -> np.ndarray:
        c = np.zeros((self.n_band, 3), np.int32)
        nb = C.c_size_t()
        self.ctx.check(self.ctx.lib.vlr_adj_band(self.ctx.handle, self.handle, ptr(c, C.c_int32), self.n_band,
                                                 C.byref(nb)), "vlr_adj_band")
        return c

    def forward(self, phi0_band=None, V=None) -> np.ndarray:
        if phi0_band is not None or V is not None:
            pb = None if phi0_band is None else np.ascontiguousarray(phi0_band, np.float32)
            vv = None if V is None else np.ascontiguousarray(V, np.float32)
            self.ctx.check(self.ctx.lib.vlr_adj_set_inputs(self.ctx.handle, self.handle,
                                                           None if pb is None else ptr(pb, C.c_float),
                                                           None if vv is None else ptr(vv, C.c_float)),
                           "vlr_adj_set_inputs")
        out = np.zeros(self.n_band, np.float32)
        self.ctx.check(self.ctx.lib.vlr_adj_forward(self.ctx.handle, self.handle, ptr(out, C.c_float)),
                       "vlr_adj_forward")
        return out

    def backward(self, grad_phik):
        g = np.ascontiguousarray(grad_phik, np.float32)
        g0 = np.zeros(self.n_band, np.float32)
        gv = np.zeros((3, self.n, self.n, self.n), np.float32) if self.n else None
        self.ctx.check(self.ctx.lib.vlr_adj_backward(self.ctx.handle, self.handle, ptr(g, C.c_float),
                                                     ptr(g0, C.c_float), None if gv is None else ptr(gv, C.c_float)),
                       "vlr_adj_backward")
        return g0, gv

    def forward_device(self, phik_ptr: int = 0):
        """Forward pass into a device buffer of n_band floats (raw pointer, or 0
        to keep phi_K only internally); enqueued on the context stream, no wait."""
        self.ctx.check(self.ctx.lib.vlr_adj_forward_device(self.ctx.handle, self.handle, phik_ptr or None),
                       "vlr_adj_forward_device")

    def backward_device(self, grad_phik_ptr: int, grad_phi0_ptr: int = 0, grad_vel_ptr: int = 0):
        """Backward pass on device buffers (raw pointers: n_band floats in,
        n_band and 3 n^3 floats out, 0 to skip an output); enqueued on the
        context stream, no wait (``Context.check_device`` reports errors)."""
        self.ctx.check(self.ctx.lib.vlr_adj_backward_device(self.ctx.handle, self.handle, grad_phik_ptr,
                                                            grad_phi0_ptr or None, grad_vel_ptr or None),
                       "vlr_adj_backward_device")

    def close(self):
        if self.handle:
            self.ctx.lib.vlr_adj_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def sphere_band(radius_vox: float, center_vox, domain: int, half_width: float = 3.0, ctx: Context | None = None):
    """Leaves (origins, masks, phi in voxels) of a sphere in a domain^3 unit cube."""
    from .method import F32, LevelSet
    vs = 1.0 / domain
    ls = LevelSet.sphere(radius_vox * vs, tuple(c * vs for c in center_vox), vs, {"kind": "constant", "c": (0, 0, 0)},
                         1.0, half_width=half_width, precision=F32, ctx=ctx)
    o, m, p = ls.arrays()
    ls.close()
    return o, m, p
