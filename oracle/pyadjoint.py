"""ORACLE — test infrastructure only.

FP64 frozen-band advection and its adjoint (oracle/adjoint_oracle.cpp), plus
central finite differences of an L2 loss, used to check the GPU adjoint.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from .pyoracle import _p, load


class AdjointOracle:
    def __init__(self, origins, masks, phi, half_width, V, n, cell, dt, period, t0, steps):
        self.lib = load()
        o = np.ascontiguousarray(origins, np.int32)
        m = np.ascontiguousarray(masks, np.uint64)
        p = np.ascontiguousarray(phi, np.float64)
        v = np.ascontiguousarray(V, np.float64).reshape(-1)
        self.n = n
        self.h = self.lib.va_create(_p(o, C.c_int32), _p(m, C.c_uint64), _p(p, C.c_double), len(o), half_width,
                                    _p(v, C.c_double), n, cell, dt, period, t0, steps)
        self.nb = self.lib.va_nband(self.h)
        self.V = v.copy()

    @classmethod
    def from_displacement(cls, origins, masks, phi, half_width, disp, steps):
        """Displacement form: phi_{k+1}(x) = trilinear(phi_k)(x + d(x)), d per band voxel."""
        self = cls.__new__(cls)
        self.lib = load()
        o = np.ascontiguousarray(origins, np.int32)
        m = np.ascontiguousarray(masks, np.uint64)
        p = np.ascontiguousarray(phi, np.float64)
        d = np.ascontiguousarray(disp, np.float64).reshape(-1)
        self.n = 0
        self.h = self.lib.va_create_disp(_p(o, C.c_int32), _p(m, C.c_uint64), _p(p, C.c_double), len(o), half_width,
                                         _p(d, C.c_double), steps)
        self.nb = self.lib.va_nband(self.h)
        self.V = np.zeros(0)
        return self

    def forward(self, phi0_band=None, V=None):
        out = np.zeros(self.nb)
        pb = None if phi0_band is None else np.ascontiguousarray(phi0_band, np.float64)
        vv = None if V is None else np.ascontiguousarray(V, np.float64).reshape(-1)
        self.lib.va_forward(self.h, None if pb is None else _p(pb, C.c_double),
                            None if vv is None else _p(vv, C.c_double), _p(out, C.c_double))
        if vv is not None:
            self.V = vv.copy()
        return out

    def backward(self, lamK):
        l = np.ascontiguousarray(lamK, np.float64)
        g0 = np.zeros(self.nb)
        gv = np.zeros(3 * self.n ** 3)
        self.lib.va_backward(self.h, _p(l, C.c_double), _p(g0, C.c_double), _p(gv, C.c_double))
        return g0, gv

    def __del__(self):
        try:
            if self.h:
                self.lib.va_free(self.h)
                self.h = None
        except Exception:
            pass


def loss(phiK, target):
    d = phiK - target
    return float(np.dot(d, d))


def fd_phi0(orc: AdjointOracle, phi0, V, target, idx, eps=1e-3):
    """Central differences of L w.r.t. phi_0 at band indices idx (FP64)."""
    out = []
    for b in idx:
        p = phi0.copy()
        p[b] += eps
        lp = loss(orc.forward(p, V), target)
        p[b] -= 2 * eps
        lm = loss(orc.forward(p, V), target)
        out.append((lp - lm) / (2 * eps))
    orc.forward(phi0, V)
    return np.array(out)


def fd_vel(orc: AdjointOracle, phi0, V, target, idx, eps=1e-3):
    """Central differences of L w.r.t. staggered velocity entries idx (flat)."""
    out = []
    V = np.ascontiguousarray(V, np.float64).reshape(-1)
    for e in idx:
        v = V.copy()
        v[e] += eps
        lp = loss(orc.forward(phi0, v), target)
        v[e] -= 2 * eps
        lm = loss(orc.forward(phi0, v), target)
        out.append((lp - lm) / (2 * eps))
    orc.forward(phi0, V)
    return np.array(out)
