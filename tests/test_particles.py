"""Particle advection (src/tools/advection.rs:58-110), position update only.

CPU: the oracle restatement (oracle_capi.cpp: vo_advect_particles) against the
crate's own particle tests (advection.rs:198-300).  GPU: bit-exact positions
against the oracle through uniform, rotating and random sparse velocity
grids, RK4 and Euler, many particles.
"""
import math

import numpy as np
import pytest


def rotating_field(oracle=None):
    """v = (-y, x, 0) on a 41 x 41 patch at voxel size 0.1 (advection.rs:239-256)."""
    from sharc.volrus_b200 import Grid, VelocityField
    vs = 0.1
    vx, vy, vz = Grid(0.0, vs), Grid(0.0, vs), Grid(0.0, vs)
    for ix in range(-20, 21):
        for iy in range(-20, 21):
            vx.set((ix, iy, 0), float(np.float32(-(iy * vs))))
            vy.set((ix, iy, 0), float(np.float32(ix * vs)))
    return VelocityField(vx, vy, vz)


def to_oracle(oracle, g):
    o, m, v = g.to_arrays()
    return oracle.OGrid.from_arrays(o, m, v, g.background, g.transform.voxel_size, g.transform.origin,
                                    g.affine.mat, g.affine.voxel_size)


def test_oracle_rk4_uniform_field(oracle):  # advection.rs:198-230
    vel = oracle.uniform_velocity(1.0, (1.0, 2.0, 3.0), (-5, -5, -5), (15, 15, 15))
    p = oracle.advect_particles(*vel, [[0.0, 0.0, 0.0]], 1.0)
    assert np.all(np.abs(p[0] - [1.0, 2.0, 3.0]) < 1e-6)


def test_oracle_rk4_beats_euler_rotating(oracle):  # advection.rs:232-300
    f = rotating_field()
    g = [to_oracle(oracle, x) for x in (f.vx, f.vy, f.vz)]
    rk, eu = np.array([[1.0, 0.0, 0.0]]), np.array([[1.0, 0.0, 0.0]])
    for _ in range(10):
        rk = oracle.advect_particles(*g, rk, 0.1, True)
        eu = oracle.advect_particles(*g, eu, 0.1, False)
    exact = np.array([math.cos(1.0), math.sin(1.0)])
    e_rk, e_eu = np.linalg.norm(rk[0, :2] - exact), np.linalg.norm(eu[0, :2] - exact)
    assert e_rk < e_eu and e_rk < 0.01


@pytest.mark.gpu
@pytest.mark.parametrize("rk4", [True, False])
def test_particles_bit_exact(ctx, oracle, rk4):
    from sharc.volrus_b200 import VelocityField, advect_particles, advect_particles_euler
    from tests.test_ref_parity import random_grid
    rng = np.random.default_rng(3)
    fields = [rotating_field(),
              VelocityField(*(random_grid(rng, 60, 3, b, vs=0.5, fill=0.7) for b in (0.25, -0.5, 0.1)))]
    for f in fields:
        og = [to_oracle(oracle, x) for x in (f.vx, f.vy, f.vz)]
        pts = rng.uniform(-2.5, 2.5, (20000, 3))
        want = pts
        got = pts
        for _ in range(3):
            want = oracle.advect_particles(*og, want, 0.07, rk4)
            got = (advect_particles if rk4 else advect_particles_euler)(got, f, 0.07, ctx=ctx)
        assert np.array_equal(got.view(np.uint64), want.view(np.uint64))


@pytest.mark.gpu
def test_particles_uniform_kat_and_empty(ctx, oracle):
    from sharc.volrus_b200 import advect_particles, make_uniform_velocity
    vel = make_uniform_velocity(1.0, (1.0, 2.0, 3.0), (-5, -5, -5), (15, 15, 15))
    p = advect_particles([[0.0, 0.0, 0.0]], vel, 1.0, ctx=ctx)
    assert np.all(np.abs(p[0] - [1.0, 2.0, 3.0]) < 1e-6)
    assert advect_particles(np.zeros((0, 3)), vel, 1.0, ctx=ctx).shape == (0, 3)
