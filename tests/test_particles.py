"""Particle advection (src/tools/advection.rs:58-110) and the point grid's
re-binning (src/points/point_grid.rs:258-266).

CPU: the oracle restatement (oracle_capi.cpp: vo_advect_particles,
vo_rebin_points) against the crate's own particle tests (advection.rs:
198-300); the host PointDataGrid mirror against the crate's point-grid tests
(point_grid.rs:268-473) and its re-binning against the oracle's on random
particles (halves, negative coordinates, a rotated map).  GPU: bit-exact
positions against the oracle through uniform, rotating and random sparse
velocity grids, RK4 and Euler, many particles; the whole crate call on a
PointDataGrid (vlr_advect_points: update, then rebin) bit-exact against the
oracle's update followed by its rebin, particle for particle and leaf for
leaf.
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


# ------------------------------------------------------------ point grid

def make_particle(id, x, y, z):
    from sharc.volrus_b200 import particle
    return particle(id, (x, y, z))


def test_point_grid_insert_kats():  # point_grid.rs:280-300, 376-392
    from sharc.volrus_b200 import PointDataGrid
    g = PointDataGrid.new(1.0)
    g.insert(make_particle(1, 3.5, 2.1, 1.9))  # index (4, 2, 2) -> leaf (0, 0, 0)
    assert g.particle_count() == 1 and g.leaf_count() == 1 and g.contains_leaf((0, 0, 0))
    g2 = PointDataGrid.new(1.0)
    g2.insert(make_particle(1, 1.0, 1.0, 1.0))
    g2.insert(make_particle(2, 10.0, 1.0, 1.0))
    assert g2.particle_count() == 2 and g2.leaf_count() == 2
    g3 = PointDataGrid.new(1.0)
    g3.insert_batch([make_particle(1, 0, 0, 0), make_particle(2, 1, 1, 1), make_particle(3, 10, 10, 10)])
    assert g3.particle_count() == 3 and g3.leaf_count() == 2
    assert PointDataGrid.new(1.0).particle_count() == 0 and PointDataGrid.new(1.0).leaf_count() == 0


def test_point_grid_voxel_query_rebin_affine():  # point_grid.rs:302-324, 415-446
    from sharc.volrus_b200 import AffineMap, PointDataGrid
    g = PointDataGrid.new(1.0)
    g.insert(make_particle(1, 2.1, 2.2, 2.3))
    g.insert(make_particle(2, 1.6, 1.7, 1.8))
    g.insert(make_particle(3, 5.0, 5.0, 5.0))
    assert sorted(int(p["id"]) for p in g.particles_in_voxel((2, 2, 2))) == [1, 2]
    assert [int(p["id"]) for p in g.particles_in_voxel((5, 5, 5))] == [3]
    assert g.particles_in_voxel((0, 0, 0)) == []
    r = PointDataGrid.new(1.0)
    r.insert(make_particle(1, 1.0, 1.0, 1.0))
    assert r.contains_leaf((0, 0, 0))
    r.particles["position"][:] = (20.0, 20.0, 20.0)
    assert r.contains_leaf((0, 0, 0))
    r.rebin()
    assert r.particle_count() == 1 and r.leaf_count() == 1 and r.contains_leaf((16, 16, 16))
    a = PointDataGrid.with_affine(AffineMap.from_uniform_scale(0.5))
    a.insert(make_particle(1, 1.0, 1.0, 1.0))
    assert a.particle_count() == 1 and a.voxel_size == 0.5 and a.leaf_origin_for((1.0, 1.0, 1.0)) == (0, 0, 0)


def _random_points(rng, n, affine=None):
    from sharc.volrus_b200 import PARTICLE, PointDataGrid
    g = PointDataGrid(1.0, affine) if affine is not None else PointDataGrid.new(0.5)
    parts = np.zeros(n, PARTICLE)
    pos = rng.uniform(-12.0, 12.0, (n, 3))
    # exact halves and quarters: the rounding rule decides their voxel
    pos[: n // 8] = np.round(pos[: n // 8] * 2.0) / 2.0
    pos[n // 8: n // 4] = np.round(pos[n // 8: n // 4] * 4.0) / 4.0
    parts["position"] = pos
    parts["velocity"] = rng.normal(size=(n, 3))
    parts["id"] = rng.permutation(n).astype(np.uint64) + 1000
    g.insert_batch(parts)
    return g


def test_point_grid_rebin_matches_oracle(oracle):
    from sharc.volrus_b200 import AffineMap
    rng = np.random.default_rng(11)
    rot = np.array([[0.0, -1.0, 0.0], [1.0, 0.0, 0.0], [0.0, 0.0, 1.0]])
    for aff in (None, AffineMap.from_scale_rotate_translate((0.5, 0.5, 0.5), rot, (0.25, -1.5, 3.0))):
        g = _random_points(rng, 4000, aff)
        moved = g.particles.copy()
        moved["position"] += rng.uniform(-6.0, 6.0, (len(moved), 3))
        g.particles = moved.copy()
        g.rebin()
        perm, org, start = oracle.rebin_points(moved["position"], g.inverse_rows())
        assert np.array_equal(g.particles.view(np.uint8), moved[perm].view(np.uint8))
        assert np.array_equal(g.leaf_origins, org) and np.array_equal(g.leaf_start, start)


@pytest.mark.gpu
@pytest.mark.parametrize("rk4", [True, False])
def test_advect_point_grid_bit_exact(ctx, oracle, rk4):
    from sharc.volrus_b200 import AffineMap, VelocityField, advect_particles, advect_particles_euler
    from tests.test_ref_parity import random_grid
    rng = np.random.default_rng(21)
    rot = np.array([[0.0, 0.0, 1.0], [0.0, 1.0, 0.0], [-1.0, 0.0, 0.0]])
    fields = [rotating_field(),
              VelocityField(*(random_grid(rng, 60, 3, b, vs=0.5, fill=0.7) for b in (0.75, -0.5, 0.3)))]
    for f in fields:
        og = [to_oracle(oracle, x) for x in (f.vx, f.vy, f.vz)]
        for aff in (None, AffineMap.from_scale_rotate_translate((0.25, 0.25, 0.25), rot, (1.0, 0.5, -2.0))):
            g = _random_points(rng, 30000, aff)
            for _ in range(2):
                want = g.particles.copy()
                want["position"] = oracle.advect_particles(*og, want["position"], 0.6, rk4)
                perm, org, start = oracle.rebin_points(want["position"], g.inverse_rows())
                (advect_particles if rk4 else advect_particles_euler)(g, f, 0.6, ctx=ctx)
                assert np.array_equal(g.particles.view(np.uint8), want[perm].view(np.uint8))
                assert np.array_equal(g.leaf_origins, org) and np.array_equal(g.leaf_start, start)
                assert g.leaf_count() > 1


@pytest.mark.gpu
def test_advect_point_grid_empty_and_capacity(ctx):
    import ctypes as C
    from sharc.volrus_b200 import PointDataGrid, advect_particles, make_uniform_velocity, particle
    from sharc.volrus_b200._lib import ptr
    from sharc.volrus_b200.tools import _as_device
    vel = make_uniform_velocity(1.0, (1.0, 2.0, 3.0), (-5, -5, -5), (15, 15, 15))
    g = PointDataGrid.new(1.0)
    assert advect_particles(g, vel, 1.0, ctx=ctx).particle_count() == 0
    g.insert_batch([particle(1, (0.0, 0.0, 0.0)), particle(2, (9.0, 0.0, 0.0))])
    advect_particles(g, vel, 1.0, ctx=ctx)
    assert g.leaf_count() == 2 and np.allclose(g.particles["position"][0], (1.0, 2.0, 3.0), atol=1e-6)
    # too small a leaf capacity: VLR_ERR_CAPACITY with the count, particles untouched
    parts = g.particles.copy()
    ds = [_as_device(c, ctx)[0] for c in (vel.vx, vel.vy, vel.vz)]
    org = np.zeros((1, 3), np.int32)
    start = np.zeros(2, np.uint32)
    nl = C.c_size_t()
    inv = g.inverse_rows()
    rc = ctx.lib.vlr_advect_points(ctx.handle, ds[0].handle, ds[1].handle, ds[2].handle, ptr(inv, C.c_double),
                                   parts.ctypes.data_as(C.c_void_p), len(parts), 1.0, 1, ptr(org, C.c_int32),
                                   ptr(start, C.c_uint32), 1, C.byref(nl))
    assert rc == 3 and nl.value == 2
    assert np.array_equal(parts.view(np.uint8), g.particles.view(np.uint8))
    for d in ds:
        d.close()
