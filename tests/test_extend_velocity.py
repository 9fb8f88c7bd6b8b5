"""extend_velocity (src/tools/level_set_track.rs:115-160).

CPU: the oracle restatement (oracle/ref_tree.hpp) against the crate's own tests
(level_set_track.rs:271-308).  GPU: vx, vy, vz bit-exact against the oracle
(leaf origins, masks, all 512 values per leaf) for a sphere, for random
velocity grids over a multi-tile SDF (integer squared distances tie often,
so the iteration-order tie rule is exercised), and for a sparse interface far
from the band, which takes the search beyond the 27-leaf neighbourhood.
"""
import numpy as np
import pytest


def to_oracle(oracle, g):
    o, m, v = g.to_arrays()
    return oracle.OGrid.from_arrays(o, m, v, g.background, g.transform.voxel_size, g.transform.origin,
                                    g.affine.mat, g.affine.voxel_size)


def same(g, og):
    o1, m1, v1 = g.to_arrays()
    o2, m2, v2 = og.arrays()
    assert np.array_equal(o1, o2), "leaf origins differ"
    assert np.array_equal(m1, m2), "masks differ"
    assert np.array_equal(v1.view(np.uint32), v2.view(np.uint32)), "values differ"


def sphere_case(oracle):
    from sharc.volrus_b200 import Grid
    og = oracle.OGrid.sphere(5.0, (0.0, 0.0, 0.0), 1.0, 3.0)
    o, m, v = og.arrays()
    sdf = Grid.from_arrays(o, m, v, 3.0, None)
    vel = [Grid(0.0, 1.0) for _ in range(3)]
    for c, val in sdf.iter_active():
        if abs(val) < 1.0:
            for g, x in zip(vel, (1.0, 2.0, 3.0)):
                g.set(c, x)
    return sdf, vel


def test_oracle_fills_band_voxels(oracle):  # level_set_track.rs:271-296
    sdf, vel = sphere_case(oracle)
    osdf = to_oracle(oracle, sdf)
    ov = [to_oracle(oracle, g) for g in vel]
    before = ov[0].active_voxel_count()
    osdf.extend_velocity(*ov, 3.0)
    assert ov[0].active_voxel_count() >= before and ov[0].active_voxel_count() > before


def test_oracle_empty_sdf_noop(oracle):  # level_set_track.rs:298-307
    e = oracle.OGrid.new(3.0, 1.0)
    ov = [oracle.OGrid.new(0.0, 1.0) for _ in range(3)]
    e.extend_velocity(*ov, 3.0)
    assert ov[0].active_voxel_count() == 0


@pytest.mark.gpu
def test_extend_velocity_sphere_bit_exact(ctx, oracle):
    from sharc.volrus_b200 import extend_velocity
    sdf, vel = sphere_case(oracle)
    osdf = to_oracle(oracle, sdf)
    ov = [to_oracle(oracle, g) for g in vel]
    extend_velocity(sdf, *vel, 3.0, ctx=ctx)
    osdf.extend_velocity(*ov, 3.0)
    for g, o in zip(vel, ov):
        same(g, o)


@pytest.mark.gpu
def test_extend_velocity_random_multi_tile_bit_exact(ctx, oracle):
    from sharc.volrus_b200 import extend_velocity
    from tests.test_ref_parity import random_grid
    rng = np.random.default_rng(17)
    og = oracle.OGrid.sphere(23.0, (-20.0, 31.0, 5.0), 1.0, 3.0)
    o, m, v = og.arrays()
    from sharc.volrus_b200 import Grid
    sdf = Grid.from_arrays(o, m, v, 3.0, None)
    vel = [random_grid(rng, 80, 6, b, fill=0.4) for b in (0.5, -0.25, 0.0)]
    osdf = to_oracle(oracle, sdf)
    ov = [to_oracle(oracle, g) for g in vel]
    extend_velocity(sdf, *vel, 3.0, ctx=ctx)
    osdf.extend_velocity(*ov, 3.0)
    for g, o in zip(vel, ov):
        same(g, o)


@pytest.mark.gpu
def test_extend_velocity_far_interface_fallback(ctx, oracle):
    """A few interface voxels and band voxels 10-40 voxels away (half width 50)."""
    from sharc.volrus_b200 import Grid, extend_velocity
    rng = np.random.default_rng(5)
    sdf = Grid(50.0, 1.0)
    for c in ((0, 0, 0), (3, 40, -7), (-30, 2, 12)):
        sdf.set(c, 0.25)
    for _ in range(300):
        c = tuple(int(x) for x in rng.integers(-45, 45, 3))
        if sdf.is_active(c):
            continue
        sdf.set(c, float(rng.uniform(1.0, 49.0)))
    vel = [Grid(b, 1.0) for b in (0.0, 1.0, -1.0)]
    for g in vel:
        for c in ((0, 0, 0), (3, 40, -7), (-30, 2, 12)):
            g.set(c, float(rng.normal()))
    osdf = to_oracle(oracle, sdf)
    ov = [to_oracle(oracle, g) for g in vel]
    extend_velocity(sdf, *vel, 50.0, ctx=ctx)
    osdf.extend_velocity(*ov, 50.0)
    for g, o in zip(vel, ov):
        same(g, o)
