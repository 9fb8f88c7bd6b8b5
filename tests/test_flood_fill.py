"""flood_fill_sign (src/tools/flood_fill.rs:18-107).

CPU: the oracle restatement (oracle/ref_tree.hpp) against the crate's own
tests (flood_fill.rs:113-164).  GPU: origins, masks and all 512 values per
leaf bit-exact against the oracle for a sphere level set (inactive voxels
inside and outside the band), random masks and values (ties between
negative and non-negative neighbour counts, leaves without active voxels),
and the crate's plane case; the mesh of a filled sphere loses most of its
inner surface and matches the oracle's.
"""
import numpy as np
import pytest


def to_oracle(oracle, g):
    o, m, v = g.to_arrays()
    return oracle.OGrid.from_arrays(o, m, v, g.background, g.transform.voxel_size, g.transform.origin,
                                    g.affine.mat, g.affine.voxel_size)


def plane(og):
    for x in range(8):
        for y in range(8):
            og.set((x, y, 3), -1.0)
            og.set((x, y, 4), 0.0)
            og.set((x, y, 5), 1.0)
    return og


def test_oracle_inside_negative(oracle):  # flood_fill.rs:113-156
    og = plane(oracle.OGrid.new(3.0, 1.0))
    og.flood_fill_sign()
    assert og.get((0, 0, 2)) < 0.0
    assert og.get((0, 0, 6)) > 0.0


def test_oracle_all_positive_stays_positive(oracle):  # flood_fill.rs:158-164
    og = oracle.OGrid.new(3.0, 1.0)
    og.set((0, 0, 0), 1.0)
    og.set((1, 0, 0), 2.0)
    og.flood_fill_sign()
    assert og.get((2, 0, 0)) > 0.0


def _same(g, og):
    o1, m1, v1 = g.to_arrays()
    o2, m2, v2 = og.arrays()
    assert np.array_equal(o1, o2) and np.array_equal(m1, m2)
    assert np.array_equal(v1.view(np.uint32), v2.view(np.uint32)), "values differ"


def _check(oracle, g):
    from sharc.volrus_b200 import flood_fill_sign
    og = to_oracle(oracle, g)
    flood_fill_sign(g)
    og.flood_fill_sign()
    _same(g, og)


@pytest.mark.gpu
def test_plane_bit_exact(ctx, oracle):
    from sharc.volrus_b200 import Grid
    og = plane(oracle.OGrid.new(3.0, 1.0))
    o, m, v = og.arrays()
    _check(oracle, Grid.from_arrays(o, m, v, 3.0, None))


@pytest.mark.gpu
def test_sphere_bit_exact(ctx, oracle):
    from sharc.volrus_b200 import make_level_set_sphere
    _check(oracle, make_level_set_sphere(14.0, (0.3, -1.2, 2.5), 1.0, 3.0))


@pytest.mark.gpu
def test_random_leaves_bit_exact(ctx, oracle):
    from sharc.volrus_b200 import Grid
    rng = np.random.default_rng(17)
    n = 300
    origins = (rng.integers(-20, 20, (n, 3)) * 8).astype(np.int32)
    origins = np.unique(origins, axis=0)
    n = len(origins)
    masks = rng.integers(0, 2**63, (n, 8), dtype=np.uint64) & rng.integers(0, 2**63, (n, 8), dtype=np.uint64)
    masks[::7] = 0  # leaves without active voxels stay as they are
    vals = rng.choice(np.array([-2.0, -0.5, 0.0, 0.5, 2.0], np.float32), (n, 512))
    _check(oracle, Grid.from_arrays(origins, masks, vals, 2.5, None))


@pytest.mark.gpu
def test_filled_sphere_mesh(ctx, oracle):
    """Unfilled, the band's inner edge meets +background voxels and the mesh
    holds a second, inner surface; the leaf-local fill removes most of it
    (the crate's fill is an approximation: a leaf's majority sign decides
    voxels with no active neighbour in the leaf).  The filled mesh is
    bit-exact against the oracle's."""
    from sharc.volrus_b200 import flood_fill_sign, make_level_set_sphere, volume_to_mesh
    g = make_level_set_sphere(10.0, (0.0, 0.0, 0.0), 1.0, 3.0)
    before = volume_to_mesh(g, 0.0)
    og = to_oracle(oracle, g)
    flood_fill_sign(g)
    og.flood_fill_sign()
    after = volume_to_mesh(g, 0.0)
    v2, t2 = og.volume_to_mesh(0.0)
    assert np.array_equal(after.vertices.view(np.uint64), v2.view(np.uint64))
    assert np.array_equal(after.triangles, t2)
    r = np.linalg.norm(after.vertices, axis=1)
    assert after.vertex_count() < before.vertex_count() and after.is_watertight()
    assert np.mean(np.abs(r - 10.0) < 1.0) > 0.95
