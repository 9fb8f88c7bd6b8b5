"""The crate's grid and transform unit tests (src/grid.rs, its test module)
against the library's host mirror of ``Grid`` / ``VoxelTransform`` /
``AffineMap`` (sharc/volrus_b200/grid.py), which builds the transforms the
C ABI receives.  Not ported: ``eval_min_max``, ``active_bbox`` and
``mem_bytes``, grid statistics off the advection path."""
import numpy as np
import pytest

from sharc.volrus_b200.grid import AffineMap, Grid, GridClass, VoxelTransform, invert_4x4

EPS = 1e-10
ROT_Z = [[0.0, -1.0, 0.0], [1.0, 0.0, 0.0], [0.0, 0.0, 1.0]]


def approx(a, b, eps=EPS):
    return all(abs(x - y) < eps for x, y in zip(a, b))


def _inv_times_fwd_is_identity(inv, fwd, eps=EPS):
    return np.abs(np.asarray(inv) @ np.asarray(fwd) - np.eye(4)).max() < eps


def test_grid_new_empty_and_set_get():  # grid_new_empty, grid_set_get_index_space
    g = Grid(0.0, 0.5)
    assert g.leaf_count() == 0 and g.active_voxel_count() == 0 and g.grid_class == GridClass.UNKNOWN
    h = Grid(-1.0, 1.0)
    h.set((5, 5, 5), 42.0)
    assert h.get((5, 5, 5)) == 42.0 and h.get((0, 0, 0)) == -1.0


def test_grid_world_space_roundtrip():  # grid_world_space_roundtrip
    g = Grid(0.0, 0.25)
    g.set_world((1.0, 2.0, 3.0), 7.0)
    assert g.get((4, 8, 12)) == 7.0 and g.get_world((1.0, 2.0, 3.0)) == 7.0


def test_grid_transform_with_origin():  # grid_transform_with_origin
    t = VoxelTransform.with_origin(0.5, (10.0, 20.0, 30.0))
    w = t.index_to_world((2, 4, 6))
    assert w == (11.0, 22.0, 33.0)
    assert t.world_to_index(w) == (2, 4, 6)


def test_grid_level_set_constructor_and_metadata():  # grid_level_set_constructor, grid_metadata
    g = Grid.level_set(0.1, 3.0)
    assert g.grid_class == GridClass.LEVEL_SET and g.name == "sdf" and abs(g.background - 0.3) < 1e-6
    h = Grid(0.0, 1.0)
    h.name, h.grid_class = "density", GridClass.FOG_VOLUME
    assert h.name == "density" and h.grid_class == GridClass.FOG_VOLUME


def test_affine_identity_roundtrip():  # affine_identity_roundtrip
    m = AffineMap.identity()
    w = m.index_to_world((3, -7, 11))
    assert approx(w, (3.0, -7.0, 11.0)) and m.world_to_index(w) == (3, -7, 11)


def test_affine_uniform_scale():  # affine_uniform_scale
    m = AffineMap.from_uniform_scale(0.25)
    assert abs(m.voxel_size - 0.25) < EPS
    w = m.index_to_world((4, 8, 12))
    assert approx(w, (1.0, 2.0, 3.0)) and m.world_to_index(w) == (4, 8, 12)


def test_affine_from_voxel_transform():  # affine_from_voxel_transform
    m = AffineMap.from_voxel_transform(VoxelTransform.with_origin(0.5, (10.0, 20.0, 30.0)))
    w = m.index_to_world((2, 4, 6))
    assert approx(w, (11.0, 22.0, 33.0)) and m.world_to_index(w) == (2, 4, 6)


def test_affine_world_to_index_f64_no_rounding():  # affine_world_to_index_f64_no_rounding
    m = AffineMap.from_uniform_scale(2.0)
    assert approx(m.world_to_index_f64((3.0, 5.0, 7.0)), (1.5, 2.5, 3.5))


def test_affine_scale_rotate_translate():  # affine_scale_rotate_translate
    m = AffineMap.from_scale_rotate_translate((2.0, 2.0, 2.0), ROT_Z, (10.0, 20.0, 30.0))
    w = m.index_to_world((1, 0, 0))
    assert approx(w, (10.0, 22.0, 30.0)) and m.world_to_index(w) == (1, 0, 0)


def test_affine_non_uniform_scale():  # affine_non_uniform_scale
    m = AffineMap.from_scale_rotate_translate((1.0, 2.0, 3.0), np.eye(3), (0.0, 0.0, 0.0))
    w = m.index_to_world((1, 1, 1))
    assert approx(w, (1.0, 2.0, 3.0)) and m.world_to_index(w) == (1, 1, 1)


def test_affine_inverses():  # affine_inverse_is_correct, affine_general_inverse_roundtrip
    m = AffineMap.from_uniform_scale(0.5)
    assert _inv_times_fwd_is_identity(m.inverse(), m.forward())
    g = AffineMap.from_scale_rotate_translate((0.5, 0.5, 0.5), ROT_Z, (100.0, -50.0, 25.0))
    assert _inv_times_fwd_is_identity(g.inverse(), g.forward(), 1e-9)


def test_invert_4x4():  # invert_4x4_identity, invert_4x4_scale_translate
    assert np.array_equal(invert_4x4(np.eye(4)), np.eye(4))
    m = [[2.0, 0.0, 0.0, 5.0], [0.0, 3.0, 0.0, 7.0], [0.0, 0.0, 4.0, 9.0], [0.0, 0.0, 0.0, 1.0]]
    assert _inv_times_fwd_is_identity(invert_4x4(m), m)
    with pytest.raises(ValueError):
        invert_4x4(np.zeros((4, 4)))


def test_grid_with_affine():  # grid_with_affine_constructor, grid_with_affine_rotated
    g = Grid.with_affine(0.0, AffineMap.from_uniform_scale(0.25))
    g.set_world((1.0, 2.0, 3.0), 7.0)
    assert g.get((4, 8, 12)) == 7.0 and g.get_world((1.0, 2.0, 3.0)) == 7.0
    assert g.transform.voxel_size == 0.25 and g.transform.origin == (0.0, 0.0, 0.0)
    r = Grid.with_affine(0.0, AffineMap.from_scale_rotate_translate((1.0, 1.0, 1.0), ROT_Z, (0.0, 0.0, 0.0)))
    r.set((1, 0, 0), 99.0)
    assert r.get_world((0.0, 1.0, 0.0)) == 99.0


def test_round_half_away_from_zero_and_saturation():
    """``f64::round`` (halves away from zero) and the saturating ``as i32`` cast."""
    t = VoxelTransform.identity()
    assert t.world_to_index((2.5, -2.5, 0.5)) == (3, -3, 1)
    assert t.world_to_index((-0.5, 1.49999, -1.5)) == (-1, 1, -2)
    assert t.world_to_index((1e30, -1e30, float("nan"))) == (2 ** 31 - 1, -2 ** 31, 0)
