"""Pin the CPU oracle to the reference crate's own known-answer tests.

The Sharc.Volrus crate ships no golden files; its tests are inline
assertions.  Every assertion on the advection path is restated here against
the oracle (C++ restatement in oracle/ref_tree.hpp), each citing the
reference test it ports.  An independent numpy restatement of the sphere
generator cross-checks the oracle's input construction at the parity config.
"""
import numpy as np
import pytest


# ---- src/tools/sphere.rs:65-123 ----------------------------------------

def test_sphere_has_active_voxels(oracle):  # sphere.rs:74-79
    g = oracle.OGrid.sphere(5.0, [0, 0, 0], 1.0, 3.0)
    assert g.active_voxel_count() > 0


def test_sphere_sdf_value_at_center_is_negative(oracle):  # sphere.rs:81-89
    g = oracle.OGrid.sphere(5.0, [0, 0, 0], 1.0, 3.0)
    assert g.get((3, 0, 0)) < 0.0


def test_sphere_sdf_value_outside_is_positive(oracle):  # sphere.rs:91-97
    g = oracle.OGrid.sphere(5.0, [0, 0, 0], 1.0, 3.0)
    assert g.get((7, 0, 0)) > 0.0


def test_sphere_sdf_value_on_surface_is_near_zero(oracle):  # sphere.rs:99-107
    g = oracle.OGrid.sphere(5.0, [0, 0, 0], 1.0, 3.0)
    assert abs(g.get((5, 0, 0))) < 0.5


def test_sphere_narrow_band_width(oracle):  # sphere.rs:109-116
    g = oracle.OGrid.sphere(10.0, [0, 0, 0], 1.0, 3.0)
    bg = g.meta()[0]
    assert g.get((20, 0, 0)) == bg


def test_sphere_with_offset_center(oracle):  # sphere.rs:118-131
    g = oracle.OGrid.sphere(3.0, [10.0, 20.0, 30.0], 0.5, 3.0)
    assert g.active_voxel_count() > 0
    assert abs(g.get((26, 40, 60))) < 1.0


# ---- src/tools/interpolation.rs:55-114 ---------------------------------

def test_trilinear_at_voxel_center_returns_exact(oracle):  # interpolation.rs:55-66
    g = oracle.OGrid.new(0.0, 1.0)
    g.set((5, 5, 5), 42.0)
    assert abs(g.sample_trilinear([5.0, 5.0, 5.0])[0] - 42.0) < 1e-6


def test_trilinear_midpoint_interpolates(oracle):  # interpolation.rs:68-77
    g = oracle.OGrid.new(0.0, 1.0)
    g.set((0, 0, 0), 0.0)
    g.set((1, 0, 0), 10.0)
    assert abs(g.sample_trilinear([0.5, 0.0, 0.0])[0] - 5.0) < 1e-5


def test_trilinear_respects_voxel_size(oracle):  # interpolation.rs:79-90
    g = oracle.OGrid.new(0.0, 0.5)
    g.set((0, 0, 0), 0.0)
    g.set((1, 0, 0), 10.0)
    assert abs(g.sample_trilinear([0.25, 0.0, 0.0])[0] - 5.0) < 1e-5


def test_trilinear_on_sphere_sdf_smooth(oracle):  # interpolation.rs:92-114
    g = oracle.OGrid.sphere(5.0, [0, 0, 0], 0.5, 3.0)
    assert abs(g.sample_trilinear([5.0, 0.0, 0.0])[0]) < 1.0
    assert g.sample_trilinear([4.0, 0.0, 0.0])[0] < 0.0


# ---- src/tools/advection.rs:151-197 ------------------------------------

def test_uniform_velocity_moves_sphere_sdf(oracle):
    g = oracle.OGrid.sphere(5.0, [0, 0, 0], 0.5, 3.0)
    vx, vy, vz = oracle.uniform_velocity(0.5, [1.0, 0.0, 0.0], (-30, -30, -30), (30, 30, 30))
    a = g.advect(vx, vy, vz, 1.0)
    assert abs(a.sample_trilinear([6.0, 0.0, 0.0])[0]) < 1.0
    assert a.sample_trilinear([5.0, 0.0, 0.0])[0] < 0.0
    assert a.sample_trilinear([7.0, 0.0, 0.0])[0] > 0.0
    # advection never changes the active set (advection.rs:39-53)
    assert a.active_voxel_count() == g.active_voxel_count()


# ---- src/tools/level_set_track.rs:185-270 ------------------------------

def test_find_zero_crossings_sphere_nonempty(oracle):  # level_set_track.rs:185-202
    g = oracle.OGrid.sphere(5.0, [0, 0, 0], 1.0, 3.0)
    c = g.zero_crossings()
    assert len(c) > 0
    r = np.sqrt((c.astype(np.float64) ** 2).sum(axis=1))
    assert np.all(np.abs(r - 5.0) < 2.5)


def test_find_zero_crossings_empty_grid(oracle):  # level_set_track.rs:204-208
    g = oracle.OGrid.new(3.0, 1.0)
    assert len(g.zero_crossings()) == 0


def test_trim_narrow_band_shrinks_count(oracle):  # level_set_track.rs:210-232
    g = oracle.OGrid.sphere(5.0, [0, 0, 0], 1.0, 5.0)
    before = g.active_voxel_count()
    g.trim(2.0)
    after = g.active_voxel_count()
    assert after < before
    o, m, v = g.arrays()
    bits = np.unpackbits(m.view(np.uint8).reshape(-1, 64), axis=1, bitorder="little").astype(bool)
    assert np.all(np.abs(v[bits]) < 2.0)


def test_trim_narrow_band_empty_grid_noop(oracle):  # level_set_track.rs:234-239
    g = oracle.OGrid.new(3.0, 1.0)
    g.trim(2.0)
    assert g.active_voxel_count() == 0


@pytest.mark.parametrize("brute", [True, False])
def test_rebuild_narrow_band_preserves_sign(oracle, brute):  # level_set_track.rs:241-262
    g = oracle.OGrid.sphere(5.0, [0, 0, 0], 1.0, 3.0)
    o, m, v = g.arrays()
    before = {}
    bits = np.unpackbits(m.view(np.uint8).reshape(-1, 64), axis=1, bitorder="little").astype(bool)
    for i in range(len(o)):
        for off in np.nonzero(bits[i])[0]:
            before[(o[i, 0] + (off >> 6), o[i, 1] + ((off >> 3) & 7), o[i, 2] + (off & 7))] = v[i, off]
    g.rebuild(3.0, brute=brute)
    for c, old in before.items():
        if g.is_active(c) and abs(old) > 0.1:
            # Rust f32::signum: +1 for +0.0, -1 for -0.0
            assert np.copysign(1.0, old) == np.copysign(1.0, g.get(c))


def test_rebuild_narrow_band_empty_grid_noop(oracle):  # level_set_track.rs:264-269
    g = oracle.OGrid.new(3.0, 1.0)
    g.rebuild(3.0)
    assert g.active_voxel_count() == 0


# ---- src/tools/morphology.rs:88-111 ------------------------------------

def test_dilate_single_voxel_produces_7_active(oracle):
    g = oracle.OGrid.new(0.0, 1.0)
    g.set((0, 0, 0), 1.0)
    g.dilate(1)
    assert g.active_voxel_count() == 7
    for off in [(1, 0, 0), (-1, 0, 0), (0, 1, 0), (0, -1, 0), (0, 0, 1), (0, 0, -1)]:
        assert g.is_active(off)


# ---- tree semantics: src/tree/leaf.rs:29-82, internal.rs:118-166,231-247, root.rs:55-72

def test_tree_get_set_deactivate_semantics(oracle):
    g = oracle.OGrid.new(2.5, 1.0)
    assert g.get((100, -7, 3)) == 2.5                # unallocated -> background
    g.set((-1, -1, -1), 4.0)                         # negative coords align down
    assert g.is_active((-1, -1, -1)) and g.get((-1, -1, -1)) == 4.0
    assert g.get((-8, -8, -8)) == 2.5 and not g.is_active((-8, -8, -8))  # same leaf, inactive -> bg fill
    assert g.leaf_count() == 1
    g.deactivate((-1, -1, -1))
    assert not g.is_active((-1, -1, -1)) and g.get((-1, -1, -1)) == 2.5
    assert g.leaf_count() == 1                       # deactivate keeps the leaf
    g.remove_empty_leaves()
    assert g.leaf_count() == 0


# ---- the oracle's fast rebuild equals the literal loop -------------------

@pytest.mark.parametrize("hw", [1.0, 2.5, 3.0, 4.0])
def test_window_rebuild_equals_brute(oracle, hw):
    base = oracle.OGrid.sphere(7.3, [0.4, -1.2, 2.0], 1.0, 4.0)
    vx, vy, vz = oracle.uniform_velocity(1.0, [0.7, -0.35, 0.2])
    a1 = base.advect(vx, vy, vz, 1.0)
    a2 = base.advect(vx, vy, vz, 1.0)
    a1.rebuild(hw, brute=True)
    a2.rebuild(hw, brute=False)
    o1, m1, v1 = a1.arrays()
    o2, m2, v2 = a2.arrays()
    assert np.array_equal(o1, o2) and np.array_equal(m1, m2)
    assert np.array_equal(v1.view(np.uint32), v2.view(np.uint32))


# ---- independent numpy restatement of the sphere generator ---------------

def numpy_sphere_count(radius, center, vs, hw):
    band = hw * vs
    bg = np.float32(band)
    ext = radius + band
    inv = 1.0 / vs
    lo = [int(np.floor((center[a] - ext) * inv)) for a in range(3)]
    hi = [int(np.ceil((center[a] + ext) * inv)) for a in range(3)]
    i = np.arange(lo[0], hi[0] + 1, dtype=np.float64)[:, None, None]
    j = np.arange(lo[1], hi[1] + 1, dtype=np.float64)[None, :, None]
    k = np.arange(lo[2], hi[2] + 1, dtype=np.float64)[None, None, :]
    wx, wy, wz = i * vs - center[0], j * vs - center[1], k * vs - center[2]
    d = np.sqrt(wx * wx + wy * wy + wz * wz)
    sdf = (d - radius).astype(np.float32)
    on = np.abs(sdf) < bg
    ii, jj, kk = np.nonzero(on)
    leaves = set(zip((ii + lo[0]) >> 3, (jj + lo[1]) >> 3, (kk + lo[2]) >> 3))
    return int(on.sum()), len(leaves), sdf, on, lo


def test_parity_config_sphere_matches_numpy(oracle):
    """Sphere r=32 at (64,64,64), vs=1, hw=3: 77,366 active voxels in 434 leaves."""
    n, nl, sdf, on, lo = numpy_sphere_count(32.0, [64.0, 64.0, 64.0], 1.0, 3.0)
    g = oracle.OGrid.sphere(32.0, [64.0, 64.0, 64.0], 1.0, 3.0)
    assert (n, nl) == (77366, 434)
    assert g.active_voxel_count() == n and g.leaf_count() == nl
    o, m, v = g.arrays()
    bits = np.unpackbits(m.view(np.uint8).reshape(-1, 64), axis=1, bitorder="little").astype(bool)
    offs = np.arange(512)
    for li in range(0, len(o), 37):
        for off in offs[bits[li]]:
            x, y, z = o[li, 0] + (off >> 6), o[li, 1] + ((off >> 3) & 7), o[li, 2] + (off & 7)
            assert v[li, off] == sdf[x - lo[0], y - lo[1], z - lo[2]]
