"""GPU parity of the reference-semantics path against the CPU oracle.

Every comparison is bit-exact: leaf topology, activity masks and the f32
bit patterns of all 512 values of every leaf (inactive voxels included),
because the CUDA kernels keep the reference's operation order and rounding.
Inputs are seeded; sizes keep the oracle to seconds.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def assert_same(dev_grid, og):
    o1, m1, v1 = dev_grid.to_arrays() if hasattr(dev_grid, "to_arrays") else dev_grid
    o2, m2, v2 = og.arrays()
    assert o1.shape == o2.shape, f"leaf count {len(o1)} vs oracle {len(o2)}"
    assert np.array_equal(o1, o2), "leaf origins differ"
    assert np.array_equal(m1, m2), "activity masks differ"
    bad = np.nonzero(v1.view(np.uint32) != v2.view(np.uint32))
    assert bad[0].size == 0, (f"{bad[0].size} values differ, first leaf {o1[bad[0][0]]} off {bad[1][0]}: "
                              f"{v1[bad][0]!r} vs {v2[bad][0]!r}")


def to_oracle(oracle, g):
    o, m, v = g.to_arrays()
    return oracle.OGrid.from_arrays(o, m, v, g.background, g.transform.voxel_size, g.transform.origin,
                                    g.affine.mat, g.affine.voxel_size)


def random_grid(rng, n_leaves, spread, bg, vs=1.0, fill=0.5):
    from sharc.volrus_b200 import Grid
    origins = set()
    while len(origins) < n_leaves:
        origins.add(tuple(int(x) * 8 for x in rng.integers(-spread, spread, 3)))
    o = np.array(sorted(origins), np.int32)
    on = rng.random((n_leaves, 512)) < fill
    m = np.packbits(on, axis=1, bitorder="little").view(np.uint64)
    v = np.where(on, rng.normal(0, 2.0, (n_leaves, 512)), bg).astype(np.float32)
    return Grid.from_arrays(o, m, v, bg, None)


SPHERES = [
    (5.0, (0.0, 0.0, 0.0), 1.0, 3.0),
    (5.0, (0.0, 0.0, 0.0), 0.5, 3.0),
    (3.0, (10.0, 20.0, 30.0), 0.5, 3.0),
    (32.0, (64.0, 64.0, 64.0), 1.0, 3.0),
    (11.7, (-40.3, 17.1, -3.9), 0.75, 2.5),
]


@pytest.mark.parametrize("args", SPHERES)
def test_sphere_generator_bit_exact(oracle, args):
    from sharc.volrus_b200 import make_level_set_sphere
    g = make_level_set_sphere(*args)
    og = oracle.OGrid.sphere(*args)
    assert_same(g, og)
    assert g.background == og.meta()[0]


def test_sample_trilinear_bit_exact(oracle):
    from sharc.volrus_b200 import make_level_set_sphere, sample_trilinear
    rng = np.random.default_rng(1)
    g = make_level_set_sphere(9.0, (1.0, 2.0, -3.0), 0.5, 3.0)
    og = to_oracle(oracle, g)
    pts = rng.uniform(-8, 8, (20000, 3)) + np.array([1.0, 2.0, -3.0])
    gpu = sample_trilinear(g, pts)
    cpu = og.sample_trilinear(pts)
    assert np.array_equal(gpu.view(np.uint32), cpu.view(np.uint32))


def test_reference_trilinear_kats():  # src/tools/interpolation.rs:55-90
    from sharc.volrus_b200 import Grid, sample_trilinear
    g = Grid(0.0, 1.0)
    g.set((5, 5, 5), 42.0)
    assert abs(sample_trilinear(g, [5.0, 5.0, 5.0]) - 42.0) < 1e-6
    g = Grid(0.0, 1.0)
    g.set((0, 0, 0), 0.0)
    g.set((1, 0, 0), 10.0)
    assert abs(sample_trilinear(g, [0.5, 0.0, 0.0]) - 5.0) < 1e-5
    g = Grid(0.0, 0.5)
    g.set((0, 0, 0), 0.0)
    g.set((1, 0, 0), 10.0)
    assert abs(sample_trilinear(g, [0.25, 0.0, 0.0]) - 5.0) < 1e-5


def test_reference_advection_kat():  # src/tools/advection.rs:151-197
    from sharc.volrus_b200 import advect_level_set, make_level_set_sphere, make_uniform_velocity, sample_trilinear
    grid = make_level_set_sphere(5.0, [0.0, 0.0, 0.0], 0.5, 3.0)
    vel = make_uniform_velocity(0.5, [1.0, 0.0, 0.0], (-30, -30, -30), (30, 30, 30))
    adv = advect_level_set(grid, vel, 1.0)
    assert abs(sample_trilinear(adv, [6.0, 0.0, 0.0])) < 1.0
    assert sample_trilinear(adv, [5.0, 0.0, 0.0]) < 0.0
    assert sample_trilinear(adv, [7.0, 0.0, 0.0]) > 0.0


@pytest.mark.parametrize("vel,dt", [((1.0, 0.5, 0.25), 1.0), ((0.3, -1.7, 0.9), 0.8), ((2.5, 0.0, -3.25), 1.0)])
def test_advect_constant_velocity_bit_exact(oracle, vel, dt):
    from sharc.volrus_b200 import advect_level_set, make_level_set_sphere, make_uniform_velocity
    g = make_level_set_sphere(12.0, (3.0, -2.0, 5.0), 1.0, 3.0)
    v = make_uniform_velocity(1.0, vel)
    out = advect_level_set(g, v, dt)
    og = to_oracle(oracle, g)
    ov = oracle.uniform_velocity(1.0, vel)
    assert_same(out, og.advect(*ov, dt))


def test_advect_sparse_velocity_grids_bit_exact(oracle):
    """Velocity from three sparse grids with their own leaves and transforms."""
    from sharc.volrus_b200 import (Grid, VelocityField, VoxelTransform, advect_level_set,
                                   make_level_set_sphere)
    rng = np.random.default_rng(7)
    g = make_level_set_sphere(10.0, (0.0, 0.0, 0.0), 0.5, 3.0)
    comps, ocomps = [], []
    for a in range(3):
        c = random_grid(rng, 60, 4, float(rng.normal()), fill=0.9)
        c.set_transform(VoxelTransform.with_origin(0.7, (0.1 * a, -0.2, 0.3)))
        c._v *= 0.4
        comps.append(c)
        ocomps.append(to_oracle(oracle, c))
    out = advect_level_set(g, VelocityField(*comps), 1.3)
    og = to_oracle(oracle, g)
    assert_same(out, og.advect(*ocomps, 1.3))


def test_advect_transform_with_translation(oracle):
    """with_affine drops the translation from the legacy transform (src/grid.rs:378-388)."""
    from sharc.volrus_b200 import VoxelTransform, advect_level_set, make_level_set_sphere, make_uniform_velocity
    g = make_level_set_sphere(6.0, (0.0, 0.0, 0.0), 1.0, 3.0)
    g.set_transform(VoxelTransform.with_origin(1.0, (0.25, -0.5, 0.125)))
    v = make_uniform_velocity(1.0, (0.5, 0.25, -0.75))
    out = advect_level_set(g, v, 1.0)
    og = to_oracle(oracle, g)
    ref = og.advect(*oracle.uniform_velocity(1.0, (0.5, 0.25, -0.75)), 1.0)
    assert_same(out, ref)
    assert out.transform.origin == (0.0, 0.0, 0.0)
    assert tuple(ref.meta()[2]) == (0.0, 0.0, 0.0)


def test_advect_random_leaves_and_empty_leaves(oracle):
    """Random values, negative coordinates, and allocated leaves with no active
    voxel (not allocated in the advected output)."""
    from sharc.volrus_b200 import advect_level_set, make_uniform_velocity
    rng = np.random.default_rng(3)
    g = random_grid(rng, 200, 6, 1.5, fill=0.3)
    g._m[:10] = 0
    out = advect_level_set(g, make_uniform_velocity(1.0, (1.3, -0.6, 2.2)), 1.0)
    og = to_oracle(oracle, g)
    assert_same(out, og.advect(*oracle.uniform_velocity(1.0, (1.3, -0.6, 2.2)), 1.0))
    assert out.leaf_count() == 190


def test_advect_far_backtrace_uses_hash(oracle):
    """Backtraces several leaves away fall outside the neighbour table."""
    from sharc.volrus_b200 import advect_level_set, make_level_set_sphere, make_uniform_velocity
    g = make_level_set_sphere(20.0, (0.0, 0.0, 0.0), 1.0, 3.0)
    vel = (13.0, -21.5, 9.25)
    out = advect_level_set(g, make_uniform_velocity(1.0, vel), 1.0)
    assert_same(out, to_oracle(oracle, g).advect(*oracle.uniform_velocity(1.0, vel), 1.0))


def test_empty_grid_ops(oracle):
    from sharc.volrus_b200 import (Grid, advect_level_set, find_zero_crossings, make_uniform_velocity,
                                   rebuild_narrow_band, trim_narrow_band)
    g = Grid.level_set(1.0, 3.0)
    out = advect_level_set(g, make_uniform_velocity(1.0, (1, 0, 0)), 1.0)
    assert out.leaf_count() == 0
    assert len(find_zero_crossings(g)) == 0
    trim_narrow_band(g, 2.0)
    rebuild_narrow_band(g, 3.0)
    assert g.active_voxel_count() == 0


@pytest.mark.parametrize("args", SPHERES[:4])
def test_zero_crossings_exact(oracle, args):
    from sharc.volrus_b200 import find_zero_crossings, make_level_set_sphere
    g = make_level_set_sphere(*args)
    assert np.array_equal(find_zero_crossings(g), to_oracle(oracle, g).zero_crossings())


def test_zero_crossings_exact_zero_and_inactive_neighbours(oracle):
    """val == 0 is a crossing; inactive neighbours never count (level_set_track.rs:27-43)."""
    from sharc.volrus_b200 import find_zero_crossings
    rng = np.random.default_rng(11)
    g = random_grid(rng, 80, 3, 2.0, fill=0.6)
    g._v[g._v.__abs__() < 0.3] = 0.0
    g._v[5, :64] = -0.0
    assert np.array_equal(find_zero_crossings(g), to_oracle(oracle, g).zero_crossings())


@pytest.mark.parametrize("hw", [2.0, 3.0, 5.0])
def test_trim_bit_exact(oracle, hw):
    from sharc.volrus_b200 import make_level_set_sphere, trim_narrow_band
    g = make_level_set_sphere(9.0, (0.5, 0.25, -1.0), 1.0, 5.0)
    og = to_oracle(oracle, g)
    trim_narrow_band(g, hw)
    og.trim(hw)
    assert_same(g, og)


def test_dilate_single_voxel_kat(oracle):  # src/tools/morphology.rs:88-111
    from sharc.volrus_b200 import Grid, dilate
    g = Grid(0.0, 1.0)
    g.set((0, 0, 0), 1.0)
    dilate(g, 1)
    assert g.active_voxel_count() == 7
    for c in ((1, 0, 0), (-1, 0, 0), (0, 1, 0), (0, -1, 0), (0, 0, 1), (0, 0, -1)):
        assert g.is_active(c) and g.get(c) == 1.0


@pytest.mark.parametrize("iterations", [1, 3])
def test_dilate_sphere_bit_exact(oracle, iterations):
    from sharc.volrus_b200 import dilate, make_level_set_sphere
    g = make_level_set_sphere(9.0, (0.5, 0.25, -1.0), 1.0, 2.0)
    og = to_oracle(oracle, g)
    dilate(g, iterations)
    og.dilate(iterations)
    assert_same(g, og)


@pytest.mark.parametrize("seed", [0, 1])
def test_dilate_order_dependent_values_bit_exact(oracle, seed):
    """Sparse voxels with distinct values over several 128^3 tiles (negative
    coordinates included): a new voxel between active voxels takes the value
    of the one first in iteration order, so values pin the order."""
    from sharc.volrus_b200 import dilate
    g = random_grid(np.random.default_rng(seed), 120, 24, -2.5, fill=0.08)
    og = to_oracle(oracle, g)
    dilate(g, 2)
    og.dilate(2)
    assert_same(g, og)


@pytest.mark.parametrize("hw", [0.0, 1.0, 2.5, 3.0, 7.5, 9.0, 12.0])
def test_rebuild_bit_exact(oracle, hw):
    """Window path (hw <= 9) and literal O(N x M) path (hw > 9)."""
    from sharc.volrus_b200 import (advect_level_set, make_level_set_sphere, make_uniform_velocity,
                                   rebuild_narrow_band)
    g = make_level_set_sphere(10.0, (0.3, -0.7, 1.1), 1.0, max(hw, 3.0) + 1.0)
    a = advect_level_set(g, make_uniform_velocity(1.0, (0.6, -0.4, 0.3)), 1.0)
    oa = to_oracle(oracle, a)
    rebuild_narrow_band(a, hw)
    oa.rebuild(hw, brute=True)
    assert_same(a, oa)


def test_reference_pipeline_config1_20_steps(oracle):
    """Sphere r=32 in a 128^3 domain, v=(1, 0.5, 0.25), dt=1, hw=3: 20 steps of
    advect_level_set + rebuild_narrow_band, compared to the oracle after every
    step on the same input."""
    from sharc.volrus_b200 import (DeviceGrid, advect_level_set, make_level_set_sphere, make_uniform_velocity,
                                   rebuild_narrow_band)
    g = make_level_set_sphere(32.0, (64.0, 64.0, 64.0), 1.0, 3.0, device=True)
    vel = make_uniform_velocity(1.0, (1.0, 0.5, 0.25))
    dvel = [DeviceGrid.upload(c, g.ctx) for c in (vel.vx, vel.vy, vel.vz)]
    ovel = oracle.uniform_velocity(1.0, (1.0, 0.5, 0.25))
    from sharc.volrus_b200 import VelocityField
    for step in range(20):
        host_in = g.download()
        og = to_oracle(oracle, host_in)
        g = advect_level_set(g, VelocityField(*dvel), 1.0)
        rebuild_narrow_band(g, 3.0)
        ref = og.advect(*ovel, 1.0)
        ref.rebuild(3.0)
        assert_same(g.download(), ref)
        if g.leaf_count() == 0:
            break


def test_host_buffer_entry_point(oracle):
    """vlr_advect_rebuild_host: the whole reference step from host arrays."""
    import ctypes as C
    from sharc.volrus_b200 import Context, make_level_set_sphere
    from sharc.volrus_b200._lib import ptr
    ctx = Context.default()
    g = make_level_set_sphere(16.0, (0.0, 0.0, 0.0), 1.0, 3.0)
    o, m, v = g.to_arrays()
    cap = len(o) + 64
    oo = np.zeros((cap, 3), np.int32)
    om = np.zeros((cap, 8), np.uint64)
    ov = np.zeros((cap, 512), np.float32)
    nout = C.c_size_t()
    vel = np.array([0.75, -0.5, 0.25], np.float32)
    t = g.c_transform()
    ctx.check(ctx.lib.vlr_advect_rebuild_host(ctx.handle, C.byref(t), C.c_float(g.background), ptr(o, C.c_int32),
                                              ptr(m, C.c_uint64), ptr(v, C.c_float), len(o), ptr(vel, C.c_float),
                                              1.0, C.c_float(3.0), ptr(oo, C.c_int32), ptr(om, C.c_uint64),
                                              ptr(ov, C.c_float), cap, C.byref(nout)))
    n = nout.value
    og = to_oracle(oracle, g)
    ref = og.advect(*oracle.uniform_velocity(1.0, vel), 1.0)
    ref.rebuild(3.0)
    assert_same((oo[:n], om[:n], ov[:n]), ref)


def test_invalid_inputs_raise():
    from sharc.volrus_b200 import Grid, VolrusError
    from sharc.volrus_b200.tools import DeviceGrid
    g = Grid.from_arrays(np.array([[0, 0, 3]], np.int32), np.zeros((1, 8), np.uint64),
                         np.zeros((1, 512), np.float32), 1.0)
    with pytest.raises(VolrusError, match="INVALID"):
        DeviceGrid.upload(g)
    g = Grid.from_arrays(np.array([[0, 0, 8], [0, 0, 8]], np.int32), np.zeros((2, 8), np.uint64),
                         np.zeros((2, 512), np.float32), 1.0)
    with pytest.raises(VolrusError, match="INVALID"):
        DeviceGrid.upload(g)
    g = Grid.from_arrays(np.array([[0, 0, 0], [1 << 26, 0, 0]], np.int32), np.zeros((2, 8), np.uint64),
                         np.zeros((2, 512), np.float32), 1.0)
    with pytest.raises(VolrusError, match="EXTENT"):
        DeviceGrid.upload(g)
