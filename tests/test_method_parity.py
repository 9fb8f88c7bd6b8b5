"""GPU narrow-band method against the FP64 method oracle.

The method (RK backtrace, Godunov reinitialisation, re-tracking) has no
counterpart in the reference crate; the oracle (oracle/method_oracle.hpp)
defines it in FP64 and the GPU must agree to f32 / f16 rounding:
  * initial state: identical leaves and masks, values equal to the f32
    rounding of the oracle's f64 values;
  * after steps: identical leaf sets, mask differences only at voxels whose
    oracle value lies within 1e-3 of the half width (threshold flips),
    value errors within the tolerances written below.
"""
import numpy as np
import pytest

from tests.method_compare import compare

pytestmark = pytest.mark.gpu

TOL_F32 = 2e-4   # voxels, max |phi_gpu - phi_fp64| over 8 steps in FP32
TOL_F16 = 8e-3   # voxels, same in FP16 storage (half ulp at 3 voxels is 1e-3)


def run_pair(oracle, vel, integrator, steps, precision, radius=10.0, center=(3.2, -1.7, 0.6), vs=1.0, dt=1.0, w0=(0, 0, 0)):
    from sharc.volrus_b200.method import LevelSet
    ls = LevelSet.sphere(radius, center, vs, vel, dt, half_width=3.0, precision=precision, integrator=integrator,
                         w0=w0)
    og = oracle.MOGrid.sphere(radius, center, vs, 3.0, w0)
    stats = []
    for s in range(steps):
        ls.step(1)
        ok = og.step(vel, integrator, 2, s * dt, dt, 8)
        assert ok
        stats.append(compare(ls.arrays(), og.arrays(), 3.0))
    return ls, og, stats


def test_initial_sphere_exact(oracle):
    from sharc.volrus_b200.method import F32, LevelSet
    vel = {"kind": "constant", "c": (0.3, 0.2, 0.1)}
    ls = LevelSet.sphere(0.15, (0.35, 0.35, 0.35), 1 / 512, vel, 1.0, precision=F32)
    og = oracle.MOGrid.sphere(0.15, (0.35, 0.35, 0.35), 1 / 512, 3.0)
    go, gm, gv = ls.arrays()
    oo, om, ov = og.arrays()
    assert np.array_equal(go, oo) and np.array_equal(gm, om)
    assert np.array_equal(gv, ov.astype(np.float32))
    assert ls.active_voxel_count() == 444838


@pytest.mark.parametrize("precision,tol", [(0, TOL_F32), (1, TOL_F16)])
def test_constant_velocity_euler(oracle, precision, tol):
    _, _, st = run_pair(oracle, {"kind": "constant", "c": (0.7, -0.45, 0.3)}, 1, 8, precision)
    for s in st:
        assert s["only_gpu"] == 0 and s["only_oracle"] == 0, s
        assert s["unexplained_flips"] == 0, s
        assert s["max_err"] < tol, s


@pytest.mark.parametrize("precision,tol", [(0, TOL_F32), (1, TOL_F16)])
def test_vortex_rk2(oracle, precision, tol):
    vel = {"kind": "vortex", "vs": 1 / 128, "period": 3.0}
    _, _, st = run_pair(oracle, vel, 2, 8, precision, radius=0.15, center=(0.35, 0.35, 0.35), vs=1 / 128,
                        dt=0.5 / (128 * 2))
    for s in st:
        assert s["only_gpu"] == 0 and s["only_oracle"] == 0, s
        assert s["unexplained_flips"] == 0, s
        assert s["max_err"] < tol, s


@pytest.mark.parametrize("precision,tol", [(0, TOL_F32), (1, TOL_F16)])
def test_curl_noise_rk3(oracle, precision, tol):
    from sharc.volrus_b200.method import curl_noise
    vel = curl_noise(5, 64.0, amplitude=1.0)
    _, _, st = run_pair(oracle, vel, 3, 8, precision, radius=12.0, center=(30.0, 33.0, 29.0))
    for s in st:
        assert s["only_gpu"] == 0 and s["only_oracle"] == 0, s
        assert s["unexplained_flips"] == 0, s
        assert s["max_err"] < tol, s


@pytest.mark.parametrize("precision,tol", [(0, TOL_F32), (1, TOL_F16)])
def test_batched_uneven_grids_rk3(oracle, precision, tol):
    """Several grids of unions of spheres with their own curl noise in one pool:
    every grid matches its own FP64 oracle run."""
    from sharc.volrus_b200.method import LevelSet, random_sphere_grids
    grids = random_sphere_grids(5, seed=11, extent_log2=(5.0, 6.5), spheres=(1, 6), radius=(3.0, 9.0))
    ls = LevelSet.spheres([(s, v) for s, v, _ in grids], 1.0, precision=precision, integrator=3)
    og = [oracle.MOGrid.spheres(s, 3.0) for s, _, _ in grids]
    for g, (_, v, _) in enumerate(grids):
        st = compare(ls.grid_arrays(g), og[g].arrays(), 3.0)
        assert st["only_gpu"] == 0 and st["only_oracle"] == 0 and st["mask_flips"] == 0, (g, st)
    for step in range(6):
        ls.step(1)
        for g, (_, v, _) in enumerate(grids):
            assert og[g].step(v, 3, 2, float(step), 1.0, 8)
    for g in range(len(grids)):
        st = compare(ls.grid_arrays(g), og[g].arrays(), 3.0)
        assert st["only_gpu"] == 0 and st["only_oracle"] == 0, (g, st)
        assert st["unexplained_flips"] == 0, (g, st)
        assert st["max_err"] < tol, (g, st)


def test_volume_fp64(oracle):
    from sharc.volrus_b200.method import F32, LevelSet
    vel = {"kind": "constant", "c": (0.3, 0.2, 0.1)}
    ls = LevelSet.sphere(0.15, (0.35, 0.35, 0.35), 1 / 512, vel, 1.0, precision=F32)
    og = oracle.MOGrid.sphere(0.15, (0.35, 0.35, 0.35), 1 / 512, 3.0)
    vg, vo = ls.volume(), og.volume()
    assert abs(vg - vo) / vo < 1e-6
    exact = 4.0 / 3.0 * np.pi * (0.15 * 512) ** 3
    assert abs(vo - exact) / exact < 1e-3
