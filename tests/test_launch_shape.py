"""Launch shapes of the stencil kernels do not change results.

The advect and reinitialisation kernels run at 128 threads per CTA over any
number of persistent CTAs, chosen on a level set's first step by the launch
autotuner (every candidate CTA count is launched on the same inputs and
timed).  Each leaf is computed by one CTA with the same arithmetic whatever
the CTA count, so every shape, and the autotuned step itself, must give
bit-identical leaves, masks and values.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

# (threads, CTAs, staging): 128 threads and staging 0 (cp.async row copies) are the only kernels built
SHAPES = [((128, 148 * 8, 0), (128, 148 * 8, 0)), ((128, 148 * 4, 0), (128, 148 * 2, 0)),
          ((128, 37, 0), (128, 19, 0)), ((128, 1, 0), (128, 1, 0)),
          ((128, 5, 0), (128, 148 * 6, 0)), ((128, 148 * 6, 0), (128, 2, 0))]


def _same(a, b):
    assert np.array_equal(a[0], b[0]), "leaf origins differ"
    assert np.array_equal(a[1], b[1]), "masks differ"
    assert np.array_equal(a[2].view(np.uint32), b[2].view(np.uint32)), "values differ"


def _vortex(precision, shape):
    from sharc.volrus_b200.method import LevelSet
    vs = 1 / 128
    ls = LevelSet.sphere(0.15, (0.35, 0.35, 0.35), vs, {"kind": "vortex", "vs": vs, "period": 3.0}, 0.5 * vs,
                         precision=precision, integrator=2)
    if shape is not None:
        ls.set_launch_shape(*shape)
    return ls


def _batched(precision, shape):
    from sharc.volrus_b200.method import LevelSet, random_sphere_grids
    gr = random_sphere_grids(6, seed=11, extent_log2=(5.0, 7.0), spheres=(1, 6), radius=(4.0, 10.0))
    ls = LevelSet.spheres([(s, v) for s, v, _ in gr], 1.0, precision=precision, integrator=3)
    if shape is not None:
        ls.set_launch_shape(*shape)
    return ls


@pytest.mark.parametrize("make", [_vortex, _batched], ids=["vortex_rk2", "batched_curl_rk3"])
@pytest.mark.parametrize("precision", [0, 1], ids=["f32", "f16"])
def test_results_independent_of_launch_shape(ctx, make, precision):
    steps = 5
    ref = make(precision, None)  # autotuned on its first step
    ref.step(steps)
    tuned = ref.launch_shape()
    assert tuned["advect"][0] == 128 and tuned["reinit"][0] == 128
    assert tuned["advect"][2] == 0 and tuned["reinit"][2] == 0
    assert all(us > 0 for *_, us in tuned["timed"])
    for k in ("k_m_advect", "k_m_reinit"):
        assert len({c for name, _, c, _, _ in tuned["timed"] if name == k}) >= 2, "several CTA counts are timed"
    want = ref.arrays()
    ref.close()
    for shape in SHAPES:
        ls = make(precision, shape)
        ls.step(steps)
        got = ls.launch_shape()
        assert got["advect"] == shape[0] and got["reinit"] == shape[1] and got["timed"] == []
        _same(ls.arrays(), want)
        ls.close()


def test_invalid_launch_shape_rejected(ctx):
    from sharc.volrus_b200._lib import VolrusError
    ls = _vortex(0, None)
    for bad in [((64, 100), (128, 100)), ((128, 0), (128, 100)), ((128, 100), (512, 100)),
                ((256, 100), (128, 100)), ((128, 100), (256, 100)), ((128, 100, 1), (128, 100, 0)),
                ((128, 100, 2), (128, 100, 0)), ((128, 100, 0), (128, 100, -1))]:
        with pytest.raises(VolrusError):
            ls.set_launch_shape(*bad)
    ls.close()


def _vortex_r(precision, radius):
    from sharc.volrus_b200.method import LevelSet
    vs = 1 / 512
    return LevelSet.sphere(radius, (0.5, 0.5, 0.5), vs, {"kind": "vortex", "vs": vs, "period": 3.0}, 0.5 * vs,
                           precision=precision, integrator=2)


@pytest.mark.parametrize("precision", [0, 1], ids=["f32", "f16"])
@pytest.mark.parametrize("radius", [None, 0.3], ids=["device_sort", "host_sort_over_8192_leaves"])
def test_host_step_matches_upload_step_download(ctx, precision, radius):
    """vlr_ls_step_host = vlr_ls_upload + vlr_ls_step + vlr_ls_download (the
    host step orders up to 8192 leaves on the device, more on the host)."""
    make = (lambda: _vortex(precision, None)) if radius is None else (lambda: _vortex_r(precision, radius))
    a = make()
    a.step(2)
    state = a.arrays()
    if radius is not None:
        assert len(state[0]) > 8192
    b = make()
    b.step(2)
    got = b.step_host(*state, n_steps=3)
    a.upload(*state)
    a.step(3)
    _same(got, a.arrays())
    a.close()
    b.close()
