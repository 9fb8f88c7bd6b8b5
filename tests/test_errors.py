"""Error paths of the level-set step, exercised without faulting or hanging a GPU.

* VLR_ERR_TIMEOUT: the look-back scan of a step waits on its predecessors'
  published prefixes with a bounded number of polls.  The test hook
  vlr_ctx_test_stall makes the first chunk withhold its prefix (a flag that
  nothing sets), and vlr_ctx_set_wait_limit shortens the bound, so the later
  chunks' waits run out: the step returns VLR_ERR_TIMEOUT, the rest of the
  step is abandoned on the device, the level set refuses further steps
  (VLR_ERR_INVALID) until a state is uploaded, and after that a step at the
  default bound is bit-identical to a clean run from the same state.
* VLR_ERR_REACH: a time step whose displacement bound exceeds the staged
  halo is refused when the level set is created; a grid that leaves its
  velocity's sampled domain reports REACH from the step instead of sampling
  a clamped table silently.
* VLR_ERR_CAPACITY: a level set created with too small a leaf capacity for
  the band it grows into reports CAPACITY from the step and then refuses
  further steps.
* VLR_ERR_NOMEM: a leaf capacity beyond the device's free memory fails the
  creation with NOMEM before the level set's arrays are allocated, and the
  temporaries allocated before the failure are released (device free memory
  is unchanged).
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _codes():
    from sharc.volrus_b200._lib import ERROR_NAMES
    return {v: k for k, v in ERROR_NAMES.items()}


def _sphere(ctx, precision, vel=None, capacity=0, radius=40.0):
    from sharc.volrus_b200.method import LevelSet
    vel = vel or {"kind": "constant", "c": (0.6, -0.35, 0.2)}
    return LevelSet.sphere(radius, (3.0, -5.0, 7.0), 1.0, vel, 1.0, half_width=3.0, precision=precision,
                           integrator=2, reinit_iters=2, capacity=capacity, ctx=ctx)


@pytest.mark.parametrize("precision", [0, 1], ids=["f32", "f16"])
def test_timeout_is_reported_and_the_next_clean_step_is_exact(ctx, precision):
    from sharc.volrus_b200 import VolrusError
    codes = _codes()
    ls = _sphere(ctx, precision, radius=60.0)
    ref = _sphere(ctx, precision, radius=60.0)
    assert ls.leaf_count() > 3 * 256  # several chunks in the look-back scan
    ls.step(1)  # the first step tunes the launch shapes
    ref.step(1)
    o, m, p = ls.arrays()
    ctx.check(ctx.lib.vlr_ctx_set_wait_limit(ctx.handle, 2000), "vlr_ctx_set_wait_limit")
    ctx.check(ctx.lib.vlr_ctx_test_stall(ctx.handle, 1), "vlr_ctx_test_stall")
    try:
        with pytest.raises(VolrusError) as e:
            ls.step(2)
        assert e.value.code == codes["VLR_ERR_TIMEOUT"]
    finally:
        ctx.check(ctx.lib.vlr_ctx_test_stall(ctx.handle, 0), "vlr_ctx_test_stall")
        ctx.check(ctx.lib.vlr_ctx_set_wait_limit(ctx.handle, 0), "vlr_ctx_set_wait_limit")
    with pytest.raises(VolrusError) as e:
        ls.step(1)
    assert e.value.code == codes["VLR_ERR_INVALID"]
    # a new state (the one before the failed step, at the same step counter)
    ls.upload(o, m, p)
    ls.set_step(1)
    ls.step(1)
    ref.step(1)
    o1, m1, p1 = ls.arrays()
    o2, m2, p2 = ref.arrays()
    assert np.array_equal(o1, o2) and np.array_equal(m1, m2)
    assert np.array_equal(p1.view(np.uint32), p2.view(np.uint32))
    ls.close()
    ref.close()


def test_reach_refused_at_creation(ctx):
    from sharc.volrus_b200 import VolrusError
    with pytest.raises(VolrusError) as e:
        _sphere(ctx, 1, vel={"kind": "constant", "c": (2.5, 0.0, 0.0)})
    assert e.value.code == _codes()["VLR_ERR_REACH"]


def test_reach_outside_velocity_domain(ctx):
    from sharc.volrus_b200 import VolrusError
    from sharc.volrus_b200.method import curl_noise
    vel = curl_noise(5, 256.0, 0.8, 3)
    vel["domain"] = ((0, 0, 0), (256, 256, 256))  # the sphere reaches negative coordinates
    ls = _sphere(ctx, 1, vel=vel, radius=20.0)
    with pytest.raises(VolrusError) as e:
        ls.step(1)
    assert e.value.code == _codes()["VLR_ERR_REACH"]
    ls.close()


def test_capacity_overflow_abandons_the_step(ctx):
    from sharc.volrus_b200 import VolrusError
    codes = _codes()
    probe = _sphere(ctx, 1, radius=12.0)
    n0 = probe.leaf_count()
    probe.close()
    ls = _sphere(ctx, 1, radius=12.0, capacity=n0 + 2, vel={"kind": "constant", "c": (0.9, 0.9, 0.9)})
    with pytest.raises(VolrusError) as e:
        ls.step(6)
    assert e.value.code == codes["VLR_ERR_CAPACITY"]
    with pytest.raises(VolrusError) as e:
        ls.step(1)
    assert e.value.code == codes["VLR_ERR_INVALID"]
    ls.close()


def test_nomem_releases_everything(ctx):
    import torch
    from sharc.volrus_b200 import VolrusError
    warm = _sphere(ctx, 1, radius=12.0)
    warm.close()
    ctx.synchronize()
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    with pytest.raises(VolrusError) as e:
        _sphere(ctx, 1, radius=12.0, capacity=1 << 30)  # ~1 TB of leaf values
    assert e.value.code == _codes()["VLR_ERR_NOMEM"]
    ctx.synchronize()
    torch.cuda.synchronize()
    assert torch.cuda.mem_get_info()[0] == free0
    ok = _sphere(ctx, 1, radius=12.0)  # the context still works
    ok.step(1)
    ok.close()
