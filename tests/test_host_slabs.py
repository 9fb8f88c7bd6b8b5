"""vlr_ls_step_host over x-slabs against the one-pass host step.

A 1,100-sphere grid in a 4096^3 extent (about 340k leaves, curl noise,
SSP-RK3, two reinitialisation iterations) steps once through the host form
with its buffers pinned: in one pass (slab count 1) and as pipelines of 2, 5
and 16 slabs and of the automatic count.  The results are bit for bit the
one pass's, and so is the level set's state afterwards (downloaded, and
stepped once more on the device).  Unsorted input and pageable buffers take
the one pass; output buffers too small fail with VLR_ERR_CAPACITY and leave
the state to the next upload.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

_TORCH = {np.int32: "int32", np.uint64: "int64", np.float32: "float32"}


def _pinned(a):
    import torch
    t = torch.empty(a.shape, dtype=getattr(torch, _TORCH[a.dtype.type]), pin_memory=True).numpy()
    if a.dtype == np.uint64:
        t = t.view(np.uint64)
    t[:] = a
    return t


def _out(cap, pinned=True):
    z = (np.zeros((cap, 3), np.int32), np.zeros((cap, 8), np.uint64), np.zeros((cap, 512), np.float32))
    return tuple(_pinned(a) for a in z) if pinned else z


def _same(a, b):
    return (len(a[0]) == len(b[0]) and np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1])
            and np.array_equal(a[2].view(np.uint32), b[2].view(np.uint32)))


@pytest.fixture(scope="module", params=[1, 0], ids=["f16", "f32"])
def grid(request):
    from sharc.volrus_b200.method import LevelSet, large_sphere_grid
    sph, vel = large_sphere_grid(1100, seed=11, extent=4096.0)
    ls = LevelSet.spheres([(sph, vel)], 1.0, half_width=3.0, precision=request.param, integrator=3, reinit_iters=2)
    o, m, v = ls.arrays()
    assert len(o) > 1 << 18  # the automatic count takes at least two slabs
    yield ls, (_pinned(o), _pinned(m), _pinned(v))
    ls.close()


def _host_step(ls, inp, slabs, out=None):
    ls.set_host_slabs(slabs)
    ls.set_step(0)
    n = len(inp[0])
    r = ls.step_host(*inp, 1, out=out if out is not None else _out(2 * n + 64))
    return tuple(np.array(a) for a in r)


def test_slabs_equal_one_pass(grid):
    ls, inp = grid
    ref = _host_step(ls, inp, 1)
    ref_state = ls.arrays()
    assert _same(ref, ref_state)
    ls.step(1)
    ref_next = ls.arrays()
    for slabs in (2, 5, 16, 0):
        got = _host_step(ls, inp, slabs)
        assert _same(got, ref), slabs
        assert _same(ls.arrays(), ref), slabs  # the pool holds the stepped state
        ls.step(1)
        assert _same(ls.arrays(), ref_next), slabs


def test_unsorted_and_pageable_take_one_pass(grid):
    ls, inp = grid
    ref = _host_step(ls, inp, 1)
    rev = tuple(_pinned(np.ascontiguousarray(a[::-1])) for a in inp)
    assert _same(_host_step(ls, rev, 4), ref)
    page = tuple(np.array(a) for a in inp)
    assert _same(_host_step(ls, page, 4, out=_out(2 * len(inp[0]) + 64, pinned=False)), ref)


def test_slabs_output_too_small(grid):
    from sharc.volrus_b200 import VolrusError
    ls, inp = grid
    n = len(inp[0])
    with pytest.raises(VolrusError):
        _host_step(ls, inp, 4, out=_out(n // 2))
    with pytest.raises(VolrusError):
        ls.step(1)  # the state waits for an upload
    ref = _host_step(ls, inp, 1)
    assert _same(_host_step(ls, inp, 4), ref)


def test_slabs_on_a_fresh_level_set(grid):
    """A level set whose first step is a slab pipeline (the launch autotuner
    runs inside the first slab) gives the one pass's result."""
    from sharc.volrus_b200.method import LevelSet, large_sphere_grid
    ls, inp = grid
    ref = _host_step(ls, inp, 1)
    sph, vel = large_sphere_grid(1100, seed=11, extent=4096.0)
    fresh = LevelSet.spheres([(sph, vel)], 1.0, half_width=3.0, precision=ls.precision, integrator=3,
                             reinit_iters=2)
    try:
        assert _same(_host_step(fresh, inp, 4), ref)
    finally:
        fresh.close()


def test_slabs_on_library_pinned_buffers(grid):
    """Buffers from vlr_host_alloc (what a caller without a CUDA runtime of
    its own uses) take the slab pipeline and give the one pass's result."""
    ls, inp = grid
    ref = _host_step(ls, inp, 1)
    ctx = ls.ctx
    lib_in = []
    for a in inp:
        b = ctx.pinned(a.shape, a.dtype)
        b[:] = a
        lib_in.append(b)
    cap = 2 * len(inp[0]) + 64
    out = tuple(ctx.pinned((cap,) + a.shape[1:], a.dtype) for a in inp)
    assert _same(_host_step(ls, tuple(lib_in), 4, out=out), ref)
