"""The allocation-free crossing search matches the regular entry point.

``vlr_find_zero_crossings_noalloc`` serves callers that cannot allocate
device memory when they need the crossings (inside a stream capture, in a
real-time loop, or when another allocator owns the device memory).  It keeps
its scratch in one fixed device array shared by all calls, so this test calls
it twice in a row on different grids through the C ABI and checks each
result against ``vlr_find_zero_crossings`` and against the CPU oracle's
restatement of the crate's ``find_zero_crossings`` on the same leaves (exact:
all are integer coordinates), which also shows that the second call does not
see the first call's leftovers.  It also checks that a call leaves the
calling thread's current device unchanged.  The file name makes pytest
collect it last.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def crossings_noalloc(ctx, dev_grid, cap):
    import torch
    coords = torch.full((max(cap, 1), 3), -7, dtype=torch.int32, device="cuda")
    count = torch.zeros(1, dtype=torch.int64, device="cuda")
    torch.cuda.synchronize()
    ctx.check(ctx.lib.vlr_find_zero_crossings_noalloc(ctx.handle, dev_grid.handle, C.c_void_p(coords.data_ptr()),
                                                      cap, C.c_void_p(count.data_ptr())),
              "vlr_find_zero_crossings_noalloc")
    ctx.synchronize()
    n = int(count.item())
    return coords[: min(n, cap)].cpu().numpy(), n


def sorted_rows(a):
    a = np.asarray(a).reshape(-1, 3)
    return a[np.lexsort((a[:, 2], a[:, 1], a[:, 0]))]


def test_noalloc_matches_regular_entry_point_twice_in_a_row():
    from sharc.volrus_b200 import (Context, advect_level_set, find_zero_crossings, make_level_set_sphere,
                                   make_uniform_velocity)
    ctx = Context.default(0)
    big = make_level_set_sphere(32.0, (64.0, 64.0, 64.0), 1.0, 3.0, ctx=ctx, device=True)
    small = advect_level_set(make_level_set_sphere(9.0, (-3.0, 5.0, 1.5), 0.5, 3.0, ctx=ctx, device=True),
                             make_uniform_velocity(0.5, (0.3, -0.2, 0.7)), 1.0)
    import torch
    from oracle import pyoracle
    for g in (big, small):
        ref = find_zero_crossings(g)
        host = g.download()
        o, m, v = host.to_arrays()
        og = pyoracle.OGrid.from_arrays(o, m, v, host.background, host.transform.voxel_size)
        dev_before = torch.cuda.current_device()
        got, n = crossings_noalloc(ctx, g, len(ref) + 16)
        assert torch.cuda.current_device() == dev_before
        assert n == len(ref) > 0
        assert np.array_equal(sorted_rows(got), ref)
        assert np.array_equal(sorted_rows(got), sorted_rows(og.zero_crossings()))


def test_noalloc_reports_total_beyond_cap_and_rejects_large_grids():
    from sharc.volrus_b200 import Context, VolrusError, find_zero_crossings, make_level_set_sphere
    ctx = Context.default(0)
    g = make_level_set_sphere(12.0, (0.0, 0.0, 0.0), 1.0, 3.0, ctx=ctx, device=True)
    ref = find_zero_crossings(g)
    got, n = crossings_noalloc(ctx, g, 10)
    assert n == len(ref) and len(got) == 10
    assert set(map(tuple, got)) <= set(map(tuple, ref))
    huge = make_level_set_sphere(520.0, (0.0, 0.0, 0.0), 1.0, 3.0, ctx=ctx, device=True)
    assert huge.leaf_count() > 65536
    with pytest.raises(VolrusError, match="CAPACITY"):
        crossings_noalloc(ctx, huge, 16)
