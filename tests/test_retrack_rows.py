"""Neighbour rows carried across steps against rows rebuilt whole.

A step keeps every survivor's 27-neighbour row and updates it only where a
neighbour was dropped or is new (k_t_nbr).  Here one level set steps on the
device, so its rows are carried from step to step, and a second one is
uploaded from the first's downloaded state before each step, so its rows are
built whole from the hash; after every step both states are bit for bit the
same (origins, masks, values).  The grids move about a voxel per step, so
every step drops and adds leaves: a 300-sphere curl-noise grid, FP16 and
FP32.  (Batches cannot be uploaded; their rows are checked by the batched
parity tests against the FP64 oracle.)
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

STEPS = 6


def _same(a, b):
    return (len(a[0]) == len(b[0]) and np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1])
            and np.array_equal(a[2].view(np.uint32), b[2].view(np.uint32)))


@pytest.mark.parametrize("precision", [1, 0], ids=["f16", "f32"])
def test_carried_rows_equal_rebuilt_rows(precision):
    from sharc.volrus_b200.method import LevelSet, large_sphere_grid
    sph, vel = large_sphere_grid(300, seed=5, extent=2048.0)
    kw = dict(half_width=3.0, precision=precision, integrator=3, reinit_iters=2)
    carried = LevelSet.spheres([(sph, vel)], 1.0, **kw)
    rebuilt = LevelSet.spheres([(sph, vel)], 1.0, **kw)
    try:
        changed = 0
        for k in range(STEPS):
            state = carried.arrays()
            rebuilt.upload(*state)
            rebuilt.set_step(k)
            carried.step(1)
            rebuilt.step(1)
            a, b = carried.arrays(), rebuilt.arrays()
            assert _same(a, b), k
            changed += len(set(map(tuple, a[0])) ^ set(map(tuple, state[0])))
        assert changed > 100  # leaves were dropped and added along the way
    finally:
        carried.close()
        rebuilt.close()

