"""The narrow-band method at bench scale against the FP64 method oracle.

large8192: the whole 8,000-sphere grid (2.5 M leaves, 384 M active voxels)
steps on the GPU.  The oracle steps only the spheres whose band comes within
8 voxels of a 1536^3 box at the grid's centre (56 spheres), and the leaves
inside the box shrunk by a 40-voxel ring (~13.6k leaves, 2.1 M active
voxels) are compared.  One step
moves information by less than 8 voxels (RK3 backtrace of at most 1 voxel,
trilinear and Godunov stencils, one leaf of dilation), so over 4 steps the
spheres left out of the subset, whose bands stay at least 48 voxels from the
compared leaves, cannot reach them (two oracle runs over this subset and
over the spheres near a box 100 voxels wider agree bit for bit on the
compared leaves after 4 steps).

batched256: all 256 grids of the batched workload step in one pool, and 8 of
them, the largest by sphere area among them, are compared with the oracle
stepping each grid alone.

The bars are those of the small parity tests (FP32 trajectory within 2e-4
voxel, FP16 within 4e-3 per step from a common state, FP16 trajectory RMS and
outlier fraction), applied to both workloads per step and over 4 steps.
"""
import numpy as np
import pytest

from tests.method_compare import compare
from tests.test_method_parity import check

pytestmark = pytest.mark.gpu

BOX = 1536
RING = 40
MARGIN = 3.0 + 8.0   # half width + the reach of one step's ghost dependence
STEPS = 4


def _box():
    lo = np.full(3, 4096 - BOX // 2, np.int64)
    return lo, lo + BOX


def _device_box_arrays(ls, lo, hi):
    """The level set's leaves inside [lo, hi)^3 (origins, masks, phi), sorted
    (x, y, z), selected on the device from a full device download."""
    import torch
    n = ls.leaf_count()
    o = torch.empty((n, 3), dtype=torch.int32, device="cuda")
    m = torch.empty((n, 8), dtype=torch.int64, device="cuda")
    p = torch.empty((n, 512), dtype=torch.float32, device="cuda")
    k = ls.download_device(o.data_ptr(), m.data_ptr(), p.data_ptr(), n)
    o, m, p = o[:k], m[:k], p[:k]
    lo_t = torch.tensor([int(x) for x in lo], dtype=torch.int32, device="cuda")
    hi_t = torch.tensor([int(x) for x in hi], dtype=torch.int32, device="cuda")
    sel = ((o >= lo_t) & (o + 8 <= hi_t)).all(dim=1)
    oo = o[sel].cpu().numpy()
    mm = m[sel].cpu().numpy().view(np.uint64)
    pp = p[sel].cpu().numpy()
    del o, m, p
    order = np.lexsort((oo[:, 2], oo[:, 1], oo[:, 0]))
    return oo[order], mm[order], pp[order]


def _select(arrays, lo, hi):
    from sharc.volrus_b200.method import leaves_in_box
    o, m, p = arrays
    s = leaves_in_box(o, lo, hi)
    return o[s], m[s], p[s]


CASES = [(0, False), (1, True), (1, False)]
CASE_IDS = ["f32", "f16-per-step", "f16-trajectory"]


@pytest.mark.parametrize("precision,per_step", CASES, ids=CASE_IDS)
def test_large8192_box_against_fp64(oracle, precision, per_step):
    from sharc.volrus_b200.method import LevelSet, large_sphere_grid, spheres_near_box
    sph, vel = large_sphere_grid()
    lo, hi = _box()
    clo, chi = lo + RING, hi - RING
    ls = LevelSet.spheres([(sph, vel)], 1.0, half_width=3.0, precision=precision, integrator=3, reinit_iters=2)
    try:
        assert ls.leaf_count() > 2_000_000
        sub = spheres_near_box(sph, lo, hi, MARGIN)
        og = oracle.MOGrid.spheres(sub, 3.0)
        s0 = compare(_device_box_arrays(ls, clo, chi), _select(og.arrays(), clo, chi), 3.0)
        assert s0["leaves_gpu"] > 10_000, s0
        assert s0["only_gpu"] == 0 and s0["only_oracle"] == 0 and s0["mask_flips"] == 0, s0
        assert s0["max_err"] < (1e-6 if precision == 0 else 1e-3), s0
        for step in range(STEPS):
            if per_step:
                og = oracle.MOGrid.from_arrays(*_device_box_arrays(ls, lo, hi), 3.0)
            ls.step(1)
            assert og.step(vel, 3, 2, float(step), 1.0, 8)
            if per_step or step == STEPS - 1:
                st = compare(_device_box_arrays(ls, clo, chi), _select(og.arrays(), clo, chi), 3.0)
                assert st["leaves_gpu"] > 10_000, st
                check(st, precision, per_step)
    finally:
        ls.close()


def _batched_selection(grids, k=8):
    """Indices of k grids spread over the batch's sizes, the largest included."""
    area = np.array([float((4 * np.pi * s[:, 3] ** 2).sum()) for s, _, _ in grids])
    order = np.argsort(area)
    pick = order[np.linspace(0, len(order) - 1, k).round().astype(int)]
    assert order[-1] in pick
    return [int(i) for i in pick]


@pytest.mark.parametrize("precision,per_step", CASES, ids=CASE_IDS)
def test_batched256_grids_against_fp64(oracle, precision, per_step):
    from sharc.volrus_b200.method import LevelSet, random_sphere_grids
    grids = random_sphere_grids(256, seed=3)
    pick = _batched_selection(grids)
    ls = LevelSet.spheres([(s, v) for s, v, _ in grids], 1.0, half_width=3.0, precision=precision, integrator=3,
                          reinit_iters=2)
    try:
        og = {g: oracle.MOGrid.spheres(grids[g][0], 3.0) for g in pick}
        for g in pick:
            st = compare(ls.grid_arrays(g), og[g].arrays(), 3.0)
            assert st["only_gpu"] == 0 and st["only_oracle"] == 0 and st["mask_flips"] == 0, (g, st)
        for step in range(STEPS):
            if per_step:
                og = {g: oracle.MOGrid.from_arrays(*ls.grid_arrays(g), 3.0) for g in pick}
            ls.step(1)
            for g in pick:
                assert og[g].step(grids[g][1], 3, 2, float(step), 1.0, 8)
            if per_step or step == STEPS - 1:
                for g in pick:
                    st = compare(ls.grid_arrays(g), og[g].arrays(), 3.0)
                    assert st["leaves_gpu"] > 0, (g, st)
                    check(st, precision, per_step)
    finally:
        ls.close()
