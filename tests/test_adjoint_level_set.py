"""Frozen-band adjoint of a level set's own step (vlr_adj_create_level_set).

A single curl-noise grid stepped with SSP-RK3: the displacement the library
computes for each band voxel (the advect kernel's backtrace arithmetic) is
checked against an FP64 RK3 backtrace through the oracle's velocity; the
forward map and the adjoint are checked against the FP64 oracle adjoint
(oracle/adjoint_oracle.cpp) driven by the same displacements, and the
oracle's gradient against FP64 central differences.  A time-dependent
velocity is refused.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _level_set(precision, amplitude=1.0):
    from sharc.volrus_b200.method import LevelSet, random_sphere_grids
    gr = random_sphere_grids(1, seed=21, extent_log2=(6.0, 6.5), spheres=(3, 5), radius=(6.0, 12.0),
                             amplitude=amplitude)
    sph, vel, _ = gr[0]
    ls = LevelSet.spheres([(sph, vel)], 1.0, half_width=3.0, precision=precision, integrator=3)
    return ls, vel


def _band_keys(coords):
    c = np.asarray(coords, np.int64) + (1 << 20)
    return (c[:, 0] << 42) | (c[:, 1] << 21) | c[:, 2]


def _oracle_band(o, m):
    """Band coordinates in the oracle's order (leaf order, then ZYX)."""
    out = []
    for (x, y, z), mm in zip(o, m):
        for off in range(512):
            if (int(mm[off >> 6]) >> (off & 63)) & 1:
                out.append((int(x) + (off >> 6), int(y) + ((off >> 3) & 7), int(z) + (off & 7)))
    return np.array(out, np.int32).reshape(-1, 3)


@pytest.mark.parametrize("precision,amplitude", [(0, 1.0), (1, 1.0), (0, 1.8)], ids=["f32", "f16", "f32_fast"])
def test_level_set_adjoint_matches_fp64(ctx, precision, amplitude):
    from oracle import pyoracle
    from oracle.pyadjoint import AdjointOracle
    from sharc.volrus_b200.adjoint import AdvectionFunction

    ls, vel = _level_set(precision, amplitude)
    ls.step(2)  # an evolved state: the adjoint starts from whatever the level set holds
    o, m, phi = ls.arrays()
    K, C = 6, 2
    fn = AdvectionFunction.from_level_set(ls, K, C)
    coords = fn.band()
    d = fn.displacement()
    assert len(coords) == int(sum(bin(int(w)).count("1") for w in m.reshape(-1)))

    # displacement = SSP-RK3 backtrace over one step, FP64 through the oracle's velocity
    dt = 1.0
    rng = np.random.default_rng(3)
    for i in rng.choice(len(coords), 64, replace=False):
        x = coords[i].astype(np.float64)
        h = -dt
        k1 = pyoracle.velocity_at(vel, x, 0.0)
        a = h * k1
        k2 = pyoracle.velocity_at(vel, x + a, 0.0)
        b = 0.25 * (a + h * k2)
        k3 = pyoracle.velocity_at(vel, x + b, 0.0)
        ref = (2.0 / 3.0) * (b + h * k3)
        assert np.abs(d[i] - ref).max() < 2e-4, (i, d[i], ref)

    # the oracle in its own band order, fed the library's displacements
    ob = _oracle_band(o, m)
    kg, ko = _band_keys(coords), _band_keys(ob)
    gi, oi = np.argsort(kg), np.argsort(ko)
    assert np.array_equal(kg[gi], ko[oi])
    to_o = np.empty(len(ko), np.int64)
    to_o[oi] = gi  # oracle band index -> library band index
    orc = AdjointOracle.from_displacement(o, m, phi.astype(np.float64), 3.0, d[to_o].astype(np.float64), K)

    phiK_gpu = fn.forward()
    phiK_orc = orc.forward()
    assert np.abs(phiK_gpu[to_o] - phiK_orc).max() < 1e-4

    lamK = rng.standard_normal(len(coords)).astype(np.float32)
    g0, gv = fn.backward(lamK)
    assert gv is None
    g0_orc, _ = orc.backward(lamK[to_o].astype(np.float64))
    err = np.linalg.norm(g0[to_o] - g0_orc) / np.linalg.norm(g0_orc)
    assert err < 5e-5, err

    # the oracle's gradient against central differences of L = <lamK, phi_K>
    # (phi_K is affine in phi_0, so the differences are exact up to rounding)
    lam_o = lamK[to_o].astype(np.float64)
    # band values of phi_0 in oracle order
    p0 = []
    for (x, y, z), mm, vv in zip(o, m, phi):
        for off in range(512):
            if (int(mm[off >> 6]) >> (off & 63)) & 1:
                p0.append(float(vv[off]))
    p0 = np.array(p0)
    for b in rng.choice(len(p0), 12, replace=False):
        q = p0.copy()
        q[b] += 1e-3
        lp = float(np.dot(lam_o, orc.forward(q)))
        q[b] -= 2e-3
        lm = float(np.dot(lam_o, orc.forward(q)))
        fd = (lp - lm) / 2e-3
        assert abs(fd - g0_orc[b]) <= 1e-6 * max(1.0, abs(g0_orc[b])), (b, fd, g0_orc[b])
    fn.close()
    ls.close()


def test_shifted_phi0_target(ctx):
    """vlr_adj_shifted_phi0 = phi_0(x - s) on the band, missing leaves read as
    copysign(hw, the clamped position's value in the voxel's own leaf)."""
    import torch
    from sharc.volrus_b200.adjoint import AdvectionFunction
    ls, _ = _level_set(0)
    o, m, phi = ls.arrays()
    fn = AdvectionFunction.from_level_set(ls, 2, 1)
    coords = fn.band()
    shift = (4, -1, 2)
    out = torch.empty(fn.n_band, dtype=torch.float32, device="cuda")
    fn.shifted_phi0_device(shift, out.data_ptr())
    ls.ctx.synchronize()
    got = out.cpu().numpy()
    leaf = {tuple(int(v) for v in oo): i for i, oo in enumerate(o)}
    for b in np.random.default_rng(7).choice(len(coords), 200, replace=False):
        x, y, z = (int(c) for c in coords[b])
        q = (x - shift[0], y - shift[1], z - shift[2])
        key = tuple(c & ~7 for c in q)
        if key in leaf:
            want = phi[leaf[key], ((q[0] & 7) << 6) | ((q[1] & 7) << 3) | (q[2] & 7)]
        else:
            own = leaf[tuple(c & ~7 for c in (x, y, z))]
            lo = [c & ~7 for c in (x, y, z)]
            cl = [min(max(qq - l, 0), 7) for qq, l in zip(q, lo)]
            want = np.copysign(np.float32(3.0), phi[own, (cl[0] << 6) | (cl[1] << 3) | cl[2]])
        assert got[b] == want, (b, got[b], want)
    fn.close()
    ls.close()


def test_level_set_adjoint_refuses_time_dependent_velocity(ctx):
    from sharc.volrus_b200._lib import VolrusError
    from sharc.volrus_b200.adjoint import AdvectionFunction
    from sharc.volrus_b200.method import LevelSet
    vs = 1 / 64
    ls = LevelSet.sphere(0.2, (0.5, 0.5, 0.5), vs, {"kind": "vortex", "vs": vs, "period": 3.0}, 0.5 * vs)
    with pytest.raises(VolrusError):
        AdvectionFunction.from_level_set(ls, 4, 2)
    ls.close()
