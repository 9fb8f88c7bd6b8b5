"""GPU adjoint of frozen-band advection against the FP64 oracle adjoint and
FP64 central finite differences (eps = 1e-3).

Tolerances: forward phi_K within 2e-4 voxel of FP64 (FP32 arithmetic over K
steps); adjoint gradients within 1e-4 relative (2-norm) of the FP64 adjoint;
the FP64 adjoint within 1e-6 relative of central differences (the map is
affine in phi_0 and smooth in V away from floor() jumps); two backward runs
bitwise identical (no float atomics).
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def setup_problem(domain=64, radius=12.0, n_stag=32, steps=16, chk=4, dt_scale=1.0):
    from sharc.volrus_b200.adjoint import AdvectionFunction, sphere_band, staggered_vortex
    o, m, p = sphere_band(radius, (domain / 2, domain / 2, domain / 2), domain)
    vs = 1.0 / domain
    cell = domain / n_stag
    V = staggered_vortex(n_stag, cell, vs)
    dt = dt_scale * 0.5 / (2.0 / vs)
    fn = AdvectionFunction(o, m, p, V, cell, dt, 2.0, steps, chk)
    band = fn.band()
    c = np.array([domain / 2 + 8.0, domain / 2, domain / 2])
    target = (np.sqrt(((band - c) ** 2).sum(axis=1)) - radius).astype(np.float64)
    return fn, (o, m, p, V, cell, dt, steps), band, target


def test_adjoint_matches_fp64_and_fd():
    from oracle.pyadjoint import AdjointOracle, fd_phi0, fd_vel, loss
    fn, (o, m, p, V, cell, dt, steps), band, target = setup_problem()
    orc = AdjointOracle(o, m, p.astype(np.float64), 3.0, V.astype(np.float64), V.shape[-1], cell, dt, 2.0, 0.0, steps)
    assert orc.nb == fn.n_band
    phiK = fn.forward()
    phiK64 = orc.forward()
    assert np.max(np.abs(phiK - phiK64)) < 2e-4
    lamK = 2.0 * (phiK64 - target)
    g0, gv = fn.backward(lamK.astype(np.float32))
    g0_64, gv_64 = orc.backward(lamK)
    assert np.linalg.norm(g0 - g0_64) / np.linalg.norm(g0_64) < 1e-4
    assert np.linalg.norm(gv.reshape(-1) - gv_64) / np.linalg.norm(gv_64) < 1e-4
    # FP64 adjoint vs central differences at seeded band voxels and velocity nodes
    rng = np.random.default_rng(4)
    bidx = rng.choice(orc.nb, 16, replace=False)
    phi0_band = _band_values(o, m, p)
    fd0 = fd_phi0(orc, phi0_band, V.astype(np.float64), target, bidx)
    assert np.linalg.norm(fd0 - g0_64[bidx]) / np.linalg.norm(fd0) < 1e-6
    strong = smooth_nodes(np.argsort(-np.abs(gv_64))[:4000], V.shape[-1], cell, 64)
    vidx = rng.choice(strong, 16, replace=False)
    fdv = fd_vel(orc, phi0_band, V.astype(np.float64), target, vidx)
    assert np.linalg.norm(fdv - gv_64[vidx]) / np.linalg.norm(fdv) < 1e-6
    # GPU vs FD directly
    assert np.linalg.norm(fd0 - g0[bidx]) / np.linalg.norm(fd0) < 1e-4
    assert np.linalg.norm(fdv - gv.reshape(-1)[vidx]) / np.linalg.norm(fdv) < 1e-4


def test_adjoint_steps_beyond_one_voxel():
    """dt * max|V| = 2.5 voxels: reach 3, where the backward gather visits each
    leaf's narrowed window of candidate offsets; still the exact transpose."""
    from oracle.pyadjoint import AdjointOracle
    fn, (o, m, p, V, cell, dt, steps), band, target = setup_problem(steps=8, chk=3, dt_scale=5.0)
    orc = AdjointOracle(o, m, p.astype(np.float64), 3.0, V.astype(np.float64), V.shape[-1], cell, dt, 2.0, 0.0, steps)
    phiK = fn.forward()
    phiK64 = orc.forward()
    assert np.max(np.abs(phiK - phiK64)) < 2e-4
    lamK = 2.0 * (phiK64 - target)
    g0, gv = fn.backward(lamK.astype(np.float32))
    g0_64, gv_64 = orc.backward(lamK)
    assert np.linalg.norm(g0 - g0_64) / np.linalg.norm(g0_64) < 1e-4
    assert np.linalg.norm(gv.reshape(-1) - gv_64) / np.linalg.norm(gv_64) < 1e-4
    g0b, gvb = fn.backward(lamK.astype(np.float32))
    assert np.array_equal(g0.view(np.uint32), g0b.view(np.uint32)) and np.array_equal(gv.view(np.uint32),
                                                                                        gvb.view(np.uint32))
    fn.close()


def smooth_nodes(nodes, n, cell, domain):
    """Drop staggered nodes whose influence reaches a plane where the vortex
    component vanishes identically (its two other coordinates at 0, domain/2
    or domain): voxels there have feet exactly on cell faces, where the
    trilinear interpolant has a kink and central differences average the two
    one-sided slopes."""
    keep = []
    zero = np.array([0.0, domain / 2.0, float(domain)])
    for e in nodes:
        a, r = divmod(int(e), n ** 3)
        idx = (r // (n * n), (r // n) % n, r % n)
        ok = True
        for b in range(3):
            if b == a:
                continue
            lo, hi = cell * (idx[b] + 0.5 - 1.0), cell * (idx[b] + 0.5 + 1.0)
            if np.any((zero >= lo - 1.0) & (zero <= hi + 1.0)):
                ok = False
        if ok:
            keep.append(e)
    return np.array(keep)


def _band_values(o, m, p):
    bits = np.unpackbits(np.ascontiguousarray(m).view(np.uint8).reshape(-1, 64), axis=1, bitorder="little").astype(bool)
    return p.reshape(-1, 512)[bits].astype(np.float64)


def test_backward_is_deterministic():
    fn, _, band, target = setup_problem(steps=8, chk=3)
    phiK = fn.forward()
    lam = (2.0 * (phiK - target)).astype(np.float32)
    a0, av = fn.backward(lam)
    fn.forward()
    b0, bv = fn.backward(lam)
    assert np.array_equal(a0.view(np.uint32), b0.view(np.uint32))
    assert np.array_equal(av.view(np.uint32), bv.view(np.uint32))


def _fd_worker(args):
    """Central differences for a slice of (kind, index) entries in a spawned process."""
    o, m, p, V, cell, dt, steps, target, entries, eps = args
    from oracle.pyadjoint import AdjointOracle, loss
    orc = AdjointOracle(o, m, p, 3.0, V, V.shape[-1], cell, dt, 2.0, 0.0, steps)
    phi0 = _band_values(o, m, p)
    Vf = V.reshape(-1).copy()
    out = []
    for kind, e in entries:
        if kind == 0:
            q = phi0.copy()
            q[e] += eps
            lp = loss(orc.forward(q, Vf), target)
            q[e] -= 2 * eps
            lm = loss(orc.forward(q, Vf), target)
        else:
            v = Vf.copy()
            v[e] += eps
            lp = loss(orc.forward(phi0, v), target)
            v[e] -= 2 * eps
            lm = loss(orc.forward(phi0, v), target)
        out.append((lp - lm) / (2 * eps))
    return out


def test_config4_adjoint_256():
    """The adjoint configuration: sphere r=32 centred in 256^3, FP32, K=64 steps of
    the deformation field (T=2), checkpoints every 8 steps, loss against the
    sphere shifted +8 voxels in x, gradients w.r.t. phi_0 and a 128^3 staggered
    field; FP64 central differences (eps=1e-3) at 64 seeded band voxels and 64
    seeded velocity nodes, and the FP64 adjoint everywhere."""
    import multiprocessing as mp
    from oracle.pyadjoint import AdjointOracle
    from sharc.volrus_b200.adjoint import AdvectionFunction, sphere_band, staggered_vortex
    domain, radius, n, steps = 256, 32.0, 128, 64
    cell, vs = domain / n, 1.0 / domain
    dt = 0.5 / (2.0 / vs)
    o, m, p = sphere_band(radius, (128.0, 128.0, 128.0), domain)
    V = staggered_vortex(n, cell, vs)
    fn = AdvectionFunction(o, m, p, V, cell, dt, 2.0, steps, 8)
    band = fn.band()
    target = np.sqrt(((band - np.array([136.0, 128.0, 128.0])) ** 2).sum(axis=1)) - radius
    phiK = fn.forward()
    g0, gv = fn.backward((2.0 * (phiK - target)).astype(np.float32))
    orc = AdjointOracle(o, m, p.astype(np.float64), 3.0, V.astype(np.float64), n, cell, dt, 2.0, 0.0, steps)
    phiK64 = orc.forward()
    assert np.max(np.abs(phiK - phiK64)) < 5e-4
    g0_64, gv_64 = orc.backward(2.0 * (phiK64 - target))
    assert np.linalg.norm(g0 - g0_64) / np.linalg.norm(g0_64) < 1e-4
    assert np.linalg.norm(gv.reshape(-1) - gv_64) / np.linalg.norm(gv_64) < 1e-4
    rng = np.random.default_rng(2024)
    bidx = rng.choice(len(band), 64, replace=False)
    vidx = rng.choice(smooth_nodes(np.argsort(-np.abs(gv_64))[:20000], n, cell, domain), 64, replace=False)
    entries = [(0, int(b)) for b in bidx] + [(1, int(e)) for e in vidx]
    workers = min(16, mp.cpu_count())
    chunks = [entries[i::workers] for i in range(workers)]
    ctx = mp.get_context("spawn")
    with ctx.Pool(workers) as pool:
        res = pool.map(_fd_worker, [(o, m, p.astype(np.float64), V.astype(np.float64), cell, dt, steps, target, c,
                                     1e-3) for c in chunks])
    fd = np.zeros(len(entries))
    for i in range(workers):
        fd[i::workers] = res[i]
    fd0, fdv = fd[:64], fd[64:]
    assert np.linalg.norm(fd0 - g0[bidx]) / np.linalg.norm(fd0) < 1e-4
    assert np.linalg.norm(fdv - gv.reshape(-1)[vidx]) / np.linalg.norm(fdv) < 1e-4
    assert np.linalg.norm(fd0 - g0_64[bidx]) / np.linalg.norm(fd0) < 1e-6
    assert np.linalg.norm(fdv - gv_64[vidx]) / np.linalg.norm(fdv) < 1e-6
