"""Spatial decomposition of one level set over ranks (sharc/volrus_b200/spatial.py).

CPU: Morton keys against a bit-by-bit interleave, balanced key ranges, the
ghost sends against a brute-force neighbourhood search, the active counts,
and the whole decomposition with the FP64 method oracle as the per-rank
stepper: 2-4 emulated ranks with rebalancing, and two gloo processes over
torch.distributed, each bit-identical to the undivided oracle run (curl noise
with RK3, and the time-dependent vortex).

Resident shards (each rank's owned leaves kept in its pool between steps,
only ghosts and routed outputs moved) against the same undivided runs: on
the CPU with a pool stepped by the FP64 oracle (emulated ranks and two gloo
processes), on the device with the library's pool edits.

GPU: the same decomposition with the library's step on each emulated rank
(one device, ranks stepped in turn, exchanges in process) is bit-identical to
the undivided run on the device, in FP32 and FP16, with the leaves moved
into and out of each rank's level set by the device-resident C ABI, and with
level sets re-created mid-run with their step counter carried over; the
resident form likewise, with ghosts exchanged in FP16 for FP16 leaves.
"""
import os
import socket

import numpy as np
import pytest
import torch
import torch.multiprocessing as mp

from sharc.volrus_b200 import spatial
from sharc.volrus_b200.spatial import GHOST_DEPTH, Leaves, Partition


def _slow_key(c):
    x, y, z = (int(v) + (1 << 20) for v in c)
    k = 0
    for b in range(21):
        k |= ((x >> b) & 1) << (3 * b + 2)
        k |= ((y >> b) & 1) << (3 * b + 1)
        k |= ((z >> b) & 1) << (3 * b)
    return k


def test_morton_keys_interleave_bits():
    rng = np.random.default_rng(1)
    c = np.concatenate([rng.integers(-(1 << 20), 1 << 20, (200, 3)), [[0, 0, 0], [-1, -1, -1], [(1 << 20) - 1] * 3,
                                                                     [-(1 << 20)] * 3]])
    got = spatial.morton_keys_of_leaf_coords(torch.from_numpy(c))
    assert got.tolist() == [_slow_key(v) for v in c]
    assert min(got.tolist()) >= 0
    lv = Leaves.from_numpy(c * 8, np.zeros((len(c), 8), np.uint64), np.zeros((len(c), 512), np.float32))
    assert torch.equal(lv.keys(), got)
    with pytest.raises(ValueError):
        spatial.morton_keys_of_leaf_coords(torch.tensor([[1 << 20, 0, 0]]))


def _random_leaves(n, seed, span=12, dtype=np.float32):
    rng = np.random.default_rng(seed)
    c = np.unique(rng.integers(-span, span, (n, 3)), axis=0)
    o = (c * 8).astype(np.int32)
    m = rng.integers(0, 2 ** 63, (len(o), 8), dtype=np.uint64)
    p = rng.standard_normal((len(o), 512)).astype(dtype)
    return Leaves.from_numpy(o, m, p)


def test_active_counts_and_host_round_trip():
    lv = _random_leaves(40, 5)
    o, m, p = lv.numpy()
    want = np.unpackbits(m.view(np.uint8).reshape(-1, 64), axis=1).sum(axis=1)
    assert lv.active_per_leaf().tolist() == want.tolist()
    assert lv.active_voxels() == int(want.sum())
    back = Leaves.from_numpy(o, m, p)
    assert torch.equal(back.masks, lv.masks) and torch.equal(back.phi, lv.phi) and torch.equal(back.origins,
                                                                                              lv.origins)


def test_partition_is_balanced_and_deterministic():
    lv = _random_leaves(3000, 2)
    k = lv.keys()
    cost = spatial.leaf_cost(lv)
    for world in (1, 2, 3, 5, 8):
        p1 = Partition.balanced(k, cost, world)
        p2 = Partition.balanced(k.flip(0), cost.flip(0), world)
        assert torch.equal(p1.splitters, p2.splitters)
        own = p1.owner(k)
        assert int(own.min()) >= 0 and int(own.max()) < world
        loads = torch.bincount(own, weights=cost, minlength=world)
        assert float(loads.max() - loads.min()) <= 2 * float(cost.max()) + 1e-9, (world, loads)
        # ranges are contiguous in key order
        assert bool((torch.diff(own[torch.argsort(k)]) >= 0).all())


def test_ghost_sends_cover_the_two_leaf_neighbourhood():
    lv = _random_leaves(1500, 3, span=8)
    world = 3
    part, shares = spatial.split(lv, world)
    shards = [spatial.Shard(r, part, shares[r], None) for r in range(world)]
    sends = [s.ghost_sends() for s in shards]
    for r in range(world):
        recv = Leaves.concat([sends[q][r] for q in range(world) if r in sends[q]], lv)
        got = {tuple(v) for v in recv.origins.tolist()}
        mine = shares[r].coords().numpy()
        need = set()
        for q in range(world):
            if q == r:
                continue
            oc = shares[q].coords().numpy()
            d = np.abs(oc[:, None, :] - mine[None, :, :]).max(axis=2)
            near = (d <= GHOST_DEPTH).any(axis=1)
            need |= {tuple(v) for v in shares[q].origins.numpy()[near].tolist()}
        assert need <= got
        # nothing is sent that lies farther than GHOST_DEPTH from every coordinate rank r owns
        for c in recv.coords():
            nb = c + spatial._offsets(GHOST_DEPTH)
            assert bool((part.owner(spatial.morton_keys_of_leaf_coords(nb)) == r).any())
        assert not got & {tuple(v) for v in shares[r].origins.tolist()}


# ------------------------------------------------------------------ oracle-stepped decomposition

class OracleStepper:
    """One FP64 method-oracle step of a rank's local leaves (test checker)."""

    def __init__(self, vel, integrator, reinit_iters, dt, hw, t0=0.0):
        self.vel, self.integrator, self.reinit_iters, self.dt, self.hw, self.t0 = vel, integrator, reinit_iters, dt, \
            hw, t0
        self.steps = 0

    def __call__(self, lv):
        from oracle import pyoracle
        t = self.t0 + self.steps * self.dt
        self.steps += 1
        if len(lv) == 0:
            return Leaves.empty(torch.float64)
        o, m, p = lv.numpy()
        g = pyoracle.MOGrid.from_arrays(o, m, p, self.hw)
        assert g.step(self.vel, self.integrator, self.reinit_iters, t, self.dt, nthreads=4)
        return Leaves.from_numpy(*g.arrays())


def _curl_case():
    from oracle import pyoracle
    from sharc.volrus_b200.method import curl_noise
    rng = np.random.default_rng(11)
    sph = np.column_stack([rng.uniform(0, 96, (14, 3)), rng.uniform(4, 12, 14)])
    g = pyoracle.MOGrid.spheres(sph, 3.0)
    return Leaves.from_numpy(*g.arrays()), curl_noise(5, 96.0, 1.0), 3, 1.0, 3.0


def _vortex_case():
    from oracle import pyoracle
    vs = 1.0 / 128
    g = pyoracle.MOGrid.sphere(0.15, (0.35, 0.35, 0.35), vs, 3.0)
    return Leaves.from_numpy(*g.arrays()), {"kind": "vortex", "vs": vs, "period": 3.0}, 2, 0.5 * vs, 3.0


def _undivided(lv, stepper, steps):
    for _ in range(steps):
        lv = stepper(lv)
    return lv.sorted_xyz()


def _assert_same(a, b):
    (ao, am, ap), (bo, bm, bp) = a.numpy(), b.numpy()
    assert np.array_equal(ao, bo), (len(ao), len(bo))
    assert np.array_equal(am, bm)
    assert np.array_equal(ap.view(np.uint8), bp.view(np.uint8))


@pytest.mark.parametrize("world,rebalance", [(2, 0), (3, 2), (4, 1)])
def test_emulated_ranks_match_undivided_oracle_curl(oracle, world, rebalance):
    lv, vel, integ, dt, hw = _curl_case()
    steps = 4
    ref = _undivided(lv, OracleStepper(vel, integ, 2, dt, hw), steps)
    got, shards = spatial.emulate(lv, world, lambda r: OracleStepper(vel, integ, 2, dt, hw), steps, rebalance)
    _assert_same(got, ref)
    assert sum(len(s.owned) for s in shards) == len(ref)
    assert all(len(s.owned) for s in shards)


def test_emulated_ranks_match_undivided_oracle_vortex(oracle):
    lv, vel, integ, dt, hw = _vortex_case()
    steps = 3
    ref = _undivided(lv, OracleStepper(vel, integ, 2, dt, hw), steps)
    got, _ = spatial.emulate(lv, 3, lambda r: OracleStepper(vel, integ, 2, dt, hw), steps, 2)
    _assert_same(got, ref)


def test_emulated_ranks_some_owning_nothing(oracle):
    """More ranks than leaves: empty ranks step nothing, send and receive
    nothing, and may own leaves after a step or a rebalance."""
    from oracle import pyoracle
    g = pyoracle.MOGrid.spheres(np.array([[20.0, 20.0, 20.0, 4.0]]), 3.0)
    lv = Leaves.from_numpy(*g.arrays())
    vel = {"kind": "constant", "c": (0.7, 0.3, -0.2)}
    ref = _undivided(lv, OracleStepper(vel, 1, 2, 1.0, 3.0), 3)
    for world in (9, 40):
        got, shards = spatial.emulate(lv, world, lambda r: OracleStepper(vel, 1, 2, 1.0, 3.0), 3, 1)
        _assert_same(got, ref)
        assert world <= len(lv) or any(len(s.owned) == 0 for s in shards)


class OraclePool:
    """A rank's leaves held in list order on the CPU (FP64 values) with the
    pool methods of spatial.DevicePool, stepped by the FP64 method oracle: the
    host logic of the resident shards without a device (test checker)."""

    device = torch.device("cpu")
    dtype = torch.float64

    def __init__(self, lv, vel, integrator, reinit_iters, dt, hw, t0=0.0):
        self.lv = Leaves(lv.origins.clone(), lv.masks.clone(), lv.phi.to(torch.float64).clone())
        self.stepper = OracleStepper(vel, integrator, reinit_iters, dt, hw, t0)

    def count(self):
        return len(self.lv)

    def origins(self):
        return self.lv.origins.clone()

    def gather(self, pos=None):
        if pos is None:
            return Leaves(self.lv.origins.clone(), self.lv.masks.clone(), self.lv.phi.clone())
        return self.lv.take(pos)

    def edit(self, drop, add):
        keep = self.lv if drop is None else self.lv.take(~drop)
        self.lv = Leaves.concat([keep, add], self.lv)
        ks = self.lv.keys()
        assert len(torch.unique(ks)) == len(ks), "a leaf listed twice"

    def step(self):
        self.lv = self.stepper(self.lv)

    def skip(self):
        self.stepper.steps += 1


@pytest.mark.parametrize("world,rebalance", [(2, 0), (3, 2), (4, 1)])
def test_resident_emulated_ranks_match_undivided_oracle(oracle, world, rebalance):
    """The resident shards (leaves kept in each rank's pool, only ghosts and
    routed outputs moved) give the undivided run bit for bit."""
    lv, vel, integ, dt, hw = _curl_case()
    steps = 4
    ref = _undivided(lv, OracleStepper(vel, integ, 2, dt, hw), steps)
    got, shards = spatial.emulate_resident(lv, world, lambda r, own: OraclePool(own, vel, integ, 2, dt, hw), steps,
                                           rebalance)
    _assert_same(got, ref)
    assert sum(s.pool.count() for s in shards) == len(ref)


def test_resident_emulated_ranks_some_owning_nothing(oracle):
    from oracle import pyoracle
    g = pyoracle.MOGrid.spheres(np.array([[20.0, 20.0, 20.0, 4.0]]), 3.0)
    lv = Leaves.from_numpy(*g.arrays())
    vel = {"kind": "constant", "c": (0.7, 0.3, -0.2)}
    ref = _undivided(lv, OracleStepper(vel, 1, 2, 1.0, 3.0), 3)
    got, shards = spatial.emulate_resident(lv, 9, lambda r, own: OraclePool(own, vel, 1, 2, 1.0, 3.0), 3, 1)
    _assert_same(got, ref)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, steps, q):
    import torch.distributed as dist
    from datetime import timedelta
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    try:
        lv, vel, integ, dt, hw = _curl_case()
        sls = spatial.SpatialLevelSet(lv, OracleStepper(vel, integ, 2, dt, hw), check_duplicates=True)
        sls.step(2)
        sls.rebalance()
        sls.step(steps - 2)
        whole = sls.gather()
        q.put((rank, whole.numpy(), len(sls.arrays()), sls.active_voxels()))
    finally:
        dist.destroy_process_group()


def _rank_main_resident(rank, world, port, steps, q):
    import torch.distributed as dist
    from datetime import timedelta
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    try:
        lv, vel, integ, dt, hw = _curl_case()
        sls = spatial.SpatialLevelSet(lv, check_duplicates=True,
                                      make_pool=lambda own: OraclePool(own, vel, integ, 2, dt, hw))
        sls.step(2)
        sls.rebalance()
        sls.step(steps - 2)
        whole = sls.gather()
        q.put((rank, whole.numpy(), len(sls.arrays()), sls.active_voxels()))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("main", [_rank_main, _rank_main_resident], ids=["copied", "resident"])
def test_two_gloo_ranks_match_undivided_oracle(oracle, main):
    world, steps = 2, 3
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=main, args=(r, world, port, steps, q)) for r in range(world)]
    for p in procs:
        p.start()
    out = sorted([q.get(timeout=300) for _ in range(world)], key=lambda t: t[0])
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    lv, vel, integ, dt, hw = _curl_case()
    ref = _undivided(lv, OracleStepper(vel, integ, 2, dt, hw), steps)
    for rank, arrays, n_owned, active in out:
        _assert_same(Leaves.from_numpy(*arrays), ref)
        assert active == ref.active_voxels()
    assert out[0][2] + out[1][2] == len(ref) and min(out[0][2], out[1][2]) > 0


# ------------------------------------------------------------------ device

class _AlwaysRecreate(spatial.DeviceStepper):
    def _fits(self, lv):
        return False


def _device_case(kind):
    from sharc.volrus_b200.method import LevelSet, random_sphere_grids
    if kind == "curl":
        gr = random_sphere_grids(1, seed=17, extent_log2=(7.0, 7.2), spheres=(24, 28), radius=(5.0, 14.0))
        sph, vel, _ = gr[0]
        ls = LevelSet.spheres([(sph, vel)], 1.0, half_width=3.0, precision=0, integrator=3)
        arrays = ls.arrays()
        ls.close()
        return arrays, vel, 3, 1.0
    vs = 1.0 / 256
    ls = LevelSet.sphere(0.15, (0.35, 0.35, 0.35), vs, {"kind": "vortex", "vs": vs, "period": 3.0}, 0.5 * vs)
    arrays = ls.arrays()
    ls.close()
    return arrays, {"kind": "vortex", "vs": vs, "period": 3.0}, 2, 0.5 * vs


@pytest.mark.gpu
@pytest.mark.parametrize("kind,precision,world,recreate", [("curl", 0, 2, False), ("curl", 1, 3, False),
                                                           ("curl", 1, 2, True), ("vortex", 1, 3, True)],
                         ids=["curl_f32_2", "curl_f16_3", "curl_f16_2_recreate", "vortex_f16_3_recreate"])
def test_device_ranks_match_undivided_device_run(ctx, kind, precision, world, recreate):
    from sharc.volrus_b200.method import LevelSet
    (o, m, p), vel, integ, dt = _device_case(kind)
    steps = 6
    ls = LevelSet.from_leaves(o, m, p, vel, dt, 3.0, precision, integ, 2, 0.0)
    o, m, p = ls.arrays()  # the start state as stored (FP16-rounded for FP16 leaves)
    ls.step(steps)
    ref = Leaves.from_numpy(*ls.arrays())
    ls.close()
    cls = _AlwaysRecreate if recreate else spatial.DeviceStepper
    steppers = []

    def make(r):
        s = cls(vel, dt, 3.0, precision, integ, 2, 0.0)
        steppers.append(s)
        return s

    got, shards = spatial.emulate(Leaves.from_numpy(o, m, p, "cuda"), world, make, steps, rebalance_every=3)
    _assert_same(got, ref)
    assert all(len(s.owned) for s in shards)
    assert got.device.type == "cuda"
    # FP64 volume: the ranks' owned-leaf sums against the undivided level set's
    ls = LevelSet.from_leaves(*ref.numpy(), vel, dt, 3.0, precision, integ, 2, 0.0)
    v_ref = ls.volume((1.0, 2.0, 3.0))
    ls.close()
    v = sum(spatial.volume_shards(shards, spatial.LocalExchange(), (1.0, 2.0, 3.0)))
    assert abs(v - v_ref) <= 1e-12 * abs(v_ref), (v, v_ref)
    for s in steppers:
        s.close()


@pytest.mark.gpu
def test_device_upload_download_round_trip_and_errors(ctx):
    """vlr_ls_upload_device / vlr_ls_download_device: the same leaves back (list
    order, so compared sorted), an origin off the 8-voxel lattice refused with
    the context still usable, and a download into too few records refused."""
    from sharc.volrus_b200._lib import VolrusError
    from sharc.volrus_b200.method import LevelSet
    (o, m, p), vel, integ, dt = _device_case("curl")
    ls = LevelSet.from_leaves(o[:10], m[:10], p[:10], vel, dt, 3.0, 0, integ, 2, 0.0, capacity=2 * len(o))
    lv = Leaves.from_numpy(o, m, p, "cuda")
    ls.upload_device(lv.origins.data_ptr(), lv.masks.data_ptr(), lv.phi.data_ptr(), len(lv))
    out = Leaves(torch.empty((len(lv), 3), dtype=torch.int32, device="cuda"),
                 torch.empty((len(lv), 8), dtype=torch.int64, device="cuda"),
                 torch.empty((len(lv), 512), dtype=torch.float32, device="cuda"))
    n = ls.download_device(out.origins.data_ptr(), out.masks.data_ptr(), out.phi.data_ptr(), len(lv))
    assert n == len(lv)
    _assert_same(out.sorted_xyz(), lv.sorted_xyz())
    with pytest.raises(VolrusError):
        ls.download_device(out.origins.data_ptr(), out.masks.data_ptr(), out.phi.data_ptr(), len(lv) - 1)
    bad = lv.origins.clone()
    bad[3, 1] += 4
    with pytest.raises(VolrusError):
        ls.upload_device(bad.data_ptr(), lv.masks.data_ptr(), lv.phi.data_ptr(), len(lv))
    # the next valid upload restores a usable state
    ls.upload_device(lv.origins.data_ptr(), lv.masks.data_ptr(), lv.phi.data_ptr(), len(lv))
    ls.step(1)
    assert ls.leaf_count() > 0
    ls.close()


@pytest.mark.gpu
@pytest.mark.parametrize("kind,precision,world", [("curl", 0, 2), ("curl", 1, 3), ("vortex", 1, 3)],
                         ids=["curl_f32_2", "curl_f16_3", "vortex_f16_3"])
def test_resident_device_ranks_match_undivided_device_run(ctx, kind, precision, world):
    """Owned leaves resident in each rank's pool, ghosts and routed outputs in
    the pool's type (FP16 for FP16 leaves): bit-identical to the undivided
    device run, with a rebalance mid-run; FP64 volume over the owned leaves."""
    from sharc.volrus_b200.method import LevelSet
    (o, m, p), vel, integ, dt = _device_case(kind)
    steps = 6
    ls = LevelSet.from_leaves(o, m, p, vel, dt, 3.0, precision, integ, 2, 0.0)
    o, m, p = ls.arrays()
    ls.step(steps)
    ref = Leaves.from_numpy(*ls.arrays())
    ls.close()
    pools = []

    def make(r, own):
        pool = spatial.DevicePool(own, vel, dt, 3.0, precision, integ, 2, 0.0)
        pools.append(pool)
        return pool

    got, shards = spatial.emulate_resident(Leaves.from_numpy(o, m, p, "cuda"), world, make, steps,
                                           rebalance_every=3)
    assert got.phi.dtype == (torch.float16 if precision == 1 else torch.float32)
    got = Leaves(got.origins, got.masks, got.phi.to(torch.float32))
    _assert_same(got, ref)
    assert all(s.pool.count() for s in shards)
    ls = LevelSet.from_leaves(*ref.numpy(), vel, dt, 3.0, precision, integ, 2, 0.0)
    v_ref = ls.volume((1.0, 2.0, 3.0))
    ls.close()
    v = sum(spatial.volume_shards(shards, spatial.LocalExchange(), (1.0, 2.0, 3.0)))
    assert abs(v - v_ref) <= 1e-12 * abs(v_ref), (v, v_ref)
    for pool in pools:
        pool.close()


@pytest.mark.gpu
@pytest.mark.parametrize("precision", [0, 1], ids=["f32", "f16"])
def test_pool_edits_and_their_errors(ctx, precision):
    """vlr_ls_gather_device / vlr_ls_edit_device: a drop-and-append edit holds
    exactly the kept and added leaves (values in the pool's type, bit for
    bit); no room is refused before anything changes; a leaf added twice is
    refused and the state stays refused until an upload; a gather position
    outside the list is refused."""
    from sharc.volrus_b200._lib import VolrusError
    from sharc.volrus_b200.method import LevelSet
    (o, m, p), vel, integ, dt = _device_case("curl")
    n = len(o)
    half = n // 2
    ls = LevelSet.from_leaves(o[:half], m[:half], p[:half], vel, dt, 3.0, precision, integ, 2, 0.0, capacity=n + 8)
    pool_dtype = torch.float16 if precision == 1 else torch.float32
    add = Leaves.from_numpy(o[half:], m[half:], p[half:], "cuda")
    add = Leaves(add.origins, add.masks, add.phi.to(pool_dtype))
    drop = torch.zeros(half, dtype=torch.uint8, device="cuda")
    drop[::3] = 1
    torch.cuda.synchronize()
    ls.edit_device(drop.data_ptr(), half, add.origins.data_ptr(), add.masks.data_ptr(), add.phi.data_ptr(), len(add))
    cnt = ls.leaf_count()
    assert cnt == half - int(drop.sum()) + len(add)
    go = torch.empty((cnt, 3), dtype=torch.int32, device="cuda")
    gm = torch.empty((cnt, 8), dtype=torch.int64, device="cuda")
    gp = torch.empty((cnt, 512), dtype=pool_dtype, device="cuda")
    ls.gather_device(None, cnt, go.data_ptr(), gm.data_ptr(), gp.data_ptr())
    keep = np.nonzero(drop.cpu().numpy() == 0)[0]
    want_o = np.concatenate([o[keep], o[half:]])
    want_m = np.concatenate([m[keep], m[half:]])
    want_p = torch.from_numpy(np.concatenate([p[keep], p[half:]])).to(pool_dtype)
    assert np.array_equal(go.cpu().numpy(), want_o)
    assert np.array_equal(gm.cpu().numpy().view(np.uint64), want_m)
    assert torch.equal(gp.cpu().view(torch.uint8 if precision == 0 else torch.int16),
                       want_p.view(torch.uint8 if precision == 0 else torch.int16))
    # positions: the same leaves picked one by one
    pos = torch.tensor([cnt - 1, 0, 5], dtype=torch.int32, device="cuda")
    po = torch.empty((3, 3), dtype=torch.int32, device="cuda")
    ls.gather_device(pos.data_ptr(), 3, po.data_ptr())
    assert np.array_equal(po.cpu().numpy(), want_o[[cnt - 1, 0, 5]])
    bad = torch.tensor([cnt], dtype=torch.int32, device="cuda")
    with pytest.raises(VolrusError):
        ls.gather_device(bad.data_ptr(), 1, po.data_ptr())
    # no room: refused, nothing changed
    none = torch.zeros(cnt, dtype=torch.uint8, device="cuda")
    big = Leaves.from_numpy(o, m, p, "cuda")
    big = Leaves(big.origins + 8 * 4096, big.masks, big.phi.to(pool_dtype))
    with pytest.raises(VolrusError) as e:
        ls.edit_device(none.data_ptr(), cnt, big.origins.data_ptr(), big.masks.data_ptr(), big.phi.data_ptr(),
                       len(big))
    assert "room" in str(e.value)
    assert ls.leaf_count() == cnt
    ls.step(1)  # still a usable state
    # a leaf added twice: refused, then refused until an upload
    cnt = ls.leaf_count()
    one = ls.leaf_count()
    go = torch.empty((1, 3), dtype=torch.int32, device="cuda")
    gm = torch.empty((1, 8), dtype=torch.int64, device="cuda")
    gp = torch.empty((1, 512), dtype=pool_dtype, device="cuda")
    ls.gather_device(None, 1, go.data_ptr(), gm.data_ptr(), gp.data_ptr())
    none = torch.zeros(one, dtype=torch.uint8, device="cuda")
    with pytest.raises(VolrusError):
        ls.edit_device(none.data_ptr(), one, go.data_ptr(), gm.data_ptr(), gp.data_ptr(), 1)
    with pytest.raises(VolrusError):
        ls.step(1)
    ls.upload(o, m, p)
    ls.step(1)
    ls.close()


# ------------------------------------------------------------------ divided adjoint

ADJ_STEPS = 6


def _adj_disp(coords):
    """A smooth per-voxel displacement (voxels, |d| < 1) standing in for a backtrace."""
    x, y, z = (coords[:, a].astype(np.float64) for a in range(3))
    return np.stack([0.8 * np.sin(0.11 * y + 0.07 * z), 0.6 * np.sin(0.09 * z + 0.05 * x),
                     -0.7 * np.sin(0.13 * x + 0.03 * y)], axis=1)


def _adj_target(coords):
    x, y, z = (coords[:, a].astype(np.float64) for a in range(3))
    return 0.3 * np.sin(0.05 * x) * np.cos(0.04 * y) + 0.1 * z / 256.0


class OracleAdjointEngine:
    """The FP64 oracle's frozen-band adjoint over a rank's local leaves, band in
    leaf then offset order, driven by _adj_disp (test checker)."""

    def __init__(self, lv, steps):
        from oracle.pyadjoint import AdjointOracle
        o, m, p = lv.numpy()
        bits = np.unpackbits(m.view(np.uint8).reshape(-1, 64), axis=1, bitorder="little").astype(bool)
        li, vi = np.nonzero(bits)
        rel = np.stack([vi >> 6, (vi >> 3) & 7, vi & 7], axis=1)
        self.coords = o[li].astype(np.int64) + rel
        self.orc = AdjointOracle.from_displacement(o, m, p, 3.0, _adj_disp(self.coords), steps)

    def band_coords(self):
        return torch.from_numpy(self.coords)

    def forward(self):
        return torch.from_numpy(self.orc.forward())

    def backward(self, lam):
        return torch.from_numpy(self.orc.backward(lam.numpy())[0])


def _adj_loss_grad(engine, phik, mask):
    return 2.0 * (phik[mask] - torch.from_numpy(_adj_target(engine.coords[mask.numpy()])))


def _adj_case():
    from oracle import pyoracle
    rng = np.random.default_rng(23)
    sph = np.column_stack([rng.uniform(0, 256, (24, 3)), rng.uniform(6, 14, 24)])
    return Leaves.from_numpy(*pyoracle.MOGrid.spheres(sph, 3.0).arrays())


def _adj_undivided(lv):
    e = OracleAdjointEngine(lv.sorted_xyz(), ADJ_STEPS)
    phik = e.forward()
    mask = torch.ones(len(phik), dtype=torch.bool)
    g0 = e.backward(_adj_loss_grad(e, phik, mask))
    keys = spatial._voxel_keys(e.band_coords())
    return {int(k): (float(a), float(b)) for k, a, b in zip(keys, phik, g0)}


def _adj_check(results, ref, exact=True):
    n = 0
    bad = 0
    for coords, phik, g0 in results:
        for k, a, b in zip(spatial._voxel_keys(coords).tolist(), phik.tolist(), g0.tolist()):
            ra, rb = ref[k]
            bad += (a != ra) or (b != rb)
            n += 1
    assert n == len(ref), (n, len(ref))
    return bad


@pytest.mark.parametrize("world", [2, 3])
def test_divided_adjoint_matches_undivided_oracle(oracle, world):
    """Each rank's forward phi_K and dL/dphi_0 on its owned band voxels equal
    the undivided FP64 adjoint's bit for bit (ghost ring of
    adjoint_ghost_depth leaves, no exchange between steps, the loss gradient
    sent the reverse way once); a ring of one leaf over twice the steps
    changes them (the dependency cone is wider than the ring)."""
    lv = _adj_case()
    ref = _adj_undivided(lv)
    part, shares = spatial.split(lv, world)
    mk = lambda r, local: OracleAdjointEngine(local, ADJ_STEPS)  # noqa: E731
    res, _ = spatial.divided_adjoint(shares, part, mk, _adj_loss_grad, spatial.LocalExchange(), ADJ_STEPS, reach=1)
    assert _adj_check(res, ref) == 0
    assert spatial.adjoint_ghost_depth(ADJ_STEPS, 1) == 3
    if world == 2:
        steps = 3 * ADJ_STEPS
        e = OracleAdjointEngine(lv.sorted_xyz(), steps)
        phik = e.forward()
        g0 = e.backward(_adj_loss_grad(e, phik, torch.ones(len(phik), dtype=torch.bool)))
        ref2 = {int(k): (float(a), float(b)) for k, a, b in zip(spatial._voxel_keys(e.band_coords()), phik, g0)}
        mk2 = lambda r, local: OracleAdjointEngine(local, steps)  # noqa: E731
        thin, _ = spatial.divided_adjoint(shares, part, mk2, _adj_loss_grad, spatial.LocalExchange(), steps, reach=1,
                                          depth=1)
        assert _adj_check(thin, ref2) > 0


def _rank_main_adjoint(rank, world, port, q):
    import torch.distributed as dist
    from datetime import timedelta
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    try:
        lv = _adj_case()
        part, shares = spatial.split(lv, world)
        ex = spatial.DistExchange(Leaves.empty(torch.float64), None)
        res, _ = spatial.divided_adjoint([shares[rank]], part, lambda r, local: OracleAdjointEngine(local, ADJ_STEPS),
                                         _adj_loss_grad, ex, ADJ_STEPS, reach=1, ranks=[rank])
        (coords, phik, g0), = res
        q.put((rank, coords.numpy(), phik.numpy(), g0.numpy()))
    finally:
        dist.destroy_process_group()


def test_divided_adjoint_two_gloo_ranks(oracle):
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main_adjoint, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    out = sorted([q.get(timeout=300) for _ in range(world)], key=lambda t: t[0])
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    ref = _adj_undivided(_adj_case())
    res = [(torch.from_numpy(c), torch.from_numpy(a), torch.from_numpy(b)) for _, c, a, b in out]
    assert _adj_check(res, ref) == 0
    assert min(len(c) for _, c, _, _ in out) > 0


@pytest.mark.gpu
@pytest.mark.parametrize("precision,world", [(1, 2), (0, 3)], ids=["f16_2", "f32_3"])
def test_divided_level_set_adjoint_matches_undivided_device_run(ctx, precision, world):
    """The level-set adjoint of a grid divided over emulated ranks (one device,
    a DeviceAdjointEngine per rank over its owned leaves and ghost ring): phi_K
    and dL/dphi_0 on every rank's owned band voxels equal the undivided
    device adjoint's bit for bit (both with the windowed lambda transpose),
    for an L2 loss against phi_0 translated by 4 voxels in x."""
    (o, m, p), vel, integ, dt = _device_case("curl")
    steps, chk = 6, 2
    lv = Leaves.from_numpy(o, m, p, "cuda").sorted_xyz()

    def loss_grad(engine, phik, mask):
        return 2.0 * (phik[mask] - engine.shifted_phi0((4, 0, 0))[mask])

    full = spatial.DeviceAdjointEngine(lv, vel, dt, steps, chk, precision=precision, integrator=integ)
    phik = full.forward()
    g0 = full.backward(loss_grad(full, phik, torch.ones(len(phik), dtype=torch.bool, device="cuda")))
    ref = {int(k): (float(a), float(b)) for k, a, b in zip(spatial._voxel_keys(full.band_coords()).tolist(),
                                                            phik.tolist(), g0.tolist())}
    full.close()
    part, shares = spatial.split(lv, world)
    engines = []

    def make(r, local):
        e = spatial.DeviceAdjointEngine(local, vel, dt, steps, chk, precision=precision, integrator=integ)
        engines.append(e)
        return e

    res, _ = spatial.divided_adjoint(shares, part, make, loss_grad, spatial.LocalExchange(), steps, reach=2)
    n = 0
    for coords, a, b in res:
        for k, x, y in zip(spatial._voxel_keys(coords).tolist(), a.tolist(), b.tolist()):
            assert ref[k] == (x, y), k
            n += 1
    assert n == len(ref)
    assert any(float(torch.abs(b).max()) > 0 for _, _, b in res)
    for e in engines:
        e.close()


@pytest.mark.gpu
def test_adjoint_gather_modes(ctx):
    """vlr_adj_set_gather: the windowed and quad transposes agree to rounding,
    each is deterministic, and the quad is refused above a reach of one."""
    from sharc.volrus_b200._lib import VolrusError
    (o, m, p), vel, integ, dt = _device_case("curl")
    e = spatial.DeviceAdjointEngine(Leaves.from_numpy(o, m, p, "cuda").sorted_xyz(), vel, dt, 4, 2, precision=0,
                                    integrator=integ)
    lam = torch.linspace(-1.0, 1.0, e.fn.n_band, device="cuda")
    outs = {}
    for mode in (1, 2, 1):
        e.fn.set_gather(mode)
        outs.setdefault(mode, []).append(e.backward(lam))
    assert torch.equal(outs[1][0], outs[1][1])
    assert torch.allclose(outs[1][0], outs[2][0], rtol=1e-5, atol=1e-6)
    with pytest.raises(VolrusError):
        e.fn.set_gather(3)
    e.close()
