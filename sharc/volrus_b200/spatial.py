"""Spatial decomposition of one level set over ranks (one GPU per rank).

A grid too large for one device is split by the Morton (Z-order) key of its
leaves: rank r owns the leaves whose key lies in its range ``[s_{r-1}, s_r)``
of the splitters, leaves that a step allocates included, so ownership is a
pure function of a leaf's coordinate.  The ranges are cut at equal cumulative
cost (one unit per leaf plus its fraction of active voxels) and re-cut on
request (``rebalance``).

A step on rank r runs the single-device method step (``LevelSet``) on its
owned leaves plus a ghost ring: every leaf of another rank within two leaves
(Chebyshev distance in leaf units) of an owned leaf, sent by its owner before
the step.  Two leaves suffice.  One method step reads within 5 voxels of a
voxel (a backtrace of at most 3 voxels inside the advect kernel's staged
halo, then two reinitialisation sweeps of one voxel each; the 26-voxel
dilation D and the missing-leaf rule read 1 voxel and the voxel's own leaf),
so the new values and mask of a leaf, whether the re-track keeps or
allocates it, and the neighbour that fills a new leaf depend only on the
input leaves within one leaf of it.  Every leaf of the step's output lies
within one leaf of an input leaf (the active set after a step lies inside
allocated leaves and the re-track allocates only face, edge and corner
neighbours of those), and the output leaves within one leaf of rank r's owned
leaves are computed from a local input that holds every input leaf within
two leaves of them: exactly as on one device, bit for bit.  Rank r keeps
those outputs and sends each to the owner of its key; a leaf that reaches its
owner from two ranks carries the same bits (checked on request).  The ghost
ring's own outputs are dropped.

Exchanges go through ``torch.distributed`` point-to-point transfers (NCCL on
GPUs, gloo on CPU), leaf records packed as bytes; ``emulate`` runs all ranks
in one process with the same logic and in-process delivery, which is how a
single device checks the decomposition against the undivided run.  The
exchange is staged through host memory (each step uploads the local leaves
and downloads the result through the C ABI's host step); the decomposition
does not change a voxel of the result, only where it is computed.

The crate has no multi-device path: this is the decomposition of the
single-grid step (src/tools/advection.rs:32-56 with the method's re-tracking)
over devices, leaf records as in src/nano/layout.rs:89-170 (origin, mask,
512 values in ZYX order).
"""
from __future__ import annotations

from dataclasses import dataclass
from typing import Callable, Sequence

import numpy as np

GHOST_DEPTH = 2  # leaves; derivation in the module docstring
_BIAS = 1 << 20  # leaf coordinates (origin >> 3) are biased to 21-bit non-negative fields
_M = np.uint64


@dataclass
class Leaves:
    """Leaf records: origins (n, 3) i32, masks (n, 8) u64, phi (n, 512) f32 or f64."""
    origins: np.ndarray
    masks: np.ndarray
    phi: np.ndarray

    def __len__(self) -> int:
        return len(self.origins)

    @classmethod
    def empty(cls, dtype=np.float32) -> "Leaves":
        return cls(np.zeros((0, 3), np.int32), np.zeros((0, 8), np.uint64), np.zeros((0, 512), dtype))

    def take(self, idx) -> "Leaves":
        return Leaves(self.origins[idx], self.masks[idx], self.phi[idx])

    @staticmethod
    def concat(parts: Sequence["Leaves"], dtype=np.float32) -> "Leaves":
        parts = [p for p in parts if len(p)]
        if not parts:
            return Leaves.empty(dtype)
        return Leaves(np.concatenate([p.origins for p in parts]), np.concatenate([p.masks for p in parts]),
                      np.concatenate([p.phi for p in parts]))

    def keys(self) -> np.ndarray:
        return morton_keys(self.origins)

    def sorted_xyz(self) -> "Leaves":
        """Records in (x, y, z) order of the origin, as ``LevelSet.arrays``."""
        o = self.origins.astype(np.int64)
        return self.take(np.lexsort((o[:, 2], o[:, 1], o[:, 0])))

    def active_voxels(self) -> int:
        return int(np.unpackbits(np.ascontiguousarray(self.masks).view(np.uint8)).sum())

    # byte records for the wire: masks, values, origins (each segment aligned)
    def pack(self) -> np.ndarray:
        return np.concatenate([np.ascontiguousarray(self.masks).view(np.uint8).reshape(-1),
                               np.ascontiguousarray(self.phi).view(np.uint8).reshape(-1),
                               np.ascontiguousarray(self.origins, np.int32).view(np.uint8).reshape(-1)])

    @staticmethod
    def unpack(buf: np.ndarray, dtype) -> "Leaves":
        isz = np.dtype(dtype).itemsize
        rec = 64 + 512 * isz + 12
        if buf.size % rec:
            raise ValueError("leaf record buffer of %d bytes is not a whole number of records" % buf.size)
        n = buf.size // rec
        b = np.ascontiguousarray(buf, np.uint8)
        m = np.frombuffer(b, np.uint64, 8 * n, 0).reshape(n, 8).copy()
        p = np.frombuffer(b, dtype, 512 * n, 64 * n).reshape(n, 512).copy()
        o = np.frombuffer(b, np.int32, 3 * n, (64 + 512 * isz) * n).reshape(n, 3).copy()
        return Leaves(o, m, p)


def _spread(v: np.ndarray) -> np.ndarray:
    """21-bit integers with their bits moved to every third position (bit b -> 3b)."""
    x = v.astype(_M) & _M(0x1FFFFF)
    x = (x | (x << _M(32))) & _M(0x1F00000000FFFF)
    x = (x | (x << _M(16))) & _M(0x1F0000FF0000FF)
    x = (x | (x << _M(8))) & _M(0x100F00F00F00F00F)
    x = (x | (x << _M(4))) & _M(0x10C30C30C30C30C3)
    x = (x | (x << _M(2))) & _M(0x1249249249249249)
    return x


def morton_keys_of_leaf_coords(c: np.ndarray) -> np.ndarray:
    """63-bit Z-order keys of leaf coordinates (origin >> 3), x in the highest
    bit of each triple.  Coordinates are biased by 2^20 (|origin| < 2^23)."""
    c = np.asarray(c, np.int64).reshape(-1, 3) + _BIAS
    if c.size and (c.min() < 0 or c.max() >= (1 << 21)):
        raise ValueError("leaf coordinate outside the 21-bit key range (|origin| >= 2^23 voxels)")
    return (_spread(c[:, 0]) << _M(2)) | (_spread(c[:, 1]) << _M(1)) | _spread(c[:, 2])


def morton_keys(origins: np.ndarray) -> np.ndarray:
    return morton_keys_of_leaf_coords(np.asarray(origins, np.int64).reshape(-1, 3) >> 3)


def leaf_cost(masks: np.ndarray) -> np.ndarray:
    """Per-leaf cost for balancing: 1 per leaf (the stencils stage whole leaves)
    plus its fraction of active voxels."""
    act = np.unpackbits(np.ascontiguousarray(masks).view(np.uint8).reshape(-1, 64), axis=1).sum(axis=1)
    return 1.0 + act / 512.0


class Partition:
    """Key ranges of ``world`` ranks: rank r owns keys in [s[r-1], s[r]) (s[-1] = 0,
    s[world-1] = 2^63), ``s`` the world - 1 non-decreasing splitters."""

    def __init__(self, splitters: np.ndarray, world: int):
        s = np.asarray(splitters, np.uint64).reshape(-1)
        if len(s) != world - 1 or (len(s) > 1 and np.any(s[1:] < s[:-1])):
            raise ValueError("need world - 1 non-decreasing splitters")
        self.splitters = s
        self.world = world

    @classmethod
    def balanced(cls, keys: np.ndarray, cost: np.ndarray, world: int) -> "Partition":
        """Cut the key-sorted leaves at equal cumulative cost; every rank
        computes the same splitters from the same (keys, cost)."""
        if world < 1:
            raise ValueError("world must be >= 1")
        k = np.asarray(keys, np.uint64)
        order = np.argsort(k, kind="stable")
        ks, cs = k[order], np.cumsum(np.asarray(cost, np.float64)[order])
        total = cs[-1] if len(cs) else 0.0
        spl = []
        for j in range(1, world):
            i = int(np.searchsorted(cs, total * j / world, side="left"))
            spl.append(ks[i] if i < len(ks) else np.uint64(1 << 63))
        return cls(np.array(spl, np.uint64), world)

    def owner(self, keys: np.ndarray) -> np.ndarray:
        return np.searchsorted(self.splitters, np.asarray(keys, np.uint64), side="right").astype(np.int64)


def _offsets(d: int) -> np.ndarray:
    r = np.arange(-d, d + 1)
    return np.stack(np.meshgrid(r, r, r, indexing="ij"), -1).reshape(-1, 3)


def _near_keys(coords: np.ndarray, d: int) -> np.ndarray:
    """Sorted unique keys of every leaf coordinate within Chebyshev distance d of ``coords``."""
    if len(coords) == 0:
        return np.zeros(0, np.uint64)
    return np.unique(np.concatenate([morton_keys_of_leaf_coords(coords + o) for o in _offsets(d)]))


def _member(keys: np.ndarray, sorted_set: np.ndarray) -> np.ndarray:
    if len(sorted_set) == 0:
        return np.zeros(len(keys), bool)
    i = np.minimum(np.searchsorted(sorted_set, keys), len(sorted_set) - 1)
    return sorted_set[i] == keys


class Shard:
    """The leaves one rank owns and the three local phases of a decomposed step."""

    def __init__(self, rank: int, part: Partition, owned: Leaves, stepper: Callable[[Leaves], Leaves],
                 check_duplicates: bool = False):
        self.rank = rank
        self.part = part
        self.stepper = stepper
        self.check_duplicates = check_duplicates
        self.dtype = owned.phi.dtype
        self.owned = Leaves.empty(self.dtype)
        self.absorb([owned])

    # phase 1: ghost leaves for the other ranks
    def ghost_sends(self) -> dict[int, Leaves]:
        """Owned leaves within GHOST_DEPTH leaves of a coordinate another rank owns, per rank."""
        if len(self.owned) == 0 or self.part.world == 1:
            return {}
        if self.part.world > 64:
            raise NotImplementedError("more than 64 ranks")
        c = self.owned.origins.astype(np.int64) >> 3
        bits = np.zeros(len(c), np.uint64)
        for o in _offsets(GHOST_DEPTH):
            bits |= np.left_shift(np.uint64(1), self.part.owner(morton_keys_of_leaf_coords(c + o)).astype(np.uint64))
        out = {}
        for q in range(self.part.world):
            if q == self.rank:
                continue
            sel = np.nonzero((bits >> np.uint64(q)) & np.uint64(1))[0]
            if len(sel):
                out[q] = self.owned.take(sel)
        return out

    # phase 2: the single-device step on owned + ghost leaves
    def step_local(self, ghosts: Sequence[Leaves]) -> Leaves:
        local = Leaves.concat([self.owned, *ghosts], self.dtype)
        return self.stepper(local)

    # phase 3: exact outputs to the owners of their keys
    def route(self, out: Leaves) -> dict[int, Leaves]:
        exact = _near_keys(self.owned.origins.astype(np.int64) >> 3, 1)
        k = out.keys()
        sel = np.nonzero(_member(k, exact))[0]
        own = self.part.owner(k[sel])
        return {int(q): out.take(sel[own == q]) for q in np.unique(own)}

    def absorb(self, parts: Sequence[Leaves]):
        """New owned set: the union of routed parts (first copy of a key wins), key-sorted."""
        allp = Leaves.concat(parts, self.dtype)
        k = allp.keys()
        uk, first = np.unique(k, return_index=True)
        if self.check_duplicates and len(uk) < len(k):
            order = np.argsort(k, kind="stable")
            ks = k[order]
            dup = np.nonzero(ks[1:] == ks[:-1])[0]
            for i in dup:
                a, b = order[i], order[i + 1]
                if not (np.array_equal(allp.masks[a], allp.masks[b]) and
                        np.array_equal(allp.phi[a].view(np.uint8), allp.phi[b].view(np.uint8))):
                    raise AssertionError("leaf %s arrived with different contents" % (allp.origins[a].tolist(),))
        self.owned = allp.take(first)

    def migrate(self, part: Partition) -> dict[int, Leaves]:
        """Owned leaves grouped by their owner under a new partition."""
        self.part = part
        own = part.owner(self.owned.keys())
        return {int(q): self.owned.take(own == q) for q in np.unique(own)}


# ------------------------------------------------------------------ exchanges

class LocalExchange:
    """In-process delivery between shards of one process (all ranks emulated)."""

    def __call__(self, sends: Sequence[dict[int, Leaves]]) -> list[list[Leaves]]:
        n = len(sends)
        return [[sends[q][r] for q in range(n) if r in sends[q]] for r in range(n)]

    def all_keys_and_cost(self, shards: Sequence[Shard]):
        k = np.concatenate([s.owned.keys() for s in shards])
        c = np.concatenate([leaf_cost(s.owned.masks) for s in shards])
        return k, c


class DistExchange:
    """Point-to-point leaf exchange over torch.distributed for the one shard of
    this process: a world x world count matrix (all_gather), then the packed
    records (batch_isend_irecv), in rank order on the receiving side."""

    def __init__(self, dtype, group=None, device=None):
        import torch
        import torch.distributed as dist
        self.torch, self.dist, self.group = torch, dist, group
        self.rank = dist.get_rank(group)
        self.world = dist.get_world_size(group)
        if device is None:
            device = (torch.device("cuda", torch.cuda.current_device()) if dist.get_backend(group) == "nccl"
                      else torch.device("cpu"))
        self.device = device
        self.dtype = np.dtype(dtype)

    def __call__(self, sends: Sequence[dict[int, Leaves]]) -> list[list[Leaves]]:
        (mine,) = sends
        torch, dist = self.torch, self.dist
        packed = {q: l.pack() for q, l in mine.items() if q != self.rank and len(l)}
        cnt = torch.zeros(self.world, dtype=torch.int64)
        for q, b in packed.items():
            cnt[q] = b.size
        cnt = cnt.to(self.device)
        rows = [torch.zeros_like(cnt) for _ in range(self.world)]
        dist.all_gather(rows, cnt, group=self.group)
        mat = torch.stack(rows).cpu().numpy()  # mat[src, dst] bytes
        ops, bufs = [], {}
        for q in range(self.world):
            if q != self.rank and mat[self.rank, q] > 0:
                ops.append(dist.P2POp(dist.isend, torch.from_numpy(packed[q]).to(self.device), q, self.group))
        for q in range(self.world):
            if q != self.rank and mat[q, self.rank] > 0:
                bufs[q] = torch.empty(int(mat[q, self.rank]), dtype=torch.uint8, device=self.device)
                ops.append(dist.P2POp(dist.irecv, bufs[q], q, self.group))
        if ops:
            for req in dist.batch_isend_irecv(ops):
                req.wait()
        out = []
        for q in range(self.world):
            if q == self.rank:
                if self.rank in mine:
                    out.append(mine[self.rank])
            elif q in bufs:
                out.append(Leaves.unpack(bufs[q].cpu().numpy(), self.dtype))
        return [out]

    def all_keys_and_cost(self, shards: Sequence[Shard]):
        (s,) = shards
        k = s.owned.keys().view(np.int64)
        c = leaf_cost(s.owned.masks)
        parts = self.all_gather_arrays([k, c])
        return (np.concatenate([p[0] for p in parts]).view(np.uint64), np.concatenate([p[1] for p in parts]))

    def all_gather_arrays(self, arrays: list[np.ndarray]) -> list[list[np.ndarray]]:
        """Every rank's list of 1-D arrays (same dtypes on all ranks), in rank order."""
        torch, dist = self.torch, self.dist
        n = torch.tensor([len(arrays[0])], dtype=torch.int64, device=self.device)
        ns = [torch.zeros_like(n) for _ in range(self.world)]
        dist.all_gather(ns, n, group=self.group)
        ns = [int(x.item()) for x in ns]
        mx = max(ns)
        per = [[None] * len(arrays) for _ in range(self.world)]
        for j, a in enumerate(arrays):
            t = torch.zeros(mx, dtype=torch.from_numpy(a[:0]).dtype, device=self.device)
            t[: len(a)] = torch.from_numpy(np.ascontiguousarray(a)).to(self.device)
            ts = [torch.zeros_like(t) for _ in range(self.world)]
            dist.all_gather(ts, t, group=self.group)
            for r in range(self.world):
                per[r][j] = ts[r][: ns[r]].cpu().numpy()
        return per


# ------------------------------------------------------------------ drivers

def step_shards(shards: Sequence[Shard], exchange) -> None:
    """One decomposed step of every shard of this process."""
    ghosts = exchange([s.ghost_sends() for s in shards])
    outs = [s.step_local(g) for s, g in zip(shards, ghosts)]
    parts = exchange([s.route(o) for s, o in zip(shards, outs)])
    for s, p in zip(shards, parts):
        s.absorb(p)


def rebalance_shards(shards: Sequence[Shard], exchange) -> Partition:
    """Re-cut the key ranges at equal cost over the current leaves and move
    leaves to their new owners."""
    k, c = exchange.all_keys_and_cost(shards)
    part = Partition.balanced(k, c, shards[0].part.world)
    parts = exchange([s.migrate(part) for s in shards])
    for s, p in zip(shards, parts):
        s.owned = Leaves.empty(s.dtype)
        s.absorb(p)
    return part


class DeviceStepper:
    """One method step of a rank's local leaves on this process's device: a
    single-grid ``LevelSet`` kept across steps, fed through the host step of
    the C ABI (upload, step, download in one call).  It is re-created, with
    its step counter carried over (so the time of every step is the same f32
    value as in an undivided run), when the local leaves outgrow its
    capacity or leave the box its velocity tables cover."""

    def __init__(self, velocity: dict, dt: float, half_width: float = 3.0, precision: int = 1, integrator: int = 3,
                 reinit_iters: int = 2, t0: float = 0.0, reinit_mode: int = 0, ctx=None, margin: int = 512):
        self.velocity, self.dt, self.hw = dict(velocity), dt, half_width
        self.precision, self.integrator, self.reinit_iters = precision, integrator, reinit_iters
        self.t0, self.reinit_mode, self.ctx, self.margin = t0, reinit_mode, ctx, margin
        self.steps = 0
        self.ls = None
        self.cap = 0
        self.box = None

    def _fits(self, lv: Leaves) -> bool:
        if self.ls is None or 2 * len(lv) + 64 > self.cap:
            return False
        if self.box is None:
            return True
        lo, hi = lv.origins.min(axis=0), lv.origins.max(axis=0) + 7
        return bool(np.all(lo >= self.box[0] + 64) and np.all(hi <= self.box[1] - 64))

    def _create(self, lv: Leaves):
        from .method import LevelSet
        if self.ls is not None:
            self.ls.close()
        vel = dict(self.velocity)
        self.box = None
        if vel["kind"] == "curl" and "domain" not in vel:
            # tables of sin/cos per integer index: the same values whatever box they cover
            lo = lv.origins.min(axis=0) - self.margin
            hi = lv.origins.max(axis=0) + 7 + self.margin
            vel["domain"] = (tuple(int(v) for v in lo), tuple(int(v) for v in hi))
            self.box = (lo, hi)
        self.cap = 4 * len(lv) + 4096
        self.ls = LevelSet.from_leaves(lv.origins, lv.masks, lv.phi.astype(np.float32), vel, self.dt, self.hw,
                                       self.precision, self.integrator, self.reinit_iters, self.t0, self.cap,
                                       self.reinit_mode, ctx=self.ctx)
        self.ls.set_step(self.steps)

    def __call__(self, lv: Leaves) -> Leaves:
        if len(lv) == 0:
            self.steps += 1
            return Leaves.empty(np.float32)
        if not self._fits(lv):
            self._create(lv)
            self.ls.step(1)
            o, m, p = self.ls.arrays()
        else:
            o, m, p = self.ls.step_host(lv.origins, lv.masks, lv.phi.astype(np.float32), 1)
            o, m, p = o.copy(), m.copy(), p.copy()
        self.steps += 1
        return Leaves(o, m, p)

    def close(self):
        if self.ls is not None:
            self.ls.close()
            self.ls = None


def split(leaves: Leaves, world: int) -> tuple[Partition, list[Leaves]]:
    """Balanced key ranges over ``leaves`` and each rank's share."""
    k = leaves.keys()
    part = Partition.balanced(k, leaf_cost(leaves.masks), world)
    own = part.owner(k)
    return part, [leaves.take(own == r) for r in range(world)]


def emulate(leaves: Leaves, world: int, make_stepper: Callable[[int], Callable[[Leaves], Leaves]], steps: int,
            rebalance_every: int = 0, check_duplicates: bool = True) -> tuple[Leaves, list[Shard]]:
    """Run ``world`` ranks of the decomposition in this process for ``steps``
    steps; returns the union of the owned leaves in (x, y, z) order and the
    shards."""
    part, shares = split(leaves, world)
    shards = [Shard(r, part, shares[r], make_stepper(r), check_duplicates) for r in range(world)]
    ex = LocalExchange()
    for s in range(steps):
        step_shards(shards, ex)
        if rebalance_every and (s + 1) % rebalance_every == 0:
            rebalance_shards(shards, ex)
    return Leaves.concat([sh.owned for sh in shards], shards[0].dtype).sorted_xyz(), shards


class SpatialLevelSet:
    """One rank of a level set divided over the ranks of a process group.

    Every rank passes the same global leaves (or at least the same keys to cut
    at: each keeps only its own share) and a stepper for its device
    (``DeviceStepper``); ``step`` runs decomposed steps, ``arrays`` returns the
    owned leaves, ``gather`` the whole grid on every rank."""

    def __init__(self, leaves: Leaves, stepper: Callable[[Leaves], Leaves], group=None, device=None,
                 check_duplicates: bool = False):
        self.ex = DistExchange(leaves.phi.dtype, group, device)
        part, shares = split(leaves, self.ex.world)
        self.shard = Shard(self.ex.rank, part, shares[self.ex.rank], stepper, check_duplicates)

    def step(self, n: int = 1):
        for _ in range(n):
            step_shards([self.shard], self.ex)

    def rebalance(self):
        rebalance_shards([self.shard], self.ex)

    def arrays(self) -> Leaves:
        return self.shard.owned

    def gather(self) -> Leaves:
        s = self.shard
        (parts,) = self.ex([{q: s.owned for q in range(self.ex.world)}])
        return Leaves.concat(parts, s.dtype).sorted_xyz()

    def active_voxels(self) -> int:
        per = self.ex.all_gather_arrays([np.array([self.shard.owned.active_voxels()], np.int64)])
        return int(sum(int(p[0][0]) for p in per))
