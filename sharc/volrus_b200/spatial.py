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

Leaf records live in torch tensors on the rank's device (origins i32 (n, 3),
masks as i64 (n, 8) holding the u64 bits, values (n, 512)); keys, owners and
selections are computed there too.  Exchanges are ``torch.distributed``
point-to-point transfers of those tensors (NCCL between GPUs, straight from
device memory; gloo on CPU); ``DeviceStepper`` moves the local leaves into
and out of its level set with the device-resident C ABI
(``vlr_ls_upload_device`` / ``vlr_ls_download_device``), so no value crosses
the host.  ``emulate`` runs all ranks in one process with the same logic and
in-process delivery, which is how a single device checks the decomposition
against the undivided run.

The crate has no multi-device path: this is the decomposition of the
single-grid step (src/tools/advection.rs:32-56 with the method's re-tracking)
over devices, leaf records as in src/nano/layout.rs:89-170 (origin, mask,
512 values in ZYX order).
"""
from __future__ import annotations

from dataclasses import dataclass
from typing import Callable, Sequence

import numpy as np
import torch

GHOST_DEPTH = 2  # leaves; derivation in the module docstring
_CHUNK = 1 << 24  # neighbour coordinates evaluated per batch (bounds the temporaries)
_BIAS = 1 << 20  # leaf coordinates (origin >> 3) are biased to 21-bit non-negative fields
_POP8 = torch.tensor([bin(i).count("1") for i in range(256)], dtype=torch.int64)


@dataclass
class Leaves:
    """Leaf records on one device: origins (n, 3) i32, masks (n, 8) i64 (u64
    bits), phi (n, 512) f32 or f64."""
    origins: torch.Tensor
    masks: torch.Tensor
    phi: torch.Tensor

    def __len__(self) -> int:
        return int(self.origins.shape[0])

    @property
    def device(self):
        return self.origins.device

    @classmethod
    def empty(cls, dtype=torch.float32, device="cpu") -> "Leaves":
        return cls(torch.zeros((0, 3), dtype=torch.int32, device=device),
                   torch.zeros((0, 8), dtype=torch.int64, device=device),
                   torch.zeros((0, 512), dtype=dtype, device=device))

    @classmethod
    def from_numpy(cls, origins, masks, phi, device="cpu") -> "Leaves":
        return cls(torch.from_numpy(np.ascontiguousarray(origins, np.int32)).to(device),
                   torch.from_numpy(np.ascontiguousarray(masks, np.uint64).view(np.int64)).to(device),
                   torch.from_numpy(np.ascontiguousarray(phi)).to(device))

    def numpy(self):
        """(origins i32, masks u64, phi) on the host."""
        return (self.origins.cpu().numpy(), self.masks.cpu().numpy().view(np.uint64), self.phi.cpu().numpy())

    def to(self, device) -> "Leaves":
        return Leaves(self.origins.to(device), self.masks.to(device), self.phi.to(device))

    def take(self, idx) -> "Leaves":
        return Leaves(self.origins[idx], self.masks[idx], self.phi[idx])

    @staticmethod
    def concat(parts: Sequence["Leaves"], like: "Leaves") -> "Leaves":
        parts = [p for p in parts if len(p)]
        if not parts:
            return Leaves.empty(like.phi.dtype, like.device)
        return Leaves(torch.cat([p.origins for p in parts]), torch.cat([p.masks for p in parts]),
                      torch.cat([p.phi for p in parts]))

    def coords(self) -> torch.Tensor:
        return self.origins.to(torch.int64) >> 3

    def keys(self) -> torch.Tensor:
        return morton_keys_of_leaf_coords(self.coords())

    def sorted_xyz(self) -> "Leaves":
        """Records in (x, y, z) order of the origin, as ``LevelSet.arrays``."""
        c = self.coords() + _BIAS
        return self.take(torch.argsort((c[:, 0] << 42) | (c[:, 1] << 21) | c[:, 2]))

    def active_per_leaf(self) -> torch.Tensor:
        b = self.masks.contiguous().view(torch.uint8).reshape(len(self), 64).to(torch.int64)
        return _POP8.to(b.device)[b].sum(dim=1)

    def active_voxels(self) -> int:
        return int(self.active_per_leaf().sum().item()) if len(self) else 0


def _spread(v: torch.Tensor) -> torch.Tensor:
    """21-bit integers with their bits moved to every third position (bit b -> 3b)."""
    x = v & 0x1FFFFF
    x = (x | (x << 32)) & 0x1F00000000FFFF
    x = (x | (x << 16)) & 0x1F0000FF0000FF
    x = (x | (x << 8)) & 0x100F00F00F00F00F
    x = (x | (x << 4)) & 0x10C30C30C30C30C3
    x = (x | (x << 2)) & 0x1249249249249249
    return x


def morton_keys_of_leaf_coords(c: torch.Tensor, check: bool = True) -> torch.Tensor:
    """63-bit Z-order keys (i64, non-negative) of leaf coordinates (origin >> 3),
    x in the highest bit of each triple.  Coordinates are biased by 2^20
    (|origin| < 2^23 voxels).  A key grows with each coordinate when the other
    two are fixed (it is 4 spread(x) + 2 spread(y) + spread(z)), so over a box
    the smallest and largest keys are those of its low and high corners."""
    c = c.to(torch.int64).reshape(-1, 3) + _BIAS
    if check and c.numel() and (int(c.min()) < 0 or int(c.max()) >= (1 << 21)):
        raise ValueError("leaf coordinate outside the 21-bit key range (|origin| >= 2^23 voxels)")
    return (_spread(c[:, 0]) << 2) | (_spread(c[:, 1]) << 1) | _spread(c[:, 2])


def leaf_cost(leaves: Leaves) -> torch.Tensor:
    """Per-leaf cost for balancing: 1 per leaf (the stencils stage whole leaves)
    plus its fraction of active voxels."""
    return 1.0 + leaves.active_per_leaf().to(torch.float64) / 512.0


class Partition:
    """Key ranges of ``world`` ranks: rank r owns keys in [s[r-1], s[r]) (s[-1] = 0,
    s[world-1] = 2^63), ``s`` the world - 1 non-decreasing splitters."""

    def __init__(self, splitters, world: int):
        s = torch.as_tensor(splitters, dtype=torch.int64).reshape(-1).cpu()
        if len(s) != world - 1 or (len(s) > 1 and bool((s[1:] < s[:-1]).any())):
            raise ValueError("need world - 1 non-decreasing splitters")
        self.splitters = s
        self.world = world
        self._on = {}

    @classmethod
    def balanced(cls, keys: torch.Tensor, cost: torch.Tensor, world: int) -> "Partition":
        """Cut the key-sorted leaves at equal cumulative cost; every rank
        computes the same splitters from the same (keys, cost)."""
        if world < 1:
            raise ValueError("world must be >= 1")
        k = keys.to(torch.int64).cpu()
        ks, order = torch.sort(k, stable=True)
        cs = torch.cumsum(cost.to(torch.float64).cpu()[order], 0)
        total = float(cs[-1]) if len(cs) else 0.0
        spl = []
        for j in range(1, world):
            i = int(torch.searchsorted(cs, torch.tensor([total * j / world], dtype=torch.float64)))
            spl.append(int(ks[i]) if i < len(ks) else (1 << 63) - 1)
        return cls(spl, world)

    def owner(self, keys: torch.Tensor) -> torch.Tensor:
        dev = keys.device
        if self.world == 1:
            return torch.zeros(len(keys), dtype=torch.int64, device=dev)
        if dev not in self._on:
            self._on[dev] = self.splitters.to(dev)
        return torch.searchsorted(self._on[dev], keys.to(torch.int64), right=True)


def _offsets(d: int, device="cpu") -> torch.Tensor:
    r = torch.arange(-d, d + 1, device=device)
    return torch.stack(torch.meshgrid(r, r, r, indexing="ij"), -1).reshape(-1, 3)


def _member(keys: torch.Tensor, sorted_set: torch.Tensor) -> torch.Tensor:
    if len(sorted_set) == 0:
        return torch.zeros(len(keys), dtype=torch.bool, device=keys.device)
    i = torch.clamp(torch.searchsorted(sorted_set, keys), max=len(sorted_set) - 1)
    return sorted_set[i] == keys


class Shard:
    """The leaves one rank owns and the three local phases of a decomposed step."""

    def __init__(self, rank: int, part: Partition, owned: Leaves, stepper: Callable[[Leaves], Leaves],
                 check_duplicates: bool = False):
        self.rank = rank
        self.part = part
        self.stepper = stepper
        self.check_duplicates = check_duplicates
        self.like = Leaves.empty(owned.phi.dtype, owned.device)
        self.owned = self.like
        self.owned_keys = torch.zeros(0, dtype=torch.int64, device=owned.device)
        self.absorb([owned])

    # phase 1: ghost leaves for the other ranks
    def ghost_sends(self) -> dict[int, Leaves]:
        """Owned leaves within GHOST_DEPTH leaves of a coordinate another rank owns, per rank."""
        if len(self.owned) == 0 or self.part.world == 1:
            return {}
        if self.part.world > 63:
            raise NotImplementedError("more than 63 ranks")
        c = self.owned.coords()
        d = GHOST_DEPTH
        # the owners over a leaf's box lie between those of its corner keys (keys
        # grow along each axis, owners along the keys): leaves whose whole box
        # is this rank's send nothing
        lo = self.part.owner(morton_keys_of_leaf_coords(c - d))
        hi = self.part.owner(morton_keys_of_leaf_coords(c + d))
        cand = torch.nonzero((lo != self.rank) | (hi != self.rank)).reshape(-1)
        out = {}
        if len(cand) == 0:
            return out
        offs = _offsets(d, c.device)
        hits = {q: [] for q in range(self.part.world) if q != self.rank}
        step = max(1, _CHUNK // len(offs))
        for i in range(0, len(cand), step):
            ci = cand[i:i + step]
            box = (c[ci][:, None, :] + offs[None]).reshape(-1, 3)
            own = self.part.owner(morton_keys_of_leaf_coords(box, False)).reshape(len(ci), len(offs))
            for q in hits:
                hits[q].append(ci[(own == q).any(dim=1)])
        for q, parts in hits.items():
            sel = torch.cat(parts)
            if len(sel):
                out[q] = self.owned.take(sel)
        return out

    # phase 2: the single-device step on owned + ghost leaves
    def step_local(self, ghosts: Sequence[Leaves]) -> Leaves:
        return self.stepper(Leaves.concat([self.owned, *ghosts], self.like))

    # phase 3: exact outputs to the owners of their keys
    def route(self, out: Leaves) -> dict[int, Leaves]:
        """Outputs within one leaf of an owned input leaf, by the owner of their key:
        an output that is itself an owned input leaf, or one with an owned
        input leaf among its 26 neighbours."""
        k = out.keys()
        exact = _member(k, self.owned_keys)
        rest = torch.nonzero(~exact).reshape(-1)
        if len(rest):
            cr = out.coords()[rest]
            morton_keys_of_leaf_coords(torch.cat([cr - 1, cr + 1]))  # range check of the whole 3^3 box
            offs = _offsets(1, k.device)
            step = max(1, _CHUNK // len(offs))
            near = []
            for i in range(0, len(cr), step):
                box = (cr[i:i + step][:, None, :] + offs[None]).reshape(-1, 3)
                near.append(_member(morton_keys_of_leaf_coords(box, False), self.owned_keys).reshape(-1, len(offs))
                            .any(dim=1))
            exact[rest] = torch.cat(near)
        sel = torch.nonzero(exact).reshape(-1)
        own = self.part.owner(k[sel])
        return {int(q): out.take(sel[own == q]) for q in torch.unique(own).tolist()}

    def absorb(self, parts: Sequence[Leaves]):
        """New owned set: the union of routed parts (first copy of a key wins), key-sorted."""
        allp = Leaves.concat(parts, self.like)
        if len(allp) == 0:
            self.owned = self.like
            self.owned_keys = torch.zeros(0, dtype=torch.int64, device=self.like.device)
            return
        ks, order = torch.sort(allp.keys(), stable=True)
        first = torch.ones(len(ks), dtype=torch.bool, device=ks.device)
        first[1:] = ks[1:] != ks[:-1]
        if self.check_duplicates and not bool(first.all()):
            dup = torch.nonzero(~first).reshape(-1)
            a, b = order[dup - 1], order[dup]
            same = torch.equal(allp.masks[a], allp.masks[b]) and torch.equal(
                allp.phi[a].contiguous().view(torch.uint8), allp.phi[b].contiguous().view(torch.uint8))
            if not same:
                raise AssertionError("a leaf arrived from two ranks with different contents")
        self.owned = allp.take(order[first])
        self.owned_keys = ks[first]

    def migrate(self, part: Partition) -> dict[int, Leaves]:
        """Owned leaves grouped by their owner under a new partition."""
        self.part = part
        own = part.owner(self.owned.keys())
        return {int(q): self.owned.take(own == q) for q in torch.unique(own).tolist()}


# ------------------------------------------------------------------ exchanges

class LocalExchange:
    """In-process delivery between the shards of one process (all ranks emulated)."""

    def __call__(self, sends: Sequence[dict[int, Leaves]]) -> list[list[Leaves]]:
        n = len(sends)
        return [[sends[q][r] for q in range(n) if r in sends[q]] for r in range(n)]

    def all_keys_and_cost(self, shards: Sequence[Shard]):
        return (torch.cat([s.owned.keys().cpu() for s in shards]), torch.cat([leaf_cost(s.owned).cpu() for s in shards]))


class DistExchange:
    """Point-to-point leaf exchange over torch.distributed for the one shard of
    this process: a world x world count matrix (all_gather), then each peer's
    origins, masks and values (batch_isend_irecv), in rank order on the
    receiving side.  Tensors stay on the shard's device (CUDA for NCCL)."""

    def __init__(self, like: Leaves, group=None):
        import torch.distributed as dist
        self.dist, self.group = dist, group
        self.rank = dist.get_rank(group)
        self.world = dist.get_world_size(group)
        self.like = like

    def __call__(self, sends: Sequence[dict[int, Leaves]]) -> list[list[Leaves]]:
        (mine,) = sends
        dist, dev = self.dist, self.like.device
        cnt = torch.zeros(self.world, dtype=torch.int64, device=dev)
        for q, l in mine.items():
            if q != self.rank:
                cnt[q] = len(l)
        rows = [torch.zeros_like(cnt) for _ in range(self.world)]
        dist.all_gather(rows, cnt, group=self.group)
        mat = torch.stack(rows).cpu()  # mat[src, dst] leaves
        ops, bufs = [], {}
        for q in range(self.world):
            if q != self.rank and int(mat[self.rank, q]) > 0:
                l = mine[q]
                for t in (l.origins, l.masks, l.phi):
                    ops.append(dist.P2POp(dist.isend, t.contiguous(), q, self.group))
        for q in range(self.world):
            n = int(mat[q, self.rank])
            if q != self.rank and n > 0:
                b = Leaves(torch.empty((n, 3), dtype=torch.int32, device=dev),
                           torch.empty((n, 8), dtype=torch.int64, device=dev),
                           torch.empty((n, 512), dtype=self.like.phi.dtype, device=dev))
                bufs[q] = b
                for t in (b.origins, b.masks, b.phi):
                    ops.append(dist.P2POp(dist.irecv, t, q, self.group))
        if ops:
            for req in dist.batch_isend_irecv(ops):
                req.wait()
        out = []
        for q in range(self.world):
            if q == self.rank and self.rank in mine:
                out.append(mine[self.rank])
            elif q in bufs:
                out.append(bufs[q])
        return [out]

    def all_gather_1d(self, t: torch.Tensor) -> list[torch.Tensor]:
        """Every rank's 1-D tensor (same dtype on all ranks), in rank order."""
        dist, dev = self.dist, self.like.device
        n = torch.tensor([len(t)], dtype=torch.int64, device=dev)
        ns = [torch.zeros_like(n) for _ in range(self.world)]
        dist.all_gather(ns, n, group=self.group)
        ns = [int(x.item()) for x in ns]
        pad = torch.zeros(max(ns), dtype=t.dtype, device=dev)
        pad[: len(t)] = t.to(dev)
        got = [torch.zeros_like(pad) for _ in range(self.world)]
        dist.all_gather(got, pad, group=self.group)
        return [g[:m] for g, m in zip(got, ns)]

    def all_keys_and_cost(self, shards: Sequence[Shard]):
        (s,) = shards
        k = torch.cat(self.all_gather_1d(s.owned.keys())).cpu()
        c = torch.cat(self.all_gather_1d(leaf_cost(s.owned))).cpu()
        return k, c


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
        s.absorb(p)
    return part


class DeviceStepper:
    """One method step of a rank's local leaves (CUDA tensors on the context's
    device): a single-grid ``LevelSet`` kept across steps, its state replaced
    and read back through the device-resident C ABI, so values stay in HBM.
    It is re-created, with its step counter carried over (every step's time is
    then the same f32 value as in an undivided run), when the local leaves
    outgrow its capacity or leave the box its velocity tables cover.  The
    returned leaves are views of its output buffers, valid until the next call."""

    def __init__(self, velocity: dict, dt: float, half_width: float = 3.0, precision: int = 1, integrator: int = 3,
                 reinit_iters: int = 2, t0: float = 0.0, reinit_mode: int = 0, ctx=None, margin: int = 512):
        self.velocity, self.dt, self.hw = dict(velocity), dt, half_width
        self.precision, self.integrator, self.reinit_iters = precision, integrator, reinit_iters
        self.t0, self.reinit_mode, self.ctx, self.margin = t0, reinit_mode, ctx, margin
        self.steps = 0
        self.ls = None
        self.cap = 0
        self.box = None
        self.out = None

    def _fits(self, lv: Leaves) -> bool:
        if self.ls is None or 2 * len(lv) + 64 > self.cap:
            return False
        if self.box is None:
            return True
        lo = lv.origins.min(dim=0).values.cpu().numpy()
        hi = lv.origins.max(dim=0).values.cpu().numpy() + 7
        return bool(np.all(lo >= self.box[0] + 64) and np.all(hi <= self.box[1] - 64))

    def _create(self, lv: Leaves):
        from .method import LevelSet
        if self.ls is not None:
            self.ls.close()
        o, m, p = lv.numpy()
        vel = dict(self.velocity)
        self.box = None
        if vel["kind"] == "curl" and "domain" not in vel:
            # tables of sin/cos per integer index: the same values whatever box they cover
            lo, hi = o.min(axis=0) - self.margin, o.max(axis=0) + 7 + self.margin
            vel["domain"] = (tuple(int(v) for v in lo), tuple(int(v) for v in hi))
            self.box = (lo, hi)
        self.cap = 3 * len(lv) + 4096
        self.ls = LevelSet.from_leaves(o, m, p.astype(np.float32), vel, self.dt, self.hw, self.precision,
                                       self.integrator, self.reinit_iters, self.t0, self.cap, self.reinit_mode,
                                       ctx=self.ctx)
        self.ls.set_step(self.steps)
        dev = lv.device
        self.out = Leaves(torch.empty((self.cap, 3), dtype=torch.int32, device=dev),
                          torch.empty((self.cap, 8), dtype=torch.int64, device=dev),
                          torch.empty((self.cap, 512), dtype=torch.float32, device=dev))

    def __call__(self, lv: Leaves) -> Leaves:
        if len(lv) == 0:
            self.steps += 1
            return Leaves.empty(torch.float32, lv.device)
        if not self._fits(lv):
            self._create(lv)  # its counter = the steps taken so far
        else:
            lv = Leaves(lv.origins.contiguous(), lv.masks.contiguous(), lv.phi.to(torch.float32).contiguous())
            torch.cuda.current_stream(lv.device).synchronize()  # the library runs on its own stream
            self.ls.upload_device(lv.origins.data_ptr(), lv.masks.data_ptr(), lv.phi.data_ptr(), len(lv))
        self.ls.step(1)
        self.steps += 1
        n = self.ls.download_device(self.out.origins.data_ptr(), self.out.masks.data_ptr(),
                                    self.out.phi.data_ptr(), self.cap)
        return self.out.take(slice(0, n))

    def volume(self, lv: Leaves, n_first: int, ref=(0.0, 0.0, 0.0)) -> float:
        """FP64 enclosed volume over the first ``n_first`` leaves of ``lv`` (the
        owned ones; the ghosts after them supply the gradients): the sum of
        their per-leaf terms (``vlr_ls_volume_partials``) in leaf order."""
        if n_first == 0:
            return 0.0
        if not self._fits(lv):
            self._create(lv)  # the level set lists leaves in the order given
        else:
            lv = Leaves(lv.origins.contiguous(), lv.masks.contiguous(), lv.phi.to(torch.float32).contiguous())
            torch.cuda.current_stream(lv.device).synchronize()
            self.ls.upload_device(lv.origins.data_ptr(), lv.masks.data_ptr(), lv.phi.data_ptr(), len(lv))
        buf = torch.empty(self.cap, dtype=torch.float64, device=lv.device)
        self.ls.volume_partials(buf.data_ptr(), self.cap, ref)
        return float(buf[:n_first].sum())

    def close(self):
        if self.ls is not None:
            self.ls.close()
            self.ls = None


def volume_shards(shards: Sequence[Shard], exchange, ref=(0.0, 0.0, 0.0)) -> list[float]:
    """Each shard's FP64 volume over its owned leaves, with the ghost ring
    exchanged first so the gradients at the range edges are the undivided
    grid's.  The stepper must provide ``volume(leaves, n_owned, ref)``."""
    ghosts = exchange([s.ghost_sends() for s in shards])
    return [s.stepper.volume(Leaves.concat([s.owned, *g], s.like), len(s.owned), ref) for s, g in zip(shards, ghosts)]


def split(leaves: Leaves, world: int) -> tuple[Partition, list[Leaves]]:
    """Balanced key ranges over ``leaves`` and each rank's share."""
    k = leaves.keys()
    part = Partition.balanced(k, leaf_cost(leaves), world)
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
    return Leaves.concat([sh.owned for sh in shards], shards[0].like).sorted_xyz(), shards


class SpatialLevelSet:
    """One rank of a level set divided over the ranks of a process group.

    Every rank passes the same global leaves (on its own device; each keeps
    only its share) and a stepper for its device (``DeviceStepper``);
    ``step`` runs decomposed steps, ``arrays`` returns the owned leaves,
    ``gather`` the whole grid on every rank.  With NCCL, each process sets its
    device (``torch.cuda.set_device``) before the process group is used; the
    first transfer of a group is an all_gather that every rank joins, so the
    point-to-point batches that follow may leave a rank out."""

    def __init__(self, leaves: Leaves, stepper: Callable[[Leaves], Leaves], group=None,
                 check_duplicates: bool = False):
        self.ex = DistExchange(Leaves.empty(leaves.phi.dtype, leaves.device), group)
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
        return Leaves.concat(parts, s.like).sorted_xyz()

    def volume(self, ref=(0.0, 0.0, 0.0)) -> float:
        """FP64 enclosed volume of the whole grid: the ranks' sums added in rank order."""
        (v,) = volume_shards([self.shard], self.ex, ref)
        return float(sum(float(t[0]) for t in self.ex.all_gather_1d(torch.tensor([v], dtype=torch.float64))))

    def active_voxels(self) -> int:
        return int(sum(int(t[0]) for t in self.ex.all_gather_1d(
            torch.tensor([self.shard.owned.active_voxels()], dtype=torch.int64))))
