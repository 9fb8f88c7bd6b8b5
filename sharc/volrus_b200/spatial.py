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


def ghost_positions(c: torch.Tensor, part: Partition, rank: int, depth: int = GHOST_DEPTH) -> dict[int, torch.Tensor]:
    """Per other rank q, the indices of the leaves at coordinates ``c`` (owned
    by ``rank``) within ``depth`` leaves of a coordinate q owns."""
    if len(c) == 0 or part.world == 1:
        return {}
    if part.world > 63:
        raise NotImplementedError("more than 63 ranks")
    d = depth
    # the owners over a leaf's box lie between those of its corner keys (keys
    # grow along each axis, owners along the keys): leaves whose whole box
    # is this rank's send nothing
    lo = part.owner(morton_keys_of_leaf_coords(c - d))
    hi = part.owner(morton_keys_of_leaf_coords(c + d))
    cand = torch.nonzero((lo != rank) | (hi != rank)).reshape(-1)
    if len(cand) == 0:
        return {}
    offs = _offsets(d, c.device)
    hits = {q: [] for q in range(part.world) if q != rank}
    step = max(1, _CHUNK // len(offs))
    for i in range(0, len(cand), step):
        ci = cand[i:i + step]
        box = (c[ci][:, None, :] + offs[None]).reshape(-1, 3)
        own = part.owner(morton_keys_of_leaf_coords(box, False)).reshape(len(ci), len(offs))
        for q in hits:
            hits[q].append(ci[(own == q).any(dim=1)])
    out = {}
    for q, parts in hits.items():
        sel = torch.cat(parts)
        if len(sel):
            out[q] = sel
    return out


def exact_outputs(k: torch.Tensor, c: torch.Tensor, owned_keys: torch.Tensor) -> torch.Tensor:
    """Which outputs (keys ``k``, coordinates ``c``) of a local step are exact:
    an owned input leaf itself, or a leaf with an owned input leaf
    (``owned_keys``, sorted) among its 26 neighbours."""
    exact = _member(k, owned_keys)
    rest = torch.nonzero(~exact).reshape(-1)
    if len(rest):
        cr = c[rest]
        morton_keys_of_leaf_coords(torch.cat([cr - 1, cr + 1]))  # range check of the whole 3^3 box
        offs = _offsets(1, k.device)
        step = max(1, _CHUNK // len(offs))
        near = []
        for i in range(0, len(cr), step):
            box = (cr[i:i + step][:, None, :] + offs[None]).reshape(-1, 3)
            near.append(_member(morton_keys_of_leaf_coords(box, False), owned_keys).reshape(-1, len(offs))
                        .any(dim=1))
        exact[rest] = torch.cat(near)
    return exact


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
        return {q: self.owned.take(sel) for q, sel in ghost_positions(self.owned.coords(), self.part, self.rank).items()}

    # phase 2: the single-device step on owned + ghost leaves
    def step_local(self, ghosts: Sequence[Leaves]) -> Leaves:
        return self.stepper(Leaves.concat([self.owned, *ghosts], self.like))

    # phase 3: exact outputs to the owners of their keys
    def route(self, out: Leaves) -> dict[int, Leaves]:
        """Outputs within one leaf of an owned input leaf, by the owner of their key:
        an output that is itself an owned input leaf, or one with an owned
        input leaf among its 26 neighbours."""
        k = out.keys()
        sel = torch.nonzero(exact_outputs(k, out.coords(), self.owned_keys)).reshape(-1)
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


class DevicePool:
    """A rank's leaves resident in a single-grid ``LevelSet`` on its device.

    Between steps the pool holds exactly the rank's owned leaves; during a
    step it also holds the ghost ring.  Leaves come in and go out through the
    pool edits of the C ABI (``vlr_ls_gather_device``, ``vlr_ls_edit_device``)
    with values in the pool's own type (FP16 for an FP16 level set), so a
    ghost is its owner's copy bit for bit and the owned leaves never leave
    HBM.  The level set is re-created from its own leaves (step counter
    carried over, values converted f16 -> f32 -> f16 exactly) when the leaves
    it must hold outgrow half its capacity, or, for a curl velocity without a
    domain, come within 64 voxels of the box its tables cover."""

    def __init__(self, leaves: Leaves, velocity: dict, dt: float, half_width: float = 3.0, precision: int = 1,
                 integrator: int = 3, reinit_iters: int = 2, t0: float = 0.0, reinit_mode: int = 0, ctx=None,
                 margin: int = 512):
        self.velocity, self.dt, self.hw = dict(velocity), dt, half_width
        self.precision, self.integrator, self.reinit_iters = precision, integrator, reinit_iters
        self.t0, self.reinit_mode, self.ctx, self.margin = t0, reinit_mode, ctx, margin
        self.device = leaves.device
        self.dtype = torch.float16 if precision == 1 else torch.float32
        self.steps = 0
        self.ls = None
        self.box = None
        self._create(leaves, 2 * len(leaves))

    def _create(self, lv: Leaves, room: int):
        from .method import LevelSet
        if self.ls is not None:
            self.ls.close()
        o, m, p = lv.numpy()
        vel = dict(self.velocity)
        self.box = None
        if vel["kind"] == "curl" and "domain" not in vel:
            # tables of sin/cos per integer index: the same values whatever box they cover
            lo = (o.min(axis=0) if len(o) else np.zeros(3, np.int64)) - self.margin
            hi = (o.max(axis=0) if len(o) else np.zeros(3, np.int64)) + 7 + self.margin
            vel["domain"] = (tuple(int(v) for v in lo), tuple(int(v) for v in hi))
            self.box = (lo, hi)
        self.cap = 2 * max(room, len(lv)) + 4096
        self.ls = LevelSet.from_leaves(o, m, p.astype(np.float32), vel, self.dt, self.hw, self.precision,
                                       self.integrator, self.reinit_iters, self.t0, self.cap, self.reinit_mode,
                                       ctx=self.ctx)
        self.ls.set_step(self.steps)

    def _sync(self):
        if self.device.type == "cuda":
            torch.cuda.current_stream(self.device).synchronize()  # the library runs on its own stream

    def count(self) -> int:
        return self.ls.leaf_count()

    def origins(self) -> torch.Tensor:
        n = self.count()
        o = torch.empty((n, 3), dtype=torch.int32, device=self.device)
        self._sync()
        self.ls.gather_device(None, n, o.data_ptr())
        return o

    def gather(self, pos: torch.Tensor | None = None) -> Leaves:
        """Leaves at list positions ``pos`` (all when None), values in the pool's type."""
        n = self.count() if pos is None else len(pos)
        out = Leaves(torch.empty((n, 3), dtype=torch.int32, device=self.device),
                     torch.empty((n, 8), dtype=torch.int64, device=self.device),
                     torch.empty((n, 512), dtype=self.dtype, device=self.device))
        if n:
            p = None if pos is None else pos.to(device=self.device, dtype=torch.int32).contiguous()
            self._sync()
            self.ls.gather_device(None if p is None else p.data_ptr(), n, out.origins.data_ptr(),
                                  out.masks.data_ptr(), out.phi.data_ptr())
        return out

    def _room(self, n_new: int):
        """Re-create the level set if ``n_new`` leaves (and the step's growth)
        would not fit, or would leave the velocity tables' box."""
        if 2 * n_new + 64 <= self.cap and self.box is None:
            return
        o = self.origins()
        inside = True
        if self.box is not None and len(o):
            lo = o.min(dim=0).values.cpu().numpy()
            hi = o.max(dim=0).values.cpu().numpy() + 7
            inside = bool(np.all(lo >= self.box[0] + 64) and np.all(hi <= self.box[1] - 64))
        if 2 * n_new + 64 > self.cap or not inside:
            self._create(self.gather(), n_new)

    def edit(self, drop: torch.Tensor | None, add: Leaves):
        """Drop the listed leaves flagged in ``drop`` (bool per list position;
        None drops none), keep the rest in order, append ``add``."""
        n = self.count()
        keep_n = n if drop is None else n - int(drop.sum())
        self._room(keep_n + len(add))
        n = self.count()  # unchanged by a re-creation, which keeps the list order
        d = torch.zeros(n, dtype=torch.uint8, device=self.device) if drop is None else \
            drop.to(device=self.device, dtype=torch.uint8).contiguous()
        a = Leaves(add.origins.to(self.device, torch.int32).contiguous(),
                   add.masks.to(self.device, torch.int64).contiguous(),
                   add.phi.to(self.device, self.dtype).contiguous())
        self._sync()
        self.ls.edit_device(d.data_ptr() if n else None, n, a.origins.data_ptr() if len(a) else None,
                            a.masks.data_ptr() if len(a) else None, a.phi.data_ptr() if len(a) else None, len(a))

    def step(self):
        self._room(self.count())
        self.ls.step(1)
        self.steps += 1

    def skip(self):
        """A step of a rank with no leaves: only the counter moves."""
        self.steps += 1
        self.ls.set_step(self.steps)

    def volume_partials(self, ref=(0.0, 0.0, 0.0)) -> torch.Tensor:
        n = self.count()
        buf = torch.empty(max(n, 1), dtype=torch.float64, device=self.device)
        self._sync()
        self.ls.volume_partials(buf.data_ptr(), len(buf), ref)
        return buf[:n]

    def close(self):
        if self.ls is not None:
            self.ls.close()
            self.ls = None


class ResidentShard:
    """A shard whose owned leaves stay in a leaf pool (``DevicePool``) between
    steps.  The phases are those of ``Shard`` with the same selections
    (``ghost_positions``, ``exact_outputs``) over the pool's list: ghosts are
    gathered from the pool and added to the receiving pool in place; after
    the step the pool drops what the rank does not own and appends the exact
    outputs other ranks computed for it (a key it already holds keeps its own
    copy, which is the same bits).  Any object with the pool's methods
    (count, origins, gather, edit, step, skip, volume_partials, device,
    dtype) serves."""

    def __init__(self, rank: int, part: Partition, pool, check_duplicates: bool = False):
        self.rank, self.part, self.pool = rank, part, pool
        self.check_duplicates = check_duplicates
        self.like = Leaves.empty(pool.dtype, pool.device)
        self.owned_keys = torch.sort(morton_keys_of_leaf_coords(pool.origins() >> 3)).values
        self._keep = None
        self._keys = None

    @property
    def owned(self) -> Leaves:
        """The owned leaves (gathered from the pool; values in its type)."""
        return self.pool.gather()

    def ghost_sends(self) -> dict[int, Leaves]:
        c = self.pool.origins() >> 3
        return {q: self.pool.gather(sel) for q, sel in ghost_positions(c, self.part, self.rank).items()}

    def step_local(self, ghosts: Sequence[Leaves]):
        self.pool.edit(None, Leaves.concat(list(ghosts), self.like))
        if self.pool.count():
            self.pool.step()
        else:
            self.pool.skip()

    def route(self, _out=None) -> dict[int, Leaves]:
        o = self.pool.origins()
        c = o >> 3
        k = morton_keys_of_leaf_coords(c)
        exact = exact_outputs(k, c, self.owned_keys)
        own = self.part.owner(k)
        self._keep = exact & (own == self.rank)
        self._keys = k
        sel = torch.nonzero(exact & (own != self.rank)).reshape(-1)
        own_s = own[sel]
        return {int(q): self.pool.gather(sel[own_s == q]) for q in torch.unique(own_s).tolist()}

    def absorb(self, parts: Sequence[Leaves]):
        recv = Leaves.concat(list(parts), self.like)
        kept_keys = torch.sort(self._keys[self._keep]).values
        if len(recv):
            rk = recv.keys()
            ks, order = torch.sort(rk, stable=True)
            first = torch.ones(len(ks), dtype=torch.bool, device=ks.device)
            first[1:] = ks[1:] != ks[:-1]
            new = first & ~_member(ks, kept_keys)
            if self.check_duplicates:
                self._check_copies(recv, ks, order, first, kept_keys)
            recv = recv.take(order[new])
            add_keys = ks[new]
        else:
            add_keys = torch.zeros(0, dtype=torch.int64, device=kept_keys.device)
        self.pool.edit(~self._keep, recv)
        self.owned_keys = torch.sort(torch.cat([kept_keys, add_keys.to(kept_keys.device)])).values
        self._keep = self._keys = None

    def _check_copies(self, recv, ks, order, first, kept_keys):
        """A key that arrives twice, or that this rank keeps too, must carry the same bits."""
        dup = torch.nonzero(~first).reshape(-1)
        a, b = order[dup - 1], order[dup]
        same = torch.equal(recv.masks[a], recv.masks[b]) and torch.equal(
            recv.phi[a].contiguous().view(torch.uint8), recv.phi[b].contiguous().view(torch.uint8))
        held = torch.nonzero(first & _member(ks, kept_keys)).reshape(-1)
        if len(held):
            pos = torch.nonzero(self._keep).reshape(-1)
            mine = self.pool.gather(pos)
            mk, mo = torch.sort(mine.keys())
            j = torch.searchsorted(mk, ks[held])
            r, m = recv.take(order[held]), mine.take(mo[j])
            same = same and torch.equal(r.masks, m.masks) and torch.equal(
                r.phi.contiguous().view(torch.uint8), m.phi.contiguous().view(torch.uint8))
        if not same:
            raise AssertionError("a leaf arrived from two ranks with different contents")

    def migrate(self, part: Partition) -> dict[int, Leaves]:
        """All pool leaves grouped by their owner under a new partition; the
        following absorb replaces the pool with what arrives."""
        self.part = part
        o = self.pool.origins()
        k = morton_keys_of_leaf_coords(o >> 3)
        own = part.owner(k)
        self._keep = torch.zeros(len(k), dtype=torch.bool, device=k.device)
        self._keys = k
        return {int(q): self.pool.gather(torch.nonzero(own == q).reshape(-1)) for q in torch.unique(own).tolist()}

    def volume(self, ghosts: Sequence[Leaves], ref=(0.0, 0.0, 0.0)) -> float:
        """FP64 enclosed volume of the owned leaves, the ghosts supplying the
        gradients at the range's edges (added for the call, dropped after)."""
        n_owned = self.pool.count()
        add = Leaves.concat(list(ghosts), self.like)
        self.pool.edit(None, add)
        v = float(self.pool.volume_partials(ref)[:n_owned].sum()) if n_owned else 0.0
        drop = torch.zeros(self.pool.count(), dtype=torch.bool, device=self.pool.device)
        drop[n_owned:] = True
        self.pool.edit(drop, Leaves.empty(self.pool.dtype, self.pool.device))
        return v


def emulate_resident(leaves: Leaves, world: int, make_pool: Callable[[int, Leaves], object], steps: int,
                     rebalance_every: int = 0, check_duplicates: bool = True):
    """``emulate`` with resident shards: ``make_pool(rank, owned leaves)``
    builds each rank's pool.  Returns the union of the owned leaves in
    (x, y, z) order (values in the pools' type) and the shards."""
    part, shares = split(leaves, world)
    shards = [ResidentShard(r, part, make_pool(r, shares[r]), check_duplicates) for r in range(world)]
    ex = LocalExchange()
    for s in range(steps):
        step_shards(shards, ex)
        if rebalance_every and (s + 1) % rebalance_every == 0:
            rebalance_shards(shards, ex)
    return Leaves.concat([sh.owned for sh in shards], shards[0].like).sorted_xyz(), shards


def volume_shards(shards: Sequence[Shard], exchange, ref=(0.0, 0.0, 0.0)) -> list[float]:
    """Each shard's FP64 volume over its owned leaves, with the ghost ring
    exchanged first so the gradients at the range edges are the undivided
    grid's.  The stepper must provide ``volume(leaves, n_owned, ref)``."""
    ghosts = exchange([s.ghost_sends() for s in shards])
    return [s.volume(g, ref) if isinstance(s, ResidentShard) else
            s.stepper.volume(Leaves.concat([s.owned, *g], s.like), len(s.owned), ref) for s, g in zip(shards, ghosts)]


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


# ------------------------------------------------------------------ divided adjoint

def adjoint_ghost_depth(steps: int, reach: int = 2) -> int:
    """Leaves of ghost ring that make a rank's K-step frozen-band adjoint exact
    on its owned voxels without exchanges between steps.  One step reads phi
    (forward) or lambda (backward) within reach + 1 voxels of a voxel, so K
    steps reach K (reach + 1) voxels; one more leaf covers the 27-leaf
    neighbourhood lookups at the ring's inner edge."""
    return -(-steps * (reach + 1) // 8) + 1


def adjoint_locals(owned: Sequence[Leaves], part: Partition, depth: int, exchange,
                   ranks: Sequence[int] | None = None):
    """Each rank's local leaves for the divided adjoint, its owned leaves and
    every other rank's leaf within ``depth`` leaves of them, sorted (x, y, z)
    (the order fixes the adjoint's band order, and a sorted subset keeps the
    undivided band's relative order); also each rank's ghost sends (rank q ->
    indices into its owned leaves), which the gradient exchange reuses."""
    ranks = list(range(len(owned))) if ranks is None else list(ranks)
    sends_idx = [ghost_positions(o.coords(), part, r, depth) for r, o in zip(ranks, owned)]
    got = exchange([{q: o.take(sel) for q, sel in si.items()} for o, si in zip(owned, sends_idx)])
    locals_ = [Leaves.concat([o, *g], o).sorted_xyz() for o, g in zip(owned, got)]
    return locals_, sends_idx


def _voxel_keys(coords: torch.Tensor) -> torch.Tensor:
    """Packed 63-bit keys of voxel coordinates (21 bits per axis, biased)."""
    c = coords.to(torch.int64) + (1 << 20)
    return (c[:, 0] << 42) | (c[:, 1] << 21) | c[:, 2]


def _band_grad_leaves(leaves: Leaves, coords: torch.Tensor, grad: torch.Tensor) -> Leaves:
    """Leaf records carrying a band function: phi holds grad at the band voxels
    (coords, a subset of the leaves' voxels) and 0 elsewhere."""
    phi = torch.zeros((len(leaves), 512), dtype=leaves.phi.dtype, device=leaves.device)
    if len(coords):
        lk = morton_keys_of_leaf_coords(leaves.coords())
        order = torch.argsort(lk)
        ck = morton_keys_of_leaf_coords(torch.div(coords, 8, rounding_mode="floor"))
        li = order[torch.searchsorted(lk[order], ck)]
        loc = coords - torch.div(coords, 8, rounding_mode="floor") * 8
        off = (loc[:, 0] << 6) | (loc[:, 1] << 3) | loc[:, 2]
        phi[li, off] = grad.to(phi.dtype)
    return Leaves(leaves.origins, leaves.masks, phi)


def divided_adjoint(owned: Sequence[Leaves], part: Partition, make_engine: Callable[[int, Leaves], object],
                    loss_grad: Callable[[object, torch.Tensor, torch.Tensor], torch.Tensor], exchange,
                    steps: int, reach: int = 2, ranks: Sequence[int] | None = None, depth: int | None = None):
    """The frozen-band adjoint of a level set divided over ranks, exact on
    every rank's owned band voxels: forward phi_K and dL/dphi_0 equal the
    undivided adjoint's bit for bit when the engines sum each voxel's terms
    in the same order (a band order that is a sorted subset of the undivided
    one, and the same transpose kernel).

    Each rank builds its engine over its owned leaves plus a ghost ring of
    ``adjoint_ghost_depth(steps, reach)`` leaves and runs the K forward steps
    with no exchange between them.  The loss gradient dL/dphi_K is taken on
    the owned band voxels only (``loss_grad(engine, phi_K, owned_mask)``
    returns it for the masked band voxels), then sent the reverse way to the ranks that hold those
    voxels as ghosts, so every local band voxel starts the backward pass with
    the undivided lambda_K; the K backward steps again need no exchange.

    ``make_engine(rank, local leaves)`` returns an object with
    ``band_coords()`` (band voxel coordinates, (n, 3) int tensor),
    ``forward()`` (phi_K on the band) and ``backward(lambda_K)``
    (dL/dphi_0 on the band).  Returns per rank (coords, phi_K, dL/dphi_0) of
    its owned band voxels, and the engines.  ``owned`` holds the shards of
    this process, of ranks ``ranks`` (all ranks, 0..n-1, when emulated; this
    process's one rank with a ``DistExchange``).  ``depth`` overrides the
    ghost ring's depth in leaves."""
    ranks = list(range(len(owned))) if ranks is None else list(ranks)
    depth = adjoint_ghost_depth(steps, reach) if depth is None else depth
    locals_, sends_idx = adjoint_locals(owned, part, depth, exchange, ranks)
    engines = [make_engine(r, lv) for r, lv in zip(ranks, locals_)]
    coords = [e.band_coords() for e in engines]
    own = [part.owner(morton_keys_of_leaf_coords(torch.div(c, 8, rounding_mode="floor"))) == r
           for r, c in zip(ranks, coords)]
    phik = [e.forward() for e in engines]
    grads = []
    for e, c, m, p in zip(engines, coords, own, phik):
        g = torch.zeros(len(c), dtype=p.dtype, device=p.device)
        g[m] = loss_grad(e, p, m).to(p.dtype)
        grads.append(g)
    # dL/dphi_K of owned voxels to the ranks holding them as ghosts (the
    # leaves of the ghost sends, carrying the gradient in place of values)
    sends = []
    for o, si, c, m, g in zip(owned, sends_idx, coords, own, grads):
        gl = _band_grad_leaves(o, c[m], g[m])
        sends.append({q: gl.take(sel) for q, sel in si.items()})
    got = exchange(sends)
    results = []
    for e, c, m, g, p, parts in zip(engines, coords, own, grads, phik, got):
        lam = g.clone()
        ghost = torch.nonzero(~m).reshape(-1)
        if len(ghost) and parts:
            rl = Leaves.concat(list(parts), parts[0])
            rk = morton_keys_of_leaf_coords(rl.coords())
            order = torch.argsort(rk)
            cg = c[ghost]
            cl = torch.div(cg, 8, rounding_mode="floor")
            want = morton_keys_of_leaf_coords(cl)
            pos = torch.clamp(torch.searchsorted(rk[order], want), max=len(rk) - 1)
            if not bool((rk[order][pos] == want).all()):
                raise AssertionError("a ghost band voxel's gradient did not arrive with its leaf")
            li = order[pos]
            loc = cg - cl * 8
            off = (loc[:, 0] << 6) | (loc[:, 1] << 3) | loc[:, 2]
            lam[ghost] = rl.phi[li, off].to(lam.dtype)
        g0 = e.backward(lam)
        results.append((c[m], p[m], g0[m]))
    return results, engines


class DeviceAdjointEngine:
    """A rank's frozen-band adjoint of its local leaves on its device: a
    single-grid ``LevelSet`` over them (the level set's velocity must be
    time-independent) and its adjoint (``vlr_adj_create_level_set``), with the
    lambda transpose pinned to the windowed gather so every rank and the
    undivided run sum each voxel's terms in the same order.  Tensors stay on
    the device; calls return after their work."""

    def __init__(self, leaves: Leaves, velocity: dict, dt: float, steps: int, checkpoint_every: int,
                 half_width: float = 3.0, precision: int = 1, integrator: int = 3, ctx=None, gather: int = 1):
        from .adjoint import AdvectionFunction
        from .method import LevelSet
        o, m, p = leaves.numpy()
        self.device = leaves.device
        self.ls = LevelSet.from_leaves(o, m, p.astype(np.float32), velocity, dt, half_width, precision, integrator,
                                       2, 0.0, 0, 0, ctx=ctx)
        self.ctx = self.ls.ctx
        self.fn = AdvectionFunction.from_level_set(self.ls, steps, checkpoint_every)
        self.fn.set_gather(gather)

    def _sync(self):
        if self.device.type == "cuda":
            torch.cuda.current_stream(self.device).synchronize()

    def band_coords(self) -> torch.Tensor:
        return torch.from_numpy(self.fn.band().astype(np.int64)).to(self.device)

    def forward(self) -> torch.Tensor:
        out = torch.empty(self.fn.n_band, dtype=torch.float32, device=self.device)
        self._sync()
        self.fn.forward_device(out.data_ptr())
        self.ctx.check_device()
        return out

    def backward(self, lam_k: torch.Tensor) -> torch.Tensor:
        lam = lam_k.to(device=self.device, dtype=torch.float32).contiguous()
        out = torch.empty(self.fn.n_band, dtype=torch.float32, device=self.device)
        self._sync()
        self.fn.backward_device(lam.data_ptr(), out.data_ptr(), 0)
        self.ctx.check_device()
        return out

    def shifted_phi0(self, shift) -> torch.Tensor:
        """phi_0 translated by ``shift`` voxels, on the band (a loss target)."""
        out = torch.empty(self.fn.n_band, dtype=torch.float32, device=self.device)
        self._sync()
        self.fn.shifted_phi0_device(shift, out.data_ptr())
        self.ctx.check_device()
        return out

    def close(self):
        self.fn.close()
        self.ls.close()


class SpatialLevelSet:
    """One rank of a level set divided over the ranks of a process group.

    Every rank passes the same global leaves (on its own device; each keeps
    only its share) and a stepper for its device (``DeviceStepper``);
    ``step`` runs decomposed steps, ``arrays`` returns the owned leaves,
    ``gather`` the whole grid on every rank.  With NCCL, each process sets its
    device (``torch.cuda.set_device``) before the process group is used; the
    first transfer of a group is an all_gather that every rank joins, so the
    point-to-point batches that follow may leave a rank out."""

    def __init__(self, leaves: Leaves, stepper: Callable[[Leaves], Leaves] | None = None, group=None,
                 check_duplicates: bool = False, make_pool: Callable[[Leaves], object] | None = None):
        """``stepper`` steps the local leaves copied in and out each step
        (``DeviceStepper``); ``make_pool(owned leaves)`` instead keeps them
        resident in a leaf pool (``DevicePool``) and moves only ghosts and
        routed outputs."""
        import torch.distributed as dist
        world, rank = dist.get_world_size(group), dist.get_rank(group)
        part, shares = split(leaves, world)
        if make_pool is not None:
            pool = make_pool(shares[rank])
            self.ex = DistExchange(Leaves.empty(pool.dtype, pool.device), group)
            self.shard = ResidentShard(rank, part, pool, check_duplicates)
        else:
            self.ex = DistExchange(Leaves.empty(leaves.phi.dtype, leaves.device), group)
            self.shard = Shard(rank, part, shares[rank], stepper, check_duplicates)

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
