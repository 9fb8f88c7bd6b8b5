"""Host mirror of the crate's ``PointDataGrid`` (src/points/point_grid.rs:50-266).

Particles (world position, velocity attribute, id: ``Particle``,
src/points/point_grid.rs:9-17) are binned into 8^3 leaves by
``AffineMap::world_to_index(position)`` aligned to 8.  The crate keeps its
leaves in a ``HashMap`` whose iteration order is unspecified; this mirror
keeps them in ascending (x, y, z) origin order, so iteration, ``rebin`` and
the GPU advection (``vlr_advect_points``) are deterministic.  Particles are
held as one structured array in binned order (leaf by leaf, each leaf's
particles in insertion order) plus the leaf origins and the index of each
leaf's first particle, which is the layout ``vlr_advect_points`` takes and
returns.
"""
from __future__ import annotations

import numpy as np

from .grid import AffineMap

PARTICLE = np.dtype([("position", "<f8", (3,)), ("velocity", "<f8", (3,)), ("id", "<u8")])
assert PARTICLE.itemsize == 56


def particle(id: int, position, velocity=(0.0, 0.0, 0.0)) -> np.ndarray:
    """One ``Particle`` record."""
    p = np.zeros((), PARTICLE)
    p["position"] = position
    p["velocity"] = velocity
    p["id"] = id
    return p


def _rust_round(f: np.ndarray) -> np.ndarray:
    """f64::round (halves away from zero), exactly: x - trunc(x) is exact."""
    t = np.trunc(f)
    frac = f - t
    return t + np.where(np.abs(frac) >= 0.5, np.sign(f), 0.0)


def _saturate_i32(r: np.ndarray) -> np.ndarray:
    r = np.where(np.isnan(r), 0.0, r)
    return np.clip(r, -2147483648.0, 2147483647.0).astype(np.int64).astype(np.int32)


class PointDataGrid:
    """Sparse grid of particles binned into 8^3 leaves (leaves in ascending origin order)."""

    def __init__(self, voxel_size: float = 1.0, affine: AffineMap | None = None):
        self.transform = affine if affine is not None else AffineMap.from_uniform_scale(voxel_size)
        self.voxel_size = float(self.transform.voxel_size) if affine is not None else float(voxel_size)
        self.particles = np.zeros(0, PARTICLE)
        self.leaf_origins = np.zeros((0, 3), np.int32)
        self.leaf_start = np.zeros(1, np.uint32)

    @staticmethod
    def new(voxel_size: float) -> "PointDataGrid":
        return PointDataGrid(voxel_size)

    @staticmethod
    def with_affine(m: AffineMap) -> "PointDataGrid":
        return PointDataGrid(m.voxel_size, m)

    # -- binning ------------------------------------------------------------
    def inverse_rows(self) -> np.ndarray:
        """Rows 0..2 of the world -> index map, as ``vlr_advect_points`` takes them."""
        return np.ascontiguousarray(self.transform.inverse()[:3], np.float64).reshape(12)

    def leaf_origin_for(self, position) -> tuple:
        """Leaf origin of a world position (``leaf_origin_for``, point_grid.rs:84-88)."""
        c = self.transform.world_to_index(position)
        return (c[0] & ~7, c[1] & ~7, c[2] & ~7)

    def _leaf_keys(self, pos: np.ndarray) -> np.ndarray:
        inv = self.transform.inverse()
        out = np.empty((len(pos), 3), np.int32)
        for a in range(3):
            r = inv[a]
            f = ((r[0] * pos[:, 0] + r[1] * pos[:, 1]) + r[2] * pos[:, 2]) + r[3]
            out[:, a] = _saturate_i32(_rust_round(f)) & ~7
        return out

    def _set_binned(self, parts: np.ndarray, leaves: np.ndarray):
        """Stable sort of `parts` by leaf origin (ascending), recording the leaves."""
        order = np.lexsort((leaves[:, 2], leaves[:, 1], leaves[:, 0]))  # stable
        self.particles = np.ascontiguousarray(parts[order])
        lv = leaves[order]
        if len(lv):
            head = np.ones(len(lv), bool)
            head[1:] = np.any(lv[1:] != lv[:-1], axis=1)
            starts = np.nonzero(head)[0]
            self.leaf_origins = np.ascontiguousarray(lv[starts], np.int32)
            self.leaf_start = np.append(starts, len(lv)).astype(np.uint32)
        else:
            self.leaf_origins = np.zeros((0, 3), np.int32)
            self.leaf_start = np.zeros(1, np.uint32)

    def _leaves_of_binned(self) -> np.ndarray:
        n = np.diff(self.leaf_start.astype(np.int64))
        return np.repeat(self.leaf_origins, n, axis=0).reshape(-1, 3)

    def insert(self, p):
        """``insert`` (point_grid.rs:96-103): append to the particle's leaf."""
        self.insert_batch(np.asarray(p, PARTICLE).reshape(1))

    def insert_batch(self, parts):
        """``insert_batch`` (point_grid.rs:106-110): each particle appended to its leaf in order."""
        parts = np.asarray(parts, PARTICLE).reshape(-1)
        if not len(parts):
            return
        old = self.particles
        old_leaves = self._leaves_of_binned()
        new_leaves = self._leaf_keys(parts["position"])
        self._set_binned(np.concatenate([old, parts]), np.concatenate([old_leaves, new_leaves]))

    def rebin(self):
        """``rebin`` (point_grid.rs:258-266): drain the leaves (ascending origin
        order) and re-insert every particle by its current position."""
        self._set_binned(self.particles.copy(), self._leaf_keys(self.particles["position"]))

    # -- queries --------------------------------------------------------------
    def particle_count(self) -> int:
        return int(len(self.particles))

    def leaf_count(self) -> int:
        return int(len(self.leaf_origins))

    def leaves(self):
        """[(origin tuple, particles of that leaf)] in ascending origin order."""
        s = self.leaf_start.astype(np.int64)
        return [(tuple(int(v) for v in self.leaf_origins[k]), self.particles[s[k]:s[k + 1]])
                for k in range(len(self.leaf_origins))]

    def contains_leaf(self, origin) -> bool:
        o = np.asarray(origin, np.int32)
        return bool(np.any(np.all(self.leaf_origins == o, axis=1)))

    def iter_particles(self):
        return iter(self.particles)

    def particles_in_voxel(self, coord):
        """``particles_in_voxel`` (point_grid.rs:136-147)."""
        c = tuple(int(v) for v in coord)
        return [p for p in self.particles if self.transform.world_to_index(tuple(p["position"])) == c]


__all__ = ["PARTICLE", "PointDataGrid", "particle"]
