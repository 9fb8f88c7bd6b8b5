"""Host-side mirror of the Sharc.Volrus ``Grid<f32>`` facade for the advection path.

The reference grid is a pointer tree (``src/tree/root.rs``: HashMap root ->
16^3 internal node -> boxed 8^3 leaf) behind ``Grid<T>`` (``src/grid.rs:349-514``).
This mirror stores the same information flat, as the reference's own
``NanoGrid`` does (``src/nano/layout.rs:41-52``): one row per allocated leaf
with its origin, 512-bit activity mask and 512 values in ZYX order.  The
voxel-level accessors (``get``/``set``/``is_active``/``deactivate``) follow the
tree semantics of ``src/tree/leaf.rs:29-82`` and ``src/tree/internal.rs:118-166``:
reads of unallocated voxels return the background, ``set`` allocates a leaf
filled with the background and marks the voxel active, ``deactivate`` writes
the background and clears the bit.  Compute runs on the GPU through
:mod:`sharc.volrus_b200.tools`; this class only holds data.
"""
from __future__ import annotations

import enum
from dataclasses import dataclass, field

import math

import numpy as np

from . import _lib


class GridClass(enum.IntEnum):
    """``GridClass`` (src/grid.rs:10-20)."""
    UNKNOWN = 0
    LEVEL_SET = 1
    FOG_VOLUME = 2


@dataclass
class VoxelTransform:
    """Legacy uniform transform used by ``sample_trilinear`` (src/grid.rs:62-122)."""
    voxel_size: float = 1.0
    origin: tuple = (0.0, 0.0, 0.0)

    @staticmethod
    def uniform(voxel_size: float) -> "VoxelTransform":
        return VoxelTransform(float(voxel_size), (0.0, 0.0, 0.0))

    @staticmethod
    def with_origin(voxel_size: float, origin) -> "VoxelTransform":
        return VoxelTransform(float(voxel_size), tuple(float(o) for o in origin))

    @staticmethod
    def identity() -> "VoxelTransform":
        return VoxelTransform(1.0, (0.0, 0.0, 0.0))

    def index_to_world(self, c):
        return tuple(c[i] * self.voxel_size + self.origin[i] for i in range(3))

    def world_to_index_f64(self, w):
        inv = 1.0 / self.voxel_size
        return tuple((w[i] - self.origin[i]) * inv for i in range(3))

    def world_to_index(self, w):
        """Nearest index, halves away from zero (src/grid.rs:103-110)."""
        return tuple(_round_i32(f) for f in self.world_to_index_f64(w))


def _round_i32(f: float) -> int:
    """Rust's ``f.round() as i32``: halves away from zero, then a saturating
    cast (NaN -> 0)."""
    if f != f:
        return 0
    r = math.floor(f + 0.5) if f >= 0.0 else -math.floor(-f + 0.5)
    return int(min(max(r, -2 ** 31), 2 ** 31 - 1))


def invert_4x4(m) -> np.ndarray:
    """Inverse of a 4x4 matrix by the Laplace expansion in 2x2 minors of rows
    (0, 1) and (2, 3): the adjugate's entries are sums of three products of an
    entry and a minor, scaled by 1/det (the method of src/grid.rs:301-345, so
    the bits match the crate's)."""
    m = [[float(v) for v in r] for r in np.asarray(m, np.float64).reshape(4, 4)]
    s = [m[0][0] * m[1][1] - m[1][0] * m[0][1], m[0][0] * m[1][2] - m[1][0] * m[0][2],
         m[0][0] * m[1][3] - m[1][0] * m[0][3], m[0][1] * m[1][2] - m[1][1] * m[0][2],
         m[0][1] * m[1][3] - m[1][1] * m[0][3], m[0][2] * m[1][3] - m[1][2] * m[0][3]]
    c = [m[2][0] * m[3][1] - m[3][0] * m[2][1], m[2][0] * m[3][2] - m[3][0] * m[2][2],
         m[2][0] * m[3][3] - m[3][0] * m[2][3], m[2][1] * m[3][2] - m[3][1] * m[2][2],
         m[2][1] * m[3][3] - m[3][1] * m[2][3], m[2][2] * m[3][3] - m[3][2] * m[2][3]]
    det = s[0] * c[5] - s[1] * c[4] + s[2] * c[3] + s[3] * c[2] - s[4] * c[1] + s[5] * c[0]
    if not abs(det) > 1e-30:
        raise ValueError("singular matrix")
    k = 1.0 / det
    a = [[(m[1][1] * c[5] - m[1][2] * c[4] + m[1][3] * c[3]), (-m[0][1] * c[5] + m[0][2] * c[4] - m[0][3] * c[3]),
          (m[3][1] * s[5] - m[3][2] * s[4] + m[3][3] * s[3]), (-m[2][1] * s[5] + m[2][2] * s[4] - m[2][3] * s[3])],
         [(-m[1][0] * c[5] + m[1][2] * c[2] - m[1][3] * c[1]), (m[0][0] * c[5] - m[0][2] * c[2] + m[0][3] * c[1]),
          (-m[3][0] * s[5] + m[3][2] * s[2] - m[3][3] * s[1]), (m[2][0] * s[5] - m[2][2] * s[2] + m[2][3] * s[1])],
         [(m[1][0] * c[4] - m[1][1] * c[2] + m[1][3] * c[0]), (-m[0][0] * c[4] + m[0][1] * c[2] - m[0][3] * c[0]),
          (m[3][0] * s[4] - m[3][1] * s[2] + m[3][3] * s[0]), (-m[2][0] * s[4] + m[2][1] * s[2] - m[2][3] * s[0])],
         [(-m[1][0] * c[3] + m[1][1] * c[1] - m[1][2] * c[0]), (m[0][0] * c[3] - m[0][1] * c[1] + m[0][2] * c[0]),
          (-m[3][0] * s[3] + m[3][1] * s[1] - m[3][2] * s[0]), (m[2][0] * s[3] - m[2][1] * s[1] + m[2][2] * s[0])]]
    return np.array([[v * k for v in r] for r in a], np.float64)


@dataclass
class AffineMap:
    """Forward rows of the 4x4 ``AffineMap`` (src/grid.rs:131-296)."""
    mat: np.ndarray = field(default_factory=lambda: np.eye(3, 4, dtype=np.float64))
    voxel_size: float = 1.0
    # rows of the inverse as the crate stores them at construction (None:
    # computed from ``mat`` by invert_4x4, as for a general map)
    inv: np.ndarray | None = None

    @staticmethod
    def from_uniform_scale(s: float) -> "AffineMap":
        m = np.zeros((3, 4), np.float64)
        m[0, 0] = m[1, 1] = m[2, 2] = s
        i = np.zeros((3, 4), np.float64)
        i[0, 0] = i[1, 1] = i[2, 2] = 1.0 / float(s)
        return AffineMap(m, float(s), i)

    @staticmethod
    def from_voxel_transform(vt: VoxelTransform) -> "AffineMap":
        m = np.zeros((3, 4), np.float64)
        m[0, 0] = m[1, 1] = m[2, 2] = vt.voxel_size
        m[:, 3] = vt.origin
        inv_s = 1.0 / float(vt.voxel_size)
        i = np.zeros((3, 4), np.float64)
        i[0, 0] = i[1, 1] = i[2, 2] = inv_s
        i[:, 3] = [-float(t) * inv_s for t in vt.origin]
        return AffineMap(m, float(vt.voxel_size), i)

    @staticmethod
    def identity() -> "AffineMap":
        return AffineMap(np.eye(3, 4, dtype=np.float64), 1.0, np.eye(3, 4, dtype=np.float64))

    @staticmethod
    def from_scale_rotate_translate(scale, rotation, translate) -> "AffineMap":
        """Forward = T R S (src/grid.rs:205-234); voxel size = length of the
        linear part's first column."""
        m = np.zeros((3, 4), np.float64)
        for r in range(3):
            for c in range(3):
                m[r, c] = float(rotation[r][c]) * float(scale[c])
            m[r, 3] = float(translate[r])
        vs = math.sqrt(m[0, 0] * m[0, 0] + m[1, 0] * m[1, 0] + m[2, 0] * m[2, 0])
        a = AffineMap(m, vs)
        a.inv = a.inverse()[:3].copy()
        return a

    def forward(self) -> np.ndarray:
        """The 4x4 index-to-world matrix."""
        f = np.zeros((4, 4), np.float64)
        f[:3] = self.mat
        f[3, 3] = 1.0
        return f

    def inverse(self) -> np.ndarray:
        """The 4x4 world-to-index matrix, as the crate holds it."""
        if self.inv is None:
            return invert_4x4(self.forward())
        i = np.zeros((4, 4), np.float64)
        i[:3] = self.inv
        i[3, 3] = 1.0
        return i

    def index_to_world(self, c):
        x, y, z = (float(v) for v in c)
        m = self.mat
        return tuple(m[r, 0] * x + m[r, 1] * y + m[r, 2] * z + m[r, 3] for r in range(3))

    def world_to_index_f64(self, w):
        """Continuous index of a world position through the inverse (src/grid.rs:268-277)."""
        x, y, z = (float(v) for v in w)
        i = self.inverse()
        return tuple(i[r, 0] * x + i[r, 1] * y + i[r, 2] * z + i[r, 3] for r in range(3))

    def world_to_index(self, w):
        """Nearest index, halves away from zero (src/grid.rs:261-264)."""
        return tuple(_round_i32(f) for f in self.world_to_index_f64(w))


def _leaf_origin(c):
    return (int(c[0]) & ~7, int(c[1]) & ~7, int(c[2]) & ~7)


def _offset(c):
    return ((int(c[0]) & 7) << 6) | ((int(c[1]) & 7) << 3) | (int(c[2]) & 7)


class Grid:
    """``Grid<f32>`` with flat leaf storage (see module docstring)."""

    def __init__(self, background: float = 0.0, voxel_size: float = 1.0):
        self.background = float(np.float32(background))
        self.transform = VoxelTransform.uniform(voxel_size)
        self.affine = AffineMap.from_uniform_scale(voxel_size)
        self.name = ""
        self.grid_class = GridClass.UNKNOWN
        self._o = np.zeros((0, 3), np.int32)
        self._m = np.zeros((0, 8), np.uint64)
        self._v = np.zeros((0, 512), np.float32)
        self._n = 0
        self._index: dict = {}

    # ---- construction helpers ---------------------------------------
    @classmethod
    def level_set(cls, voxel_size: float, half_width: float) -> "Grid":
        """``Grid::level_set`` (src/grid.rs:391-404): background = f32(hw * vs)."""
        g = cls(float(np.float32(half_width * voxel_size)), voxel_size)
        g.name = "sdf"
        g.grid_class = GridClass.LEVEL_SET
        return g

    @classmethod
    def with_affine(cls, background: float, map: AffineMap) -> "Grid":
        """``Grid::with_affine`` (src/grid.rs:378-388): the uniform transform
        takes the map's voxel size and no translation."""
        g = cls(background, map.voxel_size)
        g.affine = map
        return g

    @classmethod
    def from_arrays(cls, origins, masks, values, background: float, transform: VoxelTransform | None = None,
                    affine: AffineMap | None = None) -> "Grid":
        g = cls(background, transform.voxel_size if transform else 1.0)
        if transform is not None:
            g.transform = transform
        if affine is not None:
            g.affine = affine
        elif transform is not None:
            g.affine = AffineMap.from_voxel_transform(transform)
        o = np.ascontiguousarray(origins, np.int32).reshape(-1, 3)
        g._o = o.copy()
        g._m = np.ascontiguousarray(masks, np.uint64).reshape(-1, 8).copy()
        g._v = np.ascontiguousarray(values, np.float32).reshape(-1, 512).copy()
        g._n = len(o)
        g._index = {tuple(int(v) for v in o[i]): i for i in range(g._n)}
        return g

    def add_tiles(self, origins, values, active):
        """Insert the tiles of a pruned tree as leaf records.

        ``RootNode::prune`` (src/tree/root.rs:151-158, src/tree/internal.rs:253-299)
        collapses a leaf whose 512 values lie within a tolerance of its first
        value into a tile holding that value, active when the leaf had an active
        voxel.  The tree then reads the tile's value at each of its voxels
        (``get``, src/tree/internal.rs:118-124) and iterates an active tile as
        512 active voxels of that value (``iter_active``,
        src/tree/internal.rs:319-349).  A leaf record holding the tile's value in
        all 512 voxels, with all bits set for an active tile and none for an
        inactive one, reads and iterates the same, so a pruned tree crosses the
        C ABI as these records beside its leaves.

        Tile origins must be leaf-aligned and must not hold a leaf (a slot of the
        internal node is either a child or a tile); ValueError otherwise.
        """
        o = np.ascontiguousarray(origins, np.int64).reshape(-1, 3)
        val = np.ascontiguousarray(values, np.float32).reshape(-1)
        act = np.ascontiguousarray(active, bool).reshape(-1)
        if not (len(o) == len(val) == len(act)):
            raise ValueError("tile origins, values and flags differ in length")
        if np.any(o & 7):
            raise ValueError("tile origins must be multiples of 8")
        keys = [tuple(int(x) for x in r) for r in o]
        if len(set(keys)) != len(keys) or any(k in self._index for k in keys):
            raise ValueError("a tile overlaps a leaf or another tile")
        full = np.uint64(0xFFFFFFFFFFFFFFFF)
        for k, v, a in zip(keys, val, act):
            if self._n == len(self._o):
                self._grow()
            row = self._n
            self._n += 1
            self._o[row] = k
            self._m[row] = full if a else np.uint64(0)
            self._v[row] = v
            self._index[k] = row

    def set_transform(self, vt: VoxelTransform):
        """``Grid::set_transform`` (src/grid.rs:432-435): also resets the affine map."""
        self.transform = vt
        self.affine = AffineMap.from_voxel_transform(vt)

    def set_affine_map(self, am: AffineMap):
        """``Grid::set_affine_map`` (src/grid.rs:443-446)."""
        self.transform = VoxelTransform.uniform(am.voxel_size)
        self.affine = am

    # ---- tree accessors ---------------------------------------------
    def _grow(self):
        cap = max(16, 2 * len(self._o))
        for name, shape, dt in (("_o", 3, np.int32), ("_m", 8, np.uint64), ("_v", 512, np.float32)):
            a = getattr(self, name)
            b = np.zeros((cap, shape), dt)
            b[: self._n] = a[: self._n]
            setattr(self, name, b)

    def _leaf_row(self, c, create: bool):
        key = _leaf_origin(c)
        row = self._index.get(key)
        if row is None and create:
            if self._n == len(self._o):
                self._grow()
            row = self._n
            self._n += 1
            self._o[row] = key
            self._m[row] = 0
            self._v[row] = self.background
            self._index[key] = row
        return row

    def get(self, c) -> float:
        row = self._leaf_row(c, False)
        return self.background if row is None else float(self._v[row, _offset(c)])

    def is_active(self, c) -> bool:
        row = self._leaf_row(c, False)
        if row is None:
            return False
        off = _offset(c)
        return bool((int(self._m[row, off >> 6]) >> (off & 63)) & 1)

    def get_world(self, pos) -> float:
        """Value at the voxel nearest a world position, through the affine map (src/grid.rs:494-497)."""
        return self.get(self.affine.world_to_index(pos))

    def set_world(self, pos, value: float):
        """Set the voxel nearest a world position (src/grid.rs:500-503)."""
        self.set(self.affine.world_to_index(pos), value)

    def set(self, c, value: float):
        row = self._leaf_row(c, True)
        off = _offset(c)
        self._v[row, off] = np.float32(value)
        self._m[row, off >> 6] = np.uint64(int(self._m[row, off >> 6]) | (1 << (off & 63)))

    def deactivate(self, c):
        row = self._leaf_row(c, False)
        if row is None:
            return
        off = _offset(c)
        self._v[row, off] = np.float32(self.background)
        self._m[row, off >> 6] = np.uint64(int(self._m[row, off >> 6]) & ~(1 << (off & 63)))

    def leaf_count(self) -> int:
        return self._n

    def active_voxel_count(self) -> int:
        m = self._m[: self._n]
        return int(np.unpackbits(m.view(np.uint8)).sum()) if self._n else 0

    def iter_active(self):
        """Active voxels as (coord, value); leaves in (x, y, z) order, voxels ZYX."""
        o, m, v = self.to_arrays()
        bits = np.unpackbits(m.view(np.uint8).reshape(-1, 64), axis=1, bitorder="little").astype(bool)
        for i in range(len(o)):
            for off in np.nonzero(bits[i])[0]:
                yield ((int(o[i, 0]) + (off >> 6), int(o[i, 1]) + ((off >> 3) & 7), int(o[i, 2]) + (off & 7)),
                       float(v[i, off]))

    def remove_empty_leaves(self):
        """``RootNode::remove_empty_leaves`` (src/tree/root.rs:161-165)."""
        o, m, v = self._o[: self._n], self._m[: self._n], self._v[: self._n]
        keep = m.any(axis=1)
        self._o, self._m, self._v = o[keep].copy(), m[keep].copy(), v[keep].copy()
        self._n = len(self._o)
        self._index = {tuple(int(x) for x in self._o[i]): i for i in range(self._n)}

    def to_arrays(self):
        """(origins, masks, values) sorted by origin (x, y, z), NanoGrid order."""
        o, m, v = self._o[: self._n], self._m[: self._n], self._v[: self._n]
        order = np.lexsort((o[:, 2], o[:, 1], o[:, 0])) if self._n else np.zeros(0, np.int64)
        return (np.ascontiguousarray(o[order]), np.ascontiguousarray(m[order]), np.ascontiguousarray(v[order]))

    def c_transform(self) -> "_lib.vlr_transform":
        t = _lib.vlr_transform()
        t.voxel_size = self.transform.voxel_size
        for i in range(3):
            t.origin[i] = self.transform.origin[i]
        flat = np.asarray(self.affine.mat, np.float64).reshape(12)
        for i in range(12):
            t.affine[i] = float(flat[i])
        t.affine_voxel_size = self.affine.voxel_size
        return t

    def copy_meta_from(self, other: "Grid"):
        self.name = other.name
        self.grid_class = other.grid_class

    def __repr__(self):
        return (f"Grid(leaves={self._n}, active={self.active_voxel_count()}, bg={self.background}, "
                f"vs={self.transform.voxel_size})")
