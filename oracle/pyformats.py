"""ORACLE — test infrastructure only.  Byte-level restatement of the
reference's serialised grid formats on the host ``Grid`` mirror, used to check
the device readers and writers (``vlr_grid_{from,to}_{vol,nano}``).

    write_vol / read_vol            src/io/vol_format.rs:53-150
    nano_from_grid                  src/nano/layout.rs:89-170  (NanoGrid::from_grid)
    nano_from_bytes / nano_to_grid  src/nano/layout.rs:208-286
    nano_get / nano_is_active       src/nano/lookup.rs:11-31, 57-80

The reference writes .vol leaves in its tree's iteration order (a HashMap of
128^3 tiles, then child index order inside a tile); ``write_vol`` takes an
explicit leaf order and defaults to (x, y, z) order of origin, which is the
tree order of a single-tile grid.  The reader does not depend on the order.
"""
from __future__ import annotations

import struct

import numpy as np

from sharc.volrus_b200.grid import AffineMap, Grid, GridClass

VOL_HEADER = 32
VOL_LEAF = 12 + 64 + 2048
NANO_HEADER = 320
NANO_LEAF = 2128


class FormatError(ValueError):
    pass


def _sorted_rows(g: Grid):
    o = g._o[: g._n]
    return list(np.lexsort((o[:, 2], o[:, 1], o[:, 0]))) if g._n else []


def write_vol(g: Grid, order=None) -> bytes:
    """src/io/vol_format.rs:53-83: header, then (origin, mask, values) per leaf."""
    rows = _sorted_rows(g) if order is None else list(order)
    out = bytearray()
    out += b"VOLR" + struct.pack("<IIdfI", 1, int(g.grid_class), g.transform.voxel_size, g.background, len(rows))
    out += b"\0" * 4
    for r in rows:
        out += struct.pack("<3i", *(int(v) for v in g._o[r]))
        out += np.ascontiguousarray(g._m[r], "<u8").tobytes()
        out += np.ascontiguousarray(g._v[r], "<f4").tobytes()
    return bytes(out)


def read_vol(data: bytes) -> Grid:
    """src/io/vol_format.rs:85-150: validate, then per record grid.set(origin,
    values[0]) (allocating the leaf holding origin) and a bulk write of the
    record's values and mask into that leaf."""
    if len(data) < VOL_HEADER:
        raise FormatError("unexpected end of file")
    if data[0:4] != b"VOLR":
        raise FormatError("not a .vol file (bad magic)")
    version, cls, vs, bg, count = struct.unpack_from("<IIdfI", data, 4)
    if version != 1:
        raise FormatError(f"unsupported .vol version: {version}")
    if cls > 2:
        raise FormatError(f"unknown grid class: {cls}")
    g = Grid(bg, vs)
    g.grid_class = GridClass(cls)
    pos = VOL_HEADER
    for _ in range(count):
        if pos + VOL_LEAF > len(data):
            raise FormatError("unexpected end of file")
        origin = struct.unpack_from("<3i", data, pos)
        mask = np.frombuffer(data, "<u8", 8, pos + 12).astype(np.uint64)
        vals = np.frombuffer(data, "<f4", 512, pos + 76).astype(np.float32)
        g.set(origin, float(vals[0]))
        row = g._leaf_row(origin, False)
        g._v[row] = vals
        g._m[row] = mask
        pos += VOL_LEAF
    return g


def nano_from_grid(g: Grid, affine_inv=None) -> bytes:
    """src/nano/layout.rs:89-170: repr(C) NanoHeader (320 B) + NanoLeaf (2,128 B)
    per leaf sorted by origin; bbox over active voxels ((0,0,0) if none);
    forward matrix from the affine map, inverse as the map stores it (1 / vs on
    the diagonal for a uniform scale)."""
    rows = _sorted_rows(g)
    act = [c for c, _ in g.iter_active()]
    if act:
        a = np.array(act)
        lo, hi = a.min(axis=0), a.max(axis=0)
    else:
        lo = hi = np.zeros(3, np.int64)
    mat = np.zeros((4, 4))
    mat[:3] = g.affine.mat
    mat[3, 3] = 1.0
    inv = np.zeros((4, 4))
    if affine_inv is None:
        inv[0, 0] = inv[1, 1] = inv[2, 2] = 1.0 / g.affine.voxel_size
    else:
        inv[:3] = np.asarray(affine_inv, np.float64).reshape(3, 4)
    inv[3, 3] = 1.0
    out = bytearray(NANO_HEADER)
    struct.pack_into("<4sII", out, 0, b"NANO", 1, int(g.grid_class))
    struct.pack_into("<dfI", out, 16, g.affine.voxel_size, g.background, len(rows))
    struct.pack_into("<3i3i", out, 32, *(int(v) for v in lo), *(int(v) for v in hi))
    out[56:184] = mat.astype("<f8").tobytes()
    out[184:312] = inv.astype("<f8").tobytes()
    for r in rows:
        leaf = bytearray(NANO_LEAF)
        struct.pack_into("<3ii", leaf, 0, *(int(v) for v in g._o[r]), 0)
        leaf[16:80] = np.ascontiguousarray(g._m[r], "<u8").tobytes()
        leaf[80:] = np.ascontiguousarray(g._v[r], "<f4").tobytes()
        out += leaf
    return bytes(out)


def nano_header(data: bytes) -> dict:
    magic, version, cls = struct.unpack_from("<4sII", data, 0)
    vs, bg, count = struct.unpack_from("<dfI", data, 16)
    bb = struct.unpack_from("<3i3i", data, 32)
    mat = np.frombuffer(data, "<f8", 16, 56).reshape(4, 4)
    inv = np.frombuffer(data, "<f8", 16, 184).reshape(4, 4)
    return {"magic": magic, "version": version, "grid_class": cls, "voxel_size": vs, "background": bg,
            "leaf_count": count, "bbox_min": list(bb[:3]), "bbox_max": list(bb[3:]), "affine_mat": mat,
            "affine_inv": inv}


def _nano_origins(data: bytes):
    n = nano_header(data)["leaf_count"]
    return [struct.unpack_from("<3i", data, NANO_HEADER + i * NANO_LEAF) for i in range(n)]


def nano_from_bytes(data: bytes) -> bytes:
    """src/nano/layout.rs:208-252: size, magic, version, length, sorted leaves."""
    if len(data) < NANO_HEADER:
        raise FormatError("Buffer too small for NanoHeader")
    h = nano_header(data)
    if h["magic"] != b"NANO":
        raise FormatError(f"Invalid magic: got {h['magic']!r}")
    if h["version"] != 1:
        raise FormatError(f"Unsupported version: {h['version']}")
    if len(data) < NANO_HEADER + NANO_LEAF * h["leaf_count"]:
        raise FormatError("Buffer too small")
    o = _nano_origins(data)
    for i in range(1, len(o)):
        if not tuple(o[i - 1]) < tuple(o[i]):
            raise FormatError("Leaves not sorted")
    return data


def nano_to_grid(data: bytes) -> Grid:
    """src/nano/layout.rs:255-286: a fresh grid (with_affine) holding the
    active voxels of every leaf."""
    h = nano_header(data)
    am = AffineMap(np.array(h["affine_mat"][:3]), h["voxel_size"])
    g = Grid(h["background"], h["voxel_size"])
    g.set_affine_map(am)
    g.grid_class = GridClass(h["grid_class"] if h["grid_class"] in (1, 2) else 0)
    for i in range(h["leaf_count"]):
        base = NANO_HEADER + i * NANO_LEAF
        origin = struct.unpack_from("<3i", data, base)
        mask = np.frombuffer(data, "<u8", 8, base + 16)
        vals = np.frombuffer(data, "<f4", 512, base + 80)
        for w in range(8):
            word = int(mask[w])
            while word:
                bit = (word & -word).bit_length() - 1
                word &= word - 1
                off = w * 64 + bit
                g.set((origin[0] + (off >> 6), origin[1] + ((off >> 3) & 7), origin[2] + (off & 7)), float(vals[off]))
    return g


def _find(data: bytes, c):
    key = (c[0] & ~7, c[1] & ~7, c[2] & ~7)
    o = _nano_origins(data)
    lo, hi = 0, len(o)
    while lo < hi:
        mid = (lo + hi) // 2
        if tuple(o[mid]) < key:
            lo = mid + 1
        elif tuple(o[mid]) == key:
            return NANO_HEADER + mid * NANO_LEAF
        else:
            hi = mid
    return None


def nano_get(data: bytes, c) -> float:
    """src/nano/lookup.rs:11-20."""
    base = _find(data, c)
    if base is None:
        return nano_header(data)["background"]
    off = ((c[0] & 7) << 6) | ((c[1] & 7) << 3) | (c[2] & 7)
    return float(np.frombuffer(data, "<f4", 1, base + 80 + 4 * off)[0])


def nano_is_active(data: bytes, c) -> bool:
    """src/nano/lookup.rs:23-31."""
    base = _find(data, c)
    if base is None:
        return False
    off = ((c[0] & 7) << 6) | ((c[1] & 7) << 3) | (c[2] & 7)
    word = int(np.frombuffer(data, "<u8", 1, base + 16 + 8 * (off >> 6))[0])
    return bool((word >> (off & 63)) & 1)
