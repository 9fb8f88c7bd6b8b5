"""The reference's serialised grid formats, read into and written from device grids.

    read_vol(data) -> DeviceGrid        src/io/vol_format.rs:85-150
    write_vol(grid) -> bytes            src/io/vol_format.rs:53-83
    load_vol(path) / save_vol(g, path)  src/io/vol_format.rs:153-163
    NanoGrid                            src/nano/layout.rs:13-286

The byte layouts are the reference's (little-endian): a ``.vol`` file is a
32-byte header plus one (origin, mask, values) record per leaf; a NanoGrid is
the repr(C) image of its header and of leaves sorted by origin.  Reading
validates as the reference does and moves the leaf block to the device in one
copy (``vlr_grid_from_vol`` / ``vlr_grid_from_nano``); writing packs the
device pool into records on the GPU (``vlr_grid_to_vol`` / ``vlr_grid_to_nano``).
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from ._lib import Context
from .grid import AffineMap, Grid, GridClass
from .tools import DeviceGrid


def _buf(data: bytes):
    a = np.frombuffer(bytes(data), np.uint8)
    return a, (a.ctypes.data if len(a) else None)


def read_vol(data: bytes, ctx: Context | None = None) -> DeviceGrid:
    """Parse a ``.vol`` image into a device grid (VolrusError on bad data)."""
    ctx = ctx or Context.default()
    a, p = _buf(data)
    h = C.c_void_p()
    cls = C.c_int()
    ctx.check(ctx.lib.vlr_grid_from_vol(ctx.handle, p, len(a), C.byref(h), C.byref(cls)), "vlr_grid_from_vol")
    return DeviceGrid(ctx, h, "", GridClass(cls.value))


def write_vol(grid, grid_class: int | None = None) -> bytes:
    """``.vol`` image of a device (or host) grid."""
    g = grid if isinstance(grid, DeviceGrid) else DeviceGrid.upload(grid)
    ctx = g.ctx
    cls = int(g.grid_class if grid_class is None else grid_class)
    n = C.c_size_t()
    ctx.check(ctx.lib.vlr_grid_to_vol(ctx.handle, g.handle, cls, None, 0, C.byref(n)), "vlr_grid_to_vol")
    out = np.zeros(n.value, np.uint8)
    ctx.check(ctx.lib.vlr_grid_to_vol(ctx.handle, g.handle, cls, out.ctypes.data, len(out), C.byref(n)),
              "vlr_grid_to_vol")
    return out.tobytes()


def load_vol(path: str, ctx: Context | None = None) -> DeviceGrid:
    with open(path, "rb") as f:
        return read_vol(f.read(), ctx)


def save_vol(grid, path: str):
    with open(path, "wb") as f:
        f.write(write_vol(grid))


class NanoGrid:
    """A NanoGrid byte image (``NanoGrid::as_bytes``)."""

    def __init__(self, data: bytes):
        self.data = bytes(data)

    @classmethod
    def from_grid(cls, grid, grid_class: int | None = None, affine_inv=None) -> "NanoGrid":
        """``NanoGrid::from_grid``: linearise a device (or host) grid."""
        g = grid if isinstance(grid, DeviceGrid) else DeviceGrid.upload(grid)
        ctx = g.ctx
        k = int(g.grid_class if grid_class is None else grid_class)
        inv = None
        if affine_inv is None and isinstance(getattr(grid, "affine", None), AffineMap):
            affine_inv = grid.affine.inverse()[:3]  # the inverse the crate's map holds
        if affine_inv is not None:
            inv_a = np.ascontiguousarray(np.asarray(affine_inv, np.float64).reshape(-1)[:12])
            inv = inv_a.ctypes.data_as(C.POINTER(C.c_double))
        n = C.c_size_t()
        ctx.check(ctx.lib.vlr_grid_to_nano(ctx.handle, g.handle, k, inv, None, 0, C.byref(n)), "vlr_grid_to_nano")
        out = np.zeros(n.value, np.uint8)
        ctx.check(ctx.lib.vlr_grid_to_nano(ctx.handle, g.handle, k, inv, out.ctypes.data, len(out), C.byref(n)),
                  "vlr_grid_to_nano")
        return cls(out.tobytes())

    @classmethod
    def from_bytes(cls, data: bytes) -> "NanoGrid":
        return cls(data)

    def as_bytes(self) -> bytes:
        return self.data

    def to_grid(self, ctx: Context | None = None) -> DeviceGrid:
        """``NanoGrid::from_bytes`` + ``to_grid`` on the device (VolrusError on bad data)."""
        ctx = ctx or Context.default()
        a, p = _buf(self.data)
        h = C.c_void_p()
        k = C.c_int()
        ctx.check(ctx.lib.vlr_grid_from_nano(ctx.handle, p, len(a), C.byref(h), C.byref(k)), "vlr_grid_from_nano")
        return DeviceGrid(ctx, h, "", GridClass(k.value))


__all__ = ["NanoGrid", "load_vol", "read_vol", "save_vol", "write_vol", "Grid"]
