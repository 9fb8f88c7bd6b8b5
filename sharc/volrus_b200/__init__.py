"""B200-native narrow-band level-set advection for Sharc.Volrus grids.

The public names mirror the reference crate's advection path
(``src/lib.rs:26-43``): :class:`Grid`, :class:`VelocityField`,
:func:`advect_level_set`, :func:`sample_trilinear`,
:func:`find_zero_crossings`, :func:`trim_narrow_band`,
:func:`rebuild_narrow_band`, :func:`make_level_set_sphere`.  All compute runs
in hand-written sm_100a CUDA kernels in ``lib/libvolrus_b200.so``; there is no
CPU fallback.
"""
from ._lib import Context, VolrusError
from .grid import AffineMap, Grid, GridClass, VoxelTransform
from .points import PARTICLE, PointDataGrid, particle
from .tools import (DeviceGrid, Mesh, VelocityField, advect_level_set, advect_particles, advect_particles_euler,
                    dilate, extend_velocity, find_zero_crossings, flood_fill_sign, make_level_set_sphere,
                    make_uniform_velocity, mc_triangle_table, rebuild_narrow_band, sample_trilinear,
                    trim_narrow_band, volume_to_mesh)

__all__ = [
    "AffineMap", "Context", "DeviceGrid", "Grid", "GridClass", "VelocityField", "VolrusError", "VoxelTransform",
    "advect_level_set", "advect_particles", "advect_particles_euler", "dilate", "extend_velocity", "find_zero_crossings", "make_level_set_sphere", "make_uniform_velocity",
    "rebuild_narrow_band", "sample_trilinear", "trim_narrow_band", "Mesh", "volume_to_mesh", "mc_triangle_table",
    "flood_fill_sign", "PointDataGrid", "PARTICLE", "particle",
]
