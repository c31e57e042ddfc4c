"""B200-native 2.5D FDTD vocal-tract solver: Python handles over the C ABI.

The compute path is libvocalsim_b200.so (hand-written sm_100a CUDA behind the
C ABI in include/vocalsim_b200.h); this package only binds it with ctypes.
"""
from .abi import (CELL_AIR, CELL_DEAD, CELL_EXCITATION, CELL_NOPRESSURE, CELL_WALL, ENGINE_CPU,
                  ENGINE_EIGEN, LISTENER_EXPLICIT, LISTENER_REFERENCE, SRC_GAUSS, SRC_GAUSS_STD, SRC_SINE,
                  SRC_TMM, VsDims, VsError, VsGeometry, VsParams, load_library)
from .solver import Batch, Geometry, Solver, build_maps, params, source_table, tile_shape_steps, tile_shapes

__all__ = [
    "Batch", "Geometry", "Solver", "build_maps", "params", "source_table", "tile_shape_steps", "tile_shapes",
    "load_library",
    "VsParams", "VsGeometry", "VsDims", "VsError",
    "CELL_AIR", "CELL_DEAD", "CELL_EXCITATION", "CELL_NOPRESSURE", "CELL_WALL",
    "ENGINE_CPU", "ENGINE_EIGEN", "LISTENER_EXPLICIT", "LISTENER_REFERENCE",
    "SRC_GAUSS", "SRC_GAUSS_STD", "SRC_SINE", "SRC_TMM",
]
