"""B200-native DSMC timestep (sm_100a) behind the reference solver API.

The timestep runs in libdsmc_b200.so (hand-written CUDA kernels, C ABI in
include/dsmc_b200.h); this package is its Python host binding.
"""
from ._capi import DsmcError, lib  # noqa: F401
from .solver import (CreateSolver, DSMCBatch, DSMCSolver, build_geometry_grid, mesh_capsule,  # noqa: F401
                     mesh_icosphere, read_raw_mesh, read_twisters, settings_t)
from . import stages  # noqa: F401

__all__ = ["CreateSolver", "DSMCBatch", "DSMCSolver", "settings_t", "mesh_icosphere", "mesh_capsule",
           "read_raw_mesh", "read_twisters", "build_geometry_grid", "stages", "DsmcError", "lib"]
