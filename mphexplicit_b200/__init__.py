"""B200 (sm_100a) MPH-WC explicit time step with the interface of the
Masahiro-Kondo-AIST/MphExplicit solver (files, types, step sequence).

The compute path is ``libmph_b200.so`` (hand-written CUDA for sm_100a behind the
C ABI of include/mph_b200.h); this package is the Python host mirror over it.
"""
from ._native import (MODE_FP64, MODE_MIXED, Constants, GridHeader, Info, Params)  # noqa: F401
from .batch import Batch  # noqa: F401
from .solver import (Checkpoint, Grid, MphError, Solver, compute_constants, default_params, format_e,  # noqa: F401
                     generate_cuboids, generate_grid_file, make_header, read_boid_file, read_checkpoint,
                     read_data_file, read_grid_file, run, write_checkpoint_arrays, write_grid_file, write_vtk_arrays)

__all__ = ["Solver", "Batch", "MphError", "Grid", "Checkpoint", "read_checkpoint", "write_checkpoint_arrays", "Params", "GridHeader", "Constants", "Info", "read_data_file",
           "read_grid_file", "write_grid_file", "read_boid_file", "generate_cuboids", "generate_grid_file", "write_vtk_arrays", "format_e", "compute_constants", "default_params", "make_header", "run",
           "MODE_FP64", "MODE_MIXED"]
