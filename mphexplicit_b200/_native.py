"""ctypes view of the C ABI declared in include/mph_b200.h.

The structures below mirror the header field for field.  ``load()`` opens the
in-tree ``libmph_b200.so``; there is no fallback: if the library is missing the
import of the solver fails with the build command in the message.
"""
from __future__ import annotations

import ctypes as C
import os

TYPE_COUNT = 4

MPH_OK = 0
MPH_ERR_ARG = -1
MPH_ERR_IO = -2
MPH_ERR_CUDA = -3
MPH_ERR_CAPACITY = -4
MPH_ERR_DEVICE = -5
MPH_ERR_NONFINITE = -6
MPH_ERR_STATE = -7
MPH_ERR_NOMEM = -8
MPH_ERR_GEOMETRY = -9

MODE_FP64 = 0
MODE_MIXED = 1
MODE_MIXED_P64 = 2
MODE_LEARNED = 3
MIXED_CELL_WALK = 0x100
SAMPLE_FLOATS = 12

_D4 = C.c_double * TYPE_COUNT
_D44 = (C.c_double * TYPE_COUNT) * TYPE_COUNT
_D3 = C.c_double * 3
_D43 = (C.c_double * 3) * TYPE_COUNT


class Params(C.Structure):
    """mph_params: the keys of the reference's *.data file (main.cpp:489-539)."""

    _fields_ = [
        ("dt", C.c_double),
        ("output_interval", C.c_double),
        ("vtk_output_interval", C.c_double),
        ("end_time", C.c_double),
        ("radius_ratio_a", C.c_double),
        ("radius_ratio_p", C.c_double),
        ("radius_ratio_v", C.c_double),
        ("density", _D4),
        ("bulk_modulus", _D4),
        ("bulk_viscosity", _D4),
        ("shear_viscosity", _D4),
        ("surface_tension", _D4),
        ("interaction_ratio", _D44),
        ("gravity", _D3),
        ("wall_center", _D43),
        ("wall_velocity", _D43),
        ("wall_omega", _D43),
    ]


class GridHeader(C.Structure):
    """mph_grid_header: first two lines of a *.grid / *.prof file."""

    _fields_ = [
        ("time", C.c_double),
        ("particle_count", C.c_int),
        ("particle_spacing", C.c_double),
        ("domain_min", _D3),
        ("domain_max", _D3),
    ]


class Constants(C.Structure):
    """mph_constants: derived set-up values (main.cpp:836-1084)."""

    _fields_ = [
        ("dim", C.c_int),
        ("particle_volume", C.c_double),
        ("radius_a", C.c_double),
        ("radius_g", C.c_double),
        ("radius_p", C.c_double),
        ("radius_v", C.c_double),
        ("max_radius", C.c_double),
        ("swa", C.c_double),
        ("swg", C.c_double),
        ("swp", C.c_double),
        ("swv", C.c_double),
        ("n0a", C.c_double),
        ("n0p", C.c_double),
        ("r2g", C.c_double),
        ("n0a_count", C.c_int),
        ("n0p_count", C.c_int),
        ("cof_k", C.c_double),
        ("cof_a", _D4),
        ("domain_width", _D3),
        ("cell_count", C.c_int * 3),
        ("total_cell_count", C.c_int),
        ("cell_width", _D3),
        ("wall_rotation", ((C.c_double * 3) * 3) * TYPE_COUNT),
    ]


class Info(C.Structure):
    """mph_info: run-time counters of a context."""

    _fields_ = [
        ("particle_count", C.c_int),
        ("fluid_particle_begin", C.c_int),
        ("fluid_particle_end", C.c_int),
        ("wall_particle_begin", C.c_int),
        ("wall_particle_end", C.c_int),
        ("neighbor_ind_count", C.c_longlong),
        ("max_neighbor_count", C.c_int),
        ("neighbor_capacity", C.c_int),
        ("step", C.c_longlong),
        ("rebuild_count", C.c_longlong),
        ("time", C.c_double),
        ("mode", C.c_int),
    ]


class KernelStat(C.Structure):
    """mph_kernel_stat: per-kernel launches and CUDA-event time."""

    _fields_ = [("name", C.c_char * 32), ("launches", C.c_longlong), ("total_ms", C.c_double)]


class LearnedInfo(C.Structure):
    """mph_learned_info: counters of the learned form."""

    _fields_ = [("steps", C.c_longlong), ("learned_steps", C.c_longlong), ("judged", C.c_longlong),
                ("fallbacks", C.c_longlong), ("plain_steps", C.c_longlong), ("last_force_error", C.c_double),
                ("max_force_error", C.c_double), ("last_term_error", C.c_double), ("max_term_error", C.c_double),
                ("edges", C.c_longlong), ("max_accepted_error", C.c_double)]


class BatchTrial(C.Structure):
    """mph_batch_trial: one candidate of the batch autotuner."""

    _fields_ = [("tile", C.c_int * 3), ("threads", C.c_int), ("ctas_per_sm", C.c_int), ("capacity", C.c_int),
                ("ms_per_step", C.c_double)]


class BatchInfo(C.Structure):
    """mph_batch_info: shape and counters of a batch."""

    _fields_ = [("dim", C.c_int), ("scenes", C.c_int), ("particles", C.c_int), ("fluid_particles", C.c_int),
                ("tile", C.c_int * 3), ("threads", C.c_int), ("ctas_per_sm", C.c_int), ("items", C.c_int),
                ("capacity", C.c_int),
                ("grid_a", C.c_int), ("grid_b", C.c_int), ("graph_steps", C.c_int), ("steps", C.c_longlong),
                ("scene_rebuilds", C.c_longlong), ("tile_splits", C.c_longlong), ("launches", C.c_longlong)]


class Cuboid(C.Structure):
    """mph_cuboid: one cuboid of a *.boid file (generator/generator.cpp:17-23)."""

    _fields_ = [("spacing", C.c_double), ("type", C.c_int), ("lower", _D3), ("upper", _D3), ("velocity", _D3)]


class Boid(C.Structure):
    """mph_boid: the domain keys of a *.boid file."""

    _fields_ = [("particle_distance", C.c_double), ("lower_domain", _D3), ("upper_domain", _D3),
                ("cuboid_count", C.c_int)]


BATCH_GRAPH_STEPS = 16

# every symbol the header declares, with its ctypes signature
_P = C.c_void_p
_I = C.c_int
_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int)
_fp = C.POINTER(C.c_float)
SIGNATURES = {
    "mph_params_defaults": (_I, [C.POINTER(Params)]),
    "mph_read_data_file": (_I, [C.c_char_p, C.POINTER(Params), _ip]),
    "mph_read_grid_header": (_I, [C.c_char_p, C.POINTER(GridHeader)]),
    "mph_read_grid_file": (_I, [C.c_char_p, C.POINTER(GridHeader), _I, _ip, _dp, _dp]),
    "mph_write_grid_file": (_I, [C.c_char_p, C.POINTER(GridHeader), _ip, _dp, _dp]),
    "mph_read_boid_file": (_I, [C.c_char_p, C.POINTER(Boid), C.POINTER(Cuboid), _I, _ip]),
    "mph_generate_cuboids": (_I, [C.POINTER(Cuboid), _I, _ip, _dp, _dp, C.c_longlong, C.POINTER(C.c_longlong)]),
    "mph_write_generated_grid": (_I, [C.c_char_p, C.POINTER(Boid), C.c_longlong, _ip, _dp, _dp]),
    "mph_generate_grid_file": (_I, [C.c_char_p, C.c_char_p, C.POINTER(C.c_longlong)]),
    "mph_generator_last_error": (_I, [C.c_char_p, _I]),
    "mph_compute_constants": (_I, [C.POINTER(Params), C.POINTER(GridHeader), _I, C.POINTER(Constants)]),
    "mph_create": (_I, [C.POINTER(Params), C.POINTER(GridHeader), _I, _I, _ip, _dp, _dp, C.POINTER(_P)]),
    "mph_step": (_I, [_P, _I]),
    "mph_synchronize": (_I, [_P]),
    "mph_get_info": (_I, [_P, C.POINTER(Info)]),
    "mph_get_constants": (_I, [_P, C.POINTER(Constants)]),
    "mph_get_state": (_I, [_P, _ip, _ip, _dp, _dp, _dp, _ip, _dp, _dp, _dp]),
    "mph_set_state": (_I, [_P, _dp, _dp]),
    "mph_step_read_state": (_I, [_P, C.c_int, _dp, _dp]),
    "mph_set_step_graphs": (_I, [_P, C.c_int]),
    "mph_set_sweep_layout": (_I, [_P, C.c_int]),
    "mph_get_fields": (_I, [_P, _dp, _dp, _dp, _dp]),
    "mph_get_cells": (_I, [_P, _ip, _ip, _ip, _ip, _ip]),
    "mph_get_neighbors": (_I, [_P, C.POINTER(C.c_longlong), _ip, C.c_longlong]),
    "mph_compute_virial": (_I, [_P]),
    "mph_write_vtk": (_I, [_P, C.c_char_p]),
    "mph_write_prof": (_I, [_P, C.c_char_p]),
    "mph_write_vtk_async": (_I, [_P, C.c_char_p]),
    "mph_write_prof_async": (_I, [_P, C.c_char_p]),
    "mph_output_wait": (_I, [_P]),
    "mph_format_e": (_I, [C.c_void_p, C.c_longlong, _I, C.c_char_p, C.c_longlong, C.POINTER(C.c_longlong)]),
    "mph_write_vtk_arrays": (_I, [C.c_char_p, _I, _ip, _dp, _dp, _dp, _ip, _dp, _dp, _dp]),
    "mph_conserved_sums": (_I, [_P, _dp]),
    "mph_write_checkpoint": (_I, [_P, C.c_char_p]),
    "mph_write_checkpoint_arrays": (_I, [C.c_char_p, C.POINTER(Params), C.POINTER(GridHeader), _I, C.c_longlong,
                                         _ip, _ip, _dp, _dp]),
    "mph_read_checkpoint_header": (_I, [C.c_char_p, C.POINTER(Params), C.POINTER(GridHeader), _ip,
                                        C.POINTER(C.c_longlong)]),
    "mph_read_checkpoint": (_I, [C.c_char_p, C.POINTER(Params), C.POINTER(GridHeader), _ip, C.POINTER(C.c_longlong),
                                 _I, _ip, _ip, _dp, _dp]),
    "mph_stream": (_P, [_P]),
    "mph_launch_count": (C.c_longlong, [_P]),
    "mph_profile_enable": (_I, [_P, _I]),
    "mph_profile_read": (_I, [_P, C.POINTER(KernelStat), _I, _ip]),
    "mph_check_exact_division": (_I, [C.c_longlong, C.c_ulonglong, C.POINTER(C.c_longlong), _dp]),
    "mph_cell_sort_noalloc": (_I, [C.POINTER(Constants), C.POINTER(GridHeader), _I, _P, _P, _P, _P, _P, _P]),
    "mph_model_create": (_I, [C.c_ulonglong, C.POINTER(_P)]),
    "mph_model_destroy": (None, [_P]),
    "mph_model_param_count": (_I, []),
    "mph_model_get_params": (_I, [_P, _fp]),
    "mph_model_set_params": (_I, [_P, _fp]),
    "mph_model_set_scales": (_I, [_P, C.c_double, C.c_double]),
    "mph_model_get_scales": (_I, [_P, _dp, _dp]),
    "mph_model_gradient": (_I, [_P, _fp, C.c_longlong, _fp, _dp]),
    "mph_model_predict": (_I, [_P, _fp, C.c_longlong, _fp]),
    "mph_model_fit_scales": (_I, [_P, _P]),
    "mph_model_train": (_I, [_P, _P, _I, _I, C.c_double, C.c_ulonglong, _dp]),
    "mph_model_last_error": (_I, [_P, C.c_char_p, _I]),
    "mph_model_check_wait": (_I, [_P, _I, C.c_longlong]),
    "mph_dataset_create": (_I, [C.c_longlong, C.POINTER(_P)]),
    "mph_dataset_destroy": (None, [_P]),
    "mph_dataset_size": (C.c_longlong, [_P]),
    "mph_dataset_append": (_I, [_P, _fp, C.c_longlong]),
    "mph_dataset_read": (_I, [_P, C.c_longlong, C.c_longlong, _fp]),
    "mph_collect_samples": (_I, [_P, _P, C.c_longlong, C.c_ulonglong]),
    "mph_set_learned": (_I, [_P, _P, _I, C.c_double]),
    "mph_learned_stats": (_I, [_P, C.POINTER(LearnedInfo)]),
    "mph_batch_create": (_I, [_I, C.POINTER(Params), C.POINTER(GridHeader), _I, _ip, _dp, _dp, C.POINTER(_P)]),
    "mph_batch_step": (_I, [_P, _I]),
    "mph_batch_synchronize": (_I, [_P]),
    "mph_batch_get_state": (_I, [_P, _dp, _dp]),
    "mph_batch_set_tiles": (_I, [_P, _I, _I, _I, _I, _I]),
    "mph_batch_autotune": (_I, [_P, _I, C.POINTER(BatchTrial), _I, _ip]),
    "mph_batch_get_info": (_I, [_P, C.POINTER(BatchInfo)]),
    "mph_batch_stream": (_P, [_P]),
    "mph_batch_profile_enable": (_I, [_P, _I]),
    "mph_batch_profile_read": (_I, [_P, C.POINTER(KernelStat), _I, _ip]),
    "mph_batch_last_error": (_I, [_P, C.c_char_p, _I]),
    "mph_batch_destroy": (None, [_P]),
    "mph_last_error": (_I, [_P, C.c_char_p, _I]),
    "mph_destroy": (None, [_P]),
    "mph_version": (C.c_char_p, []),
}

PKG_DIR = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(PKG_DIR, "libmph_b200.so")
_lib = None


def load() -> C.CDLL:
    """Open the in-tree sm_100a library (no fallback)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(
            f"{LIB_PATH} is missing; build it with `make -C {os.path.join(PKG_DIR, 'csrc')}` "
            "or `python -c 'import __graft_entry__ as g; g.build()'`")
    lib = C.CDLL(LIB_PATH)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib
