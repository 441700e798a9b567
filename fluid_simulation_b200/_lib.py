"""ctypes binding of ``libfluid_b200.so`` (C ABI in ``include/fluid_b200.h``).

The product path has no fallback: if the library or a CUDA device is missing,
the solvers raise instead of computing anything on the CPU.
"""

from __future__ import annotations

import ctypes as C
import os
import threading

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libfluid_b200.so")

FS_OK = 0
FS_ERR_INVALID = 1
FS_ERR_CUDA = 2
FS_ERR_CAPACITY = 3
FS_ERR_NOGRID = 4
FS_ERR_NONFINITE = 5

FS_STATUS_NONFINITE = 1
FS_STATUS_GRID_OVERFLOW = 2
FS_STATUS_BOUNDS = 4
FS_STATUS_TIMEOUT = 8

STATUS_NAMES = {FS_STATUS_NONFINITE: "NONFINITE", FS_STATUS_GRID_OVERFLOW: "GRID_OVERFLOW",
                FS_STATUS_BOUNDS: "BOUNDS", FS_STATUS_TIMEOUT: "TIMEOUT"}

P = C.c_void_p
F = C.c_float
I32 = C.c_int32
I64 = C.c_int64


class GridConfig(C.Structure):
    _fields_ = [("dim_x", I32), ("dim_y", I32), ("dim_z", I32), ("rounding", I32)]


class WorldBox(C.Structure):
    _fields_ = [("cell_lo", I32 * 3), ("dims", I32 * 3), ("bound_width", F), ("bound_height", F),
                ("bound_length", F)]


class Tuning(C.Structure):
    _fields_ = [("block_size", I32), ("particles_per_thread", I32), ("cell_ratio", F), ("list_skin", F)]


class FrameClock(C.Structure):
    _fields_ = [("remaining", C.c_double), ("dt", F), ("active", I32), ("substeps", I32), ("run_substeps", I32),
                ("fault", I32), ("maxima", F * 2), ("pad", I32)]


class CflRule(C.Structure):
    _fields_ = [("frame_dt", C.c_double), ("substep_limit", C.c_double), ("method", I32), ("use_accel", I32),
                ("h", C.c_double), ("sound_speed", C.c_double), ("viscosity", C.c_double), ("spacing", C.c_double)]


class Model(C.Structure):
    _fields_ = [("n", I64), ("n_worlds", I32)] + [(k, P) for k in (
        "particle_flags", "particle_mask", "particle_world", "particle_mass", "gravity", "rest_density",
        "surface_tension", "viscosity", "stiffness", "exponent")]


class State(C.Structure):
    _fields_ = [(k, P) for k in (
        "particle_q", "particle_qd", "rho", "pressure", "factor", "rho_star", "d_rho_dt", "kappa", "kappa_v",
        "neighbor_count", "v_star", "pbf_lambda", "delta_p")]


class WcsphParams(C.Structure):
    _fields_ = [(k, F) for k in ("dt", "smoothing_length", "particle_radius", "bound_width", "bound_height",
                                 "bound_length", "boundary_damping")] + [("clamp_negative_pressure", I32)]


class DfsphParams(C.Structure):
    _fields_ = [(k, F) for k in ("dt", "smoothing_length", "particle_radius", "bound_width", "bound_height",
                                 "bound_length", "boundary_damping")] + [
        (k, I32) for k in ("max_rho_iterations", "max_vel_iterations", "warm_start", "min_neighbors_for_factor")] + [
        (k, F) for k in ("eta_density", "eta_divergence", "max_kappa", "max_kappa_v")]


class PbfParams(C.Structure):
    _fields_ = [(k, F) for k in ("dt", "smoothing_length", "particle_radius", "bound_width", "bound_height",
                                 "bound_length", "boundary_damping", "boundary_epsilon")] + [
        (k, I32) for k in ("max_iterations", "min_neighbors_for_lambda", "rebuild_grid_each_iteration")] + [
        (k, F) for k in ("lambda_epsilon", "scorr_k", "scorr_n", "scorr_w_delta_q", "max_delta_position", "xsph_c")]


class SeparationParams(C.Structure):
    _fields_ = [("rest_dist", F), ("query_radius", F), ("strength", F), ("bound_lo", F * 3), ("bound_hi", F * 3),
                ("wall_band", F), ("wall_margin", F), ("iterations", I32)]


class DfsphInfo(C.Structure):
    _fields_ = [("rho_iterations", I32), ("vel_iterations", I32), ("density_residual", C.c_double),
                ("divergence_residual", C.c_double)]


# name -> (restype, argtypes); must match include/fluid_b200.h
SIGNATURES = {
    "fs_context_create": (C.c_int, [C.POINTER(P), I64, C.POINTER(GridConfig), I32]),
    "fs_context_destroy": (C.c_int, [P]),
    "fs_context_capacity": (I64, [P]),
    "fs_grid_build": (C.c_int, [P, P, I64, F, P]),
    "fs_grid_tables": (C.c_int, [P, P, P, P, P, P]),
    "fs_grid_candidates": (C.c_int, [P, P, I64, F, P, P, P, P]),
    "fs_context_create_worlds": (C.c_int, [C.POINTER(P), I64, C.POINTER(WorldBox), I32, I32]),
    "fs_context_worlds": (I32, [P]),
    "fs_context_set_tuning": (C.c_int, [P, C.POINTER(Tuning)]),
    "fs_frame_clock_start": (C.c_int, [P, C.c_double, P]),
    "fs_frame_metrics": (C.c_int, [P, P, P, I64, P, P, I64, I64, P, P]),
    "fs_frame_clock_advance": (C.c_int, [P, C.POINTER(CflRule), P, I64, P, I64, P]),
    "fs_wcsph_substep_clocked": (C.c_int, [P, C.POINTER(Model), C.POINTER(State), C.POINTER(State),
                                           C.POINTER(WcsphParams), P, P, P]),
    "fs_dfsph_substep_clocked": (C.c_int, [P, C.POINTER(Model), C.POINTER(State), C.POINTER(State),
                                           C.POINTER(DfsphParams), P, P, P]),
    "fs_dfsph_nonpressure_predict": (C.c_int, [P, C.POINTER(Model), P, P, P, F, F, F, P, P, P]),
    "fs_pbf_predict": (C.c_int, [P, C.POINTER(Model), P, P, C.POINTER(PbfParams), P, P, P]),
    "fs_context_get_tuning": (C.c_int, [P, C.POINTER(Tuning)]),
    "fs_context_cells": (I64, [P]),
    "fs_grid_build_worlds": (C.c_int, [P, P, P, I64, F, P]),
    "fs_grid_candidates_worlds": (C.c_int, [P, P, P, I64, F, P, P, P, P]),
    "fs_wcsph_substep_adjoint": (C.c_int, [P, C.POINTER(Model), C.POINTER(State), P, P, P, P, P, P, P, P, P, P,
                                           C.POINTER(WcsphParams), P]),
    "fs_wcsph_substep": (C.c_int, [P, C.POINTER(Model), C.POINTER(State), C.POINTER(State),
                                   C.POINTER(WcsphParams), P, P]),
    "fs_dfsph_substep": (C.c_int, [P, C.POINTER(Model), C.POINTER(State), C.POINTER(State),
                                   C.POINTER(DfsphParams), P, P]),
    "fs_dfsph_info_read": (C.c_int, [P, C.POINTER(DfsphInfo)]),
    "fs_dfsph_info_worlds": (C.c_int, [P, C.POINTER(DfsphInfo), C.c_int32]),
    "fs_apic_separation": (C.c_int, [P, P, P, C.c_int64, C.POINTER(SeparationParams), P, P]),
    "fs_pbf_substep": (C.c_int, [P, C.POINTER(Model), C.POINTER(State), C.POINTER(State),
                                 C.POINTER(PbfParams), P, P, P]),
    "fs_wcsph_density": (C.c_int, [P, C.POINTER(Model), P, F, I32, P, P, P]),
    "fs_wcsph_force_integrate": (C.c_int, [P, C.POINTER(Model), C.POINTER(State), C.POINTER(State),
                                           C.POINTER(WcsphParams), P, P]),
    "fs_dfsph_density_factor": (C.c_int, [P, C.POINTER(Model), P, F, I32, P, P, P, P]),
    "fs_dfsph_divergence": (C.c_int, [P, C.POINTER(Model), P, P, F, P, P]),
    "fs_dfsph_correct": (C.c_int, [P, C.POINTER(Model), P, P, P, P, F, F, P]),
    "fs_dfsph_residual": (C.c_int, [P, C.POINTER(Model), P, P, P, P]),
    "fs_pbf_density": (C.c_int, [P, C.POINTER(Model), P, F, P, P]),
    "fs_pbf_lambda": (C.c_int, [P, C.POINTER(Model), P, C.POINTER(PbfParams), P, P, P, P]),
    "fs_pbf_delta": (C.c_int, [P, C.POINTER(Model), P, P, C.POINTER(PbfParams), P, P]),
    "fs_pbf_xsph": (C.c_int, [P, C.POINTER(Model), P, P, P, F, F, P, P]),
    "fs_norm_maxima": (C.c_int, [P, I64, P, I64, P, P]),
    "fs_check_finite": (C.c_int, [P, P, I64, P, I64, P, P]),
    "fs_pass_count": (I32, []),
    "fs_pass_name": (C.c_char_p, [I32]),
    "fs_timer_enable": (C.c_int, [P, I32]),
    "fs_timer_read": (C.c_int, [P, P, P, I32, P]),
    "fs_launch_count": (I64, [P]),
    "fs_list_stats": (C.c_int, [P, P, I32, I32]),
    "fs_list_stats_enable": (C.c_int, [P, I32]),
    "fs_noalloc_max_particles": (I32, []),
    "fs_wcsph_density_noalloc": (C.c_int, [C.POINTER(Model), P, F, I32, P, P, P]),
    "fs_status_read": (C.c_int, [P, C.POINTER(C.c_uint32)]),
    "fs_status_clear": (C.c_int, [P, P]),
    "fs_last_error_string": (C.c_char_p, []),
    "fs_version": (C.c_char_p, []),
}

_lock = threading.Lock()
_lib = None


class FluidLibraryError(RuntimeError):
    pass


def load():
    """Load the in-tree CUDA library (built by ``__graft_entry__.build`` /
    ``python -m fluid_simulation_b200.build``).  Raises if it is missing."""
    global _lib
    with _lock:
        if _lib is None:
            if not os.path.exists(LIB_PATH):
                raise FluidLibraryError(
                    f"{LIB_PATH} is missing: build it with `python -m fluid_simulation_b200.build`; "
                    "there is no CPU implementation of the solver kernels")
            lib = C.CDLL(LIB_PATH)
            for name, (res, args) in SIGNATURES.items():
                fn = getattr(lib, name)
                fn.restype = res
                fn.argtypes = args
            _lib = lib
    return _lib


def check(rc: int, what: str = "") -> None:
    if rc != FS_OK:
        msg = load().fs_last_error_string().decode(errors="replace")
        raise FluidLibraryError(f"{what}: fluid_b200 error {rc}: {msg}")


def status_names(word: int):
    return [name for bit, name in STATUS_NAMES.items() if word & bit]
