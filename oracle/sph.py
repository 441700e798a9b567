"""ctypes wrapper of the CPU oracle (test infrastructure only; see package doc).

Model and state are plain dicts of numpy arrays named like the Newton
attributes the reference solvers read:

* model: ``particle_flags`` (i32), ``particle_mass``, ``particle_world`` (i32),
  ``gravity`` ([W,3]), ``particle_max_radius`` (float) and the ``sph``
  namespace dict: ``particle_mask`` (i32), ``rest_density``,
  ``surface_tension``, ``viscosity``, ``stiffness``, ``exponent``.
* state: ``particle_q`` ([N,3]), ``particle_qd`` ([N,3]) and ``sph`` dict.

Configs are dicts with the field names of the reference dataclasses
(``SolverWCSPH.SphConfig`` solver_wcsph.py:309-318, ``SolverDFSPH.SphConfig``
solver_dfsph.py:446-463, ``SolverPBF.PbfConfig`` solver_pbf.py:521-539).
"""

from __future__ import annotations

import ctypes as C
import os
import subprocess
import threading

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_SRC = os.path.join(_HERE, "sph_oracle.cpp")
_LIB = os.path.join(_HERE, "libsph_oracle.so")
_lock = threading.Lock()
_lib = None

# Portable ISA level: the library is built in one place and may run on
# another host.  -ffp-contract=off keeps every operation individually rounded.
CXXFLAGS = ["-O3", "-march=x86-64-v2", "-fopenmp", "-ffp-contract=off", "-fPIC", "-shared", "-std=c++17"]


def build_oracle(force: bool = False) -> str:
    """Compile ``sph_oracle.cpp`` into ``libsph_oracle.so`` (g++)."""
    if force or not os.path.exists(_LIB) or os.path.getmtime(_LIB) < os.path.getmtime(_SRC):
        tmp = _LIB + f".tmp{os.getpid()}"
        subprocess.check_call(["g++", *CXXFLAGS, "-o", tmp, _SRC])
        os.replace(tmp, _LIB)
    return _LIB


class GridCfg(C.Structure):
    _fields_ = [("dim_x", C.c_int32), ("dim_y", C.c_int32), ("dim_z", C.c_int32), ("rounding", C.c_int32)]


class _Model(C.Structure):
    _fields_ = [
        ("n", C.c_int64), ("n_worlds", C.c_int32),
        ("flags", C.c_void_p), ("mask", C.c_void_p), ("world", C.c_void_p),
        ("mass", C.c_void_p), ("gravity", C.c_void_p), ("rest_density", C.c_void_p),
        ("surface_tension", C.c_void_p), ("viscosity", C.c_void_p),
        ("stiffness", C.c_void_p), ("exponent", C.c_void_p),
    ]


class _State(C.Structure):
    _fields_ = [(k, C.c_void_p) for k in (
        "q", "qd", "rho", "pressure", "factor", "rho_star", "d_rho_dt", "kappa", "kappa_v",
        "neighbor_count", "v_star", "pbf_lambda", "delta_p")]


class _Wcsph(C.Structure):
    _fields_ = [(k, C.c_double) for k in (
        "particle_radius", "particle_max_radius", "particle_length", "smoothing_length_coff",
        "bound_width", "bound_height", "bound_length", "boundary_damping")] + [
        ("clamp_negative_pressure", C.c_int32), ("grid", GridCfg)]


class _Dfsph(C.Structure):
    _fields_ = [(k, C.c_int32) for k in (
        "max_rho_iterations", "max_vel_iterations", "warm_start", "min_neighbors_for_factor")] + [
        (k, C.c_double) for k in (
            "eta_density", "eta_divergence", "max_kappa", "max_kappa_v",
            "particle_radius", "particle_max_radius", "particle_length", "smoothing_length_coff",
            "bound_width", "bound_height", "bound_length", "boundary_damping")] + [("grid", GridCfg)]


class _Pbf(C.Structure):
    _fields_ = [(k, C.c_int32) for k in (
        "max_iterations", "min_neighbors_for_lambda", "rebuild_grid_each_iteration")] + [
        (k, C.c_double) for k in (
            "lambda_epsilon", "scorr_k", "scorr_n", "scorr_q", "max_delta_position", "xsph_c",
            "particle_radius", "particle_max_radius", "particle_length", "smoothing_length_coff",
            "bound_width", "bound_height", "bound_length", "boundary_damping", "boundary_epsilon")] + [
        ("grid", GridCfg)]


class _Separation(C.Structure):
    _fields_ = [("rest_dist", C.c_double), ("query_radius", C.c_double), ("strength", C.c_double),
                ("bound_lo", C.c_double * 3), ("bound_hi", C.c_double * 3), ("wall_band", C.c_double),
                ("wall_margin", C.c_double), ("iterations", C.c_int32), ("grid", GridCfg)]


class DfsphInfo(C.Structure):
    _fields_ = [("rho_iterations", C.c_int32), ("vel_iterations", C.c_int32),
                ("last_density_residual", C.c_double), ("last_divergence_residual", C.c_double)]


def _load():
    global _lib
    with _lock:
        if _lib is None:
            lib = C.CDLL(build_oracle())
            P = C.c_void_p
            lib.oracle_num_threads.argtypes = [C.c_int]
            lib.oracle_grid_build_f32.argtypes = [P, C.c_int64, C.c_float, C.POINTER(GridCfg), P, P, P, P]
            lib.oracle_grid_candidates_f32.argtypes = [P, C.c_int64, C.c_float, C.POINTER(GridCfg), P, C.c_int64,
                                                       C.c_float, P, P, P]
            for prec, ct in (("f32", C.c_float), ("f64", C.c_double)):
                getattr(lib, f"oracle_wcsph_step_{prec}").argtypes = [
                    C.POINTER(_Model), C.POINTER(_State), C.POINTER(_State), C.POINTER(_Wcsph), ct, P]
                getattr(lib, f"oracle_dfsph_step_{prec}").argtypes = [
                    C.POINTER(_Model), C.POINTER(_State), C.POINTER(_State), C.POINTER(_Dfsph), ct, P,
                    C.POINTER(DfsphInfo)]
                getattr(lib, f"oracle_pbf_step_{prec}").argtypes = [
                    C.POINTER(_Model), C.POINTER(_State), C.POINTER(_State), C.POINTER(_Pbf), ct, P, P]
            for prec in ("f32", "f64"):
                getattr(lib, f"oracle_apic_separation_{prec}").argtypes = [P, P, C.c_int64,
                                                                          C.POINTER(_Separation), P]
            _lib = lib
    return _lib


def num_threads(n: int = 0) -> int:
    """Set (n > 0) and return the OpenMP thread count of the oracle."""
    return int(_load().oracle_num_threads(int(n)))


def _ptr(a):
    return None if a is None else a.ctypes.data


def _grid_cfg(dims=(128, 128, 128), rounding=0) -> GridCfg:
    return GridCfg(int(dims[0]), int(dims[1]), int(dims[2]), int(rounding))


def grid_build(x, radius, dims=(128, 128, 128), rounding=0):
    """Reference hash-grid tables for points ``x`` [N,3] f32."""
    lib = _load()
    x = np.ascontiguousarray(x, dtype=np.float32)
    n = x.shape[0]
    nc = int(dims[0]) * int(dims[1]) * int(dims[2])
    out = dict(point_ids=np.empty(n, np.int32), point_cells=np.empty(n, np.int32),
               cell_starts=np.empty(nc, np.int32), cell_ends=np.empty(nc, np.int32))
    cfg = _grid_cfg(dims, rounding)
    lib.oracle_grid_build_f32(_ptr(x), n, float(np.float32(radius)), C.byref(cfg), _ptr(out["point_ids"]),
                              _ptr(out["point_cells"]), _ptr(out["cell_starts"]), _ptr(out["cell_ends"]))
    return out


def grid_candidates(x, radius, queries=None, query_radius=None, dims=(128, 128, 128), rounding=0):
    """Candidate lists of the reference query, CSR form (offsets, candidates)."""
    lib = _load()
    x = np.ascontiguousarray(x, dtype=np.float32)
    q = x if queries is None else np.ascontiguousarray(queries, dtype=np.float32)
    r = float(np.float32(radius if query_radius is None else query_radius))
    cfg = _grid_cfg(dims, rounding)
    counts = np.empty(q.shape[0], np.int64)
    lib.oracle_grid_candidates_f32(_ptr(x), x.shape[0], float(np.float32(radius)), C.byref(cfg), _ptr(q),
                                   q.shape[0], r, _ptr(counts), None, None)
    offsets = np.zeros(q.shape[0] + 1, np.int64)
    np.cumsum(counts, out=offsets[1:])
    cand = np.empty(int(offsets[-1]), np.int32)
    lib.oracle_grid_candidates_f32(_ptr(x), x.shape[0], float(np.float32(radius)), C.byref(cfg), _ptr(q),
                                   q.shape[0], r, _ptr(counts), _ptr(offsets), _ptr(cand))
    return offsets, cand


# ----------------------------------------------------------------- steps ----
def _model_struct(model, dt_np, keep):
    n = int(model["particle_q_count"]) if "particle_q_count" in model else len(model["particle_mass"])
    sph = model["sph"]

    def f(a):
        if a is None:
            return None
        a = np.ascontiguousarray(a, dtype=dt_np)
        keep.append(a)
        return a

    def i32(a):
        a = np.ascontiguousarray(a, dtype=np.int32)
        keep.append(a)
        return a

    grav = f(np.asarray(model["gravity"]).reshape(-1, 3))
    world = model.get("particle_world")
    world = i32(np.zeros(n, np.int32) if world is None else world)
    m = _Model(n, grav.shape[0], _ptr(i32(model["particle_flags"])), _ptr(i32(sph["particle_mask"])),
               _ptr(world), _ptr(f(model["particle_mass"])), _ptr(grav), _ptr(f(sph["rest_density"])),
               _ptr(f(sph["surface_tension"])), _ptr(f(sph["viscosity"])), _ptr(f(sph.get("stiffness"))),
               _ptr(f(sph.get("exponent"))))
    return m, n


def _state_in(state, dt_np, keep, names):
    st = _State()
    st.q = _ptr(_keep(keep, np.ascontiguousarray(state["particle_q"], dtype=dt_np)))
    st.qd = _ptr(_keep(keep, np.ascontiguousarray(state["particle_qd"], dtype=dt_np)))
    sph = state.get("sph", {})
    for k in names:
        if k in sph:
            dt = np.int32 if k == "neighbor_count" else dt_np
            setattr(st, k, _ptr(_keep(keep, np.ascontiguousarray(sph[k], dtype=dt))))
    return st


def _keep(keep, a):
    keep.append(a)
    return a


def _state_out(n, dt_np, names, vec_names=()):
    out = {"particle_q": np.zeros((n, 3), dt_np), "particle_qd": np.zeros((n, 3), dt_np), "sph": {}}
    st = _State(q=_ptr(out["particle_q"]), qd=_ptr(out["particle_qd"]))
    for k in names:
        if k == "neighbor_count":
            a = np.zeros(n, np.int32)
        elif k in vec_names:
            a = np.zeros((n, 3), dt_np)
        else:
            a = np.zeros(n, dt_np)
        out["sph"][k] = a
        setattr(st, k, _ptr(a))
    return out, st


def _common(cfg, model):
    return dict(particle_radius=float(cfg["particle_radius"]),
                particle_max_radius=float(model.get("particle_max_radius", 0.0)),
                particle_length=float(cfg["particle_length"]),
                smoothing_length_coff=float(cfg["smoothing_length_coff"]),
                bound_width=float(cfg["bound_width"]), bound_height=float(cfg["bound_height"]),
                bound_length=float(cfg["bound_length"]), boundary_damping=float(cfg["boundary_damping"]))


def _dtype(precision):
    return (np.float32, "f32") if precision in ("f32", np.float32, "float32") else (np.float64, "f64")


def wcsph_step(model, state_in, cfg, dt, precision="f32", dims=(128, 128, 128), rounding=0):
    """One ``SolverWCSPH.step`` (solver_wcsph.py:431-535).  Returns (state_out, accel)."""
    lib = _load()
    dt_np, p = _dtype(precision)
    keep = []
    m, n = _model_struct(model, dt_np, keep)
    si = _state_in(state_in, dt_np, keep, ())
    out, so = _state_out(n, dt_np, ("rho", "pressure"))
    c = _Wcsph(**_common(cfg, model), clamp_negative_pressure=int(bool(cfg.get("clamp_negative_pressure", True))),
               grid=_grid_cfg(dims, rounding))
    accel = np.zeros((n, 3), dt_np)
    getattr(lib, f"oracle_wcsph_step_{p}")(C.byref(m), C.byref(si), C.byref(so), C.byref(c), dt, _ptr(accel))
    return out, accel


_DFSPH_OUT = ("rho", "factor", "rho_star", "d_rho_dt", "kappa", "kappa_v", "neighbor_count", "v_star")


def dfsph_step(model, state_in, cfg, dt, precision="f32", dims=(128, 128, 128), rounding=0):
    """One ``SolverDFSPH.step`` (solver_dfsph.py:598-898).  Returns (state_out, accel, info)."""
    lib = _load()
    dt_np, p = _dtype(precision)
    keep = []
    m, n = _model_struct(model, dt_np, keep)
    si = _state_in(state_in, dt_np, keep, ("kappa", "kappa_v"))
    out, so = _state_out(n, dt_np, _DFSPH_OUT, vec_names=("v_star",))
    c = _Dfsph(max_rho_iterations=int(cfg["max_rho_iterations"]), max_vel_iterations=int(cfg["max_vel_iterations"]),
               warm_start=int(bool(cfg["warm_start"])), min_neighbors_for_factor=int(cfg["min_neighbors_for_factor"]),
               eta_density=float(cfg["eta_density"]), eta_divergence=float(cfg["eta_divergence"]),
               max_kappa=float(cfg["max_kappa"]), max_kappa_v=float(cfg["max_kappa_v"]),
               grid=_grid_cfg(dims, rounding), **_common(cfg, model))
    if cfg["warm_start"]:
        for k in ("kappa", "kappa_v"):
            if k not in state_in.get("sph", {}):
                raise ValueError(f"warm_start needs state_in.sph.{k}")
    accel = np.zeros((n, 3), dt_np)
    info = DfsphInfo()
    getattr(lib, f"oracle_dfsph_step_{p}")(C.byref(m), C.byref(si), C.byref(so), C.byref(c), dt, _ptr(accel),
                                          C.byref(info))
    return out, accel, dict(rho_iterations=info.rho_iterations, vel_iterations=info.vel_iterations,
                            density_residual=info.last_density_residual,
                            divergence_residual=info.last_divergence_residual)


def pbf_step(model, state_in, cfg, dt, precision="f32", dims=(128, 128, 128), rounding=0):
    """One ``SolverPBF.step`` (solver_pbf.py:676-954).  Returns (state_out, accel, x_pred)."""
    lib = _load()
    dt_np, p = _dtype(precision)
    keep = []
    m, n = _model_struct(model, dt_np, keep)
    si = _state_in(state_in, dt_np, keep, ())
    out, so = _state_out(n, dt_np, ("rho", "pbf_lambda", "neighbor_count", "delta_p"), vec_names=("delta_p",))
    c = _Pbf(max_iterations=int(cfg["max_iterations"]), min_neighbors_for_lambda=int(cfg["min_neighbors_for_lambda"]),
             rebuild_grid_each_iteration=int(bool(cfg.get("rebuild_grid_each_iteration", False))),
             lambda_epsilon=float(cfg["lambda_epsilon"]), scorr_k=float(cfg["scorr_k"]),
             scorr_n=float(cfg["scorr_n"]), scorr_q=float(cfg["scorr_q"]),
             max_delta_position=float(cfg["max_delta_position"]), xsph_c=float(cfg["xsph_c"]),
             boundary_epsilon=float(cfg.get("boundary_epsilon", 0.0)), grid=_grid_cfg(dims, rounding),
             **_common(cfg, model))
    accel = np.zeros((n, 3), dt_np)
    xpred = np.zeros((n, 3), dt_np)
    getattr(lib, f"oracle_pbf_step_{p}")(C.byref(m), C.byref(si), C.byref(so), C.byref(c), dt, _ptr(accel),
                                        _ptr(xpred))
    return out, accel, xpred


def apic_separation(x, flags, cfg, precision="f32"):
    """``SolverAPIC._apply_particle_separation`` (solver_apic.py:1003-1064)
    with the two kernels of lines 193-266: ``cfg`` holds rest_dist,
    query_radius, strength, iterations, bound_lo, bound_hi, wall_band,
    wall_margin and the hash-grid dims.  Returns (positions after the last
    iteration, that iteration's pushes)."""
    lib = _load()
    dt_np, p = _dtype(precision)
    xo = np.ascontiguousarray(np.asarray(x, dt_np)).copy()
    fl = np.ascontiguousarray(np.asarray(flags, np.int32))
    n = len(xo)
    delta = np.zeros((n, 3), dt_np)
    c = _Separation(rest_dist=float(cfg["rest_dist"]), query_radius=float(cfg["query_radius"]),
                    strength=float(cfg["strength"]), wall_band=float(cfg["wall_band"]),
                    wall_margin=float(cfg["wall_margin"]), iterations=int(cfg["iterations"]),
                    grid=_grid_cfg(cfg["dims"], 0))
    c.bound_lo[:] = [float(v) for v in cfg["bound_lo"]]
    c.bound_hi[:] = [float(v) for v in cfg["bound_hi"]]
    getattr(lib, f"oracle_apic_separation_{p}")(_ptr(xo), _ptr(fl), n, C.byref(c), _ptr(delta))
    return xo, delta
