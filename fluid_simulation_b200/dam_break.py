"""Dam-break driver on the drop-in solvers (reference:
examples/dam_break/simulation.py, the caller of the hot path).

``DamBreakSimulation`` keeps the reference's constructor arguments, solver
configurations (simulation.py:110-132), frame logic (fixed substeps for PBF,
CFL substeps for WCSPH/DFSPH, 155-190) and metrics (198-225).  The CFL
maxima and the finite check are device reductions in ``libfluid_b200.so``
that read back two floats / one int, like the reference's Warp kernels.
APIC is not part of the particle hot path and is not provided.
"""

from __future__ import annotations

import ctypes as C
import math
from dataclasses import asdict

import numpy as np
import torch

from . import _lib
from .newton_shim import Axis, ModelBuilder, model_from_arrays
from .scene import ParticleScene
from .solver import SolverDFSPH, SolverPBF, SolverWCSPH

SOLVERS = {"wcsph": SolverWCSPH, "dfsph": SolverDFSPH, "pbf": SolverPBF}


def solver_config(method, scene: ParticleScene, *, wcsph_smoothing_length_coff=2.0,
                  wcsph_clamp_negative_pressure=True):
    """The reference harness's solver configs (simulation.py:110-132)."""
    bounds = dict(bound_width=scene.spec.bound_hi[0], bound_height=scene.spec.bound_hi[1],
                  bound_length=scene.spec.bound_hi[2] * 0.5)
    common = dict(particle_radius=scene.radius, particle_length=scene.spacing, smoothing_length_coff=2.0,
                  boundary_damping=0.0, **bounds)
    if method == "wcsph":
        common["smoothing_length_coff"] = wcsph_smoothing_length_coff
        return SolverWCSPH.SphConfig(clamp_negative_pressure=wcsph_clamp_negative_pressure, **common)
    if method == "dfsph":
        return SolverDFSPH.SphConfig(max_rho_iterations=5, max_vel_iterations=12, warm_start=False, max_kappa=1.0,
                                     max_kappa_v=100.0, **common)
    if method == "pbf":
        return SolverPBF.PbfConfig(max_iterations=4, lambda_epsilon=100.0, min_neighbors_for_lambda=8, scorr_k=0.0,
                                   max_delta_position=scene.radius * 0.5, xsph_c=0.05, **common)
    raise ValueError(f"unknown method {method!r} (the particle path provides wcsph, dfsph, pbf)")


def percentile99_ranks(n: int):
    """Sorted positions whose values numpy.percentile(a, 99) interpolates
    for a float32 array of n values: q = float32(0.99), index (n - 1) q in
    float32 (numpy 2 keeps the array's dtype)."""
    q = np.float32(99) / np.float32(100)
    virtual = np.float32(n - 1) * q
    k = int(np.floor(virtual))
    return k, min(k + 1, n - 1)


def percentile99(a: float, b: float, n: int) -> np.float32:
    """numpy.percentile(x, 99) of a float32 array of n values from its two
    order statistics a (k-th) and b ((k+1)-th), numpy's linear method in
    float32: a + (b - a) g, or b - (b - a)(1 - g) for g >= 0.5."""
    q = np.float32(99) / np.float32(100)
    virtual = np.float32(n - 1) * q
    g = np.float32(virtual - np.float32(np.floor(virtual)))
    a, b = np.float32(a), np.float32(b)
    d = np.float32(b - a)
    return np.float32(b - d * (np.float32(1) - g)) if g >= 0.5 else np.float32(a + d * g)


def material(method, scene, wcsph_stiffness=250000.0, wcsph_viscosity=1.0e-6):
    """simulation.py:84-91."""
    m = {"rest_density": scene.spec.density, "surface_tension": 0.0, "viscosity": 1.0e-6}
    if method == "wcsph":
        m.update(stiffness=wcsph_stiffness, exponent=7.0, viscosity=wcsph_viscosity)
    return m


class DamBreakSimulation:
    def __init__(self, scene: ParticleScene, method, device="cuda:0", substeps=4, voxel_size=None,
                 enable_projection=True, *, wcsph_stiffness=250000.0, wcsph_viscosity=1.0e-6,
                 wcsph_smoothing_length_coff=2.0, wcsph_clamp_negative_pressure=True):
        if method == "apic":
            raise NotImplementedError("APIC (grid solver) is outside the particle hot path")
        if method == "wcsph":
            for name, value in (("stiffness", wcsph_stiffness), ("smoothing_length_coff", wcsph_smoothing_length_coff)):
                if not math.isfinite(value) or value <= 0.0:
                    raise ValueError(f"WCSPH {name} must be finite and positive")
            if not math.isfinite(wcsph_viscosity) or wcsph_viscosity < 0.0:
                raise ValueError("WCSPH viscosity must be finite and non-negative")
        self.scene = scene
        self.method = method
        self.frame_dt = 1.0 / scene.spec.fps
        self.substeps = substeps
        self.frame = 0
        self.sim_time = 0.0
        self.last_substeps = 0
        self.total_substeps = 0
        solver_cls = SOLVERS[method]
        self.material = material(method, scene, wcsph_stiffness, wcsph_viscosity)
        n = scene.count
        attrs = dict(self.material)
        attrs["particle_mask"] = 0
        self.model = model_from_arrays(scene.positions, np.zeros_like(scene.positions), scene.mass, device=device,
                                       radius=scene.radius, gravity=(scene.spec.gravity,), attributes=attrs,
                                       solver_cls=solver_cls)
        self.state_0, self.state_1 = self.model.state(), self.model.state()
        config = solver_config(method, scene, wcsph_smoothing_length_coff=wcsph_smoothing_length_coff,
                               wcsph_clamp_negative_pressure=wcsph_clamp_negative_pressure)
        self.solver = solver_cls(self.model, config)
        dev = self.model.device
        self._norm_maxima = torch.zeros(2, dtype=torch.float32, device=dev)
        self._invalid_state = torch.zeros(1, dtype=torch.int32, device=dev)
        self._host2 = torch.zeros(2, dtype=torch.float32).pin_memory() if dev.type == "cuda" else None
        self._metrics = None
        del n

    @property
    def _stream(self):
        return torch.cuda.current_stream(self.model.device).cuda_stream

    def _cfl_maxima(self):
        """simulation.py:140-153: device reduction, two scalars read back."""
        use_acc = self.method == "wcsph" and self.total_substeps
        acc = self.solver._particle_accel
        v = self.state_0.particle_qd
        lib = _lib.load()
        _lib.check(lib.fs_norm_maxima(v.data_ptr(), v.shape[0], acc.data_ptr() if use_acc else None,
                                      acc.shape[0] if use_acc else 0, self._norm_maxima.data_ptr(), self._stream),
                   "norm maxima")
        speed2, accel2 = self._norm_maxima.tolist()
        if not math.isfinite(speed2):
            raise RuntimeError(f"Non-finite velocity at frame {self.frame}")
        if not math.isfinite(accel2):
            raise RuntimeError("Non-finite WCSPH acceleration")
        return math.sqrt(speed2), math.sqrt(accel2)

    def cfl_dt(self, remaining, speed, accel_max):
        """The dt rule of simulation.py:167-182."""
        limit = self.frame_dt / self.substeps
        if self.method == "wcsph":
            sound_speed = math.sqrt(self.material["stiffness"] * self.material["exponent"] / self.scene.spec.density)
            limit = min(limit, 0.25 * self.solver.smoothing_length / (sound_speed + speed))
            if accel_max > 0.0:
                limit = min(limit, 0.25 * math.sqrt(self.solver.smoothing_length / accel_max))
            viscosity = self.material["viscosity"]
            if viscosity > 0.0:
                limit = min(limit, 0.025 * self.solver.smoothing_length ** 2 / viscosity)
        elif speed > 0.0:
            limit = min(limit, 0.4 * self.scene.spacing / speed)
        return min(remaining, limit)

    def step(self):
        """One display frame (simulation.py:155-190)."""
        if self.method == "pbf":
            steps = self.substeps
            dt = self.frame_dt / steps
            for _ in range(steps):
                self._substep(dt)
        else:
            remaining = self.frame_dt
            steps = 0
            while remaining > 1.0e-12:
                speed, accel_max = self._cfl_maxima()
                dt = self.cfl_dt(remaining, speed, accel_max)
                if dt < 1.0e-10 or steps >= 4096:
                    raise RuntimeError("CFL step cannot safely complete this frame")
                self._substep(dt)
                remaining -= dt
                steps += 1
        self.frame += 1
        self.sim_time = self.frame * self.frame_dt
        self.last_substeps = steps

    def _substep(self, dt):
        self.solver.step(self.state_0, self.state_1, None, None, dt)
        self.state_0, self.state_1 = self.state_1, self.state_0
        self.total_substeps += 1

    def metrics(self):
        """simulation.py:198-225, reduced on the device (fs_frame_metrics):
        14 doubles come back instead of every particle's x, v, rho and p.
        Minima, maxima, the speed maximum and the density percentile equal
        the reference's numpy reductions on host copies exactly; the means
        are double-precision sums (numpy sums float32 pairwise), equal to
        about 1e-7 relative."""
        s = self.state_0
        n = s.particle_q.shape[0]
        with_sph = bool(self.frame)
        rho = s.sph.rho if with_sph else None
        pressure = s.sph.pressure if with_sph and self.method == "wcsph" else None
        nr = n if with_sph else 0
        k, k1 = percentile99_ranks(nr) if nr else (0, 0)
        if self._metrics is None:
            self._metrics = torch.zeros(14, dtype=torch.float64, device=self.model.device)
        _lib.check(_lib.load().fs_frame_metrics(
            self.model.particle_grid._ctx, s.particle_q.data_ptr(), s.particle_qd.data_ptr(), n,
            rho.data_ptr() if rho is not None else None, pressure.data_ptr() if pressure is not None else None, nr, k,
            self._metrics.data_ptr(), self._stream), "frame metrics")
        o = self._metrics.tolist()
        if o[0]:
            raise RuntimeError(f"Non-finite particle state at frame {self.frame}")
        result = dict(frame=self.frame, simulation_time=self.sim_time, substeps=self.last_substeps,
                      total_substeps=self.total_substeps, finite=True, speed_max=o[3] if n else 0.0,
                      height_mean=o[4], height_min=o[5], height_max=o[6])
        if with_sph:
            if o[1]:
                raise RuntimeError("Non-finite density")
            result.update(density_mean=o[7], density_min=o[8], density_max=o[9])
            if self.method == "wcsph":
                if o[2]:
                    raise RuntimeError("Non-finite pressure")
                p99 = float(percentile99(o[10], o[11], nr))
                result.update(density_p99=p99,
                              density_compression_p99=max(0.0, p99 / self.scene.spec.density - 1.0),
                              pressure_min=o[12], pressure_max=o[13])
        return result

    def check_finite(self):
        """simulation.py:227-235: one device flag read back per frame."""
        s = self.state_0
        rho = s.sph.rho
        _lib.check(_lib.load().fs_check_finite(s.particle_q.data_ptr(), s.particle_qd.data_ptr(), s.particle_q.shape[0],
                                               rho.data_ptr(), rho.shape[0], self._invalid_state.data_ptr(),
                                               self._stream), "check finite")
        if int(self._invalid_state.item()):
            raise RuntimeError(f"Non-finite particle state at frame {self.frame}")

    def report(self):
        return dict(method=self.method, config=asdict(self.solver.config), material=self.material,
                    frame_dt=self.frame_dt, base_substeps=self.substeps,
                    time_step="fixed" if self.method == "pbf" else "CFL, complete frame",
                    solver_execution="plain launches")


__all__ = ["DamBreakSimulation", "SOLVERS", "solver_config", "material", "percentile99", "percentile99_ranks",
           "ModelBuilder", "Axis", "C"]
