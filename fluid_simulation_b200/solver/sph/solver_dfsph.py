"""Drop-in DFSPH solver (reference: solver/sph/solver_dfsph.py).

Same class name, config dataclass, custom attributes and ``step`` contract as
the reference ``SolverDFSPH``.  The reference reads each solver iteration's
residual back to the host (solver_dfsph.py:733, 849); here the residual and
the break test run on the device (``fs_dfsph_substep``), so a step issues no
host synchronisation and takes the same iteration decisions.
``last_iterations()`` reads the decisions back on demand.  On a batched model
(``newton_shim.WorldGrid``) each world takes its own decisions, as its scene
would alone; ``last_world_iterations()`` reads them per world.
"""

from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import torch

from ... import _lib
from ...newton_shim import Model, ModelBuilder, SolverBase, State, vec3
from .. import _common as cm

_STATE = ("rho", "factor", "rho_star", "d_rho_dt", "kappa", "kappa_v", "neighbor_count", "v_star")


class SolverDFSPH(SolverBase):
    @dataclass
    class SphConfig:  # solver_dfsph.py:446-463
        max_rho_iterations: int = 2
        max_vel_iterations: int = 1
        warm_start: bool = True
        eta_density: float = 1.0e-1
        eta_divergence: float = 1.0e-4
        max_kappa: float = 1.0e4
        max_kappa_v: float = 1.0e6
        min_neighbors_for_factor: int = 15
        particle_radius: float = 0.1
        particle_length: float = 0.2
        smoothing_length_coff: float = 1.35
        bound_width: float = 10.0
        bound_height: float = 10.0
        bound_length: float = 10.0
        boundary_damping: float = -0.1
        voxel_size: float = 0.3

    @classmethod
    def register_custom_attributes(cls, builder: ModelBuilder) -> None:
        """solver_dfsph.py:465-535."""
        cm.register(builder,
                    [("particle_mask", int, 0), ("rest_density", float, 1000.0), ("surface_tension", float, 0.01),
                     ("viscosity", float, 0.005)],
                    [("rho", float, 0.0), ("factor", float, 0.0), ("rho_star", float, 0.0), ("d_rho_dt", float, 0.0),
                     ("kappa", float, 0.0), ("kappa_v", float, 0.0), ("neighbor_count", int, 0),
                     ("v_star", vec3, (0.0, 0.0, 0.0))])

    def __init__(self, model: Model, config: "SolverDFSPH.SphConfig"):
        super().__init__(model=model)
        self.config = config
        cm.require_cuda(model, "SolverDFSPH")
        cm.attach_grid(model, "SolverDFSPH")
        self._particle_accel = torch.empty((model.particle_count, 3), dtype=torch.float32, device=model.device)

    @property
    def smoothing_length(self) -> float:
        return self.config.particle_length * self.config.smoothing_length_coff

    def params(self, dt: float) -> _lib.DfsphParams:
        c = self.config
        return _lib.DfsphParams(float(dt), float(self.smoothing_length), cm.particle_radius(c, self.model),
                                float(c.bound_width), float(c.bound_height), float(c.bound_length),
                                float(c.boundary_damping), int(c.max_rho_iterations), int(c.max_vel_iterations),
                                int(bool(c.warm_start)), int(c.min_neighbors_for_factor), float(c.eta_density),
                                float(c.eta_divergence), float(c.max_kappa), float(c.max_kappa_v))

    def step(self, state_in: State, state_out: State, control=None, contacts=None, dt: float = 0.0) -> None:
        """solver_dfsph.py:598-898."""
        del control, contacts
        cm.copy_passthrough_state(state_in, state_out)
        model = self.model
        if model.particle_count == 0:
            return
        ctx = cm.grid_ctx(model, "SolverDFSPH")
        n, dev = model.particle_count, model.device
        m = cm.model_struct(model)
        warm = bool(self.config.warm_start)
        si = cm.state_struct(state_in, n, dev, need=("kappa", "kappa_v") if warm else ())
        so = cm.state_struct(state_out, n, dev, need=_STATE)
        p = self.params(dt)
        acc = cm.ptr(self._particle_accel, "solver._particle_accel", cols=3, n=n, device=dev)
        _lib.check(_lib.load().fs_dfsph_substep(ctx, C.byref(m), C.byref(si), C.byref(so), C.byref(p), acc,
                                                cm.stream_of(dev)), "SolverDFSPH.step")

    def last_iterations(self) -> dict:
        """Iteration counts and residuals of the last step (synchronises)."""
        info = _lib.DfsphInfo()
        _lib.check(_lib.load().fs_dfsph_info_read(cm.grid_ctx(self.model, "SolverDFSPH"), C.byref(info)),
                   "SolverDFSPH.last_iterations")
        return dict(rho_iterations=info.rho_iterations, vel_iterations=info.vel_iterations,
                    density_residual=info.density_residual, divergence_residual=info.divergence_residual)

    def last_world_iterations(self) -> list:
        """Per-world iteration counts and residuals of the last step of a
        batched model (synchronises); one dict per world."""
        ctx = cm.grid_ctx(self.model, "SolverDFSPH")
        lib = _lib.load()
        nw = int(lib.fs_context_worlds(ctx))
        if nw <= 0:
            raise RuntimeError("SolverDFSPH.last_world_iterations: the model's grid is not a batched WorldGrid")
        infos = (_lib.DfsphInfo * nw)()
        _lib.check(lib.fs_dfsph_info_worlds(ctx, infos, nw), "SolverDFSPH.last_world_iterations")
        return [dict(rho_iterations=i.rho_iterations, vel_iterations=i.vel_iterations,
                     density_residual=i.density_residual, divergence_residual=i.divergence_residual) for i in infos]

    def update_contacts(self, contacts) -> None:
        del contacts
