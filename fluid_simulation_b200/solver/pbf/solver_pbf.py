"""Drop-in PBF solver (reference: solver/pbf/solver_pbf.py).

Same class name, config dataclass, custom attributes and ``step`` contract as
the reference ``SolverPBF``; the step runs through ``fs_pbf_substep``.  As in
the reference, one grid is built from the gravity-predicted positions and its
candidate set is reused by every later pass of the step (unless
``rebuild_grid_each_iteration``).
"""

from __future__ import annotations

import ctypes as C
import math
from dataclasses import dataclass

import torch

from ... import _lib
from ...newton_shim import Model, ModelBuilder, SolverBase, State, vec3
from .. import _common as cm


def poly6(r_norm: float, h: float) -> float:
    """get_cubic of solver_pbf.py:24-32 evaluated on the host (double)."""
    if h > 0.0 and r_norm < h:
        c = h * h * h
        return 315.0 / (64.0 * math.pi * (c * c * c)) * (h * h - r_norm * r_norm) ** 3
    return 0.0


class SolverPBF(SolverBase):
    @dataclass
    class PbfConfig:  # solver_pbf.py:521-539
        max_iterations: int = 10
        lambda_epsilon: float = 100.0
        min_neighbors_for_lambda: int = 0
        scorr_k: float = 1.0e-4
        scorr_n: float = 4.0
        scorr_q: float = 0.3
        max_delta_position: float = 0.0
        xsph_c: float = 0.01
        particle_radius: float = 0.1
        particle_length: float = 0.2
        smoothing_length_coff: float = 1.35
        bound_width: float = 10.0
        bound_height: float = 10.0
        bound_length: float = 10.0
        boundary_damping: float = 0.0
        boundary_epsilon: float = 0.0
        rebuild_grid_each_iteration: bool = False

    @classmethod
    def register_custom_attributes(cls, builder: ModelBuilder) -> None:
        """solver_pbf.py:541-628."""
        cm.register(builder,
                    [("particle_mask", int, 0), ("rest_density", float, 1000.0), ("surface_tension", float, 0.01),
                     ("viscosity", float, 0.005)],
                    [("rho", float, 0.0), ("pbf_lambda", float, 0.0), ("neighbor_count", int, 0),
                     ("delta_p", vec3, (0.0, 0.0, 0.0)), ("step_displacement", vec3, (0.0, 0.0, 0.0))])

    def __init__(self, model: Model, config: "SolverPBF.PbfConfig"):
        super().__init__(model=model)
        self.config = config
        cm.require_cuda(model, "SolverPBF")
        cm.attach_grid(model, "SolverPBF")
        n = model.particle_count
        self._particle_accel = torch.empty((n, 3), dtype=torch.float32, device=model.device)
        self._x_pred = torch.empty((n, 3), dtype=torch.float32, device=model.device)

    @property
    def smoothing_length(self) -> float:
        return self.config.particle_length * self.config.smoothing_length_coff

    def _w_delta_q(self, smoothing_length: float) -> float:
        """solver_pbf.py:671-674."""
        return poly6(float(self.config.scorr_q) * smoothing_length, smoothing_length)

    def params(self, dt: float) -> _lib.PbfParams:
        c = self.config
        h = float(self.smoothing_length)
        return _lib.PbfParams(float(dt), h, cm.particle_radius(c, self.model), float(c.bound_width),
                              float(c.bound_height), float(c.bound_length), float(c.boundary_damping),
                              float(c.boundary_epsilon), int(c.max_iterations), int(c.min_neighbors_for_lambda),
                              int(bool(c.rebuild_grid_each_iteration)), float(c.lambda_epsilon), float(c.scorr_k),
                              float(c.scorr_n), float(self._w_delta_q(h)), float(c.max_delta_position),
                              float(c.xsph_c))

    def step(self, state_in: State, state_out: State, control=None, contacts=None, dt: float = 0.0) -> None:
        """solver_pbf.py:676-954."""
        del control, contacts
        cm.copy_passthrough_state(state_in, state_out)
        model = self.model
        if model.particle_count == 0:
            return
        ctx = cm.grid_ctx(model, "SolverPBF")
        n, dev = model.particle_count, model.device
        m = cm.model_struct(model)
        si = cm.state_struct(state_in, n, dev)
        so = cm.state_struct(state_out, n, dev, need=("rho", "pbf_lambda", "neighbor_count", "delta_p"))
        p = self.params(dt)
        acc = cm.ptr(self._particle_accel, "solver._particle_accel", cols=3, n=n, device=dev)
        xp = cm.ptr(self._x_pred, "solver._x_pred", cols=3, n=n, device=dev)
        _lib.check(_lib.load().fs_pbf_substep(ctx, C.byref(m), C.byref(si), C.byref(so), C.byref(p), acc, xp,
                                              cm.stream_of(dev)), "SolverPBF.step")

    def update_contacts(self, contacts) -> None:
        del contacts
