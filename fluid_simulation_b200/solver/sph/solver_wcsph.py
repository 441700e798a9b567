"""Drop-in WCSPH solver (reference: solver/sph/solver_wcsph.py).

Same class name, config dataclass, custom attributes and ``step`` contract as
the reference ``SolverWCSPH``; the step runs as hand-written sm_100a kernels
through ``fs_wcsph_substep`` (grid build, density + Tait EOS, then pressure /
viscosity / cohesion forces fused with symplectic Euler and the box walls).
"""

from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import torch

from ... import _lib
from ...newton_shim import Model, ModelBuilder, SolverBase, State
from .. import _common as cm


class SolverWCSPH(SolverBase):
    @dataclass
    class SphConfig:  # solver_wcsph.py:309-318
        particle_radius: float = 0.1
        particle_length: float = 0.2
        smoothing_length_coff: float = 1.35
        bound_width: float = 10.0
        bound_height: float = 10.0
        bound_length: float = 10.0
        boundary_damping: float = -0.1
        clamp_negative_pressure: bool = True

    @classmethod
    def register_custom_attributes(cls, builder: ModelBuilder) -> None:
        """solver_wcsph.py:320-392."""
        cm.register(builder,
                    [("particle_mask", int, 0), ("rest_density", float, 1000.0), ("surface_tension", float, 0.01),
                     ("viscosity", float, 0.005), ("stiffness", float, 85000.0), ("exponent", float, 7.0)],
                    [("rho", float, 0.0), ("pressure", float, 0.0)])

    def __init__(self, model: Model, config: "SolverWCSPH.SphConfig"):
        super().__init__(model=model)
        self.config = config
        cm.require_cuda(model, "SolverWCSPH")
        cm.attach_grid(model, "SolverWCSPH")
        n = model.particle_count
        self._particle_accel = torch.empty((n, 3), dtype=torch.float32, device=model.device)

    @property
    def smoothing_length(self) -> float:
        return self.config.particle_length * self.config.smoothing_length_coff

    def params(self, dt: float) -> _lib.WcsphParams:
        c = self.config
        return _lib.WcsphParams(float(dt), float(self.smoothing_length), cm.particle_radius(c, self.model),
                                float(c.bound_width), float(c.bound_height), float(c.bound_length),
                                float(c.boundary_damping), int(bool(c.clamp_negative_pressure)))

    def step(self, state_in: State, state_out: State, control=None, contacts=None, dt: float = 0.0) -> None:
        """solver_wcsph.py:431-535."""
        del control, contacts
        cm.copy_passthrough_state(state_in, state_out)
        model = self.model
        if model.particle_count == 0:
            return
        ctx = cm.grid_ctx(model, "SolverWCSPH")
        n, dev = model.particle_count, model.device
        m = cm.model_struct(model, wcsph=True)
        si = cm.state_struct(state_in, n, dev)
        so = cm.state_struct(state_out, n, dev, need=("rho", "pressure"))
        p = self.params(dt)
        acc = cm.ptr(self._particle_accel, "solver._particle_accel", cols=3, n=n, device=dev)
        lib = _lib.load()
        _lib.check(lib.fs_wcsph_substep(ctx, C.byref(m), C.byref(si), C.byref(so), C.byref(p), acc,
                                        cm.stream_of(dev)), "SolverWCSPH.step")

    def update_contacts(self, contacts) -> None:
        del contacts
