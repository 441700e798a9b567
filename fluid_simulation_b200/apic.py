"""The particle-separation pass of the reference's APIC solver on B200.

``SolverAPIC`` (solver/apic/solver_apic.py) is a grid (FEM pressure
projection) solver; the one part of it that consumes the particle neighbour
search is ``_apply_particle_separation`` (1003-1064), run after each step to
push apart particles closer than a rest distance.  ``ParticleSeparation``
takes the same configuration fields and derives the same parameters as
``SolverAPIC.__init__`` (634-651) and that method, and runs each iteration
as a grid build plus two kernels of ``fs_apic_separation`` on the model's
device.  Its results equal the reference's bit for bit.

    sep = ParticleSeparation(model, ParticleSeparation.Config(bound_lo=..., bound_hi=...))
    sep.apply(state)          # state.particle_q updated in place
"""

from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np
import torch

from . import _lib
from .newton_shim import HashGrid


class ParticleSeparation:
    @dataclass
    class Config:  # the fields of SolverAPIC.Config that the separation pass reads (solver_apic.py:562-582)
        bound_lo: tuple = (-1.0, -1.0, 0.0)
        bound_hi: tuple = (1.0, 1.0, 2.0)
        clamp_eps: float = 1.0e-4
        wall_margin: float = -1.0        # <0 => mean particle radius
        wall_push_band: float = -1.0     # <0 => 1.5 * wall_margin
        enable_particle_separation: bool = True
        separation_rest_dist: float = -1.0  # <0 => mean particle spacing (2 * radius)
        separation_strength: float = 0.55
        separation_iterations: int = 2

    def __init__(self, model, config: "ParticleSeparation.Config"):
        self.model = model
        self.config = config
        n = int(model.particle_count)
        radii = self._radii()
        # SolverAPIC.__init__, solver_apic.py:641-650
        if n > 0 and float(config.wall_margin) < 0.0:
            self._wall_margin = float(np.mean(radii))
        elif float(config.wall_margin) < 0.0:
            self._wall_margin = float(config.clamp_eps)
        else:
            self._wall_margin = float(config.wall_margin)
        if float(config.wall_push_band) < 0.0:
            self._wall_push_band = 1.5 * self._wall_margin
        else:
            self._wall_push_band = float(config.wall_push_band)
        self._sep_hash_grid = None
        self._sep_grid_dims = None
        self._sep_delta = None

    def _radii(self) -> np.ndarray:
        r = self.model.particle_radius
        if isinstance(r, torch.Tensor):
            r = r.detach().cpu().numpy()
        r = np.asarray(r, dtype=np.float32)
        return np.full(int(self.model.particle_count), r, np.float32) if r.ndim == 0 else r

    def parameters(self) -> dict:
        """rest_dist, query_radius, strength, iterations, grid dims and the
        wall band and margin, derived as _apply_particle_separation does
        (1009-1028)."""
        c = self.config
        if float(c.separation_rest_dist) > 0.0:
            rest_dist = float(c.separation_rest_dist)
        else:
            if not hasattr(self, "_sep_rest_dist_cached"):
                self._sep_rest_dist_cached = float(2.0 * float(np.mean(self._radii())))
            rest_dist = float(self._sep_rest_dist_cached)
        query_radius = max(rest_dist, 1.0e-5)
        lo = np.asarray(c.bound_lo, dtype=np.float64)
        hi = np.asarray(c.bound_hi, dtype=np.float64)
        extent = np.maximum(hi - lo, query_radius)
        dims = np.maximum(4, np.ceil(extent / query_radius).astype(int))
        return dict(rest_dist=rest_dist, query_radius=query_radius, strength=float(c.separation_strength),
                    iterations=max(1, int(c.separation_iterations)), dims=tuple(int(d) for d in dims),
                    bound_lo=tuple(map(float, c.bound_lo)), bound_hi=tuple(map(float, c.bound_hi)),
                    wall_band=max(float(self._wall_push_band), float(self._wall_margin) * 2.0),
                    wall_margin=float(self._wall_margin))

    def apply(self, state) -> None:
        """SolverAPIC._apply_particle_separation(state): state.particle_q is
        pushed apart in place (no-op without particles or when the config
        disables separation)."""
        model = self.model
        n = int(model.particle_count)
        if n <= 0 or not bool(self.config.enable_particle_separation):
            return
        p = self.parameters()
        dev = state.particle_q.device
        if self._sep_hash_grid is None or self._sep_grid_dims != p["dims"]:
            self._sep_hash_grid = HashGrid(*p["dims"], device=dev)
            self._sep_grid_dims = p["dims"]
        self._sep_hash_grid.reserve(n)
        if self._sep_delta is None or int(self._sep_delta.shape[0]) != n:
            self._sep_delta = torch.empty((n, 3), dtype=torch.float32, device=dev)
        x = state.particle_q
        if not (x.is_contiguous() and x.dtype == torch.float32 and tuple(x.shape) == (n, 3)):
            raise ValueError("state.particle_q must be a contiguous float32 [n, 3] tensor")
        flags = model.particle_flags.to(device=dev, dtype=torch.int32).contiguous()
        sp = _lib.SeparationParams(rest_dist=p["rest_dist"], query_radius=p["query_radius"],
                                   strength=p["strength"], wall_band=p["wall_band"], wall_margin=p["wall_margin"],
                                   iterations=p["iterations"])
        sp.bound_lo[:] = p["bound_lo"]
        sp.bound_hi[:] = p["bound_hi"]
        stream = torch.cuda.current_stream(dev).cuda_stream
        _lib.check(_lib.load().fs_apic_separation(self._sep_hash_grid._ctx, x.data_ptr(), flags.data_ptr(), n,
                                                  C.byref(sp), self._sep_delta.data_ptr(), stream),
                   "ParticleSeparation.apply")

    # the reference's method name
    _apply_particle_separation = apply


__all__ = ["ParticleSeparation"]
