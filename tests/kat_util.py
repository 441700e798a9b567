"""A CPU restatement of the dam-break harness loop (simulation.py:140-196) on
the oracle, for the known-answer tests of unit_test_dam_break.py."""

import math
from dataclasses import asdict

import numpy as np

import oracle
from fluid_simulation_b200.dam_break import material, solver_config


class OracleDamBreak:
    def __init__(self, scene, method, wcsph_viscosity=1.0e-6, wcsph_clamp_negative_pressure=True, gravity=None):
        self.scene = scene
        self.method = method
        self.frame_dt = 1.0 / scene.spec.fps
        self.substeps = 4
        self.material = material(method, scene, wcsph_viscosity=wcsph_viscosity)
        n = scene.count
        sph = {k: np.full(n, v, np.float32) for k, v in self.material.items()}
        sph["particle_mask"] = np.zeros(n, np.int32)
        g = scene.spec.gravity if gravity is None else gravity
        self.model = dict(particle_flags=np.ones(n, np.int32), particle_mass=np.full(n, scene.mass, np.float32),
                          particle_world=np.zeros(n, np.int32), gravity=np.array([g], np.float32),
                          particle_max_radius=scene.radius, sph=sph)
        self.cfg = asdict(solver_config(method, scene, wcsph_clamp_negative_pressure=wcsph_clamp_negative_pressure))
        self.x = scene.positions.astype(np.float32).copy()
        self.v = np.zeros_like(self.x)
        self.accel = None
        self.sph = {}
        self.total_substeps = 0
        self.dts = []
        h = self.cfg["particle_length"] * self.cfg["smoothing_length_coff"]
        self.h = h

    def substep(self, dt):
        st = dict(particle_q=self.x, particle_qd=self.v, sph={})
        step = {"wcsph": oracle.wcsph_step, "dfsph": oracle.dfsph_step, "pbf": oracle.pbf_step}[self.method]
        res = step(self.model, st, self.cfg, dt)
        out, self.accel = res[0], res[1]
        self.x, self.v, self.sph = out["particle_q"], out["particle_qd"], out["sph"]
        self.total_substeps += 1
        self.dts.append(dt)

    def step(self):
        if self.method == "pbf":
            for _ in range(self.substeps):
                self.substep(self.frame_dt / self.substeps)
            return
        remaining = self.frame_dt
        steps = 0
        while remaining > 1.0e-12:
            v2 = float((self.v.astype(np.float64) ** 2).sum(1).max())
            a2 = float((self.accel.astype(np.float64) ** 2).sum(1).max()) if (
                self.method == "wcsph" and self.total_substeps) else 0.0
            speed, accel = math.sqrt(v2), math.sqrt(a2)
            limit = self.frame_dt / self.substeps
            if self.method == "wcsph":
                c0 = math.sqrt(self.material["stiffness"] * self.material["exponent"] / self.scene.spec.density)
                limit = min(limit, 0.25 * self.h / (c0 + speed))
                if accel > 0.0:
                    limit = min(limit, 0.25 * math.sqrt(self.h / accel))
                if self.material["viscosity"] > 0.0:
                    limit = min(limit, 0.025 * self.h ** 2 / self.material["viscosity"])
            elif speed > 0.0:
                limit = min(limit, 0.4 * self.scene.spacing / speed)
            dt = min(remaining, limit)
            assert dt >= 1.0e-10 and steps < 4096
            self.substep(dt)
            remaining -= dt
            steps += 1
