"""Dam-break scenes and the synthetic benchmark inputs.

``make_scene`` restates the reference scene generator
(examples/dam_break/scene.py:9-123: endpoint lattice, per-axis resolution
rounding, float32 positions); its output is pinned bit-for-bit by the
SHA-256 digests of the reference's own output recorded in
``tests/golden/scenes.json``.  The other generators build the seeded
synthetic inputs of the benchmark workloads.
"""

from __future__ import annotations

import hashlib
from dataclasses import asdict, dataclass

import numpy as np


@dataclass(frozen=True)
class SceneSpec:  # scene.py:9-19
    bound_lo: tuple = (-1.20, -0.28, 0.0)
    bound_hi: tuple = (1.20, 0.28, 1.20)
    fill_x_frac: float = 0.30
    fill_z_frac: float = 0.72
    margin: float = 0.03
    density: float = 1000.0
    gravity: tuple = (0.0, 0.0, -10.0)
    fps: float = 60.0
    target_count: int = 400000


DEFAULT_SPEC = SceneSpec()


def spawn_particle_block(lo, hi, res, density: float = 1000.0):
    """scene.py:25-41: endpoint lattice with res[k] points on axis k."""
    axes = [np.linspace(lo[k], hi[k], res[k]) for k in range(3)]
    grid = np.meshgrid(*axes, indexing="ij")
    positions = np.stack([g.ravel() for g in grid], axis=1).astype(np.float32)
    spacing = float(min((hi[k] - lo[k]) / max(res[k] - 1, 1) for k in range(3)))
    volume = spacing ** 3
    return positions, density * volume, 0.5 * spacing, volume, spacing


def spawn_wave_tank(tank_lo, tank_hi, target_count=400000, fill_x_frac=0.30, fill_z_frac=0.70, margin=0.03,
                    density=1000.0):
    """scene.py:44-75: water column in the low-x corner of the tank."""
    if target_count < 1:
        raise ValueError("Target particle count must be positive")
    lo = np.asarray(tank_lo, dtype=np.float32)
    hi = np.asarray(tank_hi, dtype=np.float32)
    ext = hi - lo
    w_lo = np.array([lo[0] + margin, lo[1] + margin, lo[2] + margin], dtype=np.float32)
    w_hi = np.array([lo[0] + margin + fill_x_frac * max(ext[0] - 2.0 * margin, 1.0e-3),
                     hi[1] - margin,
                     lo[2] + margin + fill_z_frac * max(ext[2] - 2.0 * margin, 1.0e-3)], dtype=np.float32)
    w_ext = np.maximum(w_hi - w_lo, 1.0e-3)
    spacing = float((float(np.prod(w_ext)) / max(target_count, 1)) ** (1.0 / 3.0))
    res = tuple(max(2, int(round(e / spacing))) for e in w_ext)
    return spawn_particle_block(tuple(w_lo), tuple(w_hi), res, density=density)


@dataclass
class ParticleScene:
    spec: SceneSpec
    positions: np.ndarray
    mass: float
    radius: float
    volume: float
    spacing: float

    @property
    def count(self):
        return len(self.positions)

    @property
    def rest_volume(self):
        return self.count * self.mass / self.spec.density

    @property
    def ideal_height(self):
        lo, hi = self.spec.bound_lo, self.spec.bound_hi
        return self.rest_volume / ((hi[0] - lo[0]) * (hi[1] - lo[1]))

    def report(self):
        return {**asdict(self.spec), "actual_count": self.count,
                "lattice_resolution": [len(np.unique(self.positions[:, i])) for i in range(3)],
                "particle_spacing": self.spacing, "particle_radius": self.radius, "particle_volume": self.volume,
                "particle_mass": self.mass, "rest_volume": self.rest_volume, "ideal_flat_height": self.ideal_height,
                "initial_position_sha256": hashlib.sha256(self.positions.tobytes()).hexdigest(),
                "water_lo": self.positions.min(axis=0).tolist(), "water_hi": self.positions.max(axis=0).tolist(),
                "units": "meters, kilograms, seconds; Z up"}


def make_scene(particle_count=DEFAULT_SPEC.target_count) -> ParticleScene:
    """scene.py:118-123."""
    spec = SceneSpec(target_count=int(particle_count))
    return ParticleScene(spec, *spawn_wave_tank(spec.bound_lo, spec.bound_hi, spec.target_count, spec.fill_x_frac,
                                                spec.fill_z_frac, spec.margin, spec.density))


# ------------------------------------------------------ synthetic inputs ----
def jittered_column(target=10000, seed=0, lo=(-1.2, -0.28, 0.0), hi=(-0.6, 0.28, 0.6), jitter=0.01):
    """Cubic lattice filling the box [lo, hi] with about ``target`` particles,
    jittered by U(-jitter, jitter) x spacing (numpy default_rng(seed))."""
    lo = np.asarray(lo, np.float64)
    hi = np.asarray(hi, np.float64)
    ext = hi - lo
    spacing = float((np.prod(ext) / target) ** (1.0 / 3.0))
    res = [max(1, int(round(e / spacing))) for e in ext]
    axes = [lo[k] + (np.arange(res[k]) + 0.5) * (ext[k] / res[k]) for k in range(3)]
    g = np.meshgrid(*axes, indexing="ij")
    x = np.stack([a.ravel() for a in g], 1)
    rng = np.random.default_rng(seed)
    x += rng.uniform(-jitter, jitter, x.shape) * spacing
    return x.astype(np.float32), spacing


def stress_lattice(cells=128, box=1.6, seed_x=0, seed_v=1, sigma_v=0.2, jitter=0.01, bcc=True):
    """Neighbour-search stress input: a jittered cubic lattice filling the
    box [-box/2, box/2]^2 x [0, box].  With ``bcc`` (default) every cubic cell
    of side a = box / cells holds a corner and a body-centre particle, so
    2 * 128^3 = 4,194,304 particles fill a 1.6 m cube at the rest spacing
    d = a / 2^(1/3) (9.92 mm; h = 2 d gives ~33 neighbours).  Jitter is
    U(-jitter, jitter) x d (default_rng(seed_x)); v ~ N(0, sigma_v) per
    component (default_rng(seed_v)).  Returns (x, v, d)."""
    a = box / cells
    c = (np.arange(cells, dtype=np.float64) + 0.25) * a
    g = np.meshgrid(c - 0.5 * box, c - 0.5 * box, c, indexing="ij")
    x = np.stack([t.ravel() for t in g], 1)
    if bcc:
        x = np.concatenate([x, x + 0.5 * a], 0)
    d = a / (2.0 ** (1.0 / 3.0)) if bcc else a
    x += np.random.default_rng(seed_x).uniform(-jitter, jitter, x.shape) * d
    v = np.random.default_rng(seed_v).normal(0.0, sigma_v, x.shape)
    return x.astype(np.float32), v.astype(np.float32), d
