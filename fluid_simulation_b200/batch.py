"""Batches of independent dam-break scenes that advance in one model.

Each scene is one Newton world (``Model.particle_world``): its own tank
[-W, W] x [-H, H] x [0, 2L] with the reference dam-break proportions
(W : H : L = 1.2 : 0.28 : 0.6, examples/dam_break/simulation.py:86-92) scaled
to the scene, its own water column (a fraction of the tank along x, full
width, height L, as the reference column x in [-1.2, -0.6], z in [0, 0.6]),
and its own stiffness and viscosity.  All scenes share the particle spacing,
hence h, mass and dt, so one solver config steps them all.  Scenes overlap in
space (every tank starts at the origin); the segmented grid
(``newton_shim.WorldGrid``) keeps them apart.

``make_batch`` draws the scene set from one seed:
  N_s = exp(U(ln n_lo, ln n_hi))  particles of scene s (before lattice rounding)
  f_s ~ U(0.2, 0.6)              column length / tank length along x
  k_s, m_s ~ U(0.8, 1.2)         stiffness and viscosity factors
then fills each column with a cell-centred cubic lattice at ``spacing``,
jittered by U(-1 %, 1 %) of the spacing from default_rng((seed, s)).
"""

from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

from . import snapshot

# reference dam-break tank proportions and material (simulation.py:86-132)
TANK = (1.2, 0.28, 0.6)
REST_DENSITY = 1000.0
STIFFNESS = 2.5e5
VISCOSITY = 1.0e-6
EXPONENT = 7.0
GRAVITY = (0.0, 0.0, -10.0)


@dataclass
class Scene:
    count: int
    walls: tuple          # (bound_width, bound_height, bound_length)
    column_fraction: float
    stiffness: float
    viscosity: float
    x: np.ndarray         # [count, 3] float32


@dataclass
class Batch:
    spacing: float
    scenes: list = field(default_factory=list)

    # shared material / solver scalars ------------------------------------
    @property
    def h(self) -> float:
        return 2.0 * self.spacing

    @property
    def mass(self) -> float:
        return REST_DENSITY * self.spacing ** 3

    @property
    def radius(self) -> float:
        return 0.5 * self.spacing

    # concatenated arrays -------------------------------------------------
    @property
    def counts(self) -> np.ndarray:
        return np.array([s.count for s in self.scenes], np.int64)

    @property
    def starts(self) -> np.ndarray:
        return np.concatenate([[0], np.cumsum(self.counts)])

    @property
    def total(self) -> int:
        return int(self.counts.sum())

    def positions(self) -> np.ndarray:
        return np.concatenate([s.x for s in self.scenes]).astype(np.float32)

    def world(self) -> np.ndarray:
        return np.repeat(np.arange(len(self.scenes), dtype=np.int32), self.counts)

    def per_particle(self, name: str) -> np.ndarray:
        return np.repeat(np.array([getattr(s, name) for s in self.scenes], np.float32), self.counts)

    def boxes(self, h: float | None = None, margin: int = 1):
        """WorldGrid boxes: the cells int(x / h) (truncating, float32 as the
        device computes them) that the tank of each scene spans, widened by
        ``margin`` cells on every side.  The margin holds particles that a
        substep carries past a wall before the walls act: DFSPH builds its
        second grid from positions integrated with v* and clamps them only
        at the end of the substep, so a particle can lie up to |v*| dt
        outside its tank there (the harness's substep rule keeps that under
        0.4 spacing = 0.2 h).  With every particle inside its box, each
        world's cells, their contents and order equal those of the plain
        hash grid of that scene alone (the grid clamps a particle beyond the
        box into the edge cell, which changes DFSPH's candidate counts)."""
        h = self.h if h is None else h
        inv = np.float32(1.0) / np.float32(h)
        out = []
        for s in self.scenes:
            w, hh, l = s.walls
            lo = [int(np.float32(v) * inv) - margin for v in (-w, -hh, 0.0)]
            hi = [int(np.float32(v) * inv) + margin for v in (w, hh, 2.0 * l)]
            out.append((tuple(lo), tuple(b - a + 1 for a, b in zip(lo, hi)), s.walls))
        return out

    def attributes(self, wcsph: bool = True) -> dict:
        n = self.total
        a = dict(particle_mask=0, rest_density=np.full(n, REST_DENSITY, np.float32),
                 surface_tension=np.zeros(n, np.float32), viscosity=self.per_particle("viscosity"))
        if wcsph:
            a.update(stiffness=self.per_particle("stiffness"), exponent=np.full(n, EXPONENT, np.float32))
        return a


def scene_column(count_target: int, fraction: float, spacing: float, rng) -> tuple:
    """Tank walls and jittered lattice of one scene."""
    a = (count_target * spacing ** 3 / (4.0 * TANK[0] * TANK[1] * TANK[2] * fraction)) ** (1.0 / 3.0)
    w, hh, l = (TANK[0] * a, TANK[1] * a, TANK[2] * a)
    lo = np.array([-w, -hh, 0.0])
    ext = np.array([2.0 * w * fraction, 2.0 * hh, l])
    res = [max(1, int(round(e / spacing))) for e in ext]
    axes = [lo[k] + (np.arange(res[k]) + 0.5) * spacing for k in range(3)]
    g = np.meshgrid(*axes, indexing="ij")
    x = np.stack([t.ravel() for t in g], 1)
    x += rng.uniform(-0.01, 0.01, x.shape) * spacing
    # the lattice may overhang the rounded column by < spacing / 2: keep it in the tank
    x[:, 0] = np.clip(x[:, 0], -w, w)
    x[:, 1] = np.clip(x[:, 1], -hh, hh)
    return (float(w), float(hh), float(l)), x.astype(np.float32)


def make_batch(n_scenes: int = 256, seed: int = 3, n_lo: int = 2000, n_hi: int = 100000,
               spacing: float = 0.01) -> Batch:
    rng = np.random.default_rng(seed)
    counts = np.exp(rng.uniform(np.log(n_lo), np.log(n_hi), n_scenes))
    frac = rng.uniform(0.2, 0.6, n_scenes)
    kf = rng.uniform(0.8, 1.2, n_scenes)
    mf = rng.uniform(0.8, 1.2, n_scenes)
    b = Batch(spacing=float(spacing))
    for s in range(n_scenes):
        walls, x = scene_column(float(counts[s]), float(frac[s]), spacing, np.random.default_rng((seed, s)))
        b.scenes.append(Scene(len(x), walls, float(frac[s]), float(STIFFNESS * kf[s]), float(VISCOSITY * mf[s]), x))
    return b


def batched_model(batch: Batch, solver_cls, device="cuda:0", v=None):
    """Model + WorldGrid of the whole batch (one world per scene)."""
    from .newton_shim import WorldGrid, model_from_arrays

    x = batch.positions()
    m = model_from_arrays(x, np.zeros_like(x) if v is None else v, batch.mass, device=device,
                          world=batch.world(), gravity=[GRAVITY] * len(batch.scenes), radius=batch.radius,
                          attributes=batch.attributes(wcsph=solver_cls.__name__ == "SolverWCSPH"),
                          solver_cls=solver_cls)
    m.particle_grid = WorldGrid(batch.boxes(), device=device)
    m.particle_grid.reserve(m.particle_count)
    return m


def scene_model(batch: Batch, k: int, solver_cls, device="cuda:0", v=None):
    """Model of scene k alone (plain hash grid), for serial runs and parity."""
    from .newton_shim import model_from_arrays

    s = batch.scenes[k]
    n = s.count
    attrs = dict(particle_mask=0, rest_density=REST_DENSITY, surface_tension=0.0, viscosity=s.viscosity)
    if solver_cls.__name__ == "SolverWCSPH":
        attrs.update(stiffness=s.stiffness, exponent=EXPONENT)
    return model_from_arrays(s.x, np.zeros_like(s.x) if v is None else v, batch.mass, device=device,
                             world=np.zeros(n, np.int32), gravity=[GRAVITY], radius=batch.radius, attributes=attrs,
                             solver_cls=solver_cls)


# ------------------------------------------------------------ on disk ----
def scene_table(batch: Batch) -> dict:
    """The batch's per-scene parameters as ``scene_*`` arrays of a snapshot."""
    sc = batch.scenes
    return dict(scene_count=np.array([s.count for s in sc], np.int64),
                scene_walls=np.array([s.walls for s in sc], np.float64).reshape(-1, 3),
                scene_column_fraction=np.array([s.column_fraction for s in sc], np.float64),
                scene_stiffness=np.array([s.stiffness for s in sc], np.float64),
                scene_viscosity=np.array([s.viscosity for s in sc], np.float64),
                scene_sha256=np.array([snapshot.positions_sha256(s.x) for s in sc]))


def save_batch(path, batch: Batch, v=None, **meta) -> dict:
    """Write a batch (its scenes' initial positions, optional velocities and
    per-scene table) as a snapshot: the initial digest covers the whole
    batch's positions, and ``scene_sha256`` each scene's own."""
    x = batch.positions()
    v = np.zeros_like(x) if v is None else v
    return snapshot.save(path, x, v, None, batch.world(), initial_positions=x, extra_arrays=scene_table(batch),
                         kind="batch", spacing=float(batch.spacing), scenes=len(batch.scenes), **meta)


def save_batch_state(path, batch: Batch, model, state, **meta) -> dict:
    """Snapshot of a batched model's state (a later frame) with the batch's
    scene table and the digest of its initial positions."""
    return snapshot.save_state(path, model, state, initial_positions=batch.positions(),
                               extra_arrays=scene_table(batch), kind="batch_state", spacing=float(batch.spacing),
                               scenes=len(batch.scenes), **meta)


def load_batch(path) -> tuple:
    """(Batch, Snapshot) from a file written by ``save_batch``; every
    scene's positions are checked against its recorded digest."""
    snap = snapshot.load(path)
    if snap.meta.get("kind") != "batch":
        raise ValueError(f"{path}: not a batch definition (kind {snap.meta.get('kind')!r})")
    a = snap.arrays
    counts = a["scene_count"]
    starts = np.concatenate([[0], np.cumsum(counts)])
    b = Batch(spacing=float(snap.meta["spacing"]))
    for k in range(len(counts)):
        x = np.ascontiguousarray(snap.particle_q[starts[k]:starts[k + 1]])
        if snapshot.positions_sha256(x) != str(a["scene_sha256"][k]):
            raise ValueError(f"{path}: scene {k} positions do not match their digest")
        b.scenes.append(Scene(count=int(counts[k]), walls=tuple(float(w) for w in a["scene_walls"][k]),
                              column_fraction=float(a["scene_column_fraction"][k]),
                              stiffness=float(a["scene_stiffness"][k]), viscosity=float(a["scene_viscosity"][k]),
                              x=x))
    if not snap.matches(b.positions()):
        raise ValueError(f"{path}: batch positions do not match initial_position_sha256")
    return b, snap


def shard_scenes(counts, world_size: int) -> list:
    """Scenes per rank for a batched run on several GPUs: scenes are
    independent, so ranks share no particles and exchange nothing.  Greedy
    longest-first assignment to the least-loaded rank balances the particle
    counts (within the largest scene of the mean)."""
    counts = np.asarray(counts, np.int64)
    load = np.zeros(world_size, np.int64)
    out = [[] for _ in range(world_size)]
    for s in np.argsort(-counts, kind="stable"):
        r = int(np.argmin(load))
        out[r].append(int(s))
        load[r] += counts[s]
    return [sorted(o) for o in out]


def sub_batch(batch: Batch, scenes) -> Batch:
    return Batch(spacing=batch.spacing, scenes=[batch.scenes[k] for k in scenes])
