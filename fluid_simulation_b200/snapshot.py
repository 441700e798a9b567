"""On-disk particle snapshots (one ``.npz`` file per frame or batch).

The reference pins a run to its initial condition by the SHA-256 of the
initial float32 positions: ``scene.report()["initial_position_sha256"]``
(examples/dam_break/scene.py:111), which its USD output also carries as
layer data (examples/dam_break/surface.py:73).  A snapshot here stores the
per-particle state of a frame next to that digest, so a file can be checked
against the scene it came from and a run resumed from it:

  particle_q      [n, 3] float32   positions
  particle_qd     [n, 3] float32   velocities
  rho             [n]    float32   density (when the solver state has one)
  particle_world  [n]    int32     world of each particle (batched models)
  scene_*                          a batch's scene table (``save_batch``)
  meta            JSON string: initial_position_sha256, frame, sim_time,
                  solver, particle_count and any caller keys

Everything is little-endian numpy; ``np.load(path)`` reads it without this
package.
"""

from __future__ import annotations

import hashlib
import json
from dataclasses import dataclass, field

import numpy as np

FORMAT = "fluid_simulation_b200.snapshot/1"


def positions_sha256(x) -> str:
    """SHA-256 of float32 C-order positions: the digest of scene.report()."""
    return hashlib.sha256(np.ascontiguousarray(np.asarray(x, dtype=np.float32)).tobytes()).hexdigest()


@dataclass
class Snapshot:
    particle_q: np.ndarray
    particle_qd: np.ndarray
    rho: np.ndarray | None = None
    particle_world: np.ndarray | None = None
    meta: dict = field(default_factory=dict)
    arrays: dict = field(default_factory=dict)  # extra arrays (a batch's scene_* table)

    @property
    def count(self) -> int:
        return int(self.particle_q.shape[0])

    def matches(self, initial_positions) -> bool:
        """Whether this snapshot was taken from a run started at these positions."""
        return self.meta.get("initial_position_sha256") == positions_sha256(initial_positions)


def _host(a, dtype, shape_tail):
    if a is None:
        return None
    if hasattr(a, "detach"):  # torch tensor (device or host)
        a = a.detach().cpu().numpy()
    a = np.ascontiguousarray(np.asarray(a, dtype=dtype))
    if a.shape[1:] != shape_tail:
        raise ValueError(f"snapshot array of shape {a.shape}, expected [n{', ' if shape_tail else ''}"
                         f"{', '.join(map(str, shape_tail))}]")
    return a


def save(path, particle_q, particle_qd, rho=None, particle_world=None, *, initial_positions=None,
         initial_position_sha256: str | None = None, extra_arrays: dict | None = None, **meta) -> dict:
    """Write one snapshot; returns its metadata.  Arrays may be numpy arrays
    or torch tensors (copied to the host).  Give the run's initial positions
    or their digest."""
    x = _host(particle_q, np.float32, (3,))
    v = _host(particle_qd, np.float32, (3,))
    n = x.shape[0]
    if v.shape[0] != n:
        raise ValueError("particle_q and particle_qd differ in length")
    arrays = dict(particle_q=x, particle_qd=v)
    if rho is not None:
        arrays["rho"] = _host(rho, np.float32, ())
    if particle_world is not None:
        arrays["particle_world"] = _host(particle_world, np.int32, ())
    for k, a in arrays.items():
        if a.shape[0] != n:
            raise ValueError(f"{k} has {a.shape[0]} rows, expected {n}")
    if initial_positions is not None:
        digest = positions_sha256(initial_positions)
        if initial_position_sha256 is not None and initial_position_sha256 != digest:
            raise ValueError("initial_positions do not match initial_position_sha256")
        initial_position_sha256 = digest
    if initial_position_sha256 is None:
        raise ValueError("a snapshot needs the run's initial positions or their SHA-256")
    info = dict(format=FORMAT, initial_position_sha256=initial_position_sha256, particle_count=int(n), **meta)
    for k, a in (extra_arrays or {}).items():
        if k in arrays or k == "meta":
            raise ValueError(f"extra array name {k!r} is reserved")
        arrays[k] = np.asarray(a)
    with open(path, "wb") as f:  # np.savez would append .npz to a path without it
        np.savez(f, meta=np.array(json.dumps(info, sort_keys=True)), **arrays)
    return info


def load(path) -> Snapshot:
    with np.load(path, allow_pickle=False) as z:
        meta = json.loads(str(z["meta"]))
        if meta.get("format") != FORMAT:
            raise ValueError(f"{path}: not a {FORMAT} file (format {meta.get('format')!r})")
        known = ("meta", "particle_q", "particle_qd", "rho", "particle_world")
        return Snapshot(particle_q=z["particle_q"], particle_qd=z["particle_qd"],
                        rho=z["rho"] if "rho" in z.files else None,
                        particle_world=z["particle_world"] if "particle_world" in z.files else None, meta=meta,
                        arrays={k: z[k] for k in z.files if k not in known})


# -------------------------------------------------------------- states ----
def save_state(path, model, state, *, initial_positions=None, initial_position_sha256=None, extra_arrays=None,
               **meta) -> dict:
    """Snapshot of a solver State (device tensors) of ``model``; models of
    several worlds also store ``particle_world``."""
    rho = getattr(getattr(state, "sph", None), "rho", None)
    world = getattr(model, "particle_world", None)
    several = world is not None and int(model.gravity.shape[0]) > 1
    return save(path, state.particle_q, state.particle_qd, rho, world if several else None,
                initial_positions=initial_positions, initial_position_sha256=initial_position_sha256,
                extra_arrays=extra_arrays, **meta)


def restore_state(snap: Snapshot, state) -> None:
    """Copy a snapshot's positions and velocities (and density, when both
    have one) into a State of the same particle count."""
    import torch
    if snap.count != state.particle_q.shape[0]:
        raise ValueError(f"snapshot of {snap.count} particles, state of {state.particle_q.shape[0]}")
    state.particle_q.copy_(torch.as_tensor(snap.particle_q))
    state.particle_qd.copy_(torch.as_tensor(snap.particle_qd))
    rho = getattr(getattr(state, "sph", None), "rho", None)
    if snap.rho is not None and rho is not None:
        rho.copy_(torch.as_tensor(snap.rho))


def save_simulation(path, sim) -> dict:
    """Snapshot of a DamBreakSimulation's current frame, tagged with its
    scene's digest, frame, time and solver.  The solver's last acceleration
    is kept too (``particle_accel``): the WCSPH substep rule reads it, so a
    resumed run takes the same substeps."""
    return save_state(path, sim.model, sim.state_0, initial_position_sha256=sim.scene.report()["initial_position_sha256"],
                      extra_arrays=dict(particle_accel=sim.solver._particle_accel.detach().cpu().numpy()),
                      frame=int(sim.frame), sim_time=float(sim.sim_time), solver=sim.method,
                      total_substeps=int(sim.total_substeps))


def restore_simulation(path, sim) -> Snapshot:
    """Resume a DamBreakSimulation from a snapshot of the same scene and
    solver: the following frames equal those of the uninterrupted run."""
    import torch
    snap = load(path)
    want = sim.scene.report()["initial_position_sha256"]
    if snap.meta.get("initial_position_sha256") != want:
        raise ValueError("snapshot was taken from another scene (initial_position_sha256 differs)")
    if snap.meta.get("solver", sim.method) != sim.method:
        raise ValueError(f"snapshot of a {snap.meta.get('solver')} run, simulation runs {sim.method}")
    restore_state(snap, sim.state_0)
    if "particle_accel" in snap.arrays:
        sim.solver._particle_accel.copy_(torch.as_tensor(snap.arrays["particle_accel"]))
    sim.frame = int(snap.meta.get("frame", 0))
    sim.sim_time = float(snap.meta.get("sim_time", sim.frame * sim.frame_dt))
    sim.total_substeps = int(snap.meta.get("total_substeps", 0))
    return snap


__all__ = ["FORMAT", "Snapshot", "positions_sha256", "save", "load", "save_state", "restore_state",
           "save_simulation", "restore_simulation"]
