"""Autotuner of the neighbour-kernel launches.

The WCSPH / DFSPH / PBF neighbour passes are bound by instruction issue and
gather latency, and how many particles a launch keeps in flight decides how
much of that latency is hidden.  Three knobs of a context (``fs_tuning``)
move that balance:

  block_size            threads per block (64, 128, 256)
  particles_per_thread  cell-sorted particles each thread walks (1, 2, 4)
  cell_ratio            grid cell width / h (WCSPH only: 1 or 0.5)

(a fourth, ``list_skin``, the skin of PBF's first density lists that lets
the first lambda pass skip its grid scan, changes no result either and
keeps its default here).

``autotune(solver, state, dt)`` times a few substeps from one saved state
under every candidate (each candidate starts from the same state, so DFSPH
runs the same iterations), keeps the fastest on the solver's context and
returns the measurements.  block_size and particles_per_thread change no
result; cell_ratio 0.5 changes the order of WCSPH's sums (not its neighbour
set), so it is offered for WCSPH only and only on hash-grid contexts (PBF
queries its grid from moved positions and DFSPH counts candidates: the cell
width is part of their results).
"""

from __future__ import annotations

import ctypes as C
import itertools
import statistics
from dataclasses import asdict, dataclass

from . import _lib

BLOCK_SIZES = (64, 128, 256)
PARTICLES_PER_THREAD = (1, 2, 4)
DEFAULT = (128, 1, 1.0)


@dataclass(frozen=True)
class Tuning:
    block_size: int = 128
    particles_per_thread: int = 1
    cell_ratio: float = 1.0
    list_skin: float = 0.02


def get_tuning(ctx) -> Tuning:
    t = _lib.Tuning()
    _lib.check(_lib.load().fs_context_get_tuning(ctx, C.byref(t)), "fs_context_get_tuning")
    f32 = lambda v: float(f"{v:.7g}")  # the decimal a float32 field was set from
    return Tuning(int(t.block_size), int(t.particles_per_thread), f32(t.cell_ratio), f32(t.list_skin))


def set_tuning(ctx, tuning: Tuning) -> None:
    t = _lib.Tuning(int(tuning.block_size), int(tuning.particles_per_thread), float(tuning.cell_ratio),
                    float(tuning.list_skin))
    _lib.check(_lib.load().fs_context_set_tuning(ctx, C.byref(t)), "fs_context_set_tuning")


def candidates(solver_kind: str, batched: bool = False):
    """Every tuning worth timing for a solver ('wcsph', 'dfsph', 'pbf'),
    the default first (it wins ties)."""
    ratios = (1.0, 0.5) if solver_kind == "wcsph" and not batched else (1.0,)
    out = [Tuning(*DEFAULT)]
    for b, p, r in itertools.product(BLOCK_SIZES, PARTICLES_PER_THREAD, ratios):
        t = Tuning(b, p, r)
        if t not in out:
            out.append(t)
    return out


def choose(times: dict) -> Tuning:
    """The fastest candidate; among equal times the first listed."""
    best = None
    for t, ms in times.items():
        if best is None or ms < times[best]:
            best = t
    return best


def _kind(solver) -> str:
    return {"SolverWCSPH": "wcsph", "SolverDFSPH": "dfsph", "SolverPBF": "pbf"}[type(solver).__name__]


def autotune(solver, state, dt: float, steps: int = 3, repeats: int = 2, timer=None) -> dict:
    """Tune ``solver``'s context on ``steps`` substeps from ``state`` (left
    unchanged).  ``timer(tuning) -> ms`` replaces the CUDA-event timing
    (tests).  Returns {"chosen": Tuning, "times_ms": {Tuning: ms}}."""
    from .newton_shim import WorldGrid

    model = solver.model
    grid = model.particle_grid
    ctx = grid._ctx
    cands = candidates(_kind(solver), batched=isinstance(grid, WorldGrid))
    if timer is None:
        timer = _device_timer(solver, state, dt, steps, repeats)
    times = {}
    for t in cands:
        set_tuning(ctx, t)
        times[t] = float(timer(t))
    best = choose(times)
    set_tuning(ctx, best)
    return {"chosen": best, "times_ms": times}


def _device_timer(solver, state, dt, steps, repeats):
    import torch

    model = solver.model
    a, b = model.state(), model.state()
    names = [k for k in vars(state.sph)] if hasattr(state, "sph") else []

    def restore(dst):
        dst.particle_q.copy_(state.particle_q)
        dst.particle_qd.copy_(state.particle_qd)
        for k in names:
            getattr(dst.sph, k).copy_(getattr(state.sph, k))

    def timer(_tuning):
        runs = []
        for r in range(repeats + 1):
            restore(a)
            x, y = a, b
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            for _ in range(steps):
                solver.step(x, y, None, None, dt)
                x, y = y, x
            e1.record()
            e1.synchronize()
            if r:  # the first run warms up
                runs.append(e0.elapsed_time(e1) / steps)
        return statistics.median(runs)

    return timer


def describe(result: dict) -> dict:
    """JSON-ready summary of an autotune() result."""
    times = sorted(result["times_ms"].items(), key=lambda kv: kv[1])
    return dict(chosen=asdict(result["chosen"]),
                ms_per_substep={f"{t.block_size}x{t.particles_per_thread}x{t.cell_ratio:g}": round(ms, 4)
                                for t, ms in times},
                default_ms=round(result["times_ms"][Tuning(*DEFAULT)], 4))
