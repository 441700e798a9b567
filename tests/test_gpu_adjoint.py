"""Gradients of the hand-written WCSPH adjoint (fs_wcsph_substep_adjoint
behind fluid_simulation_b200.diff.DiffWCSPH).

  - against tape gradients (autograd of the FP64 torch restatement, whose
    forward is pinned to the FP64 oracle in test_wcsph_tape.py) after one
    and after 20 substeps of a compressed block against the walls, with
    pressure, viscosity, cohesion and walls active: 1e-3 norm-relative;
  - checkpointing every 1, 7 or 10 substeps, with segment records kept or
    segments replayed, gives bit-identical gradients;
  - against FP64 central finite differences of the CPU oracle, loss = mean
    squared distance to the initial cloud moved by +0.3 m in x, along random
    directions of v0 (a dam-break column) and of v0, stiffness, viscosity
    and rest density (a compressed block clear of the walls), eps = 1e-4
    relative: 1e-3 relative.  Finite differences are taken away from walls:
    a wall clamps positions and damps velocities discontinuously, so a
    difference quotient across a wall contact is no derivative (the tape
    tests above cover the walls' adjoint).
"""

import os

import numpy as np
import pytest
import torch

import oracle
from adjoint_util import CFG, DT, GRAVITY, MASS, block, oracle_model, params, tape_rollout
from fluid_simulation_b200.diff import DiffWCSPH
from fluid_simulation_b200.newton_shim import model_from_arrays
from fluid_simulation_b200.scene import make_scene
from fluid_simulation_b200.solver import SolverWCSPH
from golden_io import rel_err

pytestmark = pytest.mark.gpu
GTOL = 1e-3


def diff_sim(x, prm, dev, k=10, cfg=CFG, dt=DT, mass=MASS, record_bytes=None):
    m = model_from_arrays(x, np.zeros_like(x), mass, device=dev, radius=cfg["particle_radius"],
                          gravity=(GRAVITY,), attributes=dict(prm, particle_mask=0), solver_cls=SolverWCSPH)
    c = SolverWCSPH.SphConfig(**cfg)
    return DiffWCSPH(m, c, dt, checkpoint_every=k, record_bytes=record_bytes)


def gpu_grads(sim, x, v, prm, steps, loss_fn, dev):
    leaves = [torch.tensor(a, device=dev, requires_grad=True)
              for a in (x, v, prm["stiffness"], prm["viscosity"], prm["rest_density"])]
    xT, vT = sim.rollout(*leaves, steps)
    loss_fn(xT, vT).backward()
    return [t.grad.double().cpu().numpy() for t in leaves]


def tape_grads(x, v, prm, steps, loss_fn):
    leaves = [torch.tensor(a, dtype=torch.float64, requires_grad=True)
              for a in (x, v, prm["stiffness"], prm["viscosity"], prm["rest_density"])]
    p = dict(stiffness=leaves[2], viscosity=leaves[3], rest_density=leaves[4],
             exponent=torch.tensor(prm["exponent"], dtype=torch.float64),
             surface_tension=torch.tensor(prm["surface_tension"], dtype=torch.float64))
    xT, vT = tape_rollout(leaves[0], leaves[1], p, steps)
    loss_fn(xT, vT).backward()
    return [t.grad.numpy() for t in leaves]


def weighted_loss(n, seed):
    rng = np.random.default_rng(seed)
    wx, wv = rng.normal(size=(n, 3)), rng.normal(size=(n, 3))

    def f(xT, vT):
        return (xT * torch.as_tensor(wx, dtype=xT.dtype, device=xT.device)).sum() + \
            1e-3 * (vT * torch.as_tensor(wv, dtype=vT.dtype, device=vT.device)).sum()
    return f


NAMES = ("x0", "v0", "stiffness", "viscosity", "rest_density")


@pytest.mark.parametrize("steps", [1, 20])
def test_adjoint_matches_tape(steps, cuda_device):
    x, v = block()
    prm = params(len(x))
    loss = weighted_loss(len(x), 5)
    got = gpu_grads(diff_sim(x, prm, cuda_device), x, v, prm, steps, loss, cuda_device)
    want = tape_grads(x, v, prm, steps, loss)
    errs = {nm: rel_err(g, w) for nm, g, w in zip(NAMES, got, want)}
    print(errs)
    assert all(e <= GTOL for e in errs.values()), errs
    assert np.abs(want[2]).max() > 0 and np.abs(want[3]).max() > 0  # pressure and viscosity act


def test_gradients_do_not_depend_on_checkpoint_interval(cuda_device):
    """Checkpoint intervals 1, 7, 10, each with every segment's record kept
    and with all but the last segment replayed: identical bits."""
    x, v = block(side=9, seed=3)
    prm = params(len(x), seed=4)
    loss = weighted_loss(len(x), 6)
    ref = None
    for k in (1, 7, 10):
        for record_bytes in (None, 0):
            sim = diff_sim(x, prm, cuda_device, k=k, record_bytes=record_bytes)
            assert (sim.max_records >= 25) == (record_bytes is None)
            g = gpu_grads(sim, x, v, prm, 25, loss, cuda_device)
            if ref is None:
                ref = g
            else:
                for nm, a, b in zip(NAMES, g, ref):
                    assert np.array_equal(a, b), (k, record_bytes, nm)


def test_graph_replayed_rollouts_equal_eager_ones(cuda_device):
    x, v = block(side=9, seed=7)
    prm = params(len(x), seed=8)
    loss = weighted_loss(len(x), 9)
    out = []
    for graphs in (False, True):
        sim = diff_sim(x, prm, cuda_device, k=5)
        sim.use_graphs = graphs
        for _ in range(3):  # eager first run, recording, then replays
            g = gpu_grads(sim, x, v, prm, 15, loss, cuda_device)
        out.append(g)
    for nm, a, b in zip(NAMES, out[0], out[1]):
        assert np.array_equal(a, b), nm


def test_rollout_forward_equals_plain_substeps(cuda_device):
    """The differentiable rollout runs the drop-in substep: same bits."""
    x, v = block(side=9, seed=5)
    prm = params(len(x), seed=6)
    sim = diff_sim(x, prm, cuda_device, k=4)
    t = [torch.tensor(a, device=cuda_device) for a in (x, v, prm["stiffness"], prm["viscosity"],
                                                        prm["rest_density"])]
    xT, vT = sim.rollout(*t, 9)
    m = model_from_arrays(x, v, MASS, device=cuda_device, radius=CFG["particle_radius"], gravity=(GRAVITY,),
                          attributes=dict(prm, particle_mask=0), solver_cls=SolverWCSPH)
    solver = SolverWCSPH(m, SolverWCSPH.SphConfig(**CFG))
    a, b = m.state(), m.state()
    for _ in range(9):
        solver.step(a, b, None, None, DT)
        a, b = b, a
    assert torch.equal(xT, a.particle_q) and torch.equal(vT, a.particle_qd)


# ------------------------------------------------------ finite differences --
def dam_case(target=5000, steps=40):
    s = make_scene(target)
    n = s.count
    cfg = dict(particle_radius=s.radius, particle_length=s.spacing, smoothing_length_coff=2.0, bound_width=1.2,
               bound_height=0.28, bound_length=0.6, boundary_damping=0.0, clamp_negative_pressure=True)
    prm = dict(stiffness=np.full(n, 2.5e5, np.float32), viscosity=np.full(n, 1e-6, np.float32),
               rest_density=np.full(n, 1000.0, np.float32), surface_tension=np.zeros(n, np.float32),
               exponent=np.full(n, 7.0, np.float32))
    h = 2.0 * s.spacing
    dt = 0.25 * h / (2.5e5 * 7.0 / 1000.0) ** 0.5
    return s, cfg, prm, dt, steps


def oracle_loss(x0, v0, prm, cfg, dt, steps, mass, target):
    n = len(x0)
    model = dict(particle_flags=np.ones(n, np.int32), particle_mass=np.full(n, mass, np.float32),
                 particle_world=np.zeros(n, np.int32), gravity=np.array([GRAVITY], np.float32),
                 particle_max_radius=cfg["particle_radius"], sph=dict(particle_mask=np.zeros(n, np.int32), **prm))
    state = dict(particle_q=x0, particle_qd=v0, sph={})
    for _ in range(steps):
        out, _ = oracle.wcsph_step(model, state, cfg, dt, precision="f64")
        state = dict(particle_q=out["particle_q"], particle_qd=out["particle_qd"], sph={})
    return float(np.mean(np.sum((state["particle_q"] - target) ** 2, axis=1)))


@pytest.mark.parametrize("case", ["dam", "block"])
def test_gradients_match_fp64_finite_differences(case, cuda_device):
    """dam: a make_scene(5000) column at rest, 40 substeps at the acoustic dt
    (its pressure stays clamped at zero this early, so only v0 is checked);
    block: the compressed block clear of the walls, 20 substeps, where
    stiffness, viscosity and rest density all act."""
    if case == "dam":
        s, cfg, prm, dt, steps = dam_case()
        x0, mass = s.positions, s.mass
        v0 = np.zeros_like(x0)
        fields = ()
    else:
        x0, v0 = block(at_wall=False)
        prm, cfg, dt, steps, mass = params(len(x0)), CFG, DT, 20, MASS
        fields = (("stiffness", 2), ("viscosity", 3), ("rest_density", 4))
    n = len(x0)
    target = x0.astype(np.float64) + np.array([0.3, 0.0, 0.0])
    tgt = torch.tensor(target, dtype=torch.float32, device=cuda_device)

    def loss(xT, vT):
        return ((xT - tgt) ** 2).sum(1).mean()

    g = gpu_grads(diff_sim(x0, prm, cuda_device, cfg=cfg, dt=dt, mass=mass), x0, v0, prm, steps, loss, cuda_device)
    rng = np.random.default_rng(2)
    eps = 1e-4
    checks = []
    for _ in range(6):  # random unit directions of v0 (scale 1 m/s)
        d = rng.normal(size=(n, 3))
        d /= np.linalg.norm(d)
        lp = oracle_loss(x0, v0 + eps * d, prm, cfg, dt, steps, mass, target)
        lm = oracle_loss(x0, v0 - eps * d, prm, cfg, dt, steps, mass, target)
        checks.append(("v0", float(np.sum(g[1] * d)), (lp - lm) / (2 * eps)))
    for key, gi in fields:  # the whole field scaled by 1 +- eps
        hi = dict(prm, **{key: prm[key].astype(np.float64) * (1 + eps)})
        lo = dict(prm, **{key: prm[key].astype(np.float64) * (1 - eps)})
        fd = (oracle_loss(x0, v0, hi, cfg, dt, steps, mass, target) -
              oracle_loss(x0, v0, lo, cfg, dt, steps, mass, target)) / (2 * eps)
        checks.append((key, float(np.sum(g[gi] * prm[key])), fd))
    print(case, checks)
    for name, ad, fd in checks:
        assert fd != 0.0, name
        assert abs(ad - fd) <= GTOL * abs(fd), (name, ad, fd)


def test_active_column_50k_gradients(cuda_device):
    """The differentiable workload at full size with pressure and viscosity
    acting (adjoint_util.active_column: make_scene(50000), 50,232
    particles, N(0, 0.1 m/s) initial velocities, 120 substeps, checkpoints
    every 10 with every segment but the last replayed).

    The clamped EOS max(p, 0) has a kink at rest density: the loss is
    piecewise smooth, and over 120 substeps an FP32 and an FP64 forward put
    different particles on either side of it, so their derivatives differ
    (by 0.1-1 % along v0 and 7 % for the stiffness here).  The chain of
    checks therefore keeps each derivative on its own trajectory:

    * the adjoint against FP64 tape gradients along the solver's own
      trajectory (each of the 120 substeps re-evaluated in FP64 by the torch
      restatement from the plain solver's state, on the side of the kink the
      solver took, differentiated, adjoints chained): the gradients w.r.t.
      x0, v0, stiffness, viscosity and rest density within 1e-3
      norm-relative, and the derivatives along the parameter fields (d/d log
      k) and 8 random unit directions of v0 within 1e-3 relative, all
      non-zero; the FP32 tape along the same trajectory is printed beside it;
    * the FP64 tape rollout (its own FP64 trajectory, the oracle's to 1e-12
      per substep) against FP64 central differences of the oracle (v0 along
      random unit directions, each parameter field scaled by 1 +- eps) at eps
      = 1e-5 and 3e-5, within max(1e-3 |FD|, 2 |FD(1e-5) - FD(3e-5)|): the
      spread stands for the quotient's own error across kinks.  The oracle
      needs a few seconds per FP64 rollout, so the default run checks 2 v0
      directions; FS_FD_DIRECTIONS=32 runs 32."""
    from adjoint_util import active_column, tape_along_trajectory, tape_rollout
    ndir = int(os.environ.get("FS_FD_DIRECTIONS", "2"))
    s, cfg, prm, x0, v0, dt = active_column()
    steps = 120
    n = len(x0)
    target = x0.astype(np.float64) + np.array([0.3, 0.0, 0.0])

    def loss(xT, vT):
        return ((xT - torch.as_tensor(target, dtype=xT.dtype, device=xT.device)) ** 2).sum(1).mean()

    sim = diff_sim(x0, prm, cuda_device, k=10, cfg=cfg, dt=dt, mass=s.mass, record_bytes=0)
    g = gpu_grads(sim, x0, v0, prm, steps, loss, cuda_device)
    del sim
    # the plain solver's trajectory (the rollout's forward, bit for bit)
    m = model_from_arrays(x0, v0, s.mass, device=cuda_device, radius=cfg["particle_radius"], gravity=(GRAVITY,),
                          attributes=dict(prm, particle_mask=0), solver_cls=SolverWCSPH)
    solver = SolverWCSPH(m, SolverWCSPH.SphConfig(**cfg))
    a, b = m.state(), m.state()
    xs, vs, on = [], [], []
    for _ in range(steps):
        xs.append(a.particle_q.clone())
        vs.append(a.particle_qd.clone())
        solver.step(a, b, None, None, dt)
        on.append(b.sph.pressure > 0)  # the clamp's branch this substep took
        a, b = b, a
    xT = a.particle_q.clone()
    del m, solver, b

    def leaves_of(dtype):
        lv = {k: torch.tensor(prm[k], dtype=dtype, device=cuda_device, requires_grad=True)
              for k in ("stiffness", "viscosity", "rest_density")}
        return lv, dict(lv, exponent=torch.tensor(prm["exponent"], dtype=dtype, device=cuda_device),
                        surface_tension=torch.tensor(prm["surface_tension"], dtype=dtype, device=cuda_device))

    def grads(gx, gv, lv):
        return [t.double().cpu().numpy() for t in (gx, gv)] + \
               [lv[k].grad.double().cpu().numpy() for k in ("stiffness", "viscosity", "rest_density")]

    def along_trajectory(dtype):
        lv, p = leaves_of(dtype)
        tg = torch.as_tensor(target, dtype=dtype, device=cuda_device)
        xf = xT.to(dtype)
        gx, gv = tape_along_trajectory([t.to(dtype) for t in xs], [t.to(dtype) for t in vs], p,
                                       2.0 * (xf - tg) / n, torch.zeros_like(xf), dt, cfg, s.mass, pressure_on=on)
        out = grads(gx, gv, lv)
        torch.cuda.empty_cache()
        return out

    want, t32 = along_trajectory(torch.float64), along_trajectory(torch.float32)
    del xs, vs, on
    # the FP64 tape of its own trajectory
    lv, p = leaves_of(torch.float64)
    lx = torch.tensor(x0, dtype=torch.float64, device=cuda_device, requires_grad=True)
    lvel = torch.tensor(v0, dtype=torch.float64, device=cuda_device, requires_grad=True)
    xr, vr = tape_rollout(lx, lvel, p, steps, dt=dt, cfg=cfg, mass=s.mass)
    loss(xr, vr).backward()
    own = grads(lx.grad, lvel.grad, lv)
    del lx, lvel, lv, p, xr, vr
    torch.cuda.empty_cache()
    rng = np.random.default_rng(7)
    dirs = [rng.normal(size=(n, 3)) for _ in range(8)]

    def along(gr):
        return [float(np.sum(gr[1] * d)) for d in dirs] + \
               [float(np.sum(gr[gi] * prm[key])) for key, gi in (("stiffness", 2), ("viscosity", 3), ("rest_density", 4))]

    a_ad, a_64, a_32 = along(g), along(want), along(t32)
    labels = ["v0"] * len(dirs) + ["stiffness", "viscosity", "rest_density"]
    fields = {nm: (rel_err(x, w), rel_err(y, w)) for nm, x, y, w in zip(NAMES, g, t32, want)}
    dirs_rel = [(lb, abs(x - w) / abs(w), abs(y - w) / abs(w)) for lb, x, y, w in zip(labels, a_ad, a_32, a_64)]
    print("per-particle fields, (adjoint vs FP64 tape, FP32 tape vs FP64 tape), norm-relative:", fields)
    print("directional derivatives, (adjoint vs FP64 tape, FP32 tape vs FP64 tape), relative:", dirs_rel)
    # FP64 central differences of the oracle against the FP64 tape of its own trajectory
    rng = np.random.default_rng(2)
    checks = []

    def fd(make):
        out = []
        for eps in (1e-5, 3e-5):
            (xp, vp, pp), (xm, vm, pm) = make(eps), make(-eps)
            out.append((oracle_loss(xp, vp, pp, cfg, dt, steps, s.mass, target) -
                        oracle_loss(xm, vm, pm, cfg, dt, steps, s.mass, target)) / (2 * eps))
        return out

    for _ in range(ndir):
        d = rng.normal(size=(n, 3))
        d /= np.linalg.norm(d)
        f1, f2 = fd(lambda e: (x0, v0 + e * d, prm))
        checks.append(("v0", float(np.sum(own[1] * d)), float(np.sum(g[1] * d)), f1, f2))
    for key, gi in (("stiffness", 2), ("viscosity", 3), ("rest_density", 4)):
        f1, f2 = fd(lambda e: (x0, v0, dict(prm, **{key: prm[key].astype(np.float64) * (1 + e)})))
        checks.append((key, float(np.sum(own[gi] * prm[key])), float(np.sum(g[gi] * prm[key])), f1, f2))
    print("FP64 tape rollout vs FP64 central differences (tape, adjoint, FD eps 1e-5, FD eps 3e-5):", checks)
    for nm, (e_ad, e_32) in fields.items():
        assert e_ad <= GTOL, (nm, e_ad, e_32)
    for lb, e_ad, e_32 in dirs_rel:
        assert e_ad <= GTOL, (lb, e_ad, e_32)
    for k in (2, 3, 4):
        assert np.abs(want[k]).max() > 0, NAMES[k]
    for name, tp, ad, f1, f2 in checks:
        assert f1 != 0.0, name
        assert abs(tp - f1) <= max(GTOL * abs(f1), 2.0 * abs(f1 - f2)), (name, tp, f1, f2)
