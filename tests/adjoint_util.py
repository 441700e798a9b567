"""Shared setup of the WCSPH gradient tests: a small compressed block against
a wall (pressure, walls and cohesion all active) and the oracle-form model."""

import numpy as np
import torch

import wcsph_tape

SPACING = 0.01
H = 2.0 * SPACING
MASS = 1000.0 * SPACING ** 3
CFG = dict(particle_radius=0.5 * SPACING, particle_length=SPACING, smoothing_length_coff=2.0, bound_width=0.1,
           bound_height=0.1, bound_length=0.1, boundary_damping=-0.5, clamp_negative_pressure=True)
GRAVITY = (0.0, 0.0, -10.0)
DT = 1.0e-4


def block(side=11, squeeze=0.94, seed=0, sigma=0.3, at_wall=True):
    """side^3 particles squeezed to 94 % of the spacing, velocities
    N(0, sigma); resting on the floor against the -x wall (at_wall) or
    floating in the middle of the tank, clear of every wall."""
    rng = np.random.default_rng(seed)
    g = np.arange(side) * SPACING * squeeze
    x = np.stack(np.meshgrid(g, g, g, indexing="ij"), -1).reshape(-1, 3)
    x = x + rng.uniform(-0.03, 0.03, x.shape) * SPACING
    if at_wall:
        x = x + np.array([-CFG["bound_width"] + 0.1 * SPACING, -0.5 * g[-1], 0.1 * SPACING])
    else:
        x = x + np.array([-0.5 * g[-1], -0.5 * g[-1], CFG["bound_length"] - 0.5 * g[-1]])
    v = rng.normal(size=x.shape) * sigma
    return x.astype(np.float32), v.astype(np.float32)


def params(n, seed=1):
    rng = np.random.default_rng(seed)
    return dict(stiffness=(2.5e5 * rng.uniform(0.8, 1.2, n)).astype(np.float32),
                viscosity=(2e-3 * rng.uniform(0.8, 1.2, n)).astype(np.float32),
                rest_density=(1000.0 * rng.uniform(0.98, 1.02, n)).astype(np.float32),
                surface_tension=np.full(n, 0.02, np.float32), exponent=np.full(n, 7.0, np.float32))


def oracle_model(x, prm):
    n = len(x)
    return dict(particle_flags=np.ones(n, np.int32), particle_mass=np.full(n, MASS, np.float32),
                particle_world=np.zeros(n, np.int32), gravity=np.array([GRAVITY], np.float32),
                particle_max_radius=CFG["particle_radius"],
                sph=dict(particle_mask=np.zeros(n, np.int32), **prm))


def tape_rollout(x, v, prm, steps, dt=DT, cfg=CFG, mass=MASS):
    """FP64 torch rollout; x, v, prm entries are float64 tensors (leaves),
    all on one device."""
    n = x.shape[0]
    mass = torch.full((n,), float(np.float32(mass)), dtype=torch.float64, device=x.device)  # float32 in the model
    g = torch.tensor(GRAVITY, dtype=torch.float64, device=x.device)
    cfg = dict(cfg, h=cfg["smoothing_length_coff"] * cfg["particle_length"])
    for _ in range(steps):
        x, v = wcsph_tape.substep(x, v, mass, prm["stiffness"], prm["viscosity"], prm["rest_density"],
                                  prm["exponent"], prm["surface_tension"], g, cfg, dt)
    return x, v


def active_column(target=50000, sigma=0.1, seed=21):
    """The differentiable dam-break workload at full size with pressure and
    viscosity acting: the reference scene make_scene(target) (50,232
    particles for 50,000) in the reference tank at the reference WCSPH
    defaults (B = 250 kPa, exponent 7, viscosity 1e-6, clamped EOS), with a
    seeded N(0, sigma) initial velocity field.  Over 120 substeps at
    dt = 0.25 h / (c0 + max|v0|) the velocity field compresses parts of the
    column (pressure up to ~20 kPa, ~6 % of the particles above rest
    density at the end), viscosity acts on the relative velocities, and no
    particle reaches a wall (closest approach 1.8 cm; a wall contact would
    make the loss discontinuous).  Returns (scene, cfg, prm, x0, v0, dt)."""
    from fluid_simulation_b200.scene import make_scene
    s = make_scene(target)
    n = s.count
    cfg = dict(particle_radius=s.radius, particle_length=s.spacing, smoothing_length_coff=2.0, bound_width=1.2,
               bound_height=0.28, bound_length=0.6, boundary_damping=0.0, clamp_negative_pressure=True)
    prm = dict(stiffness=np.full(n, 2.5e5, np.float32), viscosity=np.full(n, 1e-6, np.float32),
               rest_density=np.full(n, 1000.0, np.float32), surface_tension=np.zeros(n, np.float32),
               exponent=np.full(n, 7.0, np.float32))
    x0 = s.positions
    v0 = (np.random.default_rng(seed).normal(size=x0.shape) * sigma).astype(np.float32)
    c0 = (2.5e5 * 7.0 / 1000.0) ** 0.5
    dt = 0.25 * (2.0 * s.spacing) / (c0 + float(np.linalg.norm(v0, axis=1).max()))
    return s, cfg, prm, x0, v0, dt


def tape_along_trajectory(xs, vs, prm, seed_x, seed_v, dt, cfg, mass, pressure_on=None):
    """Tape gradients along a given trajectory: xs[k], vs[k] (k = 0..K-1,
    float64 or float32 tensors on one device) are the inputs of substep k as another
    forward produced them.  Each substep is re-evaluated by the torch
    restatement from its recorded input and differentiated alone; the
    adjoints are chained from (seed_x, seed_v) = dL/d(x_K, v_K) back to
    substep 0.  prm: stiffness, viscosity, rest_density (leaves of the same
    dtype, gradients accumulate in .grad), exponent, surface_tension.  Returns
    (dL/dx0, dL/dv0).  Unlike a tape rollout, the trajectory is the given
    one, so this checks another forward's derivative; pressure_on[k] (bool
    per particle, optional) fixes the clamped EOS's branch at substep k to
    the one that forward took, so that an FP64 density a rounding away from
    rest density does not switch a particle to the other side of the kink."""
    dev, dtype = xs[0].device, xs[0].dtype
    n = xs[0].shape[0]
    m = torch.full((n,), float(np.float32(mass)), dtype=dtype, device=dev)
    g = torch.tensor(GRAVITY, dtype=dtype, device=dev)
    c = dict(cfg, h=cfg["smoothing_length_coff"] * cfg["particle_length"])
    ax, av = seed_x, seed_v
    for k in range(len(xs) - 1, -1, -1):
        x = xs[k].clone().requires_grad_()
        v = vs[k].clone().requires_grad_()
        x1, v1 = wcsph_tape.substep(x, v, m, prm["stiffness"], prm["viscosity"], prm["rest_density"],
                                    prm["exponent"], prm["surface_tension"], g, c, dt,
                                    pressure_on=None if pressure_on is None else pressure_on[k])
        torch.autograd.backward([x1, v1], [ax, av])
        ax, av = x.grad, v.grad
    return ax, av
