"""FP64 torch restatement of the WCSPH substep (solver_wcsph.py:110-305) for
tape gradients: autograd through this plays the part of a wp.Tape through the
reference kernels.  Each substep's neighbour set (pairs with r < h, found
with a k-d tree at the substep's input positions) is held fixed, as in the
hand-written adjoint.  Test infrastructure only (dense torch ops; on a CUDA
device when the inputs are there, which the 50k-particle rollout needs)."""

import math

import numpy as np
import torch
from scipy.spatial import cKDTree


def cubic_w(r, h):
    k = 8.0 / (math.pi * h ** 3)
    q = r / h
    inner = k * (6.0 * q ** 3 - 6.0 * q ** 2 + 1.0)
    outer = 2.0 * k * (1.0 - q) ** 3
    return torch.where(q <= 0.5, inner, torch.where(q <= 1.0, outer, torch.zeros_like(q)))


def cubic_gs(r, h):
    """grad W(d) = gs(r) d (zero for r <= 1e-5 or r > h)."""
    k = 8.0 / (math.pi * h ** 3)
    q = r / h
    rs = torch.clamp(r, min=1e-30)
    inner = 6.0 * k / h ** 2 * (3.0 * q - 2.0)
    outer = -6.0 * k / h * (1.0 - q) ** 2 / rs
    g = torch.where(q <= 0.5, inner, outer)
    return torch.where((r > 1e-5) & (q <= 1.0), g, torch.zeros_like(g))


def walls(p, v, w, hh, l, damping):
    lo = torch.tensor([-w, -hh, 0.0], dtype=p.dtype, device=p.device)
    hi = torch.tensor([w, hh, 2.0 * l], dtype=p.dtype, device=p.device)
    below = p < lo
    v = torch.where(below & (v < 0), v * damping, v)
    p = torch.where(below, lo.expand_as(p), p)
    above = p > hi
    v = torch.where(above & (v > 0), v * damping, v)
    p = torch.where(above, hi.expand_as(p), p)
    return p, v


def substep(x, v, mass, stiffness, viscosity, rest_density, exponent, coh_st, g, cfg, dt, pressure_on=None):
    """One substep, all particles active and dynamic.  cfg: h, particle_radius,
    bound_width/height/length, boundary_damping, clamp_negative_pressure.
    pressure_on (bool per particle, optional): the clamp's branch taken from
    another evaluation of the same state (p kept where True, 0 elsewhere), so
    that the derivative follows that evaluation's side of the kink at rest
    density."""
    h = cfg["h"]
    n = x.shape[0]
    dev = x.device
    pairs = cKDTree(x.detach().cpu().numpy()).query_pairs(h, output_type="ndarray")
    i = torch.as_tensor(np.concatenate([pairs[:, 0], pairs[:, 1]]), dtype=torch.long, device=dev)
    j = torch.as_tensor(np.concatenate([pairs[:, 1], pairs[:, 0]]), dtype=torch.long, device=dev)
    vol = mass / torch.clamp(rest_density, min=1e-6)
    mv = rest_density * vol
    d = x[i] - x[j]
    r = torch.sqrt((d * d).sum(1))
    rho = mv * cubic_w(torch.zeros(n, dtype=x.dtype, device=dev), h) + torch.zeros(n, dtype=x.dtype, device=dev).index_add(
        0, i, mv[j] * cubic_w(r, h))
    p = stiffness * ((rho / torch.clamp(rest_density, min=1e-6)) ** exponent - 1.0)
    if cfg["clamp_negative_pressure"]:
        # relu: derivative 0 at p = 0, the adjoint's convention for max(p, 0)
        p = torch.relu(p) if pressure_on is None else torch.where(pressure_on, p, torch.zeros_like(p))
    P = p / torch.clamp(rho * rho, min=1e-6)
    R = 1.0 / torch.clamp(rho, min=1e-6)
    gs = cubic_gs(r, h)
    u = v[i] - v[j]
    visc = 10.0 * viscosity[i] * mass[j] * R[j] * (u * d).sum(1) / (r * r + 0.01 * h * h)
    pres = -mass[j] * (P[i] + P[j])
    wc = (coh_st[i] / mass[i]) * mass[j] * cubic_w(torch.clamp(r, min=cfg["particle_radius"]), h)
    c = (visc + pres) * gs - wc
    a = torch.zeros(n, 3, dtype=x.dtype, device=dev).index_add(0, i, c[:, None] * d) + g
    v1 = v + dt * a
    x1 = x + dt * v1
    x1, v1 = walls(x1, v1, cfg["bound_width"], cfg["bound_height"], cfg["bound_length"], cfg["boundary_damping"])
    return x1, v1
