"""The separate-pass entry points of the C ABI (each after fs_grid_build).

  - fs_wcsph_density + fs_wcsph_force_integrate reproduce fs_wcsph_substep
    bit for bit (same grid, same kernels, same visiting order);
  - fs_dfsph_density_factor at the end-of-step positions reproduces the
    rho / factor / neighbor_count the DFSPH substep leaves in state_out;
  - fs_dfsph_nonpressure_predict reproduces the substep's acceleration bit
    for bit; fs_pbf_predict follows its formula and walls;
  - fs_dfsph_divergence, fs_dfsph_correct, fs_dfsph_residual, fs_pbf_density,
    fs_pbf_lambda, fs_pbf_delta and fs_pbf_xsph agree within 1e-5
    norm-relative with an FP64 brute-force restatement of the reference
    formulas (solver_dfsph.py:246-337, 574-596; solver_pbf.py:115-141,
    246-350, 435-463) on a compressed block, where every field is well
    conditioned.
"""

import ctypes as C

import numpy as np
import pytest
import torch
from scipy.spatial import cKDTree

from fluid_simulation_b200 import _lib
from fluid_simulation_b200.newton_shim import HashGrid, model_from_arrays
from fluid_simulation_b200.solver import SolverDFSPH, SolverPBF, SolverWCSPH
from fluid_simulation_b200.solver import _common as cm
from golden_io import rel_err

pytestmark = pytest.mark.gpu
TOL = 1e-5
SPACING = 0.01
H = 2.0 * SPACING
MASS = 1000.0 * SPACING ** 3


def block(side=14, squeeze=0.93, seed=0):
    rng = np.random.default_rng(seed)
    g = np.arange(side) * SPACING * squeeze
    x = np.stack(np.meshgrid(g, g, g, indexing="ij"), -1).reshape(-1, 3)
    x = x + rng.uniform(-0.05, 0.05, x.shape) * SPACING + np.array([0.1, 0.1, 0.1])
    v = rng.normal(size=x.shape) * 0.2
    return x.astype(np.float32), v.astype(np.float32)


def model_for(cls, x, v, dev):
    attrs = dict(particle_mask=0, rest_density=1000.0, surface_tension=0.0, viscosity=1e-6)
    if cls is SolverWCSPH:
        attrs.update(stiffness=2.5e5, exponent=7.0)
    return model_from_arrays(x, v, MASS, device=dev, radius=0.5 * SPACING, attributes=attrs, solver_cls=cls)


def T(a, dev, dtype=torch.float32):
    return torch.as_tensor(np.ascontiguousarray(a), dtype=dtype, device=dev)


def stream(dev):
    return torch.cuda.current_stream(dev).cuda_stream


# ---------------------------------------------------- FP64 restatements ----
def pairs_within(x, h):
    p = cKDTree(x.astype(np.float64)).query_pairs(h, output_type="ndarray")
    i = np.concatenate([p[:, 0], p[:, 1]])
    j = np.concatenate([p[:, 1], p[:, 0]])
    return i, j


def cubic_grad(d, h):
    """grad W of the cubic spline (solver_dfsph.py:24-54) for offsets d = x_i - x_j."""
    r = np.linalg.norm(d, axis=1)
    q = r / h
    k = 8.0 / (np.pi * h ** 3)
    dw = np.where(q <= 0.5, k * (18.0 * q * q - 12.0 * q) / h, -6.0 * k * (1.0 - q) ** 2 / h)
    dw = np.where((r > 1e-5) & (q <= 1.0), dw, 0.0)
    return (dw / np.maximum(r, 1e-30))[:, None] * d


def poly6(r2, h):
    return np.where(r2 < h * h, 315.0 / (64.0 * np.pi * h ** 9) * (h * h - r2) ** 3, 0.0)


def spiky_grad(d, h):
    r = np.linalg.norm(d, axis=1)
    s = np.where((r > 1e-6) & (r < h), -45.0 / (np.pi * h ** 6) * (h - r) ** 2 / np.maximum(r, 1e-30), 0.0)
    return s[:, None] * d


def scatter(n, i, vals):
    out = np.zeros((n,) + vals.shape[1:])
    np.add.at(out, i, vals)
    return out


# --------------------------------------------------------------- WCSPH ----
def test_wcsph_passes_reproduce_substep(cuda_device):
    dev = cuda_device
    x, v = block()
    n = len(x)
    m = model_for(SolverWCSPH, x, v, dev)
    solver = SolverWCSPH(m, SolverWCSPH.SphConfig(particle_radius=0.5 * SPACING, particle_length=SPACING,
                                                 smoothing_length_coff=2.0, bound_width=0.3, bound_height=0.3,
                                                 bound_length=0.2, boundary_damping=-0.5))
    s_in, s_out = m.state(), m.state()
    solver.step(s_in, s_out, None, None, 1e-4)
    lib = _lib.load()
    ms = cm.model_struct(m, wcsph=True)
    grid = HashGrid(device=dev)
    grid.build(s_in.particle_q, H)
    s2 = m.state()
    acc = torch.zeros(n, 3, device=dev)
    _lib.check(lib.fs_wcsph_density(grid._ctx, C.byref(ms), s_in.particle_q.data_ptr(), H, 1,
                                    s2.sph.rho.data_ptr(), s2.sph.pressure.data_ptr(), stream(dev)), "density")
    si = cm.state_struct(s_in, n, m.device)
    so = cm.state_struct(s2, n, m.device, need=("rho", "pressure"))
    p = solver.params(1e-4)
    _lib.check(lib.fs_wcsph_force_integrate(grid._ctx, C.byref(ms), C.byref(si), C.byref(so), C.byref(p),
                                            acc.data_ptr(), stream(dev)), "force_integrate")
    torch.cuda.synchronize()
    assert torch.equal(s2.sph.rho, s_out.sph.rho)
    assert torch.equal(s2.sph.pressure, s_out.sph.pressure)
    assert torch.equal(acc, solver._particle_accel)
    assert torch.equal(s2.particle_q, s_out.particle_q)
    assert torch.equal(s2.particle_qd, s_out.particle_qd)
    assert float(s_out.sph.pressure.max()) > 1e4


# --------------------------------------------------------------- DFSPH ----
def test_dfsph_density_factor_reproduces_substep(cuda_device):
    dev = cuda_device
    x, v = block(seed=1)
    n = len(x)
    m = model_for(SolverDFSPH, x, v, dev)
    solver = SolverDFSPH(m, SolverDFSPH.SphConfig(particle_radius=0.5 * SPACING, particle_length=SPACING,
                                                 smoothing_length_coff=2.0, bound_width=0.3, bound_height=0.3,
                                                 bound_length=0.2))
    s_in, s_out = m.state(), m.state()
    solver.step(s_in, s_out, None, None, 1.0 / 240.0)
    lib = _lib.load()
    ms = cm.model_struct(m)
    grid = HashGrid(device=dev)
    grid.build(s_out.particle_q, H)
    rho = torch.zeros(n, device=dev)
    fac = torch.zeros(n, device=dev)
    cnt = torch.zeros(n, dtype=torch.int32, device=dev)
    _lib.check(lib.fs_dfsph_density_factor(grid._ctx, C.byref(ms), s_out.particle_q.data_ptr(), H,
                                           solver.config.min_neighbors_for_factor, rho.data_ptr(), fac.data_ptr(),
                                           cnt.data_ptr(), stream(dev)), "density_factor")
    torch.cuda.synchronize()
    assert torch.equal(rho, s_out.sph.rho)
    assert torch.equal(fac, s_out.sph.factor)
    assert torch.equal(cnt, s_out.sph.neighbor_count)


def test_dfsph_divergence_correct_residual_match_fp64(cuda_device):
    dev = cuda_device
    x, v = block(seed=2)
    n = len(x)
    m = model_for(SolverDFSPH, x, v, dev)
    lib = _lib.load()
    ms = cm.model_struct(m)
    grid = HashGrid(device=dev)
    xt, vt = T(x, dev), T(v, dev)
    grid.build(xt, H)
    i, j = pairs_within(x, H)
    d = x[i].astype(np.float64) - x[j]
    gw = cubic_grad(d, H)
    # divergence: sum_j m_j (v_i - v_j) . grad W_ij
    want = scatter(n, i, MASS * ((v[i].astype(np.float64) - v[j]) * gw).sum(1))
    got = torch.zeros(n, device=dev)
    _lib.check(lib.fs_dfsph_divergence(grid._ctx, C.byref(ms), xt.data_ptr(), vt.data_ptr(), H, got.data_ptr(),
                                       stream(dev)), "divergence")
    torch.cuda.synchronize()
    assert rel_err(got.cpu().numpy(), want) <= TOL
    # correction: v* -= dt sum_j m_j (kappa_i / rho_i + kappa_j / rho_j) grad W_ij
    rng = np.random.default_rng(3)
    rho = (1000.0 * (1.0 + 0.1 * rng.random(n))).astype(np.float32)
    kappa = (rng.random(n) * 5.0).astype(np.float32)
    dt = 1.0 / 240.0
    kr = kappa.astype(np.float64) / rho
    want_v = v - dt * scatter(n, i, MASS * (kr[i] + kr[j])[:, None] * gw)
    vs = vt.clone()
    rho_t, kappa_t = T(rho, dev), T(kappa, dev)  # held: a temporary's memory may be reused before the launch
    _lib.check(lib.fs_dfsph_correct(grid._ctx, C.byref(ms), xt.data_ptr(), vs.data_ptr(), rho_t.data_ptr(),
                                    kappa_t.data_ptr(), H, dt, stream(dev)), "correct")
    torch.cuda.synchronize()
    assert rel_err(vs.cpu().numpy() - v, want_v - v) <= TOL
    # residual: mean over dynamic particles of max(a - b, 0)
    a = (rng.random(n) * 2.0 - 0.5).astype(np.float32)
    b = (rng.random(n) * 0.5).astype(np.float32)
    out = torch.zeros(1, dtype=torch.float64, device=dev)
    a_t, b_t = T(a, dev), T(b, dev)
    _lib.check(lib.fs_dfsph_residual(grid._ctx, C.byref(ms), a_t.data_ptr(), b_t.data_ptr(), out.data_ptr(),
                                     stream(dev)), "residual")
    torch.cuda.synchronize()
    assert abs(float(out) - np.maximum(a.astype(np.float64) - b, 0.0).mean()) <= 1e-6


# ----------------------------------------------------------------- PBF ----
def test_pbf_passes_match_fp64(cuda_device):
    dev = cuda_device
    x, v = block(seed=4)
    n = len(x)
    m = model_for(SolverPBF, x, v, dev)
    lib = _lib.load()
    ms = cm.model_struct(m)
    grid = HashGrid(device=dev)
    xt, vt = T(x, dev), T(v, dev)
    grid.build(xt, H)
    i, j = pairs_within(x, H)
    d = x[i].astype(np.float64) - x[j]
    r2 = (d * d).sum(1)
    w0 = poly6(np.zeros(1), H)[0]
    rho_want = MASS * w0 + scatter(n, i, MASS * poly6(r2, H))
    rho = torch.zeros(n, device=dev)
    _lib.check(lib.fs_pbf_density(grid._ctx, C.byref(ms), xt.data_ptr(), H, rho.data_ptr(), stream(dev)), "density")
    torch.cuda.synchronize()
    assert rel_err(rho.cpu().numpy(), rho_want) <= TOL
    # lambda
    eps, min_nb = 100.0, 8
    p = _lib.PbfParams()
    p.smoothing_length, p.lambda_epsilon, p.min_neighbors_for_lambda = H, eps, min_nb
    p.max_delta_position = 0.5 * 0.5 * SPACING
    gj = -(MASS / 1000.0) * spiky_grad(d, H)
    sq = scatter(n, i, (gj * gj).sum(1)) + (scatter(n, i, -gj) ** 2).sum(1)
    cnt = np.bincount(i, minlength=n)
    c = np.maximum(rho_want / 1000.0 - 1.0, 0.0)
    lam_want = np.where(cnt < min_nb, 0.0, -c / (sq + eps))
    lam = torch.zeros(n, device=dev)
    rho2 = torch.zeros(n, device=dev)
    cnt_t = torch.zeros(n, dtype=torch.int32, device=dev)
    _lib.check(lib.fs_pbf_lambda(grid._ctx, C.byref(ms), xt.data_ptr(), C.byref(p), lam.data_ptr(), rho2.data_ptr(),
                                 cnt_t.data_ptr(), stream(dev)), "lambda")
    torch.cuda.synchronize()
    assert np.array_equal(cnt_t.cpu().numpy(), cnt)
    assert rel_err(lam.cpu().numpy(), lam_want) <= TOL
    assert (lam_want < 0.0).mean() > 0.5  # compressed: most constraints active
    # delta: (1 / rho0) sum_{j != i} (lambda_i + lambda_j) m_j grad W_ij, clamped to max_delta_position
    lam32 = lam.cpu().numpy().astype(np.float64)
    dp = scatter(n, i, ((lam32[i] + lam32[j]) * MASS)[:, None] * spiky_grad(d, H)) / 1000.0
    ln = np.linalg.norm(dp, axis=1)
    dp = np.where((ln > p.max_delta_position)[:, None], dp * (p.max_delta_position / np.maximum(ln, 1e-12))[:, None],
                  dp)
    got_dp = torch.zeros(n, 3, device=dev)
    _lib.check(lib.fs_pbf_delta(grid._ctx, C.byref(ms), xt.data_ptr(), lam.data_ptr(), C.byref(p), got_dp.data_ptr(),
                                stream(dev)), "delta")
    torch.cuda.synchronize()
    assert rel_err(got_dp.cpu().numpy(), dp) <= TOL
    # xsph: v_i + c sum_{j != i} (m_j / rho_j) (v_j - v_i) W_ij
    xc = 0.05
    rho_in = rho.cpu().numpy().astype(np.float64)
    dv = scatter(n, i, (MASS / rho_in[j] * poly6(r2, H))[:, None] * (v[j].astype(np.float64) - v[i]))
    v_want = v + xc * dv
    v_out = torch.zeros(n, 3, device=dev)
    _lib.check(lib.fs_pbf_xsph(grid._ctx, C.byref(ms), xt.data_ptr(), vt.data_ptr(), rho.data_ptr(), H, xc,
                               v_out.data_ptr(), stream(dev)), "xsph")
    torch.cuda.synchronize()
    assert rel_err(v_out.cpu().numpy() - v, v_want - v) <= TOL


def test_dfsph_nonpressure_predict_reproduces_substep_accel(cuda_device):
    """fs_dfsph_nonpressure_predict at the step's input positions, with the
    density of fs_dfsph_density_factor, gives the acceleration the substep
    reports (solver._particle_accel) bit for bit, and v* = v + dt a."""
    dev = cuda_device
    x, v = block(seed=6)
    n = len(x)
    m = model_for(SolverDFSPH, x, v, dev)
    cfg = SolverDFSPH.SphConfig(particle_radius=0.5 * SPACING, particle_length=SPACING, smoothing_length_coff=2.0,
                                bound_width=0.3, bound_height=0.3, bound_length=0.2)
    solver = SolverDFSPH(m, cfg)
    dt = 1.0 / 240.0
    s_in, s_out = m.state(), m.state()
    solver.step(s_in, s_out, None, None, dt)
    lib = _lib.load()
    ms = cm.model_struct(m)
    grid = HashGrid(device=dev)
    grid.build(s_in.particle_q, H)
    rho = torch.zeros(n, device=dev)
    fac = torch.zeros(n, device=dev)
    cnt = torch.zeros(n, dtype=torch.int32, device=dev)
    _lib.check(lib.fs_dfsph_density_factor(grid._ctx, C.byref(ms), s_in.particle_q.data_ptr(), H,
                                           cfg.min_neighbors_for_factor, rho.data_ptr(), fac.data_ptr(),
                                           cnt.data_ptr(), stream(dev)), "density_factor")
    acc = torch.zeros(n, 3, device=dev)
    vstar = torch.zeros(n, 3, device=dev)
    _lib.check(lib.fs_dfsph_nonpressure_predict(grid._ctx, C.byref(ms), s_in.particle_q.data_ptr(),
                                                s_in.particle_qd.data_ptr(), rho.data_ptr(), H, 0.5 * SPACING, dt,
                                                acc.data_ptr(), vstar.data_ptr(), stream(dev)), "nonpressure")
    torch.cuda.synchronize()
    assert torch.equal(acc, solver._particle_accel)
    want = s_in.particle_qd.double() + dt * acc.double()
    assert rel_err(vstar.cpu().numpy() - v, want.cpu().numpy() - v) <= TOL


def test_pbf_predict_matches_formula(cuda_device):
    """v_pred = v + dt g, x_pred = x + dt v_pred, clamped into the walls inset
    by the radius (solver_pbf.py:193-224, 367-399)."""
    dev = cuda_device
    x, v = block(seed=7)
    v = v * 20.0  # fast enough to cross the walls in one predict
    n = len(x)
    m = model_for(SolverPBF, x, v, dev)
    lib = _lib.load()
    ms = cm.model_struct(m)
    grid = HashGrid(device=dev)
    grid.reserve(n)
    p = _lib.PbfParams()
    p.dt, p.particle_radius = 1.0 / 240.0, 0.5 * SPACING
    p.bound_width, p.bound_height, p.bound_length = 0.2, 0.2, 0.15
    xt, vt = T(x, dev), T(v, dev)
    xp = torch.zeros(n, 3, device=dev)
    vp = torch.zeros(n, 3, device=dev)
    _lib.check(lib.fs_pbf_predict(grid._ctx, C.byref(ms), xt.data_ptr(), vt.data_ptr(), C.byref(p), xp.data_ptr(),
                                  vp.data_ptr(), stream(dev)), "predict")
    torch.cuda.synchronize()
    dt = np.float64(p.dt)
    vw = v.astype(np.float64) + dt * np.array([0.0, 0.0, -10.0])
    xw = x.astype(np.float64) + dt * vw
    r = np.float64(np.float32(0.5 * SPACING))
    lo = np.array([-0.2 + r, -0.2 + r, r])
    hi = np.array([0.2 - r, 0.2 - r, 0.3 - r])
    clamped = (xw < lo) | (xw > hi)
    xw = np.clip(xw, lo, hi)
    assert clamped.any()  # the walls act
    assert np.abs(vp.cpu().numpy() - vw).max() <= 1e-6 * np.abs(vw).max()
    assert np.abs(xp.cpu().numpy() - xw).max() <= 1e-6 * np.abs(xw).max()
