"""Edge cases of the drop-in step (reference behaviour in parentheses):

  - a model without particles: step returns at once (solver_*.py early
    return for particle_count == 0);
  - every particle inactive: positions and velocities pass through, density
    and pressure are zero (inactive particles are skipped by every kernel);
  - particles active but masked (particle_mask != 0): they do not move but
    push their neighbours (non-dynamic = active and unmasked);
  - a single particle: no grid is attached (the reference attaches one for
    more than one particle), so the step raises; with a grid, rho = m W(0);
  - positions far outside the 128^3 hash range: cells alias, and the step
    still matches the oracle (candidates are filtered by distance);
  - more particles than a context holds: a clear capacity error;
  - non-finite positions: the grid bins them apart and raises the status
    word; every finite particle's step is bit-identical to the step of the
    finite particles alone (in the reference a NaN candidate would turn its
    neighbours' sums into NaN; its harness rejects such a state).
"""

import ctypes as C

import numpy as np
import pytest
import torch

from fluid_simulation_b200 import _lib
from fluid_simulation_b200.newton_shim import HashGrid, model_from_arrays
from fluid_simulation_b200.solver import SolverDFSPH, SolverPBF, SolverWCSPH
from fluid_simulation_b200.solver import _common as cm
from golden_io import compare_fields, oracle_outputs

pytestmark = pytest.mark.gpu
SP = 0.01
KINDS = {"wcsph": (SolverWCSPH, SolverWCSPH.SphConfig, 1e-4), "dfsph": (SolverDFSPH, SolverDFSPH.SphConfig, 1e-3),
         "pbf": (SolverPBF, SolverPBF.PbfConfig, 1e-3)}


def lattice(side=8, offset=(0.0, 0.0, 0.1), seed=0):
    rng = np.random.default_rng(seed)
    g = np.arange(side) * SP
    x = np.stack(np.meshgrid(g, g, g, indexing="ij"), -1).reshape(-1, 3) + np.array(offset)
    x = x + rng.uniform(-0.02, 0.02, x.shape) * SP
    v = rng.normal(size=x.shape) * 0.1
    return x.astype(np.float32), v.astype(np.float32)


def make(kind, x, v, dev, flags=None, mask=0):
    cls, cfg_cls, dt = KINDS[kind]
    attrs = dict(particle_mask=mask, rest_density=1000.0, surface_tension=0.0, viscosity=1e-3)
    if kind == "wcsph":
        attrs.update(stiffness=2.5e5, exponent=7.0)
    m = model_from_arrays(x, v, 1000.0 * SP ** 3, device=dev, flags=flags, radius=0.5 * SP, attributes=attrs,
                          solver_cls=cls)
    cfg = cfg_cls(particle_radius=0.5 * SP, particle_length=SP, smoothing_length_coff=2.0, bound_width=1e4,
                  bound_height=1e4, bound_length=1e4, boundary_damping=0.0)
    return m, cls(m, cfg), dt


@pytest.mark.parametrize("kind", list(KINDS))
def test_empty_model_returns_at_once(kind, cuda_device):
    x = np.zeros((0, 3), np.float32)
    m, solver, dt = make(kind, x, x, cuda_device)
    a, b = m.state(), m.state()
    solver.step(a, b, None, None, dt)
    torch.cuda.synchronize()
    assert b.particle_q.shape == (0, 3)


@pytest.mark.parametrize("kind", list(KINDS))
def test_all_inactive_particles_pass_through(kind, cuda_device):
    x, v = lattice()
    m, solver, dt = make(kind, x, v, cuda_device, flags=np.zeros(len(x), np.int32))
    a, b = m.state(), m.state()
    solver.step(a, b, None, None, dt)
    torch.cuda.synchronize()
    assert torch.equal(b.particle_q, a.particle_q)
    assert torch.equal(b.particle_qd, a.particle_qd) or kind == "dfsph"  # DFSPH: v* of a non-dynamic particle is 0
    assert float(b.sph.rho.abs().max()) == 0.0


@pytest.mark.parametrize("kind", list(KINDS))
def test_masked_particles_stay_and_push(kind, cuda_device):
    """Half of a compressed lattice masked: the masked half keeps its
    positions; the free half matches the oracle (it feels the masked half)."""
    x, v = lattice(side=8)
    x = (x * 0.95).astype(np.float32)
    mask = (x[:, 0] < x[:, 0].mean()).astype(np.int32)
    m, solver, dt = make(kind, x, v, cuda_device, mask=mask)
    a, b = m.state(), m.state()
    solver.step(a, b, None, None, dt)
    torch.cuda.synchronize()
    q = b.particle_q.cpu().numpy()
    assert np.array_equal(q[mask == 1], x[mask == 1])
    assert not np.array_equal(q[mask == 0], x[mask == 0])
    n = len(x)
    cls, cfg_cls, _ = KINDS[kind]
    model = dict(particle_flags=np.ones(n, np.int32), particle_mass=np.full(n, 1000.0 * SP ** 3, np.float32),
                 particle_world=np.zeros(n, np.int32), gravity=np.array([[0, 0, -10.0]], np.float32),
                 particle_max_radius=0.5 * SP,
                 sph=dict(particle_mask=mask, rest_density=np.full(n, 1000.0, np.float32),
                          surface_tension=np.zeros(n, np.float32), viscosity=np.full(n, 1e-3, np.float32),
                          stiffness=np.full(n, 2.5e5, np.float32), exponent=np.full(n, 7.0, np.float32)))
    from dataclasses import asdict
    cfg = asdict(solver.config)
    state = dict(particle_q=x, particle_qd=v, sph=dict(kappa=np.zeros(n, np.float32), kappa_v=np.zeros(n, np.float32)))
    ref32 = oracle_outputs(kind, model, state, cfg, dt, "f32")
    ref64 = oracle_outputs(kind, model, state, cfg, dt, "f64")
    errors, _ = compare_fields([("particle_q", q, ref32["particle_q"])], ref64, kind=kind)
    assert not errors, errors


@pytest.mark.parametrize("kind", list(KINDS))
def test_single_particle_density_is_its_own_weight(kind, cuda_device):
    """A one-particle model gets no grid (the reference attaches one only for
    more than one particle), so its step raises as the reference's does; with
    a grid attached by hand, its density is m W(0)."""
    x = np.array([[0.1, 0.2, 0.3]], np.float32)
    v = np.zeros_like(x)
    m, solver, dt = make(kind, x, v, cuda_device)
    a, b = m.state(), m.state()
    with pytest.raises(RuntimeError, match="particle_grid"):
        solver.step(a, b, None, None, dt)
    m.particle_grid = HashGrid(device=cuda_device)
    solver.step(a, b, None, None, dt)
    torch.cuda.synchronize()
    h = 2.0 * SP
    mass = np.float32(1000.0 * SP ** 3)
    w0 = 315.0 / (64.0 * np.pi * h ** 9) * h ** 6 if kind == "pbf" else 8.0 / (np.pi * h ** 3)
    assert abs(float(b.sph.rho[0]) - mass * w0) <= 1e-5 * mass * w0


@pytest.mark.parametrize("kind", list(KINDS))
def test_far_positions_alias_in_the_hash_and_keep_parity(kind, cuda_device):
    """A lattice around x = 1000 m: cell coordinates far beyond 128 wrap onto
    cells of other lattice parts; candidates from aliased cells fail the
    distance test and the step matches the oracle."""
    x, v = lattice(side=8, offset=(1000.0, -300.0, 2.0))
    x2, v2 = lattice(side=6, offset=(1000.0 + 128 * 2 * SP, -300.0, 2.0), seed=1)  # 128 cells away: aliased
    x, v = np.concatenate([x, x2]), np.concatenate([v, v2])
    m, solver, dt = make(kind, x, v, cuda_device)
    a, b = m.state(), m.state()
    solver.step(a, b, None, None, dt)
    torch.cuda.synchronize()
    n = len(x)
    from dataclasses import asdict
    model = dict(particle_flags=np.ones(n, np.int32), particle_mass=np.full(n, 1000.0 * SP ** 3, np.float32),
                 particle_world=np.zeros(n, np.int32), gravity=np.array([[0, 0, -10.0]], np.float32),
                 particle_max_radius=0.5 * SP,
                 sph=dict(particle_mask=np.zeros(n, np.int32), rest_density=np.full(n, 1000.0, np.float32),
                          surface_tension=np.zeros(n, np.float32), viscosity=np.full(n, 1e-3, np.float32),
                          stiffness=np.full(n, 2.5e5, np.float32), exponent=np.full(n, 7.0, np.float32)))
    state = dict(particle_q=x, particle_qd=v, sph=dict(kappa=np.zeros(n, np.float32), kappa_v=np.zeros(n, np.float32)))
    ref32 = oracle_outputs(kind, model, state, asdict(solver.config), dt, "f32")
    ref64 = oracle_outputs(kind, model, state, asdict(solver.config), dt, "f64")
    got = dict(particle_q=b.particle_q.cpu().numpy(), particle_qd=b.particle_qd.cpu().numpy(),
               rho=b.sph.rho.cpu().numpy())
    errors, _ = compare_fields([(k, got[k], ref32[k]) for k in got], ref64, kind=kind)
    assert not errors, errors


def test_more_particles_than_capacity_is_refused(cuda_device):
    x, v = lattice(side=6)
    m, solver, dt = make("wcsph", x, v, cuda_device)
    grid = HashGrid(device=cuda_device)
    grid.reserve(10)
    lib = _lib.load()
    stream = torch.cuda.current_stream(cuda_device).cuda_stream
    xt = m.particle_q
    rc = lib.fs_grid_build(grid._ctx, xt.data_ptr(), xt.shape[0], 0.02, stream)
    assert rc == _lib.FS_ERR_CAPACITY
    assert b"capacity" in lib.fs_last_error_string()
    ms = cm.model_struct(m, wcsph=True)
    rho = torch.zeros(len(x), device=cuda_device)
    rc = lib.fs_wcsph_density(grid._ctx, C.byref(ms), xt.data_ptr(), 0.02, 1, rho.data_ptr(), rho.data_ptr(), stream)
    assert rc == _lib.FS_ERR_NOGRID  # no grid was built for these points


@pytest.mark.parametrize("kind", ["wcsph", "pbf"])
def test_nonfinite_particles_leave_the_others_bit_identical(kind, cuda_device):
    x, v = lattice(side=12, offset=(-0.05, -0.05, 0.1), seed=4)
    bad = np.array([7, 300, 1000, 1500])
    xb = x.copy()
    xb[bad[0], 0], xb[bad[1], 1], xb[bad[2], 2], xb[bad[3]] = np.nan, np.inf, -np.inf, np.nan
    ok = np.setdiff1d(np.arange(len(x)), bad)
    outs = []
    for xx, vv in ((xb, v), (x[ok], v[ok])):
        m, solver, dt = make(kind, xx, vv, cuda_device)
        a, b = m.state(), m.state()
        solver.step(a, b, None, None, dt)
        torch.cuda.synchronize()
        outs.append((m, {"q": b.particle_q.cpu().numpy(), "qd": b.particle_qd.cpu().numpy(),
                         "rho": b.sph.rho.cpu().numpy()}))
    (m_bad, with_bad), (_, alone) = outs
    for k in alone:
        np.testing.assert_array_equal(with_bad[k][ok], alone[k], err_msg=k)
    assert np.isfinite(with_bad["q"][ok]).all()
    assert m_bad.particle_grid.status() & _lib.FS_STATUS_NONFINITE
