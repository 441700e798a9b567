"""Launch tuning of the neighbour kernels (fs_context_set_tuning) and the
autotuner: block size and particles per thread change no bit of any
solver's result; WCSPH's half-width cells keep the parity rule against the
oracle; invalid tunings are refused; autotune() leaves the fastest tuning on
the context and the state untouched."""

import ctypes as C

import numpy as np
import pytest
import torch

from fluid_simulation_b200 import _lib
from fluid_simulation_b200.autotune import Tuning, autotune, candidates, get_tuning, set_tuning
from fluid_simulation_b200.batch import batched_model, make_batch
from fluid_simulation_b200.dam_break import material, solver_config
from fluid_simulation_b200.newton_shim import model_from_arrays
from fluid_simulation_b200.scene import make_scene
from fluid_simulation_b200.solver import SolverDFSPH, SolverPBF, SolverWCSPH
from golden_io import compare_fields, oracle_outputs

pytestmark = pytest.mark.gpu
SOLVERS = {"wcsph": (SolverWCSPH, 1e-4), "dfsph": (SolverDFSPH, 1.0 / 240.0), "pbf": (SolverPBF, 1.0 / 240.0)}


def setup(kind, dev, target=20000):
    s = make_scene(target)
    cls, dt = SOLVERS[kind]
    v0 = (np.random.default_rng(0).normal(size=s.positions.shape) * 0.3).astype(np.float32)
    m = model_from_arrays(s.positions, v0, s.mass, device=dev, radius=s.radius, gravity=(s.spec.gravity,),
                          attributes=dict(material(kind, s), particle_mask=0), solver_cls=cls)
    return s, m, cls(m, solver_config(kind, s)), dt


def step_outputs(m, solver, dt):
    a, b = m.state(), m.state()
    solver.step(a, b, None, None, dt)
    torch.cuda.synchronize()
    out = {"q": b.particle_q.clone(), "qd": b.particle_qd.clone()}
    out.update({k: v.clone() for k, v in vars(b.sph).items()})
    return out


@pytest.mark.parametrize("kind", ["wcsph", "dfsph", "pbf"])
def test_block_size_and_particles_per_thread_change_no_result(kind, cuda_device):
    _, m, solver, dt = setup(kind, cuda_device)
    ctx = m.particle_grid._ctx
    ref = step_outputs(m, solver, dt)
    for t in (Tuning(64, 1, 1.0), Tuning(256, 2, 1.0), Tuning(128, 4, 1.0)):
        set_tuning(ctx, t)
        assert get_tuning(ctx) == t
        got = step_outputs(m, solver, dt)
        for k in ref:
            assert torch.equal(got[k], ref[k]), (t, k)


def test_pbf_list_skin_changes_no_result(cuda_device):
    """The first lambda pass reuses the first density's lists when every
    particle moved less than list_skin h / 2 in between.  Skin off, default
    and largest: the same bits.  With a strong cohesion the non-pressure
    update moves particles past the skin and the device falls back to
    scanning: the same bits again, and no reuse counted."""
    lib = _lib.load()
    for gamma in (0.0, 1.0):
        s, m, solver, dt = setup("pbf", cuda_device)
        if gamma:
            m.sph.surface_tension.fill_(gamma)
        ctx = m.particle_grid._ctx
        _lib.check(lib.fs_list_stats_enable(ctx, 1), "stats")
        counters = (C.c_int64 * 3)()
        outs, reused = {}, {}
        for skin in (0.0, 0.02, 0.25):
            set_tuning(ctx, Tuning(128, 1, 1.0, skin))
            _lib.check(lib.fs_list_stats(ctx, counters, 3, 1), "stats")
            outs[skin] = step_outputs(m, solver, dt)
            _lib.check(lib.fs_list_stats(ctx, counters, 3, 1), "stats")
            assert counters[0] + counters[1] == s.count  # the XSPH lists of the final density
            reused[skin] = counters[2]
        for skin in (0.02, 0.25):
            for k in outs[0.0]:
                assert torch.equal(outs[skin][k], outs[0.0][k]), (gamma, skin, k)
        assert reused[0.0] == 0
        if gamma == 0.0:
            assert reused[0.02] > 0.9 * s.count, reused
        else:
            assert reused[0.02] == 0, reused
        _lib.check(lib.fs_list_stats_enable(ctx, 0), "stats")


def test_wcsph_half_cells_keep_parity(cuda_device):
    s, m, solver, dt = setup("wcsph", cuda_device, target=10000)
    set_tuning(m.particle_grid._ctx, Tuning(128, 1, 0.5))
    a, b = m.state(), m.state()
    solver.step(a, b, None, None, dt)
    torch.cuda.synchronize()
    n = s.count
    model = dict(particle_flags=np.ones(n, np.int32), particle_mass=np.full(n, s.mass, np.float32),
                 particle_world=np.zeros(n, np.int32), gravity=np.array([s.spec.gravity], np.float32),
                 particle_max_radius=s.radius,
                 sph=dict(particle_mask=np.zeros(n, np.int32),
                          **{k: np.full(n, v, np.float32) for k, v in material("wcsph", s).items()}))
    state = dict(particle_q=s.positions, particle_qd=a.particle_qd.cpu().numpy(), sph={})
    from dataclasses import asdict
    cfg = asdict(solver_config("wcsph", s))
    ref32 = oracle_outputs("wcsph", model, state, cfg, dt, "f32")
    ref64 = oracle_outputs("wcsph", model, state, cfg, dt, "f64")
    got = dict(particle_q=b.particle_q.cpu().numpy(), particle_qd=b.particle_qd.cpu().numpy(),
               accel=solver._particle_accel.cpu().numpy(), rho=b.sph.rho.cpu().numpy(),
               pressure=b.sph.pressure.cpu().numpy())
    errors, _ = compare_fields([(k, got[k], v) for k, v in ref32.items()], ref64, kind="wcsph")
    assert not errors, errors


def test_invalid_tunings_are_refused(cuda_device):
    _, m, _, _ = setup("pbf", cuda_device, target=3000)
    lib = _lib.load()
    for bad in ((96, 1, 1.0, 0.02), (128, 3, 1.0, 0.02), (128, 1, 0.7, 0.02), (128, 1, 1.0, -0.1),
                (128, 1, 1.0, 0.3)):
        rc = lib.fs_context_set_tuning(m.particle_grid._ctx, C.byref(_lib.Tuning(*bad)))
        assert rc == _lib.FS_ERR_INVALID
    b = make_batch(n_scenes=2, seed=1, n_lo=1000, n_hi=2000)
    mb = batched_model(b, SolverWCSPH, device=cuda_device)
    rc = lib.fs_context_set_tuning(mb.particle_grid._ctx, C.byref(_lib.Tuning(128, 1, 0.5)))
    assert rc == _lib.FS_ERR_INVALID


def test_autotune_keeps_the_fastest_and_leaves_the_state(cuda_device):
    _, m, solver, dt = setup("pbf", cuda_device, target=20000)
    state = m.state()
    before = state.particle_q.clone()
    res = autotune(solver, state, dt, steps=2, repeats=1)
    assert res["chosen"] in candidates("pbf")
    assert get_tuning(m.particle_grid._ctx) == res["chosen"]
    assert min(res["times_ms"].values()) == res["times_ms"][res["chosen"]]
    assert torch.equal(state.particle_q, before)
