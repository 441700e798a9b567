"""APIC particle separation on the GPU (fs_apic_separation through
ParticleSeparation): bit-for-bit equal to the golden fixture made by the
reference's own kernels, and to the oracle on a dam-break column with
clumping, inactive particles and particles in the wall bands."""

import json

import numpy as np
import pytest
import torch

import oracle
from fluid_simulation_b200 import _lib
from fluid_simulation_b200.apic import ParticleSeparation
from fluid_simulation_b200.newton_shim import model_from_arrays
from fluid_simulation_b200.scene import make_scene
from golden_io import GOLDEN

pytestmark = pytest.mark.gpu


def run(x, flags, radius, dev, **cfg):
    m = model_from_arrays(x, np.zeros_like(x), 1.0, device=dev, flags=flags, radius=radius)
    sep = ParticleSeparation(m, ParticleSeparation.Config(**cfg))
    st = m.state()
    sep.apply(st)
    torch.cuda.synchronize()
    return st.particle_q.cpu().numpy(), sep._sep_delta.cpu().numpy(), sep.parameters()


def test_golden_fixture_bit_for_bit(cuda_device):
    z = np.load(f"{GOLDEN}/apic_separation.npz")
    cfg = json.loads(str(z["config"]))
    x, d, p = run(z["in_x"], z["flags"], cfg["radius"], cuda_device, bound_lo=tuple(cfg["bound_lo"]),
                  bound_hi=tuple(cfg["bound_hi"]))
    assert list(p["dims"]) == cfg["dims"]
    assert np.array_equal(x, z["out_x"])
    assert np.array_equal(d, z["out_delta"])


def test_dam_column_matches_oracle(cuda_device):
    s = make_scene(20000)
    rng = np.random.default_rng(4)
    x = (s.positions * np.float32(0.97) + rng.uniform(-0.2, 0.2, s.positions.shape) * s.spacing).astype(np.float32)
    x[:, 2] = np.maximum(x[:, 2], 0.0)
    flags = np.ones(len(x), np.int32)
    flags[rng.choice(len(x), 50, replace=False)] = 0
    lo, hi = s.spec.bound_lo, s.spec.bound_hi
    xg, dg, p = run(x, flags, s.radius, cuda_device, bound_lo=lo, bound_hi=hi, separation_iterations=3)
    xo, do = oracle.apic_separation(x, flags, p, "f32")
    assert np.array_equal(xg, xo)
    assert np.array_equal(dg, do)
    assert np.count_nonzero(np.abs(xg - x).max(1)) > 0.5 * len(x)  # the pass acts
    assert np.array_equal(xg[flags == 0], x[flags == 0])            # inactive particles stay


def test_full_size_dam_matches_oracle(cuda_device):
    """The 401,856-particle dam-break scene, jittered by +-0.2 spacing, two
    separation iterations (the harness default): bit-for-bit equal to the
    oracle."""
    s = make_scene(400000)
    rng = np.random.default_rng(11)
    x = (s.positions + rng.uniform(-0.2, 0.2, s.positions.shape) * s.spacing).astype(np.float32)
    flags = np.ones(len(x), np.int32)
    xg, dg, p = run(x, flags, s.radius, cuda_device, bound_lo=s.spec.bound_lo, bound_hi=s.spec.bound_hi)
    xo, do = oracle.apic_separation(x, flags, p, "f32")
    assert np.array_equal(xg, xo)
    assert np.array_equal(dg, do)
    assert np.count_nonzero(np.abs(xg - x).max(1)) > 0.1 * len(x)  # the pass acts


def test_disabled_or_empty_is_a_no_op(cuda_device):
    x = np.zeros((0, 3), np.float32)
    m = model_from_arrays(x, x, 1.0, device=cuda_device, flags=np.zeros(0, np.int32), radius=0.01)
    sep = ParticleSeparation(m, ParticleSeparation.Config())
    st = m.state()
    sep.apply(st)  # no particles: returns before any launch
    assert sep._sep_delta is None
    x = np.random.default_rng(0).uniform(-0.01, 0.01, (64, 3)).astype(np.float32)
    m = model_from_arrays(x, np.zeros_like(x), 1.0, device=cuda_device, radius=0.005)
    sep = ParticleSeparation(m, ParticleSeparation.Config(enable_particle_separation=False))
    st = m.state()
    sep.apply(st)
    assert torch.equal(st.particle_q.cpu(), torch.as_tensor(x))


def test_batched_context_is_refused(cuda_device):
    from fluid_simulation_b200.batch import batched_model, make_batch
    from fluid_simulation_b200.solver import SolverWCSPH
    b = make_batch(n_scenes=2, seed=1, n_lo=500, n_hi=800)
    m = batched_model(b, SolverWCSPH, device=cuda_device)
    sp = _lib.SeparationParams(rest_dist=0.01, query_radius=0.01, strength=0.5, wall_band=0.0, wall_margin=0.0,
                               iterations=1)
    delta = torch.zeros_like(m.particle_q)
    rc = _lib.load().fs_apic_separation(m.particle_grid._ctx, m.particle_q.data_ptr(),
                                        m.particle_flags.data_ptr(), m.particle_count, sp, delta.data_ptr(), None)
    assert rc == _lib.FS_ERR_INVALID
