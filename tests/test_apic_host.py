"""APIC particle separation, host side (no GPU): the oracle restatement
against the golden fixture produced by the reference's own kernels
(solver/apic/solver_apic.py:193-266 through the loop of
_apply_particle_separation, 1003-1064, tests/golden/make_golden.py), and the
parameter derivation of ParticleSeparation against the reference's."""

import json
import types

import numpy as np

import oracle
from fluid_simulation_b200.apic import ParticleSeparation
from golden_io import GOLDEN as GOLDEN_DIR


def golden():
    z = np.load(f"{GOLDEN_DIR}/apic_separation.npz")
    return z, json.loads(str(z["config"]))


def test_oracle_equals_reference_kernels_bit_for_bit():
    z, cfg = golden()
    x, d = oracle.apic_separation(z["in_x"], z["flags"], cfg, "f32")
    assert np.array_equal(x, z["out_x"])
    assert np.array_equal(d, z["out_delta"])
    # the fixture exercises the pass: most particles move, some sit in wall bands
    assert np.count_nonzero(np.abs(z["out_x"] - z["in_x"]).max(1)) > 0.9 * len(x)


def test_oracle_f64_agrees_with_f32():
    z, cfg = golden()
    x32, _ = oracle.apic_separation(z["in_x"], z["flags"], cfg, "f32")
    x64, _ = oracle.apic_separation(z["in_x"], z["flags"], cfg, "f64")
    assert np.abs(x64 - x32).max() < 1e-6


def test_parameters_follow_the_reference_derivation():
    z, cfg = golden()
    n = len(z["in_x"])
    model = types.SimpleNamespace(particle_count=n, particle_radius=np.full(n, cfg["radius"], np.float32))
    sep = ParticleSeparation(model, ParticleSeparation.Config(bound_lo=tuple(cfg["bound_lo"]),
                                                              bound_hi=tuple(cfg["bound_hi"])))
    p = sep.parameters()
    for k in ("rest_dist", "query_radius", "strength", "iterations", "wall_band", "wall_margin"):
        assert p[k] == cfg[k], k
    assert list(p["dims"]) == cfg["dims"]
    # explicit values override the derived ones
    sep = ParticleSeparation(model, ParticleSeparation.Config(separation_rest_dist=0.02, wall_margin=0.001,
                                                              wall_push_band=0.05, separation_iterations=0))
    p = sep.parameters()
    assert p["rest_dist"] == 0.02 and p["wall_margin"] == 0.001 and p["wall_band"] == 0.05 and p["iterations"] == 1
    assert p["dims"] == (100, 100, 100)
