"""Known-answer tests of the reference (unit_test/unit_test_dam_break.py)
re-expressed on the CPU oracle.  They pin the oracle to the reference's own
behavioural tests (the GPU versions are in test_gpu_harness.py)."""

from dataclasses import replace

import numpy as np

import oracle
from fluid_simulation_b200.scene import DEFAULT_SPEC, ParticleScene, make_scene
from kat_util import OracleDamBreak


def test_underdense_block_falls_without_pressure_attraction():
    # unit_test_dam_break.py:79-91
    sim = OracleDamBreak(make_scene(512), "wcsph")
    sim.step()
    assert np.all(sim.sph["rho"] < 1000.0)
    np.testing.assert_array_equal(sim.sph["pressure"], 0.0)
    expected = np.tile(np.asarray(sim.scene.spec.gravity) * sim.frame_dt, (sim.scene.count, 1))
    np.testing.assert_allclose(sim.v, expected, atol=1e-7)
    signed = OracleDamBreak(make_scene(512), "wcsph", wcsph_clamp_negative_pressure=False)
    signed.step()
    assert np.any(signed.sph["pressure"] < 0.0)
    assert np.linalg.norm(signed.v, axis=1).max() > np.linalg.norm(sim.v, axis=1).max()


def test_compressed_particles_repel_and_conserve_momentum():
    # unit_test_dam_break.py:93-107
    d = 0.01
    center = np.asarray([0.0, 0.0, 0.5], dtype=np.float32)
    offsets = np.asarray([[1, 1, 1], [1, -1, -1], [-1, 1, -1], [-1, -1, 1]], dtype=np.float32) * (0.05 * d)
    scene = ParticleScene(replace(DEFAULT_SPEC, gravity=(0.0, 0.0, 0.0), target_count=4), center + offsets,
                          1000.0 * d ** 3, d * 0.5, d ** 3, d)
    sim = OracleDamBreak(scene, "wcsph", wcsph_viscosity=0.0)
    sim.substep(1e-6)
    assert np.all(sim.sph["rho"] > 1000.0)
    assert np.all(sim.sph["pressure"] > 0.0)
    assert np.all(np.sum(sim.v * offsets, axis=1) > 0.0)
    np.testing.assert_allclose(sim.v.sum(axis=0), 0.0, atol=1e-6)


def test_viscous_timestep_damps_velocity_and_completes_frame():
    # unit_test_dam_break.py:132-151
    sim = OracleDamBreak(make_scene(512), "wcsph", wcsph_viscosity=10.0, gravity=(0.0, 0.0, 0.0))
    v0 = np.zeros((sim.scene.count, 3), np.float32)
    v0[:, 0] = np.where(np.arange(sim.scene.count) % 2, -0.01, 0.01)
    sim.v = v0.copy()
    sim.step()
    assert max(sim.dts) <= 0.025 * sim.h ** 2 / 10.0
    assert abs(sum(sim.dts) - sim.frame_dt) < 1e-9
    assert np.sum(sim.v ** 2) < np.sum(v0 ** 2)


def test_every_method_advances_complete_frames():
    # unit_test_dam_break.py:59-75 (particle solvers)
    scene = make_scene(512)
    for method in ("wcsph", "dfsph", "pbf"):
        sim = OracleDamBreak(scene, method)
        for _ in range(2):
            sim.step()
            assert np.isfinite(sim.x).all() and np.isfinite(sim.v).all()
            assert np.all(sim.x >= np.asarray(scene.spec.bound_lo) - 1e-6)
            assert np.all(sim.x <= np.asarray(scene.spec.bound_hi) + 1e-6)
        if method == "wcsph":
            assert sim.total_substeps > 8
        else:
            assert sim.total_substeps >= 8


def test_grid_tables_match_brute_force_definition():
    # the restated warp hash grid on a case small enough to enumerate: every
    # point's cell from the truncating conversion, stable order inside cells
    rng = np.random.default_rng(1)
    x = rng.uniform(-0.3, 0.3, (500, 3)).astype(np.float32)
    h = np.float32(0.07)
    t = oracle.grid_build(x, h, (8, 8, 8), 0)
    inv = np.float32(1.0) / h
    c = np.trunc(x * inv).astype(np.int64) + (1 << 20)
    key = (c[:, 2] % 8) * 64 + (c[:, 1] % 8) * 8 + (c[:, 0] % 8)
    order = np.argsort(key, kind="stable")
    np.testing.assert_array_equal(t["point_ids"], order)
    np.testing.assert_array_equal(t["point_cells"], key[order])
