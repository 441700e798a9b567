"""The reference's dam-break known-answer tests (unit_test/unit_test_dam_break.py)
on the GPU, through the drop-in solvers and the restated DamBreakSimulation
harness (CFL maxima and finite checks as device reductions)."""

from dataclasses import replace

import numpy as np
import pytest
import torch

from fluid_simulation_b200.dam_break import DamBreakSimulation
from fluid_simulation_b200.scene import DEFAULT_SPEC, ParticleScene, make_scene
from kat_util import OracleDamBreak
from numpy_metrics import numpy_frame_metrics

pytestmark = pytest.mark.gpu


def test_finite_check_detects_invalid_state_between_metrics(cuda_device):
    # unit_test_dam_break.py:39-46 (fault injected from the host)
    sim = DamBreakSimulation(make_scene(512), "pbf", device=cuda_device)
    sim.check_finite()
    sim.state_0.particle_q[0, 0] = float("nan")
    with pytest.raises(RuntimeError, match="Non-finite"):
        sim.check_finite()


def test_solvers_share_initial_particles_and_mass(cuda_device):
    # unit_test_dam_break.py:48-57
    scene = make_scene(512)
    for method in ("wcsph", "dfsph", "pbf"):
        sim = DamBreakSimulation(scene, method, device=cuda_device)
        np.testing.assert_array_equal(sim.state_0.particle_q.cpu().numpy(), scene.positions)
        np.testing.assert_array_equal(sim.state_0.particle_qd.cpu().numpy(), 0.0)
        np.testing.assert_allclose(sim.model.particle_radius.cpu().numpy(), scene.radius)
        np.testing.assert_allclose(sim.model.particle_mass.cpu().numpy(), scene.mass)
        np.testing.assert_allclose(sim.model.gravity.cpu().numpy()[0], scene.spec.gravity)


def test_every_method_advances_complete_frames(cuda_device):
    # unit_test_dam_break.py:59-75
    scene = make_scene(512)
    for method in ("wcsph", "dfsph", "pbf"):
        sim = DamBreakSimulation(scene, method, device=cuda_device, substeps=4)
        for frame in range(1, 3):
            sim.step()
            assert sim.sim_time == frame / 60.0
            assert sim.last_substeps >= 4
            assert sim.metrics()["finite"]
            x = sim.state_0.particle_q.cpu().numpy()
            assert np.all(x >= np.asarray(scene.spec.bound_lo) - 1e-6)
            assert np.all(x <= np.asarray(scene.spec.bound_hi) + 1e-6)
        if method == "wcsph":
            assert sim.total_substeps > 8


def test_underdense_block_falls_without_pressure_attraction(cuda_device):
    # unit_test_dam_break.py:79-91
    sim = DamBreakSimulation(make_scene(512), "wcsph", device=cuda_device)
    sim.step()
    assert np.all(sim.state_0.sph.rho.cpu().numpy() < 1000.0)
    np.testing.assert_array_equal(sim.state_0.sph.pressure.cpu().numpy(), 0.0)
    expected = np.tile(np.asarray(sim.scene.spec.gravity) * sim.frame_dt, (sim.scene.count, 1))
    np.testing.assert_allclose(sim.state_0.particle_qd.cpu().numpy(), expected, atol=1e-7)
    signed = DamBreakSimulation(make_scene(512), "wcsph", device=cuda_device, wcsph_clamp_negative_pressure=False)
    signed.step()
    assert np.any(signed.state_0.sph.pressure.cpu().numpy() < 0.0)
    assert signed.metrics()["speed_max"] > sim.metrics()["speed_max"]


def test_compressed_particles_repel_and_conserve_momentum(cuda_device):
    # unit_test_dam_break.py:93-107
    d = 0.01
    center = np.asarray([0.0, 0.0, 0.5], dtype=np.float32)
    offsets = np.asarray([[1, 1, 1], [1, -1, -1], [-1, 1, -1], [-1, -1, 1]], dtype=np.float32) * (0.05 * d)
    scene = ParticleScene(replace(DEFAULT_SPEC, gravity=(0.0, 0.0, 0.0), target_count=4), center + offsets,
                          1000.0 * d ** 3, d * 0.5, d ** 3, d)
    sim = DamBreakSimulation(scene, "wcsph", device=cuda_device, wcsph_viscosity=0.0)
    sim._substep(1e-6)
    assert np.all(sim.state_0.sph.rho.cpu().numpy() > 1000.0)
    assert np.all(sim.state_0.sph.pressure.cpu().numpy() > 0.0)
    velocity = sim.state_0.particle_qd.cpu().numpy()
    assert np.all(np.sum(velocity * offsets, axis=1) > 0.0)
    np.testing.assert_allclose(velocity.sum(axis=0), 0.0, atol=1e-6)


def test_cfl_reduction_preserves_maxima_and_rejects_nonfinite_values(cuda_device):
    # unit_test_dam_break.py:109-130
    sim = DamBreakSimulation(make_scene(512), "wcsph", device=cuda_device)
    rng = np.random.default_rng(42)
    velocity = rng.normal(size=(sim.scene.count, 3)).astype(np.float32)
    acceleration = (rng.normal(size=velocity.shape) * 20).astype(np.float32)
    sim.state_0.particle_qd.copy_(torch.as_tensor(velocity))
    sim.solver._particle_accel.copy_(torch.as_tensor(acceleration))
    sim.total_substeps = 1
    speed, accel = sim._cfl_maxima()
    np.testing.assert_allclose([speed, accel], [np.linalg.norm(velocity, axis=1).max(),
                                                np.linalg.norm(acceleration, axis=1).max()], rtol=1e-6)
    velocity[0, 0] = np.nan
    sim.state_0.particle_qd.copy_(torch.as_tensor(velocity))
    with pytest.raises(RuntimeError, match="Non-finite velocity"):
        sim._cfl_maxima()
    velocity[0, 0] = 0.0
    sim.state_0.particle_qd.copy_(torch.as_tensor(velocity))
    acceleration[0, 0] = np.inf
    sim.solver._particle_accel.copy_(torch.as_tensor(acceleration))
    with pytest.raises(RuntimeError, match="Non-finite WCSPH acceleration"):
        sim._cfl_maxima()


def test_viscous_timestep_damps_velocity_and_completes_frame(cuda_device):
    # unit_test_dam_break.py:132-151
    sim = DamBreakSimulation(make_scene(512), "wcsph", device=cuda_device, wcsph_viscosity=10.0)
    velocity = np.zeros((sim.scene.count, 3), dtype=np.float32)
    velocity[:, 0] = np.where(np.arange(sim.scene.count) % 2, -0.01, 0.01)
    sim.state_0.particle_qd.copy_(torch.as_tensor(velocity))
    sim.model.set_gravity((0.0, 0.0, 0.0))
    dts = []
    advance = sim._substep

    def record_and_advance(dt):
        dts.append(dt)
        advance(dt)

    sim._substep = record_and_advance
    sim.step()
    sim.check_finite()
    assert max(dts) <= 0.025 * sim.solver.smoothing_length ** 2 / 10.0
    assert sum(dts) == pytest.approx(sim.frame_dt)
    assert np.sum(sim.state_0.particle_qd.cpu().numpy() ** 2) < np.sum(velocity ** 2)


@pytest.mark.parametrize("method", ["wcsph", "pbf", "dfsph"])
def test_multi_frame_statistics_track_oracle(method, cuda_device):
    """Chaotic trajectories diverge, so several frames are compared through
    density-error and kinetic-energy statistics (GPU harness vs CPU oracle
    harness on the same scene)."""
    scene = make_scene(2000)
    gpu = DamBreakSimulation(scene, method, device=cuda_device)
    cpu = OracleDamBreak(scene, method)
    for _ in range(3):
        gpu.step()
        cpu.step()
    assert gpu.total_substeps == cpu.total_substeps
    rho_g = gpu.state_0.sph.rho.cpu().numpy().astype(np.float64)
    rho_c = cpu.sph["rho"].astype(np.float64)
    v_g = gpu.state_0.particle_qd.cpu().numpy().astype(np.float64)
    ke_g, ke_c = 0.5 * scene.mass * (v_g ** 2).sum(), 0.5 * scene.mass * (cpu.v.astype(np.float64) ** 2).sum()
    assert abs(ke_g - ke_c) <= 1e-3 * ke_c
    for q in (1, 50, 99):
        assert abs(np.percentile(rho_g, q) - np.percentile(rho_c, q)) <= 1e-3 * 1000.0


@pytest.mark.parametrize("method", ["wcsph", "pbf", "dfsph"])
def test_device_metrics_equal_numpy_metrics(method, cuda_device):
    """fs_frame_metrics against the reference's numpy reductions on the same
    state: minima, maxima, speed maximum and the density percentile exact,
    means to 1e-6 relative."""
    from fluid_simulation_b200.dam_break import DamBreakSimulation
    from fluid_simulation_b200.scene import make_scene

    sim = DamBreakSimulation(make_scene(20000), method, device=cuda_device)
    for frame in range(2):
        dev, host = sim.metrics(), numpy_frame_metrics(sim)
        assert set(dev) == set(host)
        for k, want in host.items():
            got = dev[k]
            if k.endswith("_mean"):
                assert abs(got - want) <= 1e-6 * abs(want), k
            else:
                assert got == want, (k, got, want)
        sim.step()


def test_device_metrics_report_nonfinite_state(cuda_device):
    from fluid_simulation_b200.dam_break import DamBreakSimulation
    from fluid_simulation_b200.scene import make_scene

    sim = DamBreakSimulation(make_scene(3000), "wcsph", device=cuda_device)
    sim.step()
    sim.state_0.sph.pressure[5] = float("inf")
    with pytest.raises(RuntimeError, match="Non-finite pressure"):
        sim.metrics()
    sim.state_0.particle_q[3, 1] = float("nan")
    with pytest.raises(RuntimeError, match="Non-finite particle state"):
        sim.metrics()


@pytest.mark.parametrize("method", ["wcsph", "dfsph", "pbf"])
def test_resume_from_snapshot_equals_uninterrupted_run(method, cuda_device, tmp_path):
    """Two frames straight through against one frame, a snapshot on disk, a
    fresh simulation restored from it and one more frame: same bits, same
    substep count."""
    from fluid_simulation_b200 import snapshot
    scene = make_scene(5000)
    a = DamBreakSimulation(scene, method, device=cuda_device)
    a.step()
    path = tmp_path / f"{method}.npz"
    info = snapshot.save_simulation(path, a)
    assert info["initial_position_sha256"] == scene.report()["initial_position_sha256"] and info["frame"] == 1
    a.step()
    b = DamBreakSimulation(make_scene(5000), method, device=cuda_device)
    snapshot.restore_simulation(path, b)
    b.step()
    torch.cuda.synchronize()
    assert b.frame == a.frame == 2 and b.total_substeps == a.total_substeps
    assert torch.equal(a.state_0.particle_q, b.state_0.particle_q)
    assert torch.equal(a.state_0.particle_qd, b.state_0.particle_qd)
    other = DamBreakSimulation(make_scene(4000), method, device=cuda_device)
    with pytest.raises(ValueError, match="another scene"):
        snapshot.restore_simulation(path, other)
