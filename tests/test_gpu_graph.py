"""Whole-frame CUDA graphs: replaying a captured frame gives bit-identical
results to launching the same substeps one by one (the grid build ranks
particles inside cells deterministically, DFSPH reduces its residual in a
fixed order, so repeated runs are reproducible)."""

import numpy as np
import pytest
import torch

from fluid_simulation_b200.dam_break import material, solver_config
from fluid_simulation_b200.graph import FrameGraph
from fluid_simulation_b200.newton_shim import model_from_arrays
from fluid_simulation_b200.scene import make_scene
from fluid_simulation_b200.solver import SolverDFSPH, SolverPBF, SolverWCSPH

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("kind,cls,dt", [("pbf", SolverPBF, 1.0 / 240.0), ("dfsph", SolverDFSPH, 1.0 / 240.0),
                                         ("wcsph", SolverWCSPH, 1.0e-4)])
def test_frame_graph_matches_plain_launches(kind, cls, dt, cuda_device):
    s = make_scene(20000)
    attrs = dict(material(kind, s), particle_mask=0)
    rng = np.random.default_rng(0)
    v0 = (rng.normal(size=s.positions.shape) * 0.3).astype(np.float32)

    def fresh():
        m = model_from_arrays(s.positions, v0, s.mass, device=cuda_device, radius=s.radius,
                              gravity=(s.spec.gravity,), attributes=attrs, solver_cls=cls)
        return m, cls(m, solver_config(kind, s))

    m1, s1 = fresh()
    a, b = m1.state(), m1.state()
    for _ in range(8):
        s1.step(a, b, None, None, dt)
        a, b = b, a
    m2, s2 = fresh()
    g = FrameGraph(s2, m2.state(), m2.state(), dt, substeps=4, warmup=False)
    g.replay()
    out = g.replay()
    torch.cuda.synchronize()
    assert torch.equal(out.particle_q, a.particle_q)
    assert torch.equal(out.particle_qd, a.particle_qd)
    assert torch.equal(out.sph.rho, a.sph.rho)


@pytest.mark.parametrize("method,graph_substeps,frames", [("wcsph", 16, 2), ("dfsph", 2, 3)])
def test_device_frame_loop_equals_host_loop(method, graph_substeps, frames, cuda_device):
    """Dam-break frames with the substep rule evaluated on the device (one
    graph of clocked substeps, replayed until the frame is done) end in the
    same bits, after the same number of substeps, as the reference harness
    loop that reads the maxima back before every substep.  DFSPH starts at
    4 m/s, so that its speed limit (0.4 spacing / |v|) cuts its substeps
    below 1/240 s."""
    from fluid_simulation_b200.dam_break import DamBreakSimulation
    from fluid_simulation_b200.graph import DeviceFrameLoop

    s = make_scene(10000)
    host = DamBreakSimulation(s, method, device=cuda_device)
    dev = DamBreakSimulation(s, method, device=cuda_device)
    if method == "dfsph":
        for sim in (host, dev):
            sim.state_0.particle_qd[:, 0] = 4.0
    loop = DeviceFrameLoop(dev, graph_substeps=graph_substeps)
    counts = []
    for _ in range(frames):
        host.step()
        loop.step()
        torch.cuda.synchronize()
        assert dev.last_substeps == host.last_substeps
        counts.append(host.last_substeps)
    assert max(counts) > graph_substeps  # several replays per frame
    assert torch.equal(dev.state_0.particle_q, host.state_0.particle_q)
    assert torch.equal(dev.state_0.particle_qd, host.state_0.particle_qd)
    assert torch.equal(dev.state_0.sph.rho, host.state_0.sph.rho)
    assert dev.total_substeps == host.total_substeps


def test_device_frame_loop_reports_nonfinite_state(cuda_device):
    from fluid_simulation_b200.dam_break import DamBreakSimulation
    from fluid_simulation_b200.graph import DeviceFrameLoop

    sim = DamBreakSimulation(make_scene(3000), "wcsph", device=cuda_device)
    loop = DeviceFrameLoop(sim, graph_substeps=4)
    sim.state_0.particle_qd[7, 2] = float("nan")
    with pytest.raises(RuntimeError, match="Non-finite"):
        loop.step()
