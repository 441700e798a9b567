"""Host-side reference computation of the device frame metrics.

The reference harness (examples/dam_break/simulation.py:198-225) copies the
particle state to the host every frame and reduces it with numpy.  This
module does the same on a ``DamBreakSimulation``'s current state so that the
tests can compare ``DamBreakSimulation.metrics()`` (device reductions)
against it.  Test infrastructure only.
"""

import numpy as np


def _host(t):
    return t.detach().cpu().numpy()


def numpy_frame_metrics(sim):
    state = sim.state_0
    pos, vel = _host(state.particle_q), _host(state.particle_qd)
    if not (np.isfinite(pos).all() and np.isfinite(vel).all()):
        raise RuntimeError(f"Non-finite particle state at frame {sim.frame}")
    height = pos[:, 2]
    out = {
        "frame": sim.frame,
        "simulation_time": sim.sim_time,
        "substeps": sim.last_substeps,
        "total_substeps": sim.total_substeps,
        "finite": True,
        "speed_max": float(np.linalg.norm(vel, axis=1).max(initial=0.0)),
        "height_mean": float(height.mean()),
        "height_min": float(height.min()),
        "height_max": float(height.max()),
    }
    if not sim.frame:  # no density before the first frame
        return out
    rho = _host(state.sph.rho)
    if not np.isfinite(rho).all():
        raise RuntimeError("Non-finite density")
    out.update(density_mean=float(rho.mean()), density_min=float(rho.min()), density_max=float(rho.max()))
    if sim.method != "wcsph":
        return out
    pressure = _host(state.sph.pressure)
    if not np.isfinite(pressure).all():
        raise RuntimeError("Non-finite pressure")
    rho99 = float(np.percentile(rho, 99))
    out.update(density_p99=rho99, density_compression_p99=max(0.0, rho99 / sim.scene.spec.density - 1.0),
               pressure_min=float(pressure.min()), pressure_max=float(pressure.max()))
    return out
