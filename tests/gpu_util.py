"""Helpers of the GPU tests: models/states on CUDA from golden fixtures or
synthetic scenes, run through the drop-in solvers (C-ABI library)."""

import numpy as np
import torch

from fluid_simulation_b200.newton_shim import model_from_arrays
from fluid_simulation_b200.solver import SolverDFSPH, SolverPBF, SolverWCSPH
from golden_io import load, solver_of

SOLVERS = {"wcsph": SolverWCSPH, "dfsph": SolverDFSPH, "pbf": SolverPBF}
CONFIGS = {"wcsph": SolverWCSPH.SphConfig, "dfsph": SolverDFSPH.SphConfig, "pbf": SolverPBF.PbfConfig}


def make_solver(kind, model_np, cfg: dict, device="cuda:0"):
    """Model (from oracle-form dict) + solver on the device."""
    x = model_np.get("x")
    sph = dict(model_np["sph"])
    m = model_from_arrays(x, np.zeros_like(x), model_np["particle_mass"], device=device,
                          flags=model_np["particle_flags"], world=model_np.get("particle_world"),
                          gravity=model_np["gravity"], attributes=sph, solver_cls=SOLVERS[kind])
    m.particle_max_radius = float(model_np.get("particle_max_radius", 0.0))
    return m, SOLVERS[kind](m, CONFIGS[kind](**cfg))


def run_step(kind, model_np, state_np, cfg, dt, device="cuda:0", solver=None, model=None):
    """One step on the GPU; returns numpy outputs in oracle form."""
    if solver is None:
        model_np = dict(model_np, x=state_np["particle_q"])
        model, solver = make_solver(kind, model_np, cfg, device)
    s_in, s_out = model.state(), model.state()
    s_in.particle_q.copy_(torch.as_tensor(state_np["particle_q"]))
    s_in.particle_qd.copy_(torch.as_tensor(state_np["particle_qd"]))
    for k, val in state_np.get("sph", {}).items():
        getattr(s_in.sph, k).copy_(torch.as_tensor(val))
    solver.step(s_in, s_out, None, None, dt)
    torch.cuda.synchronize()
    out = dict(particle_q=s_out.particle_q.cpu().numpy(), particle_qd=s_out.particle_qd.cpu().numpy(),
               sph={k: v.cpu().numpy() for k, v in vars(s_out.sph).items()},
               accel=solver._particle_accel.cpu().numpy())
    if kind == "pbf":
        out["x_pred"] = solver._x_pred.cpu().numpy()
    return out, solver, model


def golden_case(name):
    model, state_in, cfg, dt, expect = load(name)
    return solver_of(name), model, state_in, cfg, dt, expect
