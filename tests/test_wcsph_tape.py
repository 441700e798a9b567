"""The FP64 torch restatement used for tape gradients reproduces the FP64
oracle (itself pinned to the reference solver) substep by substep."""

import numpy as np
import torch

import oracle
from adjoint_util import CFG, DT, block, oracle_model, params, tape_rollout


def test_tape_forward_matches_fp64_oracle():
    x, v = block(side=8)
    prm = params(len(x))
    model = oracle_model(x, prm)
    state = dict(particle_q=x.astype(np.float64), particle_qd=v.astype(np.float64), sph={})
    xt = torch.tensor(x, dtype=torch.float64)
    vt = torch.tensor(v, dtype=torch.float64)
    pt = {k: torch.tensor(a, dtype=torch.float64) for k, a in prm.items()}
    for _ in range(5):
        out, _ = oracle.wcsph_step(model, state, CFG, DT, precision="f64")
        state = dict(particle_q=out["particle_q"], particle_qd=out["particle_qd"], sph={})
        xt, vt = tape_rollout(xt, vt, pt, 1)
        assert np.abs(xt.numpy() - out["particle_q"]).max() <= 1e-12
        assert np.abs(vt.numpy() - out["particle_qd"]).max() <= 1e-9 * max(1.0, np.abs(out["particle_qd"]).max())
    # the block is compressed against the floor and the -x wall: walls and pressure act
    assert np.any(out["particle_q"][:, 0] == -CFG["bound_width"]) or np.any(out["particle_q"][:, 2] == 0.0)
