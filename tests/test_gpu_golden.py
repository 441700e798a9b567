"""GPU solvers against the golden vectors of the reference solvers.

The fixtures hold the output of the unmodified reference ``step`` (run under
a substitute FP32 Warp runtime, see tests/golden/make_golden.py).  Bar
(golden_io.compare_fields): neighbour counts and DFSPH iteration decisions
identical; every float field within 1e-5 norm-relative error of the
reference, or, for a field whose own FP32 rounding exceeds that, no farther
from the FP64 oracle solution than 4x the reference's own FP32 error.
"""

import pytest

import oracle
from golden_io import CASES, compare_fields, oracle_outputs
from gpu_util import golden_case, run_step

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name", CASES)
def test_gpu_step_matches_reference(name, cuda_device):
    kind, model, state_in, cfg, dt, expect = golden_case(name)
    out, solver, _ = run_step(kind, model, state_in, cfg, dt)
    pairs = [("particle_q", out["particle_q"], expect["particle_q"]),
             ("particle_qd", out["particle_qd"], expect["particle_qd"]),
             ("accel", out["accel"], expect["accel"])]
    if "x_pred" in expect:
        pairs.append(("x_pred", out["x_pred"], expect["x_pred"]))
    for k, ref in expect["sph"].items():
        if k != "step_displacement":  # never written by the reference step (launch commented out)
            pairs.append((k, out["sph"][k], ref))
    ref64 = oracle_outputs(kind, model, state_in, cfg, dt, "f64")
    errors, conditioned = compare_fields(pairs, ref64, kind=kind)
    assert not errors, f"{name}: " + "; ".join(errors)
    if conditioned:
        print(f"{name}: conditioned fields: " + "; ".join(conditioned))
    if kind == "dfsph":
        _, _, info = oracle.dfsph_step(model, state_in, cfg, dt)
        got = solver.last_iterations()
        assert got["rho_iterations"] == info["rho_iterations"]
        assert got["vel_iterations"] == info["vel_iterations"]
