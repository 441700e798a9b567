"""Loading of the golden fixtures (``tests/golden/*.npz``) into oracle form."""

import json
import os

import numpy as np

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
CASES = ["wcsph_block", "wcsph_block_signed", "wcsph_dam512", "dfsph_block", "dfsph_block_warm",
         "dfsph_dam512", "pbf_block", "pbf_block_scorr", "pbf_dam512"]


def load(name):
    z = np.load(os.path.join(GOLDEN, f"{name}.npz"))
    cfg = json.loads(str(z["config"]))
    mat = {k[4:]: z[k] for k in z.files if k.startswith("mat_")}
    model = dict(particle_flags=z["flags"], particle_mass=z["mass"], particle_world=z["world"],
                 gravity=z["gravity"], particle_max_radius=float(z["particle_max_radius"]),
                 sph=dict(particle_mask=z["mask"], rest_density=z["rest_density"], **mat))
    state_in = dict(particle_q=z["in_x"], particle_qd=z["in_v"],
                    sph={k[7:]: z[k] for k in z.files if k.startswith("in_sph_")})
    expect = dict(particle_q=z["out_x"], particle_qd=z["out_v"], accel=z["accel"],
                  sph={k[8:]: z[k] for k in z.files if k.startswith("out_sph_")})
    if "x_pred" in z.files:
        expect["x_pred"] = z["x_pred"]
    return model, state_in, cfg, float(z["dt"]), expect


def solver_of(name):
    return name.split("_")[0]


def rel_err(a, b, scale=None):
    """max |a-b| / max(|b|) over the array (a norm-relative error); ``scale``
    replaces max(|b|) for quantities formed by cancellation."""
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    if not b.size:
        return 0.0
    s = float(np.abs(b).max()) if scale is None else float(scale)
    return float(np.abs(a - b).max()) / max(s, 1e-30)


def compare_fields(pairs, ref64, tol=1e-5):
    """Parity rule of the GPU tests.  pairs: (name, candidate, reference FP32);
    ref64: name -> the FP64 oracle's value on the same inputs.

    * integer fields (neighbor_count): identical;
    * float fields: max|cand - ref| <= tol * max|ref|; or, for fields whose
      own FP32 rounding exceeds that (quantities formed by cancellation:
      EOS pressure near rest density, PBF lambda, DFSPH kappa_v, velocities
      derived as position differences / dt, forces of nearly balanced
      pressure), the candidate's distance from the FP64 solution is at most
      4x the FP32 reference's own distance from it, or tol * max|FP64|.
    Returns (errors, conditioned) lists of messages."""
    errors, conditioned = [], []
    for name, got, ref in pairs:
        got = np.asarray(got)
        ref = np.asarray(ref)
        if name == "neighbor_count":
            bad = int(np.count_nonzero(got != ref))
            if bad:
                errors.append(f"{name}: {bad} counts differ")
            continue
        e = rel_err(got, ref)
        if e <= tol:
            continue
        r64 = ref64.get(name)
        if r64 is None:
            errors.append(f"{name}: rel err {e:.3e} (no FP64 reference)")
            continue
        r64 = np.asarray(r64, np.float64)
        eg = float(np.abs(got.astype(np.float64) - r64).max())
        er = float(np.abs(ref.astype(np.float64) - r64).max())
        bound = max(tol * float(np.abs(r64).max()), 4.0 * er)
        msg = f"{name}: rel err {e:.3e} vs FP32; |cand-FP64| {eg:.3e}, |FP32-FP64| {er:.3e}"
        (conditioned if eg <= bound else errors).append(msg)
    return errors, conditioned


def oracle_outputs(kind, model, state_in, cfg, dt, precision):
    """Flat name -> array dict of one oracle step."""
    import oracle
    if kind == "wcsph":
        out, acc = oracle.wcsph_step(model, state_in, cfg, dt, precision=precision)
        extra = {}
    elif kind == "dfsph":
        out, acc, _ = oracle.dfsph_step(model, state_in, cfg, dt, precision=precision)
        extra = {}
    else:
        out, acc, xp = oracle.pbf_step(model, state_in, cfg, dt, precision=precision)
        extra = {"x_pred": xp}
    flat = dict(particle_q=out["particle_q"], particle_qd=out["particle_qd"], accel=acc, **extra)
    flat.update(out["sph"])
    return flat
