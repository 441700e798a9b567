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


# Float fields formed by cancellation, whose FP32 rounding alone can exceed
# the 1e-5 bar on ordinary inputs: EOS pressure near rest density; PBF
# lambda and the position correction built from it, and the velocity
# (x_pred - x_in) / dt; DFSPH kappa, kappa_v, the density-change rate and
# the factor (1 / (|sum g|^2 + sum |g|^2) over nearly balanced gradients),
# and the velocities the iterations correct.
ILL_CONDITIONED = {
    "wcsph": {"pressure"},
    "pbf": {"pbf_lambda", "delta_p", "particle_qd", "step_displacement"},
    "dfsph": {"kappa", "kappa_v", "d_rho_dt", "factor", "v_star", "particle_qd"},
}


def _log_fallback(rec):
    """Appends one JSON line per fallback use to $FS_PARITY_LOG (if set)."""
    path = os.environ.get("FS_PARITY_LOG")
    if not path:
        return
    rec = dict(rec, test=os.environ.get("PYTEST_CURRENT_TEST", "").split(" ")[0])
    with open(path, "a") as f:
        f.write(json.dumps(rec) + "\n")


def compare_fields(pairs, ref64, *, kind, tol=1e-5):
    """Parity rule of the GPU tests.  pairs: (name, candidate, reference FP32);
    ref64: name -> the FP64 oracle's value on the same inputs; kind: the
    solver ("wcsph", "dfsph", "pbf").

    * integer fields (neighbor_count): identical, except PBF's, which
      counts pairs at positions the iterations have already rounded
      differently: at most one pair off for at most 1 particle in 1,000;
    * every float field: max|cand - ref| <= tol * max|ref| (norm-relative);
    * otherwise, a field of ILL_CONDITIONED[kind] passes when the
      candidate's distance from the FP64 solution is at most 4x the FP32
      reference's own distance from it (or tol * max|FP64|);
    * any other field (positions, densities, accelerations) passes that way
      only when the FP32 reference itself misses the bar against FP64 on
      this input (FP32 cannot meet it there), and then within 2x the FP32
      reference's own distance from FP64.
    Returns (errors, conditioned) lists of messages; each fallback use is
    also appended to $FS_PARITY_LOG."""
    errors, conditioned = [], []
    named = ILL_CONDITIONED[kind]
    for name, got, ref in pairs:
        got = np.asarray(got)
        ref = np.asarray(ref)
        if name == "neighbor_count":
            diff = got.astype(np.int64) - ref.astype(np.int64)
            bad = int(np.count_nonzero(diff))
            if bad and kind == "pbf":
                # PBF counts pairs with r < h at the positions left by the
                # Jacobi updates, which differ from the FP32 oracle's in the
                # last bits (lambda is ill-conditioned); that moves a pair
                # lying within ~1e-6 h of the support boundary across it.
                # Counts taken at identical positions are compared exactly.
                ok = int(np.abs(diff).max()) <= 1 and bad <= max(2, len(diff) // 1000)
                _log_fallback(dict(kind=kind, field=name, named=True, ok=ok, counts_differing=bad,
                                   particles=int(len(diff))))
                if not ok:
                    errors.append(f"{name}: {bad} counts differ (max {int(np.abs(diff).max())})")
            elif bad:
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
        scale = max(float(np.abs(r64).max()), 1e-30)
        eg = float(np.abs(got.astype(np.float64) - r64).max())
        er = float(np.abs(ref.astype(np.float64) - r64).max())
        if name in named:
            bound = max(tol * scale, 4.0 * er)
        elif er > tol * scale:
            bound = 2.0 * er
        else:
            errors.append(f"{name}: rel err {e:.3e} vs FP32 (FP32 itself within {er / scale:.2e} of FP64)")
            continue
        msg = (f"{name}: rel err {e:.3e} vs FP32; cand-FP64 {eg / scale:.3e}, FP32-FP64 {er / scale:.3e} "
               f"(norm-relative)")
        ok = eg <= bound
        (conditioned if ok else errors).append(msg)
        _log_fallback(dict(kind=kind, field=name, named=name in named, ok=ok, err_vs_fp32=e,
                           cand_vs_fp64=eg / scale, fp32_vs_fp64=er / scale))
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
