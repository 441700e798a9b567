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


def rel_err(a, b):
    """max |a-b| / max(|b|) over the array (a norm-relative error)."""
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    scale = max(float(np.abs(b).max()) if b.size else 0.0, 1e-30)
    return float(np.abs(a - b).max()) / scale if b.size else 0.0
