"""Generate the golden fixtures in this folder from the reference's own code.

Run once in a container that holds the reference sources:

    python tests/golden/make_golden.py --reference <path to fluid_simulation checkout>

It executes the UNMODIFIED reference solvers (``solver/sph/solver_wcsph.py``,
``solver/sph/solver_dfsph.py``, ``solver/pbf/solver_pbf.py``) through their
public ``step(state_in, state_out, control, contacts, dt)``, and the APIC
solver's particle-separation kernels (``solver/apic/solver_apic.py``) through
the loop of ``_apply_particle_separation``, under the
substitute Warp/Newton runtime of ``warp_shim.py`` (FP32, one Python call per
thread), and the reference scene generator ``examples/dam_break/scene.py``.
Each case is saved as ``<case>.npz`` holding the inputs, the config (JSON)
and every array the step writes.  ``attributes.json`` records the custom
attributes each reference solver registers (the drop-in boundary names).

Nothing at test time imports this script or the reference; the tests read
only the ``.npz`` / ``.json`` files.
"""

from __future__ import annotations

import argparse
import dataclasses
import json
import os
import sys
import time
import types

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def _ns(**kw):
    return types.SimpleNamespace(**kw)


def block_scene(n_side=6, spacing=0.02, squeeze=0.97, seed=0, vel_sigma=0.1):
    """Jittered, slightly compressed lattice block with edge cases planted."""
    rng = np.random.default_rng(seed)
    g = np.arange(n_side, dtype=np.float64) * spacing * squeeze
    xx, yy, zz = np.meshgrid(g, g, g, indexing="ij")
    x = np.stack([xx.ravel(), yy.ravel(), zz.ravel()], 1)
    x += rng.uniform(-0.05, 0.05, x.shape) * spacing
    x += np.array([-0.5 * (n_side - 1) * spacing, -0.5 * (n_side - 1) * spacing, 0.004])
    x = x.astype(np.float32)
    n = len(x)
    v = (rng.normal(size=(n, 3)) * vel_sigma).astype(np.float32)
    flags = np.ones(n, np.int32)
    flags[[5, 77, 150]] = 0          # inactive particles (ParticleFlags.ACTIVE cleared)
    flags[[9]] = 3                   # active with another flag bit set
    mask = np.zeros(n, np.int32)
    mask[[11, 100, 180]] = 1         # kinematic (masked) particles
    world = (np.arange(n) % 2).astype(np.int32)
    world[[3]] = -1                  # negative world index -> world 0
    mass = np.full(n, 1000.0 * spacing ** 3, np.float32) * (1.0 + 0.05 * rng.uniform(-1, 1, n)).astype(np.float32)
    rest = np.full(n, 1000.0, np.float32)
    rest[[20, 21]] = 990.0
    return dict(x=x, v=v, flags=flags, mask=mask, world=world, mass=mass, rest_density=rest,
                gravity=np.array([[0.0, 0.0, -10.0], [0.5, 0.0, -5.0]], np.float32), spacing=spacing)


def dam_scene(target):
    from examples.dam_break.scene import make_scene
    s = make_scene(target)
    n = s.count
    return dict(x=s.positions.astype(np.float32), v=np.zeros((n, 3), np.float32),
                flags=np.ones(n, np.int32), mask=np.zeros(n, np.int32), world=np.zeros(n, np.int32),
                mass=np.full(n, s.mass, np.float32), rest_density=np.full(n, 1000.0, np.float32),
                gravity=np.array([[0.0, 0.0, -10.0]], np.float32), spacing=s.spacing, radius=s.radius,
                sha256=s.report()["initial_position_sha256"])


def make_model(wp, sc, extra):
    n = len(sc["x"])
    sph = _ns(particle_mask=wp.array(sc["mask"], dtype=int),
              rest_density=wp.array(sc["rest_density"], dtype=float))
    for k, val in extra.items():
        setattr(sph, k, wp.array(np.asarray(val, np.float32), dtype=float))
    return _ns(particle_count=n, device="cpu", particle_grid=None,
               particle_max_radius=float(sc.get("radius", 0.5 * sc["spacing"])),
               particle_flags=wp.array(sc["flags"], dtype=wp.int32),
               particle_mass=wp.array(sc["mass"], dtype=float),
               particle_world=wp.array(sc["world"], dtype=wp.int32),
               gravity=wp.array(sc["gravity"], dtype=wp.vec3), sph=sph)


def make_state(wp, sc, names_vec, names_scalar, names_int, init=None):
    n = len(sc["x"])
    init = init or {}
    sph = _ns()
    for k in names_scalar:
        setattr(sph, k, wp.array(init.get(k, np.zeros(n, np.float32)), dtype=float))
    for k in names_int:
        setattr(sph, k, wp.array(np.zeros(n, np.int32), dtype=int))
    for k in names_vec:
        setattr(sph, k, wp.array(np.zeros((n, 3), np.float32), dtype=wp.vec3))
    return _ns(particle_q=wp.array(sc["x"], dtype=wp.vec3), particle_qd=wp.array(sc["v"], dtype=wp.vec3),
               body_count=0, joint_q=None, joint_qd=None, sph=sph)


def apic_separation_kernels(wp, newton, reference):
    """The two particle-separation kernels of solver/apic/solver_apic.py
    (accumulate_particle_separation, apply_particle_separation_delta, lines
    193-266), compiled from the reference source on their own: the module
    itself needs warp.fem and warp.sparse, which the shim does not provide."""
    import ast
    path = os.path.join(reference, "solver", "apic", "solver_apic.py")
    src = open(path).read()
    tree = ast.parse(src)
    keep = [node for node in tree.body if isinstance(node, ast.FunctionDef)
            and node.name in ("accumulate_particle_separation", "apply_particle_separation_delta")]
    assert len(keep) == 2
    ns = dict(wp=wp, ParticleFlags=newton.ParticleFlags)
    exec(compile(ast.Module(body=keep, type_ignores=[]), path, "exec"), ns)
    return ns["accumulate_particle_separation"], ns["apply_particle_separation_delta"]


def run_apic_separation(wp, newton, reference, name, x, flags, radius, bound_lo, bound_hi, strength=0.55,
                        iterations=2, rest_dist_cfg=-1.0, wall_margin_cfg=-1.0, wall_push_band_cfg=-1.0):
    """SolverAPIC._apply_particle_separation (solver_apic.py:1003-1064) with
    the parameter derivation of SolverAPIC.__init__ (641-650) for a model of
    uniform particle radius."""
    accumulate, apply_delta = apic_separation_kernels(wp, newton, reference)
    n = len(x)
    radii = np.full(n, radius, np.float32)
    wall_margin = float(np.mean(radii)) if wall_margin_cfg < 0.0 else float(wall_margin_cfg)
    wall_push_band = 1.5 * wall_margin if wall_push_band_cfg < 0.0 else float(wall_push_band_cfg)
    rest_dist = float(rest_dist_cfg) if rest_dist_cfg > 0.0 else float(2.0 * float(np.mean(radii)))
    query_radius = max(rest_dist, 1.0e-5)
    lo = np.asarray(bound_lo, dtype=np.float64)
    hi = np.asarray(bound_hi, dtype=np.float64)
    extent = np.maximum(hi - lo, query_radius)
    dims = np.maximum(4, np.ceil(extent / query_radius).astype(int))
    grid = wp.HashGrid(int(dims[0]), int(dims[1]), int(dims[2]))
    pos = wp.array(x, dtype=wp.vec3)
    fl = wp.array(flags, dtype=wp.int32)
    delta = wp.array(np.zeros((n, 3), np.float32), dtype=wp.vec3)
    blo, bhi = wp.vec3(*bound_lo), wp.vec3(*bound_hi)
    band = max(float(wall_push_band), float(wall_margin) * 2.0)
    t0 = time.time()
    for _ in range(max(1, int(iterations))):
        grid.build(points=pos, radius=query_radius)
        wp.launch(kernel=accumulate, dim=n, inputs=[grid.id, pos, fl, delta, rest_dist, query_radius, strength,
                                                     blo, bhi, band])
        wp.launch(kernel=apply_delta, dim=n, inputs=[pos, fl, delta, blo, bhi, float(wall_margin)])
    cfg = dict(rest_dist=rest_dist, query_radius=query_radius, strength=strength, iterations=int(iterations),
               bound_lo=list(map(float, bound_lo)), bound_hi=list(map(float, bound_hi)), wall_band=band,
               wall_margin=wall_margin, dims=[int(d) for d in dims], radius=float(radius))
    np.savez_compressed(os.path.join(HERE, f"{name}.npz"), in_x=x, flags=flags, config=json.dumps(cfg),
                        out_x=pos.numpy(), out_delta=delta.numpy())
    print(f"{name}: n={n} {time.time() - t0:.1f}s", flush=True)


def apic_block(seed=3):
    """Clumped jittered lattice (spacing 0.8 of the rest distance) in a small
    tank, with particles inside the wall bands, outside the tank (their cells
    alias through the grid's modulo), inactive ones and a coincident pair."""
    rng = np.random.default_rng(seed)
    r = 0.005
    g = np.arange(9, dtype=np.float64) * 0.8 * (2 * r)
    xx, yy, zz = np.meshgrid(g - 0.032, g - 0.032, g + 0.001, indexing="ij")
    x = np.stack([xx.ravel(), yy.ravel(), zz.ravel()], 1)
    x += rng.uniform(-0.15, 0.15, x.shape) * r
    out = rng.uniform([0.20, -0.03, 0.0], [0.22, 0.03, 0.06], (24, 3))     # beyond x = hi: aliased cells
    x = np.concatenate([x, out]).astype(np.float32)
    x[7] = x[6]                                                              # coincident pair
    n = len(x)
    flags = np.ones(n, np.int32)
    flags[[3, 40, 41, 300]] = 0
    flags[[12]] = 5
    return x, flags, r


def run_case(wp, name, solver_cls, cfg, sc, material, dt, state_names, init=None):
    vec, scal, ints = state_names
    model = make_model(wp, sc, material)
    s_in = make_state(wp, sc, vec, scal, ints, init)
    s_out = make_state(wp, sc, vec, scal, ints)
    solver = solver_cls(model, cfg)
    t0 = time.time()
    solver.step(s_in, s_out, None, None, dt)
    out = dict(
        in_x=sc["x"], in_v=sc["v"], flags=sc["flags"], mask=sc["mask"], world=sc["world"], mass=sc["mass"],
        rest_density=sc["rest_density"], gravity=sc["gravity"],
        particle_max_radius=np.float64(model.particle_max_radius), dt=np.float64(dt),
        config=json.dumps(dataclasses.asdict(cfg)),
        out_x=s_out.particle_q.numpy(), out_v=s_out.particle_qd.numpy(),
        accel=solver._particle_accel.numpy(),
    )
    for k, val in material.items():
        out["mat_" + k] = np.asarray(val, np.float32)
    for k, val in (init or {}).items():
        out["in_sph_" + k] = np.asarray(val)
    for k in vec + scal + ints:
        out["out_sph_" + k] = getattr(s_out.sph, k).numpy()
    if hasattr(solver, "_x_pred"):
        out["x_pred"] = solver._x_pred.numpy()
    np.savez_compressed(os.path.join(HERE, f"{name}.npz"), **out)
    print(f"{name}: n={len(sc['x'])} {time.time() - t0:.1f}s", flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", required=True)
    ap.add_argument("--only", default="")
    args = ap.parse_args()
    sys.path.insert(0, HERE)
    import warp_shim
    wp, newton = warp_shim.install()
    sys.path.insert(0, os.path.abspath(args.reference))
    from solver.sph.solver_wcsph import SolverWCSPH
    from solver.sph.solver_dfsph import SolverDFSPH
    from solver.pbf.solver_pbf import SolverPBF

    # Registered custom attributes (drop-in boundary names).
    attrs = {}
    for name, cls in (("wcsph", SolverWCSPH), ("dfsph", SolverDFSPH), ("pbf", SolverPBF)):
        b = newton.ModelBuilder()
        cls.register_custom_attributes(b)
        attrs[name] = [dict(name=a.name, frequency=a.frequency.name, assignment=a.assignment.name,
                            dtype={int: "int32", float: "float32", np.float32: "float32",
                                   np.int32: "int32", wp.vec3: "vec3"}[a.dtype],
                            default=(list(map(float, a.default.c)) if isinstance(a.default, wp.vec3)
                                     else a.default), namespace=a.namespace)
                       for a in b.custom_attributes]
        attrs[name + "_config_defaults"] = dataclasses.asdict(
            (cls.SphConfig if hasattr(cls, "SphConfig") else cls.PbfConfig)())
    with open(os.path.join(HERE, "attributes.json"), "w") as f:
        json.dump(attrs, f, indent=1, sort_keys=True)

    only = set(filter(None, args.only.split(",")))

    def want(n):
        return not only or n in only

    blk = block_scene()
    d = blk["spacing"]
    n = len(blk["x"])
    rng = np.random.default_rng(7)
    box = dict(bound_width=0.05, bound_height=0.05, bound_length=0.05)   # some particles start outside

    wc_mat = dict(rest_density=blk["rest_density"], surface_tension=np.full(n, 0.3, np.float32),
                  viscosity=np.full(n, 1.0e-3, np.float32),
                  stiffness=np.full(n, 2.5e5, np.float32) * rng.uniform(0.9, 1.1, n).astype(np.float32),
                  exponent=np.full(n, 7.0, np.float32))
    wc_mat.pop("rest_density")
    wnames = ((), ("rho", "pressure"), ())
    if want("wcsph_block"):
        cfg = SolverWCSPH.SphConfig(particle_radius=0.5 * d, particle_length=d, smoothing_length_coff=2.0,
                                    boundary_damping=-0.3, **box)
        run_case(wp, "wcsph_block", SolverWCSPH, cfg, blk, wc_mat, 2.0e-4, wnames)
    if want("wcsph_block_signed"):
        cfg = SolverWCSPH.SphConfig(particle_radius=0.0, particle_length=d, smoothing_length_coff=2.0,
                                    boundary_damping=-0.3, clamp_negative_pressure=False, **box)
        run_case(wp, "wcsph_block_signed", SolverWCSPH, cfg, blk, wc_mat, 2.0e-4, wnames)

    dam = dam_scene(512)
    nd = len(dam["x"])
    hd = 2.0 * dam["spacing"]
    dam_common = dict(particle_radius=dam["radius"], particle_length=dam["spacing"], smoothing_length_coff=2.0,
                      boundary_damping=0.0, bound_width=1.2, bound_height=0.28, bound_length=0.6)
    if want("wcsph_dam512"):
        mat = dict(surface_tension=np.zeros(nd, np.float32), viscosity=np.full(nd, 1.0e-6, np.float32),
                   stiffness=np.full(nd, 2.5e5, np.float32), exponent=np.full(nd, 7.0, np.float32))
        c0 = (2.5e5 * 7.0 / 1000.0) ** 0.5
        dt = min(1.0 / 60.0 / 4.0, 0.25 * hd / c0)
        run_case(wp, "wcsph_dam512", SolverWCSPH, SolverWCSPH.SphConfig(**dam_common), dam, mat, dt, wnames)

    df_mat = dict(surface_tension=np.full(n, 0.2, np.float32), viscosity=np.full(n, 1.0e-3, np.float32))
    dnames = (("v_star",), ("rho", "factor", "rho_star", "d_rho_dt", "kappa", "kappa_v"), ("neighbor_count",))
    if want("dfsph_block"):
        cfg = SolverDFSPH.SphConfig(max_rho_iterations=5, max_vel_iterations=12, warm_start=False, max_kappa=1.0,
                                    max_kappa_v=100.0, particle_radius=0.5 * d, particle_length=d,
                                    smoothing_length_coff=2.0, boundary_damping=-0.5, **box)
        run_case(wp, "dfsph_block", SolverDFSPH, cfg, blk, df_mat, 1.0e-3, dnames)
    if want("dfsph_block_warm"):
        init = dict(kappa=rng.uniform(0, 0.05, n).astype(np.float32),
                    kappa_v=rng.uniform(0, 0.5, n).astype(np.float32))
        cfg = SolverDFSPH.SphConfig(max_rho_iterations=3, max_vel_iterations=4, warm_start=True, max_kappa=1.0,
                                    max_kappa_v=100.0, min_neighbors_for_factor=10, particle_radius=0.5 * d,
                                    particle_length=d, smoothing_length_coff=2.0, boundary_damping=-0.5, **box)
        run_case(wp, "dfsph_block_warm", SolverDFSPH, cfg, blk, df_mat, 1.0e-3, dnames, init=init)
    if want("dfsph_dam512"):
        mat = dict(surface_tension=np.zeros(nd, np.float32), viscosity=np.full(nd, 1.0e-6, np.float32))
        cfg = SolverDFSPH.SphConfig(max_rho_iterations=5, max_vel_iterations=12, warm_start=False, max_kappa=1.0,
                                    max_kappa_v=100.0, **dam_common)
        run_case(wp, "dfsph_dam512", SolverDFSPH, cfg, dam, mat, 1.0 / 240.0, dnames)

    pnames = (("delta_p", "step_displacement"), ("rho", "pbf_lambda"), ("neighbor_count",))
    pb_mat = dict(surface_tension=np.full(n, 0.2, np.float32), viscosity=np.full(n, 1.0e-3, np.float32))
    if want("pbf_block"):
        cfg = SolverPBF.PbfConfig(max_iterations=4, lambda_epsilon=100.0, min_neighbors_for_lambda=8, scorr_k=0.0,
                                  max_delta_position=0.25 * d, xsph_c=0.05, particle_radius=0.5 * d,
                                  particle_length=d, smoothing_length_coff=2.0, boundary_damping=-0.3, **box)
        run_case(wp, "pbf_block", SolverPBF, cfg, blk, pb_mat, 1.0 / 240.0, pnames)
    if want("pbf_block_scorr"):
        cfg = SolverPBF.PbfConfig(max_iterations=3, lambda_epsilon=100.0, min_neighbors_for_lambda=0, scorr_k=1.0e-3,
                                  scorr_n=4.0, scorr_q=0.3, max_delta_position=0.5 * d, xsph_c=0.01,
                                  particle_radius=0.5 * d, particle_length=d, smoothing_length_coff=2.0,
                                  boundary_damping=-0.2, boundary_epsilon=1.0e-4,
                                  rebuild_grid_each_iteration=True, **box)
        run_case(wp, "pbf_block_scorr", SolverPBF, cfg, blk, pb_mat, 1.0 / 240.0, pnames)
    if want("pbf_dam512"):
        mat = dict(surface_tension=np.zeros(nd, np.float32), viscosity=np.full(nd, 1.0e-6, np.float32))
        cfg = SolverPBF.PbfConfig(max_iterations=4, lambda_epsilon=100.0, min_neighbors_for_lambda=8, scorr_k=0.0,
                                  max_delta_position=dam["radius"] * 0.5, xsph_c=0.05, **dam_common)
        run_case(wp, "pbf_dam512", SolverPBF, cfg, dam, mat, 1.0 / 240.0, pnames)

    if want("apic_separation"):
        x, flags, r = apic_block()
        run_apic_separation(wp, newton, args.reference, "apic_separation", x, flags, r,
                            bound_lo=(-0.05, -0.05, 0.0), bound_hi=(0.05, 0.05, 0.1))

    if want("scenes"):
        scenes = {}
        for t in (512, 10000, 50000, 400000):
            s = dam_scene(t)
            scenes[str(t)] = dict(count=len(s["x"]), spacing=s["spacing"], radius=s["radius"],
                                  sha256=s["sha256"])
        with open(os.path.join(HERE, "scenes.json"), "w") as f:
            json.dump(scenes, f, indent=1, sort_keys=True)


if __name__ == "__main__":
    main()
