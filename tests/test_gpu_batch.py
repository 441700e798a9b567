"""Batched scenes: one model of many worlds on the segmented (world, cell) grid.

Checked here:
  - the segmented grid build and its candidate enumeration against a numpy
    restatement (bit-exact sorted order, cell ranges and candidate lists);
  - one batched WCSPH / PBF substep over several scenes against the CPU
    oracle run on each scene alone with that scene's walls, stiffness and
    viscosity (the parity rule of the plain solvers: golden_io.compare_fields);
  - scenes overlapping in space do not interact;
  - a batched frame replayed from a CUDA graph equals the eager steps;
  - a batched DFSPH substep takes its iteration decisions per world: every
    scene iterates as it would alone (same counts, same bits), and the scenes
    chosen here stop after different numbers of iterations;
  - the whole 256-scene batch (6,190,898 particles), one PBF or DFSPH frame:
    every scene bit-identical to the scene run alone.
"""

import numpy as np
import pytest
import torch

from fluid_simulation_b200 import _lib
from fluid_simulation_b200.batch import EXPONENT, GRAVITY, REST_DENSITY, batched_model, make_batch
from fluid_simulation_b200.graph import FrameGraph
from fluid_simulation_b200.solver import SolverDFSPH, SolverPBF, SolverWCSPH
from golden_io import compare_fields, oracle_outputs
from gpu_util import run_step

pytestmark = pytest.mark.gpu


def small_batch(n_scenes=5, seed=11):
    return make_batch(n_scenes=n_scenes, seed=seed, n_lo=1500, n_hi=6000, spacing=0.01)


def velocities(batch, seed=5, sigma=0.3):
    return (np.random.default_rng(seed).normal(size=(batch.total, 3)) * sigma).astype(np.float32)


# ----------------------------------------------------------------- grid ----
def axis_cell(v, inv, clo, d):
    """clamp(int(v / h) - cell_lo, 0, dims - 1): truncating, float32 product."""
    return np.clip(np.trunc(np.float32(v) * inv).astype(np.int64) - clo, 0, d - 1)


def world_keys(x, world, boxes, h):
    """(world, cell) key of each particle: base + (cz * dy + cy) * dx + cx."""
    inv = np.float32(1.0) / np.float32(h)
    bases = np.concatenate([[0], np.cumsum([d[0] * d[1] * d[2] for _, d, _ in boxes])])
    keys = np.empty(len(x), np.int64)
    for w, (clo, dims, _) in enumerate(boxes):
        sel = world == w
        c = [axis_cell(x[sel, k], inv, clo[k], dims[k]) for k in range(3)]
        keys[sel] = bases[w] + (c[2] * dims[1] + c[1]) * dims[0] + c[0]
    return keys, bases


def test_world_grid_tables_and_candidates(cuda_device):
    b = small_batch()
    m = batched_model(b, SolverWCSPH, device=cuda_device)
    x = b.positions()
    world = b.world()
    grid = m.particle_grid
    grid.build(m.particle_q, b.h, m.particle_world)
    ids, cells, starts, ends = [t.cpu().numpy() for t in grid.tables()]
    keys, bases = world_keys(x, world, b.boxes(), b.h)
    order = np.lexsort((np.arange(len(x)), keys))  # stable sort by key, ascending id inside a cell
    assert np.array_equal(ids, order)
    assert np.array_equal(cells, keys[order])
    ncell = int(bases[-1])
    cnt = np.bincount(keys, minlength=ncell)
    assert np.array_equal(starts, np.concatenate([[0], np.cumsum(cnt)[:-1]]))
    assert np.array_equal(ends - starts, cnt)
    # candidates of sampled queries: the world's cells overlapped by [q - h, q + h], z/y/x order
    rng = np.random.default_rng(0)
    qi = rng.choice(len(x), 300, replace=False)
    q = torch.as_tensor(x[qi], device=cuda_device)
    qw = torch.as_tensor(world[qi], device=cuda_device)
    off, cand = grid.candidates(q, b.h, qw)
    off, cand = off.cpu().numpy(), cand.cpu().numpy()
    inv = np.float32(1.0) / np.float32(b.h)
    h = np.float32(b.h)
    for k, i in enumerate(qi):
        clo, dims, _ = b.boxes()[world[i]]
        rng_ax = []
        for a in range(3):
            c0 = int(axis_cell(np.float32(x[i, a] - h), inv, clo[a], dims[a]))
            c1 = int(axis_cell(np.float32(x[i, a] + h), inv, clo[a], dims[a]))
            rng_ax.append((c0, c1))
        want = []
        for cz in range(rng_ax[2][0], rng_ax[2][1] + 1):
            for cy in range(rng_ax[1][0], rng_ax[1][1] + 1):
                for cx in range(rng_ax[0][0], rng_ax[0][1] + 1):
                    key = bases[world[i]] + (cz * dims[1] + cy) * dims[0] + cx
                    want.extend(ids[starts[key]:ends[key]].tolist())
        assert cand[off[k]:off[k + 1]].tolist() == want
        # completeness: every particle of the world within h is a candidate, no other world appears
        d2 = ((x - x[i]) ** 2).sum(1)
        near = set(np.nonzero((d2 <= h * h) & (world == world[i]))[0].tolist())
        assert near <= set(want)
        assert np.all(world[want] == world[i])


# --------------------------------------------------------------- parity ----
SHIFT = np.array([0.0, 0.0, -0.006], np.float32)  # bottom layer starts below the floor: walls act


def scene_np(b, k, v):
    """Oracle-form model/state/config pieces of scene k alone (input shifted by SHIFT)."""
    s = b.scenes[k]
    n = s.count
    a, e = b.starts[k], b.starts[k + 1]
    model = dict(particle_flags=np.ones(n, np.int32), particle_mass=np.full(n, b.mass, np.float32),
                 particle_world=np.zeros(n, np.int32), gravity=np.array([GRAVITY], np.float32),
                 particle_max_radius=b.radius,
                 sph=dict(particle_mask=np.zeros(n, np.int32), rest_density=np.full(n, REST_DENSITY, np.float32),
                          surface_tension=np.zeros(n, np.float32), viscosity=np.full(n, s.viscosity, np.float32),
                          stiffness=np.full(n, s.stiffness, np.float32), exponent=np.full(n, EXPONENT, np.float32)))
    state = dict(particle_q=s.x + SHIFT, particle_qd=v[a:e], sph={})
    walls = dict(bound_width=s.walls[0], bound_height=s.walls[1], bound_length=s.walls[2])
    return model, state, walls, slice(a, e)


COMMON = dict(particle_length=0.01, smoothing_length_coff=2.0, boundary_damping=-0.3, bound_width=9.0,
              bound_height=9.0, bound_length=9.0)


def configs(b):
    wc = dict(COMMON, particle_radius=b.radius, clamp_negative_pressure=True)
    pc = dict(COMMON, particle_radius=b.radius, max_iterations=4, lambda_epsilon=100.0, min_neighbors_for_lambda=8,
              scorr_k=0.0, scorr_n=4.0, scorr_q=0.3, max_delta_position=b.radius * 0.5, xsph_c=0.05)
    return {"wcsph": (SolverWCSPH, SolverWCSPH.SphConfig, wc, 1e-4),
            "pbf": (SolverPBF, SolverPBF.PbfConfig, pc, 1.0 / 240.0)}


@pytest.mark.parametrize("kind", ["wcsph", "pbf"])
def test_batched_step_matches_oracle_per_scene(kind, cuda_device):
    b = small_batch()
    v = velocities(b)
    cls, cfg_cls, cfg, dt = configs(b)[kind]
    m = batched_model(b, cls, device=cuda_device, v=v)
    m.particle_q += torch.as_tensor(SHIFT, device=cuda_device)
    solver = cls(m, cfg_cls(**cfg))
    s_in, s_out = m.state(), m.state()
    solver.step(s_in, s_out, None, None, dt)
    torch.cuda.synchronize()
    assert m.particle_grid.status() == 0
    got = dict(particle_q=s_out.particle_q.cpu().numpy(), particle_qd=s_out.particle_qd.cpu().numpy(),
               accel=solver._particle_accel.cpu().numpy(),
               **{k: t.cpu().numpy() for k, t in vars(s_out.sph).items()})
    if kind == "pbf":
        got["x_pred"] = solver._x_pred.cpu().numpy()
    floor = 0.0 if kind == "wcsph" else b.radius  # PBF walls are inset by the radius (+ boundary_epsilon = 0)
    assert np.sum(got["particle_q"][:, 2] == np.float32(floor)) > 0
    for k in range(len(b.scenes)):
        model, state, walls, sl = scene_np(b, k, v)
        c = dict(cfg, **walls)  # the scene's own tank, as the batched walls table gives it
        # the same scene stepped alone by the plain solver (hash grid): identical bits
        alone, _, _ = run_step(kind, model, state, c, dt, device=cuda_device)
        for name in ("particle_q", "particle_qd", "accel"):
            assert np.array_equal(alone[name], got[name][sl]), (k, name)
        for name, val in alone["sph"].items():
            assert np.array_equal(val, got[name][sl]), (k, name)
        # and the oracle's parity rule per scene
        ref32 = oracle_outputs(kind, model, state, c, dt, "f32")
        ref64 = oracle_outputs(kind, model, state, c, dt, "f64")
        cnt = ref32.pop("neighbor_count", None)
        pairs = [(name, got[name][sl], val) for name, val in ref32.items()]
        errors, _ = compare_fields(pairs, ref64, kind=kind)
        assert not errors, f"scene {k}: " + "; ".join(errors)
        if cnt is not None:
            # PBF counts pairs with r < h at the positions left by three Jacobi
            # updates; the GPU's FMA-contracted updates and the oracle's plain
            # FP32 ones differ in the last bits, which moves a pair lying within
            # ~1e-6 h of the support boundary across it: a few particles in 10^3
            # may differ by one neighbour.  (With identical positions, as in the
            # single-pass counts, the counts are compared exactly.)
            diff = got["neighbor_count"][sl].astype(np.int64) - cnt
            assert np.abs(diff).max() <= 1 and np.count_nonzero(diff) <= max(2, len(diff) // 1000), (k, diff)


def test_overlapping_scenes_do_not_interact(cuda_device):
    """Every tank starts at the origin, so scenes overlap in space; stepping
    one scene alone inside the batch layout (others deactivated) gives the
    same result for it as stepping the full batch."""
    b = small_batch(n_scenes=3, seed=12)
    v = velocities(b, seed=6)
    cls, cfg_cls, cfg, dt = configs(b)["wcsph"]
    outs = []
    for only in (None, 1):
        m = batched_model(b, cls, device=cuda_device, v=v)
        if only is not None:
            flags = torch.zeros_like(m.particle_flags)
            sl = slice(int(b.starts[only]), int(b.starts[only + 1]))
            flags[sl] = 1
            m.particle_flags = flags
        solver = cls(m, cfg_cls(**cfg))
        s_in, s_out = m.state(), m.state()
        solver.step(s_in, s_out, None, None, dt)
        outs.append((s_out.particle_q.cpu().numpy(), s_out.sph.rho.cpu().numpy()))
    sl = slice(int(b.starts[1]), int(b.starts[2]))
    assert np.array_equal(outs[0][0][sl], outs[1][0][sl])
    assert np.array_equal(outs[0][1][sl], outs[1][1][sl])


def test_batched_frame_graph_equals_eager(cuda_device):
    b = small_batch(n_scenes=4, seed=13)
    v = velocities(b, seed=7)
    cls, cfg_cls, cfg, dt = configs(b)["pbf"]
    res = []
    for graph in (False, True):
        m = batched_model(b, cls, device=cuda_device, v=v)
        solver = cls(m, cfg_cls(**cfg))
        a, c = m.state(), m.state()
        if graph:
            fg = FrameGraph(solver, a, c, dt, substeps=4, warmup=False)
            out = fg.replay()
        else:
            for _ in range(4):
                solver.step(a, c, None, None, dt)
                a, c = c, a
            out = a
        torch.cuda.synchronize()
        res.append(out.particle_q.cpu().numpy())
    assert np.array_equal(res[0], res[1])


# DFSPH with tolerances that the five scenes below (velocities scaled by
# 0.5 (k + 1)) pass after different numbers of iterations: the oracle takes
# 2, 2, 8, 8, 8 density and 8, 6, 8, 8, 8 divergence iterations on them.
DFSPH_CFG = dict(COMMON, max_rho_iterations=8, max_vel_iterations=8, warm_start=False, max_kappa=1.0,
                 max_kappa_v=100.0, eta_density=6.0, eta_divergence=48.0, min_neighbors_for_factor=8)


def dfsph_batch():
    b = small_batch(n_scenes=5, seed=14)
    v = velocities(b, seed=8)
    for k in range(len(b.scenes)):
        v[b.starts[k]:b.starts[k + 1]] *= 0.5 * (k + 1)
    return b, v


def test_batched_dfsph_decides_per_world(cuda_device):
    b, v = dfsph_batch()
    cfg = dict(DFSPH_CFG, particle_radius=b.radius)
    dt = 1e-3
    m = batched_model(b, SolverDFSPH, device=cuda_device, v=v)
    m.particle_q += torch.as_tensor(SHIFT, device=cuda_device)
    solver = SolverDFSPH(m, SolverDFSPH.SphConfig(**cfg))
    s_in, s_out = m.state(), m.state()
    solver.step(s_in, s_out, None, None, dt)
    torch.cuda.synchronize()
    assert m.particle_grid.status() == 0
    per_world = solver.last_world_iterations()
    got = dict(particle_q=s_out.particle_q.cpu().numpy(), particle_qd=s_out.particle_qd.cpu().numpy(),
               accel=solver._particle_accel.cpu().numpy(),
               **{k: t.cpu().numpy() for k, t in vars(s_out.sph).items()})
    seen = set()
    for k in range(len(b.scenes)):
        model, state, walls, sl = scene_np(b, k, v)
        c = dict(cfg, **walls)
        alone, sv, _ = run_step("dfsph", model, state, c, dt, device=cuda_device)
        it_alone = sv.last_iterations()
        for key in ("rho_iterations", "vel_iterations"):
            assert per_world[k][key] == it_alone[key], (k, key, per_world[k], it_alone)
        for key in ("density_residual", "divergence_residual"):  # same terms, summed in another order
            assert per_world[k][key] == pytest.approx(it_alone[key], rel=1e-12, abs=1e-12), (k, key)
        for name in ("particle_q", "particle_qd", "accel"):
            assert np.array_equal(alone[name], got[name][sl]), (k, name)
        for name, val in alone["sph"].items():
            assert np.array_equal(val, got[name][sl]), (k, name)
        # the oracle's decisions and parity rule per scene
        import oracle
        _, _, info = oracle.dfsph_step(model, state, c, dt, precision="f32")
        assert (info["rho_iterations"], info["vel_iterations"]) == (per_world[k]["rho_iterations"],
                                                                    per_world[k]["vel_iterations"]), k
        ref32 = oracle_outputs("dfsph", model, state, c, dt, "f32")
        ref64 = oracle_outputs("dfsph", model, state, c, dt, "f64")
        pairs = [(name, got[name][sl], val) for name, val in ref32.items()]
        errors, _ = compare_fields(pairs, ref64, kind="dfsph")
        assert not errors, f"scene {k}: " + "; ".join(errors)
        seen.add((per_world[k]["rho_iterations"], per_world[k]["vel_iterations"]))
    assert len(seen) > 1  # the worlds stopped at different iterations
    total = solver.last_iterations()  # a batched context reports the largest counts
    assert total["rho_iterations"] == max(w["rho_iterations"] for w in per_world)
    assert total["vel_iterations"] == max(w["vel_iterations"] for w in per_world)


def test_batched_dfsph_particles_past_the_walls_keep_bits(cuda_device):
    """The wall layer at x = -W thrown outward at 20 m/s: DFSPH builds its
    second grid from x + v* dt, before the walls act, and there particles of
    three of the five scenes lie a cell past their tank.  The one-cell margin
    of the world boxes keeps them in their own cells, so every scene still
    equals its plain step bit for bit."""
    b, v = dfsph_batch()
    x = b.positions()
    for k, s in enumerate(b.scenes):
        a, e = b.starts[k], b.starts[k + 1]
        edge = x[a:e, 0] < -s.walls[0] + b.spacing
        v[a:e][edge, 0] = -20.0
    cfg = dict(DFSPH_CFG, particle_radius=b.radius)
    dt = 1e-3
    m = batched_model(b, SolverDFSPH, device=cuda_device, v=v)
    solver = SolverDFSPH(m, SolverDFSPH.SphConfig(**cfg))
    s_in, s_out = m.state(), m.state()
    solver.step(s_in, s_out, None, None, dt)
    torch.cuda.synchronize()
    assert m.particle_grid.status() == 0
    vstar = s_out.sph.v_star.cpu().numpy()
    inv = np.float32(1.0) / np.float32(b.h)
    escaped = 0
    for k, s in enumerate(b.scenes):
        model, state, walls, sl = scene_np(b, k, v)
        state["particle_q"] = x[sl]  # unshifted
        mid = (x[sl] + vstar[sl] * np.float32(dt)).astype(np.float32)
        escaped += int(np.sum(np.trunc(mid[:, 0] * inv) < int(np.float32(-s.walls[0]) * inv)))
        alone, _, _ = run_step("dfsph", model, state, dict(cfg, **walls), dt, device=cuda_device)
        assert np.array_equal(alone["particle_q"], s_out.particle_q[sl].cpu().numpy()), k
        assert np.array_equal(alone["sph"]["neighbor_count"], s_out.sph.neighbor_count[sl].cpu().numpy()), k
        assert np.array_equal(alone["sph"]["rho"], s_out.sph.rho[sl].cpu().numpy()), k
    assert escaped > 0


def test_batched_dfsph_frame_graph_equals_eager(cuda_device):
    b, v = dfsph_batch()
    cfg = dict(DFSPH_CFG, particle_radius=b.radius)
    res = []
    for graph in (False, True):
        m = batched_model(b, SolverDFSPH, device=cuda_device, v=v)
        solver = SolverDFSPH(m, SolverDFSPH.SphConfig(**cfg))
        a, c = m.state(), m.state()
        if graph:
            fg = FrameGraph(solver, a, c, 1e-3, substeps=3, warmup=False)
            out = fg.replay()
        else:
            for _ in range(3):
                solver.step(a, c, None, None, 1e-3)
                a, c = c, a
            out = a
        torch.cuda.synchronize()
        res.append((out.particle_q.cpu().numpy(), solver.last_world_iterations()))
    assert np.array_equal(res[0][0], res[1][0])
    assert res[0][1] == res[1][1]


@pytest.mark.parametrize("kind", ["pbf", "dfsph"])
def test_full_batch_frame_equals_scenes_run_alone(kind, cuda_device):
    """The whole 256-scene batch (6,190,898 particles, log-uniform scene
    sizes 2,000-100,000) advanced one frame of 4 substeps as one model, from
    seeded velocities: every scene's positions and velocities are bit-identical
    to the same scene run alone with the plain solver (and, for DFSPH, so are
    its iteration counts in the last substep)."""
    from fluid_simulation_b200.batch import scene_model
    b = make_batch()
    v = velocities(b, seed=17, sigma=0.2)
    common = dict(particle_radius=b.radius, particle_length=b.spacing, smoothing_length_coff=2.0,
                  boundary_damping=0.0)
    if kind == "pbf":
        cls = SolverPBF
        cfg = lambda w: SolverPBF.PbfConfig(max_iterations=4, lambda_epsilon=100.0, min_neighbors_for_lambda=8,
                                            scorr_k=0.0, max_delta_position=b.radius * 0.5, xsph_c=0.05,
                                            bound_width=w[0], bound_height=w[1], bound_length=w[2], **common)
    else:
        cls = SolverDFSPH
        cfg = lambda w: SolverDFSPH.SphConfig(max_rho_iterations=5, max_vel_iterations=12, warm_start=False,
                                              max_kappa=1.0, max_kappa_v=100.0, bound_width=w[0],
                                              bound_height=w[1], bound_length=w[2], **common)
    dt = 1.0 / 240.0
    mb = batched_model(b, cls, device=cuda_device, v=v)
    sb = cls(mb, cfg((1.0, 1.0, 1.0)))
    a, c = mb.state(), mb.state()
    for _ in range(4):
        sb.step(a, c, None, None, dt)
        a, c = c, a
    torch.cuda.synchronize()
    xb, vb = a.particle_q.cpu().numpy(), a.particle_qd.cpu().numpy()
    per_world = sb.last_world_iterations() if kind == "dfsph" else None
    del mb, sb, c
    mismatched = []
    for k, s in enumerate(b.scenes):
        lo, hi = int(b.starts[k]), int(b.starts[k + 1])
        m = scene_model(b, k, cls, device=cuda_device, v=v[lo:hi])
        sv = cls(m, cfg(s.walls))
        p, q = m.state(), m.state()
        for _ in range(4):
            sv.step(p, q, None, None, dt)
            p, q = q, p
        ok = np.array_equal(p.particle_q.cpu().numpy(), xb[lo:hi]) and \
            np.array_equal(p.particle_qd.cpu().numpy(), vb[lo:hi])
        if kind == "dfsph":
            it, pw = sv.last_iterations(), per_world[k]
            ok = ok and (it["rho_iterations"], it["vel_iterations"]) == (pw["rho_iterations"], pw["vel_iterations"])
        if not ok:
            mismatched.append(k)
        del m, sv, p, q
    assert not mismatched, mismatched
