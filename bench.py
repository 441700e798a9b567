"""Benchmark of the particle-fluid hot path on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--workload NAME]

Metric: particle-steps/s (one particle advanced one solver substep).
Headline workload (default ``pbf_dam_401856``): the reference's PBF dam
break at 401,856 particles (make_scene(400000)), its harness config (4
constraint iterations, lambda_eps 100, min 8 neighbours, s_corr off, dx clamp
r/2, XSPH 0.05) at the fixed substep dt = 1/240 s.  That is the workload of
the only published solve time (64.65 ms per 4-substep frame on an RTX 4090,
24.86 M particle-substeps/s).  A "step" is one solver substep.

* value: device time with CUDA events around every timed step, L2 flushed by
  a 512 MB write between steps (outside the events); inputs resident in HBM.
* e2e: the same metric through the drop-in solver API with host state:
  every step copies particle_q / particle_qd from pinned host memory, runs
  SolverPBF.step and copies particle_q / particle_qd back.
* roofline: the dominant pass from the library's per-pass CUDA-event timer
  (run on up to 100 further steps after the timed loop, so that its event
  records do not sit inside the timed steps), algorithmic bytes per particle
  per pass (constants below) / its average launch time, against the measured
  HBM copy bandwidth.
* cpu_baseline: the CPU oracle (C++ restatement of the reference solver,
  OpenMP, all host threads) on a bounded number of substeps of the same
  workload.  --impl reference times the same thing as the reference arm: the
  reference (Warp + Newton) cannot be installed or run on these hosts.
* Multi-GPU (torchrun): every rank advances its own replica (weak scaling, no
  data-path collective); time = max over ranks.
* secondary (N=1): the DFSPH dam break, the 4,194,304-particle WCSPH
  lattice and the PBF dam break with s_corr on (each over the same number
  of substeps as the headline), the 256-scene batches, device-side frame
  loops, frame metrics, APIC particle separation and the WCSPH adjoint.
"""

from __future__ import annotations

import argparse
import dataclasses
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

# Algorithmic HBM bytes per particle per pass launch (compulsory traffic under
# the reference's pass dependencies: each per-particle array a pass uses is
# read once, neighbour re-reads are cache hits, outputs written once; FP32,
# vec3 = 12 B).  Per substep: PBF 728 B, WCSPH 180 B, DFSPH 328 B + 116 B per
# density iteration + 108 B per divergence iteration.  PBF's final density
# pass also does the velocity update (44 B), so its two density launches
# average 28 + 44 / 2 B.
B_ALG = {
    "grid_build": 48, "pbf_predict": 60, "pbf_density": 50, "pbf_accel": 72, "pbf_lambda": 40, "pbf_delta": 56,
    "pbf_velocity": 44, "pbf_xsph": 64, "wcsph_density": 40, "wcsph_force": 92, "dfsph_density_factor": 36,
    "dfsph_accel": 76, "dfsph_rate": 60, "dfsph_correct": 56, "dfsph_integrate": 36, "dfsph_final": 48,
}
PUBLISHED_PBF = 401856 * 4 / 0.06464700849610381   # particle-substeps/s, RTX 4090 (performance_summary.json)
# DRAM bytes (read + write) per particle per launch, cold cache, from the
# ncu captures summarised under profiles/: PBF lambda, the mean of one
# substep's four launches at 401,856 particles (the first reuses the density
# pass's lists and reads them back, 79.64 MB; the three scanning ones 38.2
# MB each); WCSPH at 524,288 particles.
TRAFFIC_PER_PARTICLE = {"pbf_lambda": 48.91e6 / 401856, "dfsph_rate": 68.17e6 / 401856,
                        "dfsph_density_factor": 36.86e6 / 401856, "wcsph_density": 62.30e6 / 524288,
                        "wcsph_force": 94.48e6 / 524288}
TRAFFIC_SOURCE = {
    "pbf_lambda": "ncu, mean of one substep's 4 launches at 401,856 particles (profiles/pbf_dam_401856.md)",
    "dfsph_rate": "ncu, one launch at 401,856 particles (profiles/dfsph_dam_401856.md)",
    "dfsph_density_factor": "ncu, one launch at 401,856 particles (profiles/dfsph_dam_401856.md)",
    "wcsph_density": "ncu at 524,288 particles (profiles/wcsph_bcc_524k.md), scaled by the particle count",
    "wcsph_force": "ncu at 524,288 particles (profiles/wcsph_bcc_524k.md), scaled by the particle count",
}
# Warp instructions per particle per launch from the ncu captures of the
# PBF, WCSPH and DFSPH workloads (PBF lambda: the mean of 36.33 M for the
# reusing launch and 90.41 M for each scanning one; PBF delta: the mean of
# its captured launches).  The neighbour passes are bound by instruction issue, so the bench reports
# the issue rate beside the HBM roofline.  Issue peak = 148 SMs x 4
# schedulers x 1 warp instruction per cycle at the SM clock sampled during
# the timed region.
WARP_INST_PER_PARTICLE = {"pbf_lambda": 76.89e6 / 401856, "pbf_delta": 24.32e6 / 401856,
                          "wcsph_density": 126.16e6 / 524288, "wcsph_force": 49.30e6 / 524288,
                          "dfsph_density_factor": 92.02e6 / 401856, "dfsph_rate": 26.87e6 / 401856}
FALLBACK_HBM_GBS = 6650.0
SUBSTEP_DT = {"pbf": 1.0 / 240.0, "dfsph": 1.0 / 240.0}


class HarnessClock:
    """The reference harness's substep sizes (simulation.py:155-190): PBF
    takes frame_dt / 4; DFSPH takes min(rest of the frame, frame_dt / 4,
    0.4 spacing / max|v|) before every substep.  The speed is a device
    max-norm reduction (fs_norm_maxima) read back between timed steps, never
    inside one; ``speed_of`` replaces it for numpy states (CPU runs)."""

    def __init__(self, kind, spacing, frame_dt=1.0 / 60.0, substeps=4):
        self.kind, self.spacing = kind, float(spacing)
        self.frame_dt, self.limit = frame_dt, frame_dt / substeps
        self.remaining = frame_dt
        self._out = None

    def _speed(self, v):
        if isinstance(v, np.ndarray):
            return float(np.sqrt((v.astype(np.float64) ** 2).sum(1).max())) if len(v) else 0.0
        import torch
        from fluid_simulation_b200 import _lib
        if self._out is None:
            self._out = torch.zeros(2, dtype=torch.float32, device=v.device)
        _lib.check(_lib.load().fs_norm_maxima(v.data_ptr(), v.shape[0], None, 0, self._out.data_ptr(),
                                              torch.cuda.current_stream(v.device).cuda_stream), "norm maxima")
        return float(self._out[0].item()) ** 0.5

    def next(self, v):
        if self.kind != "dfsph":
            return self.limit
        speed = self._speed(v)
        dt = self.limit if speed <= 0.0 else min(self.limit, 0.4 * self.spacing / speed)
        dt = min(self.remaining, dt)
        self.remaining -= dt
        if self.remaining <= 1.0e-12:
            self.remaining = self.frame_dt
        return dt


def measured_peak():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback"


# ------------------------------------------------------------- workloads ----
def build_workload(name, device):
    """(model, solver, dt, n, description)."""
    from fluid_simulation_b200.dam_break import material, solver_config
    from fluid_simulation_b200.newton_shim import model_from_arrays
    from fluid_simulation_b200.scene import make_scene
    from fluid_simulation_b200.solver import SolverDFSPH, SolverPBF, SolverWCSPH
    desc = workload_desc(name)
    if name in ("pbf_dam_401856", "dfsph_dam_401856", "pbf_dam_401856_scorr"):
        kind = name.split("_")[0]
        s = make_scene(400000)
        cls = {"pbf": SolverPBF, "dfsph": SolverDFSPH}[kind]
        attrs = dict(material(kind, s), particle_mask=0)
        m = model_from_arrays(s.positions, np.zeros_like(s.positions), s.mass, device=device, radius=s.radius,
                              gravity=(s.spec.gravity,), attributes=attrs, solver_cls=cls)
        cfg = solver_config(kind, s)
        if name.endswith("_scorr"):
            # artificial pressure on, at the solver class's defaults (k = 1e-4, n = 4, q = 0.3)
            d = SolverPBF.PbfConfig()
            cfg = dataclasses.replace(cfg, scorr_k=d.scorr_k, scorr_n=d.scorr_n, scorr_q=d.scorr_q)
        return m, cls(m, cfg), SUBSTEP_DT[kind], s.count, desc
    if name in ("wcsph_stress_4m", "wcsph_stress_524k"):
        x, v, sp, half, box, dt, cells = stress_setup(name)
        m = model_from_arrays(x, v, 1000.0 * sp ** 3, device=device, radius=0.5 * sp,
                              attributes=dict(rest_density=1000.0, surface_tension=0.0, viscosity=1e-6,
                                              stiffness=2.5e5, exponent=7.0, particle_mask=0), solver_cls=SolverWCSPH)
        solver = SolverWCSPH(m, SolverWCSPH.SphConfig(particle_radius=0.5 * sp, particle_length=sp,
                                                      smoothing_length_coff=2.0, boundary_damping=0.0,
                                                      bound_width=half, bound_height=half, bound_length=half))
        return m, solver, dt, len(x), desc
    raise SystemExit(f"unknown workload {name}")


def stress_setup(name):
    """Lattice, spacing, tank half-width and fixed acoustic dt of a WCSPH
    stress workload: BCC 2 x 128^3 = 4,194,304 particles at d = 9.92 mm in
    a 1.6 m cube, or (the small case of the profiling captures) 2 x 64^3 in
    a 0.8 m cube at the same spacing."""
    from fluid_simulation_b200.scene import stress_lattice
    cells, box = (128, 1.6) if name == "wcsph_stress_4m" else (64, 0.8)
    x, v, sp = stress_lattice(cells=cells, box=box)
    c0 = (2.5e5 * 7.0 / 1000.0) ** 0.5
    dt = 0.25 * (2.0 * sp) / (c0 + float(np.linalg.norm(v, axis=1).max()))
    return x, v, sp, 0.5 * box, box, dt, cells


def workload_desc(name):
    """The workload's description (the bench line's config), without a GPU."""
    if name.startswith("wcsph_stress"):
        x, v, sp, half, box, dt, cells = stress_setup(name)
        return dict(workload=name, particles=len(x), scene=f"jittered BCC lattice 2 x {cells}^3 filling "
                    f"[-{half},{half}]^2 x [0,{box}] m, v ~ N(0, 0.2)", solver="WCSPH", dt=dt, h=2.0 * sp,
                    spacing=sp)
    from fluid_simulation_b200.scene import make_scene
    kind = name.split("_")[0]
    s = make_scene(400000)
    desc = dict(workload=name, particles=s.count, scene="make_scene(400000) dam break", solver=kind.upper(),
                dt=SUBSTEP_DT[kind] if kind == "pbf" else "harness CFL: min(rest of frame, 1/240, 0.4 spacing / "
                "max|v|)", spacing=s.spacing)
    if kind == "pbf":
        scorr = ("on (k=0.0001, n=4, q=0.3: the solver class defaults)" if name.endswith("_scorr")
                 else "off (harness scorr_k=0)")
        desc.update(constraint_iterations=4, substeps_per_frame=4, artificial_pressure=scorr, xsph_c=0.05)
    else:
        desc.update(max_rho_iterations=5, max_vel_iterations=12, warm_start=False)
    return desc


def cpu_oracle_setup(name):
    """Oracle-form model/state/config of the same workload (numpy), and its
    substep clock."""
    from dataclasses import asdict
    if name.startswith("wcsph_stress"):
        x, v, sp, half, box, dt, cells = stress_setup(name)
        n = len(x)
        mat = dict(rest_density=1000.0, surface_tension=0.0, viscosity=1e-6, stiffness=2.5e5, exponent=7.0)
        sph = {k: np.full(n, val, np.float32) for k, val in mat.items()}
        sph["particle_mask"] = np.zeros(n, np.int32)
        model = dict(particle_flags=np.ones(n, np.int32), particle_mass=np.full(n, 1000.0 * sp ** 3, np.float32),
                     particle_world=np.zeros(n, np.int32), gravity=np.array([[0.0, 0.0, -10.0]], np.float32),
                     particle_max_radius=0.5 * sp, sph=sph)
        cfg = dict(particle_radius=0.5 * sp, particle_length=sp, smoothing_length_coff=2.0, boundary_damping=0.0,
                   bound_width=half, bound_height=half, bound_length=half, clamp_negative_pressure=True)
        clock = HarnessClock("wcsph", sp)
        clock.next = lambda v: dt  # fixed acoustic dt, as on the GPU
        return "wcsph", model, dict(particle_q=x, particle_qd=v, sph={}), cfg, n, clock
    from fluid_simulation_b200.dam_break import material, solver_config
    from fluid_simulation_b200.scene import make_scene
    kind = name.split("_")[0]
    s = make_scene(400000)
    n = s.count
    mat = material(kind, s)
    sph = {k: np.full(n, val, np.float32) for k, val in mat.items()}
    sph["particle_mask"] = np.zeros(n, np.int32)
    model = dict(particle_flags=np.ones(n, np.int32), particle_mass=np.full(n, s.mass, np.float32),
                 particle_world=np.zeros(n, np.int32), gravity=np.array([s.spec.gravity], np.float32),
                 particle_max_radius=s.radius, sph=sph)
    state = dict(particle_q=s.positions.copy(), particle_qd=np.zeros_like(s.positions), sph={})
    cfg = asdict(solver_config(kind, s))
    if name.endswith("_scorr"):  # as build_workload: artificial pressure at the class defaults
        from fluid_simulation_b200.solver import SolverPBF
        d = SolverPBF.PbfConfig()
        cfg.update(scorr_k=d.scorr_k, scorr_n=d.scorr_n, scorr_q=d.scorr_q)
    return kind, model, state, cfg, n, HarnessClock(kind, cfg["particle_length"])


def oracle_stepper(kind):
    import oracle
    step = {"pbf": oracle.pbf_step, "dfsph": oracle.dfsph_step, "wcsph": oracle.wcsph_step}[kind]

    def advance(model, state, cfg, dt):
        out = step(model, state, cfg, dt)[0]
        return dict(particle_q=out["particle_q"], particle_qd=out["particle_qd"], sph={})
    return advance


def time_cpu_baseline(name, max_seconds=20.0, max_steps=1000, min_steps=1, single_thread_seconds=8.0):
    """Substeps of the CPU oracle from the workload's initial state until
    max_seconds have passed, on all host threads; then
    (single_thread_seconds > 0) the same on one thread."""
    import oracle
    kind, model, state0, cfg, n, _ = cpu_oracle_setup(name)
    advance = oracle_stepper(kind)

    def run(seconds):
        clock = cpu_oracle_setup(name)[5] if kind == "wcsph" else HarnessClock(kind, cfg["particle_length"])
        state, k = state0, 0
        t0 = time.perf_counter()
        while k < max_steps and (k < min_steps or time.perf_counter() - t0 < seconds):
            state = advance(model, state, cfg, clock.next(state["particle_qd"]))
            k += 1
        return k, time.perf_counter() - t0

    all_threads = os.cpu_count() or 1
    cores = oracle.num_threads(all_threads)
    k, el = run(max_seconds)
    rec = dict(value=n * k / el, unit="particle-steps/s", cores=cores, kind="port",
               sample=f"the first {k} consecutive substeps of the full {n}-particle workload from its initial "
                      f"state in {el:.1f} s (C++ restatement of the reference solver, OpenMP, {cores} threads)")
    if single_thread_seconds > 0:
        oracle.num_threads(1)
        try:
            k1, el1 = run(single_thread_seconds)
        finally:
            oracle.num_threads(all_threads)
        rec["single_thread"] = dict(value=n * k1 / el1, cores=1,
                                    sample=f"the first {k1} of those substeps on one thread in {el1:.1f} s")
    return rec


# ------------------------------------------------------ batched scenes ----
def batched_configs(batch, kind):
    """Solver config and dt of a batch of dam-break scenes: the reference
    harness's PBF config (4 iterations, ...) at dt = 1/240, its DFSPH config
    (5 density / 12 divergence iterations, no warm start) at the harness's
    1/240 cap (the columns start at rest, and after the timed frames they
    fall at under 1 m/s, below the 0.4 spacing / max|v| limit), or WCSPH at
    the acoustic limit 0.25 h / c0 of the stiffest scene.  Walls come from
    each scene (the config's bound_* apply only to the plain per-scene runs)."""
    from fluid_simulation_b200.solver import SolverDFSPH, SolverPBF, SolverWCSPH
    common = dict(particle_radius=batch.radius, particle_length=batch.spacing, smoothing_length_coff=2.0,
                  boundary_damping=0.0)
    if kind == "dfsph":
        return SolverDFSPH, (lambda walls: SolverDFSPH.SphConfig(
            max_rho_iterations=5, max_vel_iterations=12, warm_start=False, max_kappa=1.0, max_kappa_v=100.0,
            bound_width=walls[0], bound_height=walls[1], bound_length=walls[2], **common)), 1.0 / 240.0, 4
    if kind == "pbf":
        return SolverPBF, (lambda walls: SolverPBF.PbfConfig(
            max_iterations=4, lambda_epsilon=100.0, min_neighbors_for_lambda=8, scorr_k=0.0,
            max_delta_position=batch.radius * 0.5, xsph_c=0.05, bound_width=walls[0], bound_height=walls[1],
            bound_length=walls[2], **common)), 1.0 / 240.0, 4
    c0 = (max(s.stiffness for s in batch.scenes) * 7.0 / 1000.0) ** 0.5
    return SolverWCSPH, (lambda walls: SolverWCSPH.SphConfig(
        bound_width=walls[0], bound_height=walls[1], bound_length=walls[2], **common)), 0.25 * batch.h / c0, 8


def time_batched(kind, dev, flush, frames=2, warm=1):
    """All scenes of make_batch() (256 dam-break scenes, ~6.2 M particles)
    advanced as one batched model, a frame of substeps replayed from one CUDA
    graph, against the same scenes run one by one with the plain solver
    (eagerly, and with one frame graph per scene).  Both start from the same
    state and run the same frames; their final states are compared bit for
    bit (equal error: the batched step reproduces each scene's plain step)."""
    import torch
    from fluid_simulation_b200 import _lib
    from fluid_simulation_b200.batch import batched_model, make_batch, scene_model
    from fluid_simulation_b200.graph import FrameGraph
    lib = _lib.load()
    b = make_batch()
    cls, cfg_of, dt, sub = batched_configs(b, kind)
    n = b.total

    def timed(run, nframes):
        tot = 0.0
        for _ in range(nframes):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            run()
            e1.record()
            flush.zero_()
            e1.synchronize()
            tot += e0.elapsed_time(e1)
        return tot

    # batched: one model, one graph per frame
    mb = batched_model(b, cls, device=dev)
    sb = cls(mb, cfg_of((1.0, 1.0, 1.0)))
    ctx_b = mb.particle_grid._ctx
    from fluid_simulation_b200.autotune import autotune, describe
    tuning = describe(autotune(sb, mb.state(), dt, steps=2, repeats=1))  # the serial solvers keep the default
    l0 = lib.fs_launch_count(ctx_b)
    fb = FrameGraph(sb, mb.state(), mb.state(), dt, substeps=sub, warmup=False)
    launches_b = lib.fs_launch_count(ctx_b) - l0   # kernels recorded in the frame graph
    timed(fb.replay, warm)
    t_batched = timed(fb.replay, frames)
    # serial: the same scenes, one plain model and solver each
    scenes = []
    for k, s in enumerate(b.scenes):
        m = scene_model(b, k, cls, device=dev)
        scenes.append((m, cls(m, cfg_of(s.walls)), m.state(), m.state()))

    def serial_frame():
        for i, (m, sv, a, c) in enumerate(scenes):
            for _ in range(sub):
                sv.step(a, c, None, None, dt)
                a, c = c, a
            scenes[i] = (m, sv, a, c)

    timed(serial_frame, warm)
    l0 = sum(lib.fs_launch_count(m.particle_grid._ctx) for m, *_ in scenes)
    t_serial = timed(serial_frame, frames)
    launches_s = sum(lib.fs_launch_count(m.particle_grid._ctx) for m, *_ in scenes) - l0
    graphs = [FrameGraph(sv, a, c, dt, substeps=sub, warmup=False) for m, sv, a, c in scenes]

    def serial_graphs():
        for g in graphs:
            g.replay()

    timed(serial_graphs, warm)
    t_serial_g = timed(serial_graphs, frames)
    # same number of frames on both sides: batched runs as many as the serial side ran
    for _ in range(warm + frames):
        fb.replay()
    torch.cuda.synchronize()
    xb = fb.result.particle_q
    same = all(torch.equal(xb[int(b.starts[k]):int(b.starts[k + 1])], g.result.particle_q)
               for k, g in enumerate(graphs))
    extra = {}
    if kind == "dfsph":  # per-world decisions: each scene's iteration counts as it took them alone
        per_world = sb.last_world_iterations()
        alone = [sv.last_iterations() for m, sv, a, c in scenes]
        key = lambda d: (d["rho_iterations"], d["vel_iterations"])
        extra = dict(iterations_equal_to_serial=all(key(p) == key(q) for p, q in zip(per_world, alone)),
                     last_substep_iterations=dict(
                         rho=dict(min=min(p["rho_iterations"] for p in per_world),
                                  max=max(p["rho_iterations"] for p in per_world)),
                         vel=dict(min=min(p["vel_iterations"] for p in per_world),
                                  max=max(p["vel_iterations"] for p in per_world))))
    rate = lambda ms: round(n * sub * frames / (ms * 1e-3), 1)
    rec = dict(workload=f"batched_{kind}_256", solver=kind.upper(), scenes=len(b.scenes), particles=n,
               scene_counts="log-uniform [2000, 100000], seed 3; column fraction U(0.2, 0.6); stiffness and "
                            "viscosity x U(0.8, 1.2)", spacing=b.spacing, dt=dt, substeps_per_frame=sub,
               frames=frames, value=rate(t_batched), unit="particle-steps/s",
               ms_per_frame=round(t_batched / frames, 3), launches_per_frame_batched=int(launches_b),
               serial_eager=dict(value=rate(t_serial), ms_per_frame=round(t_serial / frames, 3),
                                 launches_per_frame=launches_s // frames),
               serial_graph=dict(value=rate(t_serial_g), ms_per_frame=round(t_serial_g / frames, 3)),
               speedup_vs_serial_eager=round(t_serial / t_batched, 2),
               speedup_vs_serial_graph=round(t_serial_g / t_batched, 2),
               final_state_bit_identical_to_serial=bool(same), tuning_batched=tuning, **extra)
    del fb, graphs, scenes, mb, sb
    torch.cuda.empty_cache()
    return rec


# ------------------------------------------------------- APIC separation ----
def time_separation(dev, flush, reps=20, cpu_reps=2):
    """SolverAPIC's particle-separation pass (solver_apic.py:1003-1064, the
    reference defaults: 2 iterations, strength 0.55, rest distance 2 x the
    particle radius, wall margin = radius) on make_scene(400000)'s column in
    the dam-break tank, its lattice jittered by U(-0.2, 0.2) spacing (seed
    11) so that neighbours sit inside the rest distance.  Device time per
    call (CUDA events, L2 flushed between calls, each call from the same
    input) against the oracle restatement on the host cores."""
    import torch
    import oracle
    from fluid_simulation_b200.apic import ParticleSeparation
    from fluid_simulation_b200.newton_shim import model_from_arrays
    from fluid_simulation_b200.scene import make_scene
    s = make_scene(400000)
    rng = np.random.default_rng(11)
    x = (s.positions + rng.uniform(-0.2, 0.2, s.positions.shape) * s.spacing).astype(np.float32)
    m = model_from_arrays(x, np.zeros_like(x), s.mass, device=dev, radius=s.radius)
    sep = ParticleSeparation(m, ParticleSeparation.Config(bound_lo=s.spec.bound_lo, bound_hi=s.spec.bound_hi))
    st = m.state()
    x0 = st.particle_q.clone()
    times = []
    for r in range(reps + 3):
        st.particle_q.copy_(x0)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        sep.apply(st)
        e1.record()
        flush.zero_()
        e1.synchronize()
        if r >= 3:
            times.append(e0.elapsed_time(e1))
    xg = st.particle_q.cpu().numpy()
    p = sep.parameters()
    cores = oracle.num_threads(os.cpu_count() or 1)
    t0 = time.perf_counter()
    for _ in range(cpu_reps):
        xo, _ = oracle.apic_separation(x, m.particle_flags.cpu().numpy(), p, "f32")
    t_cpu = (time.perf_counter() - t0) / cpu_reps * 1e3
    ms = float(np.median(times))
    n, it = s.count, p["iterations"]
    rec = dict(workload="apic_separation_401856", particles=n, iterations=it, rest_dist=p["rest_dist"],
               grid_dims=list(p["dims"]), value=round(n * it / (ms * 1e-3), 1), unit="particle-separations/s",
               ms_per_call=round(ms, 4), cpu_oracle=dict(ms_per_call=round(t_cpu, 2), cores=cores),
               speedup_vs_cpu=round(t_cpu / ms, 1), bit_identical_to_oracle=bool(np.array_equal(xg, xo)))
    del sep, m, st
    torch.cuda.empty_cache()
    return rec


# ------------------------------------------------------------- metrics ----
def time_metrics(dev, reps=20):
    """The harness's per-frame metrics (simulation.py:198-225) on the WCSPH
    dam break at 401,856 particles after one frame: reduced on the device
    (fs_frame_metrics, 14 doubles read back) against the reference's way
    (copy x, v, rho, p to the host and reduce with numpy).  Wall time per
    call, both ending with the values on the host."""
    import torch
    from fluid_simulation_b200.dam_break import DamBreakSimulation
    from fluid_simulation_b200.scene import make_scene
    sim = DamBreakSimulation(make_scene(400000), "wcsph", device=dev)
    sim.step()
    torch.cuda.synchronize()

    def wall(fn, k):
        fn()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for _ in range(k):
            out = fn()
        return (time.perf_counter() - t0) / k * 1e3, out

    t_dev, m_dev = wall(sim.metrics, reps)
    sys.path.insert(0, os.path.join(os.path.dirname(os.path.abspath(__file__)), "tests"))
    from numpy_metrics import numpy_frame_metrics  # the reference's way, to compare against
    t_host, m_host = wall(lambda: numpy_frame_metrics(sim), max(3, reps // 4))
    exact = ("speed_max", "height_min", "height_max", "density_min", "density_max", "density_p99", "pressure_min",
             "pressure_max")
    worst_mean = max(abs(m_dev[k] - m_host[k]) / max(abs(m_host[k]), 1e-30) for k in ("height_mean", "density_mean"))
    rec = dict(workload="metrics_wcsph_dam_401856", particles=sim.scene.count, frame=sim.frame,
               device_ms=round(t_dev, 4), host_numpy_ms=round(t_host, 3), speedup=round(t_host / t_dev, 1),
               d2h_bytes_device=14 * 8, d2h_bytes_host=sim.scene.count * (12 + 12 + 4 + 4),
               extrema_and_p99_equal=all(m_dev[k] == m_host[k] for k in exact), means_max_rel_diff=worst_mean)
    del sim
    torch.cuda.empty_cache()
    return rec


# ------------------------------------------------------------- adjoint ----
def time_adjoint(dev, flush, batched=False, steps=120, k=10, reps=3):
    """Differentiable WCSPH: forward of ``steps`` substeps (the plain drop-in
    step) against forward + backward through DiffWCSPH (checkpoint every k
    substeps, segments replayed in the backward).  Loss: mean squared distance
    of the final positions to the initial ones moved by +0.3 m in x;
    gradients w.r.t. v0 [N, 3], stiffness, viscosity and rest density.
    Workload: make_scene(50000) (50,232 particles) with a seeded N(0, 0.1
    m/s) initial velocity field, so that pressure and viscosity act (the
    gradient tests' active_column), or, batched, the 256 scenes of
    make_batch() as one model (at rest)."""
    import torch
    from fluid_simulation_b200.batch import batched_model, make_batch
    from fluid_simulation_b200.dam_break import material, solver_config
    from fluid_simulation_b200.diff import DiffWCSPH
    from fluid_simulation_b200.graph import FrameGraph
    from fluid_simulation_b200.newton_shim import model_from_arrays
    from fluid_simulation_b200.solver import SolverWCSPH
    if batched:
        b = make_batch()
        _, cfg_of, dt, _ = batched_configs(b, "wcsph")
        model = batched_model(b, SolverWCSPH, device=dev)
        cfg = cfg_of((1.0, 1.0, 1.0))
        stiff = torch.as_tensor(b.per_particle("stiffness"), device=dev)
        visc = torch.as_tensor(b.per_particle("viscosity"), device=dev)
        rest = torch.full_like(stiff, 1000.0)
        desc = dict(workload="batched_adjoint_wcsph_256", scenes=len(b.scenes), particles=b.total)
        v_init = torch.zeros_like(model.particle_q)
    else:
        sys.path.insert(0, os.path.join(ROOT, "tests"))
        from adjoint_util import active_column  # the gradient tests' workload
        s, _, _, x_np, v_np, dt = active_column()
        attrs = dict(material("wcsph", s), particle_mask=0)
        model = model_from_arrays(x_np, v_np, s.mass, device=dev, radius=s.radius,
                                  gravity=(s.spec.gravity,), attributes=attrs, solver_cls=SolverWCSPH)
        cfg = solver_config("wcsph", s)
        stiff, visc, rest = (torch.tensor(v, device=dev) for v in (2.5e5, 1.0e-6, 1000.0))
        v_init = torch.as_tensor(v_np, device=dev)
        desc = dict(workload="adjoint_wcsph_50232", scene="make_scene(50000) dam-break column, v0 ~ N(0, 0.1 m/s) "
                    "(seed 21): pressure and viscosity act, no wall contact", particles=s.count)
    n = model.particle_count
    x0 = model.particle_q.clone()
    target = x0 + torch.tensor([0.3, 0.0, 0.0], device=dev)
    sim = DiffWCSPH(model, cfg, dt, checkpoint_every=k)
    sim_replay = DiffWCSPH(model, cfg, dt, checkpoint_every=k, record_bytes=0)
    solver = SolverWCSPH(model, cfg)
    fa, fc = model.state(), model.state()
    fwd_graph = FrameGraph(solver, fa, fc, dt, substeps=steps, warmup=False)

    def forward_only():  # the plain substeps, all of them in one CUDA graph
        fa.particle_q.copy_(x0)
        fa.particle_qd.copy_(v_init)
        fwd_graph.replay()

    def forward_eager():
        a, c = model.state(), model.state()
        a.particle_qd.copy_(v_init)
        for _ in range(steps):
            solver.step(a, c, None, None, dt)
            a, c = c, a

    def fwd_bwd(which=sim):
        leaves = [x0.clone().requires_grad_(), v_init.clone().requires_grad_()] + \
                 [t.clone().requires_grad_() for t in (stiff, visc, rest)]
        xT, _ = which.rollout(*leaves, steps)
        loss = ((xT - target) ** 2).sum(1).mean()
        loss.backward()
        return leaves

    def timed(fn):
        fn()  # warm-up (records the CUDA graphs)
        torch.cuda.synchronize()
        ts = []
        for _ in range(reps):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            out = fn()
            e1.record()
            flush.zero_()
            e1.synchronize()
            ts.append(e0.elapsed_time(e1))
        return statistics.median(ts), out

    t_f, _ = timed(forward_only)
    t_fe, _ = timed(forward_eager)
    t_fb, leaves = timed(fwd_bwd)
    t_fbr, _ = timed(lambda: fwd_bwd(sim_replay))
    gnorm = {nm: float(t.grad.norm()) for nm, t in zip(("x0", "v0", "stiffness", "viscosity", "rest_density"),
                                                        leaves)}
    rec = dict(desc, solver="WCSPH", dt=dt, substeps=steps, checkpoint_every=k, value=round(n * steps / (t_fb * 1e-3), 1),
               unit="particle-steps/s (forward + backward)", ms_forward=round(t_f, 3),
               ms_forward_eager=round(t_fe, 3), ms_forward_backward=round(t_fb, 3),
               ratio_fwd_bwd_to_forward=round(t_fb / t_f, 3), ratio_fwd_bwd_to_forward_eager=round(t_fb / t_fe, 3),
               segment_records_kept=min(sim.max_records, (steps + k - 1) // k),
               replay_all_but_last=dict(ms_forward_backward=round(t_fbr, 3), ratio_fwd_bwd_to_forward=round(t_fbr / t_f, 3),
                                        record_bytes=0),
               forward_value=round(n * steps / (t_f * 1e-3), 1), grad_norms=gnorm,
               forward="plain WCSPH substeps replayed from one CUDA graph (eager: one solver.step per substep)",
               backward="DiffWCSPH: checkpoints every k substeps; segment records kept within a quarter of free "
                        "device memory, other segments replayed; CUDA graph per segment")
    del sim, sim_replay, solver, model, fwd_graph
    torch.cuda.empty_cache()
    return rec


# ------------------------------------------- WCSPH dam break, 60 frames ----
def time_dam_60_frames(dev, target=10000, frames=60, cpu_seconds=20.0):
    """The reference's CPU-runnable case: the WCSPH dam break of
    make_scene(10000) (9,936 particles) for 60 display frames of 1/60 s
    with the harness's CFL substeps (simulation.py:155-196), on the GPU
    (DamBreakSimulation with the host loop, as the reference runs it, and
    graph.DeviceFrameLoop) and with the CPU oracle on all host threads (the
    harness restated over the oracle, tests/kat_util.OracleDamBreak) for as
    many frames as fit in cpu_seconds.  Trajectories diverge chaotically,
    so GPU and CPU are compared on kinetic energy and density statistics
    after the frames the CPU ran.  Wall time per frame (the CFL readback
    makes the host loop host-bound at this size)."""
    import torch
    import oracle
    from fluid_simulation_b200.dam_break import DamBreakSimulation
    from fluid_simulation_b200.graph import DeviceFrameLoop
    from fluid_simulation_b200.scene import make_scene
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    from kat_util import OracleDamBreak
    s = make_scene(target)
    n = s.count

    def stats(x, v, rho):
        ke = 0.5 * float(s.mass) * float((v.astype(np.float64) ** 2).sum())
        return dict(kinetic_energy=ke, density_p99=float(np.percentile(rho, 99)), density_mean=float(rho.mean()),
                    height_mean=float(x[:, 2].mean()))

    out = dict(workload=f"wcsph_dam_{n}_60_frames", particles=n, frames=frames)
    cores = oracle.num_threads(os.cpu_count() or 1)
    cpu = OracleDamBreak(s, "wcsph")
    t0 = time.perf_counter()
    kc = 0
    while kc < frames and (kc == 0 or time.perf_counter() - t0 < cpu_seconds):
        cpu.step()
        kc += 1
    el = time.perf_counter() - t0
    out["cpu_oracle"] = dict(frames=kc, ms_per_frame=round(el / kc * 1e3, 3), substeps=int(cpu.total_substeps),
                             value=round(n * cpu.total_substeps / el, 1), unit="particle-steps/s (wall)", cores=cores,
                             stats_at_its_last_frame=stats(cpu.x, cpu.v, cpu.sph["rho"]))
    for name, make in (("gpu_host_loop", lambda: DamBreakSimulation(s, "wcsph", device=dev)),
                       ("gpu_device_loop", lambda: DeviceFrameLoop(DamBreakSimulation(s, "wcsph", device=dev),
                                                                   graph_substeps=64))):
        run = make()
        sim = run if isinstance(run, DamBreakSimulation) else run.sim
        torch.cuda.synchronize()
        el, at_kc = 0.0, None
        for k in range(frames):
            t0 = time.perf_counter()
            run.step()
            torch.cuda.synchronize()
            el += time.perf_counter() - t0
            if k + 1 == kc:
                st = sim.state_0
                at_kc = stats(st.particle_q.cpu().numpy(), st.particle_qd.cpu().numpy(), st.sph.rho.cpu().numpy())
        st = sim.state_0
        out[name] = dict(ms_per_frame=round(el / frames * 1e3, 3), substeps=int(sim.total_substeps),
                         value=round(n * sim.total_substeps / el, 1), unit="particle-steps/s (wall)",
                         stats_after_cpu_frames=at_kc,
                         stats_after_60_frames=stats(st.particle_q.cpu().numpy(), st.particle_qd.cpu().numpy(),
                                                     st.sph.rho.cpu().numpy()))
        del run, sim
    out["speedup_gpu_device_loop_vs_cpu"] = round(out["cpu_oracle"]["ms_per_frame"] /
                                                  out["gpu_device_loop"]["ms_per_frame"], 1)
    torch.cuda.empty_cache()
    return out


# -------------------------------------------------- harness frame loop ----
def time_frame_loop(dev, flush, target=400000, frames=2, method="wcsph"):
    """WCSPH or DFSPH dam-break display frames (make_scene(target), CFL substeps of
    the reference harness) with the host loop (max |v|, |a| read back before
    every substep, as simulation.py:155-196) against graph.DeviceFrameLoop
    (the rule on the device, one graph of 64 clocked substeps replayed until
    the frame is done).  Both run the same frames from the same state; the
    line reports whether they end in the same bits."""
    import torch
    from fluid_simulation_b200.dam_break import DamBreakSimulation
    from fluid_simulation_b200.graph import DeviceFrameLoop
    from fluid_simulation_b200.scene import make_scene
    s = make_scene(target)
    host = DamBreakSimulation(s, method, device=dev)
    devs = DamBreakSimulation(s, method, device=dev)
    loop = DeviceFrameLoop(devs, graph_substeps=64 if method == "wcsph" else devs.substeps)
    host.step()
    loop.step()  # first frame: warm-up of both
    torch.cuda.synchronize()

    def timed(fn):
        tot, sub = 0.0, 0
        for _ in range(frames):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            fn()
            e1.record()
            e1.synchronize()
            tot += e0.elapsed_time(e1)
            flush.zero_()
            torch.cuda.synchronize()
        return tot

    t_host = timed(host.step)
    t_dev = timed(loop.step)
    same = bool(torch.equal(host.state_0.particle_q, devs.state_0.particle_q))
    n = s.count
    rec = dict(workload=f"{method}_dam_frames_{n}", particles=n, frames=frames,
               substeps_per_frame=host.last_substeps, ms_per_frame_host_loop=round(t_host / frames, 3),
               ms_per_frame_device_loop=round(t_dev / frames, 3), speedup=round(t_host / t_dev, 3),
               value=round(n * host.last_substeps * frames / (t_dev * 1e-3), 1), unit="particle-steps/s (device loop)",
               graph_replays=loop.replays, final_state_bit_identical=same, total_substeps=int(host.total_substeps))
    del host, devs, loop
    torch.cuda.empty_cache()
    return rec


# --------------------------------------------------------------- clocks ----
class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                                          "-lms", "100", "-i", str(self.gpu)], stdout=subprocess.PIPE,
                                         stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.t.join(timeout=2)
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for nm, val in zip(names, f[5:9]):
                if val.lower().startswith("active"):
                    reasons.add(nm)
        if not sm:
            return None
        return dict(sm_mhz=statistics.median(sm), sm_max_mhz=mx, reasons=sorted(reasons), samples=len(sm))


# ------------------------------------------------------------- our arm ----
def measure_workload(name, dev, flush, steps, warmup, args, world=1, clocks_gpu=0, cpu_baseline=False):
    """One workload timed the headline's way: W warm-up substeps, K timed
    substeps (CUDA events around each, L2 flushed between them), the
    per-pass event timer on up to 100 further substeps (dominant pass ->
    roofline), then end to end through the solver API with host buffers.
    Returns the record (without rank reduction for world == 1)."""
    import torch
    import torch.distributed as dist
    import ctypes as C
    from fluid_simulation_b200 import _lib
    lib = _lib.load()
    model, solver, dt, n, desc = build_workload(name, dev)
    ctx = model.particle_grid._ctx
    a, b = model.state(), model.state()
    clock = HarnessClock(desc["solver"].lower(), desc.get("spacing", 0.0))
    if desc["solver"] == "WCSPH":
        clock.next = lambda v: dt  # the stress lattice runs at its fixed acoustic dt
    tuning = None
    if not args.no_autotune:  # launch tuning from a few substeps of the initial state, before warm-up
        from fluid_simulation_b200.autotune import autotune, describe
        tuning = describe(autotune(solver, a, clock.limit if clock.kind == "dfsph" else dt))

    def step(dt_k):
        nonlocal a, b
        solver.step(a, b, None, None, dt_k)
        a, b = b, a

    for _ in range(warmup):
        step(clock.next(a.particle_qd))
    torch.cuda.synchronize()

    K = steps
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(K)]
    npass = lib.fs_pass_count()
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    sampler = ClockSampler(clocks_gpu)
    sampler.start()
    time.sleep(0.3)
    launches0 = lib.fs_launch_count(ctx)
    for k in range(K):
        dt_k = clock.next(a.particle_qd)  # DFSPH: reads back max|v| (outside the events)
        ev[k][0].record()
        step(dt_k)
        ev[k][1].record()
        flush.zero_()
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    launches = lib.fs_launch_count(ctx) - launches0
    clk = sampler.stop()
    step_ms = sum(e0.elapsed_time(e1) for e0, e1 in ev)
    iterations = solver.last_iterations() if hasattr(solver, "last_iterations") else None
    # per-pass breakdown: further steps with the per-pass event timer on,
    # outside the timed loop (its event records would sit between the passes)
    Kp = min(K, 100)
    evp = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(Kp)]
    _lib.check(lib.fs_timer_enable(ctx, max(64, 96 * Kp)), "timer")
    for k in range(Kp):
        dt_k = clock.next(a.particle_qd)
        evp[k][0].record()
        step(dt_k)
        evp[k][1].record()
        flush.zero_()
    torch.cuda.synchronize()
    ms = (C.c_float * npass)()
    cnt = (C.c_int32 * npass)()
    dropped = C.c_int32(0)
    _lib.check(lib.fs_timer_read(ctx, ms, cnt, npass, C.byref(dropped)), "timer read")
    instrumented_ms = sum(e0.elapsed_time(e1) for e0, e1 in evp)
    t_local = torch.tensor([step_ms], dtype=torch.float64, device=dev)
    if world > 1:
        dist.all_reduce(t_local, op=dist.ReduceOp.MAX)
    total_ms = float(t_local.item())
    value = world * n * K / (total_ms * 1e-3)

    passes = {}
    for p in range(npass):
        if cnt[p]:
            pname = lib.fs_pass_name(p).decode()
            passes[pname] = dict(ms_total=round(ms[p], 4), launches=int(cnt[p]), ms_avg=round(ms[p] / cnt[p], 5))
    dom = max(passes, key=lambda k: passes[k]["ms_total"])
    peak, peak_kind = measured_peak()
    bpl = B_ALG.get(dom, 0) * n
    achieved = bpl / (passes[dom]["ms_avg"] * 1e-3) / 1e9
    traffic = TRAFFIC_PER_PARTICLE.get(dom)
    roofline = dict(bound="hbm", kernel=dom, achieved=round(achieved, 1), peak=peak, unit="GB/s",
                    frac=round(achieved / peak, 4), peak_source=f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)",
                    traffic=(round(traffic * n) if traffic is not None else None),
                    traffic_source=TRAFFIC_SOURCE.get(dom), bytes_per_launch=bpl,
                    share_of_step=round(passes[dom]["ms_total"] / max(instrumented_ms, 1e-9), 3))
    if dom in WARP_INST_PER_PARTICLE:
        inst = WARP_INST_PER_PARTICLE[dom] * n
        mhz = (clk or {}).get("sm_mhz") or 1965.0
        peak_inst = 148 * 4 * mhz * 1e6
        rate = inst / (passes[dom]["ms_avg"] * 1e-3)
        roofline["issue"] = dict(kernel=dom, warp_instructions_per_launch=round(inst),
                                 achieved_warp_inst_per_s=round(rate), peak_warp_inst_per_s=round(peak_inst),
                                 frac=round(rate / peak_inst, 4), sm_mhz=mhz,
                                 source="warp instructions per particle from the committed ncu capture"
                                 + ("" if name.startswith("pbf") or name.startswith("dfsph") or name.endswith("524k")
                                    else " of the 524,288-particle lattice, scaled by the particle count"))
    bytes_per_step = sum(B_ALG.get(k, 0) * n * v["launches"] for k, v in passes.items()) / Kp
    gbs = bytes_per_step / (step_ms / K * 1e-3) / 1e9
    step_roofline = dict(algorithmic_bytes_per_step=bytes_per_step, achieved_gbs=round(gbs, 1),
                         frac=round(gbs / peak, 4))

    # ---- e2e through the solver API with host state
    Ke = max(3, min(K, args.e2e_steps))
    hx = a.particle_q.cpu().pin_memory()     # continue from the state the timed loop reached
    hv = a.particle_qd.cpu().pin_memory()
    ee = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(Ke)]
    s_in, s_out = model.state(), model.state()
    for k in range(Ke):
        if clock.kind == "dfsph":  # the harness reads max|v| back before each substep
            torch.cuda.current_stream(dev).synchronize()
            dt_k = clock.next(hv.numpy())
        else:
            dt_k = clock.next(None)
        ee[k][0].record()
        s_in.particle_q.copy_(hx, non_blocking=True)
        s_in.particle_qd.copy_(hv, non_blocking=True)
        solver.step(s_in, s_out, None, None, dt_k)
        hx.copy_(s_out.particle_q, non_blocking=True)
        hv.copy_(s_out.particle_qd, non_blocking=True)
        ee[k][1].record()
        flush.zero_()
    torch.cuda.synchronize()
    e2e_ms = sum(e0.elapsed_time(e1) for e0, e1 in ee)
    t_e2e = torch.tensor([e2e_ms], dtype=torch.float64, device=dev)
    if world > 1:
        dist.all_reduce(t_e2e, op=dist.ReduceOp.MAX)
    e2e_value = world * n * Ke / (float(t_e2e.item()) * 1e-3)
    rec = dict(value=round(value, 1), unit="particle-steps/s", steps=K, warmup=warmup,
               ms_per_step=round(total_ms / K, 5), desc=desc, tuning=tuning,
               e2e=dict(value=round(e2e_value, 1), unit="particle-steps/s", h2d_bytes_per_step=2 * n * 12,
                        d2h_bytes_per_step=2 * n * 12, steps=Ke,
                        path=f"host particle_q/qd (pinned) -> {type(solver).__name__}.step -> host"),
               gpu_launches=int(launches), roofline=roofline, step_roofline=step_roofline, passes=passes,
               passes_steps=Kp, passes_ms_per_step=round(instrumented_ms / Kp, 5), timer_dropped=int(dropped.value),
               clocks=clk)
    if iterations is not None:
        rec["iterations_last_timed_step"] = iterations
    del model, solver, a, b, s_in, s_out
    torch.cuda.empty_cache()
    if cpu_baseline:
        rec["cpu_baseline"] = time_cpu_baseline(name, max_seconds=args.cpu_seconds, single_thread_seconds=0)
    return rec


def run_ours(args):
    import torch
    import torch.distributed as dist

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if not torch.cuda.is_available():
        raise SystemExit("bench.py needs a CUDA device")
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120), device_id=dev)
    flush = torch.empty(512 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)
    if args.only:  # one secondary workload by itself (profiling); prints its record, not the bench line
        if args.only == "adjoint":
            rec = time_adjoint(dev, flush, reps=1)
        elif args.only == "frames":
            rec = [time_frame_loop(dev, flush), time_frame_loop(dev, flush, target=50000, frames=3),
                   time_frame_loop(dev, flush, frames=3, method="dfsph")]
        elif args.only == "metrics":
            rec = time_metrics(dev)
        elif args.only == "separation":
            rec = time_separation(dev, flush)
        else:
            rec = time_batched(args.only.split("_")[1], dev, flush, frames=1, warm=1)
        print(json.dumps(dict(only=args.only, record=rec)), flush=True)
        return

    head = measure_workload(args.workload, dev, flush, args.steps, args.warmup, args, world=world, clocks_gpu=local)

    # ---- secondary workloads (same timing rules and step counts), N=1 only
    secondary = {}
    if world == 1 and not args.no_secondary:
        for wl in ("dfsph_dam_401856", "wcsph_stress_4m", "pbf_dam_401856_scorr"):
            if wl == args.workload:
                continue
            rec = measure_workload(wl, dev, flush, args.steps, args.warmup, args, clocks_gpu=local,
                                   cpu_baseline=not args.no_cpu_baseline and wl != "pbf_dam_401856_scorr")
            desc = rec.pop("desc")
            secondary[wl] = dict(desc, **rec)

    if world == 1 and not args.no_secondary and not args.no_batched:
        for kind in ("pbf", "wcsph", "dfsph"):
            secondary[f"batched_{kind}_256"] = time_batched(kind, dev, flush)
    if world == 1 and not args.no_secondary:
        secondary["wcsph_dam_9936_60_frames"] = time_dam_60_frames(dev)
        secondary["wcsph_dam_frames_401856"] = time_frame_loop(dev, flush)
        secondary["wcsph_dam_frames_50232"] = time_frame_loop(dev, flush, target=50000, frames=3)
        secondary["dfsph_dam_frames_401856"] = time_frame_loop(dev, flush, frames=3, method="dfsph")
        secondary["metrics_wcsph_dam_401856"] = time_metrics(dev)
        secondary["apic_separation_401856"] = time_separation(dev, flush)
    if world == 1 and not args.no_secondary and not args.no_adjoint:
        secondary["adjoint_wcsph_50232"] = time_adjoint(dev, flush)
        secondary["batched_adjoint_wcsph_256"] = time_adjoint(dev, flush, batched=True)

    cpu = None
    if world == 1 and not args.no_cpu_baseline:
        cpu = time_cpu_baseline(args.workload, max_seconds=args.cpu_seconds)

    if rank == 0:
        desc = head["desc"]
        line = dict(
            metric="particle-steps/s", value=head["value"], unit="particle-steps/s", n_gpus=world, steps=head["steps"],
            warmup=args.warmup, ms_per_step=head["ms_per_step"], higher_is_better=True, scaling="weak",
            vs_baseline=round(head["value"] / PUBLISHED_PBF, 3) if args.workload == "pbf_dam_401856" else None,
            dtype="f32", data="synthetic (reference dam-break scene generator, seeded)",
            config=dict(desc, l2="flushed between timed steps (512 MB write outside the events)",
                        tuning=head["tuning"],
                        parallelism="replicas" if world > 1 else "single GPU",
                        grid="HashGrid(128,128,128), cell = h, truncating cell coordinates"),
            e2e=head["e2e"], gpu_launches=head["gpu_launches"], roofline=head["roofline"],
            step_roofline=head["step_roofline"], passes=head["passes"], passes_steps=head["passes_steps"],
            passes_ms_per_step=head["passes_ms_per_step"], timer_dropped=head["timer_dropped"],
            clocks=head["clocks"], cpu_baseline=cpu, secondary=secondary or None,
        )
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


def run_reference(args):
    """The reference arm: the reference's CPU path for this workload, which
    here is the C++ restatement of the reference solver (the reference
    itself needs warp-lang + newton, which cannot be installed on these
    hosts), on all host threads.  Same workload, config, warm-up count and
    substep count as the GPU arm: W warm-up substeps from the initial state,
    then K timed ones; only if those would run past --reference-seconds does
    it stop early, and then it times the first k of the K substeps (said in
    the line)."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    import oracle
    kind, model, state, cfg, n, clock = cpu_oracle_setup(args.workload)
    advance = oracle_stepper(kind)
    cores = oracle.num_threads(os.cpu_count() or 1)
    warmup = max(args.warmup, 3)  # the GPU arm's floor
    t_start = time.perf_counter()
    for _ in range(warmup):
        state = advance(model, state, cfg, clock.next(state["particle_qd"]))
    k = 0
    t0 = time.perf_counter()
    while k < args.steps and (k == 0 or time.perf_counter() - t_start < args.reference_seconds):
        state = advance(model, state, cfg, clock.next(state["particle_qd"]))
        k += 1
    el = time.perf_counter() - t0
    value = n * k / el
    window = (f"substeps {warmup + 1}-{warmup + k} (all {args.steps} requested)" if k == args.steps else
              f"substeps {warmup + 1}-{warmup + k}, the first {k} of the {args.steps} requested (stopped at "
              f"{args.reference_seconds:.0f} s)")
    sample = (f"{window} of the full {n}-particle workload after {warmup} warm-up substeps, in {el:.1f} s; "
              f"C++ restatement of the reference solver, OpenMP {cores} threads")
    print(json.dumps(dict(
        impl="reference", metric="particle-steps/s", value=round(value, 1), unit="particle-steps/s", n_gpus=0,
        steps=k, warmup=warmup, ms_per_step=round(el / k * 1e3, 3), higher_is_better=True,
        scaling="weak", vs_baseline=None, dtype="f32", data="synthetic (reference dam-break scene generator, seeded)",
        config=dict(workload_desc(args.workload), l2="host run (no device cache to flush)", tuning=None,
                    parallelism="host threads",
                    grid="HashGrid(128,128,128), cell = h, truncating cell coordinates"),
        cpu_baseline=dict(value=round(value, 1), unit="particle-steps/s", cores=cores, kind="port", sample=sample),
        e2e=dict(value=round(value, 1), unit="particle-steps/s", h2d_bytes_per_step=0, d2h_bytes_per_step=0),
    )), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=300)
    ap.add_argument("--warmup", type=int, default=10)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="pbf_dam_401856",
                    choices=["pbf_dam_401856", "dfsph_dam_401856", "wcsph_stress_4m", "wcsph_stress_524k",
                             "pbf_dam_401856_scorr"])
    ap.add_argument("--e2e-steps", type=int, default=50)
    ap.add_argument("--cpu-seconds", type=float, default=15.0)
    ap.add_argument("--reference-seconds", type=float, default=240.0,
                    help="reference arm: stop the timed substeps early past this many seconds in all")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-secondary", action="store_true")
    ap.add_argument("--no-batched", action="store_true")
    ap.add_argument("--no-adjoint", action="store_true")
    ap.add_argument("--no-autotune", action="store_true")
    ap.add_argument("--only", choices=["adjoint", "batched_pbf", "batched_wcsph", "batched_dfsph", "frames", "metrics", "separation"],
                    help="run one secondary workload alone (profiling); no bench line")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
