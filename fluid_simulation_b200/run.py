"""Headless dam-break runner with the reference example's command line.

``examples/dam_break/run.py`` (parse_args 43-102, main 105-233) runs a
``DamBreakSimulation`` frame by frame, prints a progress line every
``--report-every`` frames, takes the full statistics every
``--metrics-every`` frames (the finite check runs every frame) and writes
``metrics.csv`` and ``run.json`` into the output directory.  This module does
the same for the particle solvers of this package:

    python -m fluid_simulation_b200.run --solver pbf --particles 400000 --frames 300

Options that drive the reference's OpenGL viewer, its surface extraction
and USD export, and the APIC grid solver are accepted by name so that the
reference's command lines parse, but only in their off state: this package
has no graphics path and no APIC grid solver, and asking for one of them is
an error (``--viewer gl``, ``--usd``, ``--solver apic``).  The viewer
default is therefore ``none``.
"""

from __future__ import annotations

import argparse
import csv
import json
import math
import sys
import time
from pathlib import Path

SOLVERS = ("wcsph", "dfsph", "pbf")


def positive_int(text):  # run.py:20-25
    value = int(text)
    if value <= 0:
        raise argparse.ArgumentTypeError("Must be a positive integer")
    return value


def positive_float(text):  # run.py:28-32
    value = float(text)
    if not math.isfinite(value) or value <= 0.0:
        raise argparse.ArgumentTypeError("Must be a finite positive number")
    return value


def nonnegative_float(text):  # run.py:35-39
    value = float(text)
    if not math.isfinite(value) or value < 0.0:
        raise argparse.ArgumentTypeError("Must be a finite non-negative number")
    return value


def parse_args(method=None, argv=None):
    """The reference's options (run.py:43-102) with the same names, defaults
    and checks; graphics, surface, USD and APIC options only in their off
    state."""
    from .scene import DEFAULT_SPEC

    parser = argparse.ArgumentParser(description="Dam-break example on the B200 particle solvers")
    if method is None:
        parser.add_argument("--solver", choices=SOLVERS + ("apic",), default="pbf")
    else:
        parser.set_defaults(solver=method)
    parser.add_argument("--device", default="cuda:0")
    parser.add_argument("--particles", type=positive_int, default=DEFAULT_SPEC.target_count,
                        help="Target particle count of the dam-break lattice")
    parser.add_argument("--frames", type=positive_int, default=300)
    parser.add_argument("--substeps", type=positive_int, default=4,
                        help="Base substeps per 1/60 s frame; SPH may use more for CFL")
    parser.add_argument("--viewer", choices=["gl", "none"], default="none")
    parser.add_argument("--no-viewer", dest="viewer", action="store_const", const="none")
    parser.add_argument("--no-surface", action="store_true")
    parser.add_argument("--show-particles", action="store_true")
    parser.add_argument("--usd", help="not available: no USD export")
    parser.add_argument("--usd-every", type=positive_int, default=1)
    parser.add_argument("--output-dir", type=Path, default=None, help="Metrics and run metadata directory")
    parser.add_argument("--surface-voxel-size", type=positive_float, default=0.007)
    parser.add_argument("--surface-max-grid-cells", type=positive_int, default=None)
    parser.add_argument("--no-anisotropic", action="store_true")
    parser.add_argument("--water-opacity", type=float, default=0.35)
    parser.add_argument("--voxel-size", type=positive_float, default=None, help="APIC simulation voxel size")
    parser.add_argument("--no-projection", action="store_true", help="Disable APIC pressure projection")
    parser.add_argument("--wcsph-stiffness", type=positive_float, default=None,
                        help="WCSPH Tait pressure constant B in Pa (default: 250000)")
    parser.add_argument("--wcsph-viscosity", type=nonnegative_float, default=None,
                        help="WCSPH kinematic viscosity in m^2/s (default: 1e-6)")
    parser.add_argument("--wcsph-smoothing-length-coff", type=positive_float, default=None,
                        help="WCSPH kernel support radius / particle spacing (default: 2)")
    parser.add_argument("--wcsph-allow-negative-pressure", action="store_true",
                        help="Disable the pressure clamp for WCSPH comparisons")
    parser.add_argument("--report-every", type=positive_int, default=10)
    parser.add_argument("--metrics-every", type=positive_int, default=10,
                        help="Full statistics interval; finite-state checks still run every frame")
    parser.add_argument("--no-cuda-interop", action="store_true", help="(viewer option; no effect)")
    args = parser.parse_args(argv)
    if not 0.0 <= args.water_opacity <= 1.0:
        parser.error("--water-opacity must be in [0, 1]")
    if args.solver == "apic":
        parser.error("--solver apic: the APIC grid solver is not part of this package "
                     "(fluid_simulation_b200.apic provides its particle-separation pass)")
    if args.viewer != "none":
        parser.error("--viewer gl: no graphics path in this package; run headless (--viewer none)")
    if args.usd:
        parser.error("--usd: no surface or USD export in this package")
    if args.voxel_size is not None or args.no_projection:
        parser.error("--voxel-size and --no-projection apply to APIC")
    if args.solver != "wcsph" and (
        args.wcsph_stiffness is not None or args.wcsph_viscosity is not None
        or args.wcsph_smoothing_length_coff is not None or args.wcsph_allow_negative_pressure
    ):
        parser.error("--wcsph-* options apply to WCSPH")
    args.output_dir = args.output_dir or Path("output") / args.solver
    return args


def main(method=None, argv=None):
    """run.py:105-233 without the viewer and surface: frames, reports,
    metrics.csv and run.json."""
    import torch

    from .dam_break import DamBreakSimulation
    from .scene import make_scene

    args = parse_args(method, argv)
    args.output_dir.mkdir(parents=True, exist_ok=True)
    scene = make_scene(args.particles)
    print(f"{args.solver.upper()} dam_break: {scene.count} particles, "
          f"radius={scene.radius:.6g} m, spacing={scene.spacing:.6g} m", flush=True)
    print(f"tank={scene.spec.bound_lo} .. {scene.spec.bound_hi}; "
          f"{args.frames} frames at {scene.spec.fps:g} fps", flush=True)
    print(f"ideal flat height={scene.ideal_height:.6f} m; "
          f"ruler=100%, 90%, 80% of rest volume", flush=True)
    wcsph_options = {key: getattr(args, key) for key in
                     ("wcsph_stiffness", "wcsph_viscosity", "wcsph_smoothing_length_coff")
                     if getattr(args, key) is not None}
    sim = DamBreakSimulation(scene, args.solver, args.device, args.substeps,
                             wcsph_clamp_negative_pressure=not args.wcsph_allow_negative_pressure,
                             **wcsph_options)
    if args.solver == "wcsph":
        print(f"WCSPH B={sim.material['stiffness']:g} Pa, "
              f"viscosity={sim.material['viscosity']:g} m^2/s, "
              f"h={sim.solver.smoothing_length:.6g} m, "
              f"non-negative pressure={sim.solver.config.clamp_negative_pressure}", flush=True)

    rows = []
    started = time.perf_counter()
    rows.append(sim.metrics())
    while sim.frame < args.frames:
        sim.step()
        sim.check_finite()
        report_now = sim.frame % args.report_every == 0 or sim.frame == args.frames
        if sim.frame % args.metrics_every == 0 or report_now:
            metrics = sim.metrics()
            rows.append(metrics)
        if report_now:
            print(f"frame {sim.frame}/{args.frames}, t={sim.sim_time:.4f} s, "
                  f"substeps={sim.last_substeps}, vmax={metrics['speed_max']:.4g}, finite=True", flush=True)
    if rows[-1]["frame"] != sim.frame:
        rows.append(sim.metrics())
    elapsed = time.perf_counter() - started
    fieldnames = list(dict.fromkeys(key for row in rows for key in row))
    with (args.output_dir / "metrics.csv").open("w", newline="") as stream:
        writer = csv.DictWriter(stream, fieldnames=fieldnames)
        writer.writeheader()
        writer.writerows(rows)
    dev = sim.model.device
    report = dict(scene=scene.report(), simulation=sim.report(), completed_frames=sim.frame,
                  simulation_seconds=sim.sim_time, elapsed_seconds=elapsed,
                  diagnostics=dict(metrics_every=args.metrics_every, finite_check_every=1),
                  environment=dict(python=sys.version.split()[0], torch=torch.__version__,
                                   device=str(dev), device_name=torch.cuda.get_device_name(dev)),
                  surface=dict(enabled=False), final_metrics=rows[-1])
    (args.output_dir / "run.json").write_text(json.dumps(report, indent=2) + "\n")
    print(f"Finished in {elapsed:.2f} s. Metrics: {args.output_dir}", flush=True)
    return report


if __name__ == "__main__":
    main()
