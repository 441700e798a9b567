"""The headless runner's command line (fluid_simulation_b200.run) against
the reference example's (examples/dam_break/run.py:20-102): same names,
defaults and checks; graphics, USD and APIC options refused."""

import pytest

from fluid_simulation_b200.run import parse_args


def test_reference_command_lines_parse(tmp_path):
    a = parse_args(argv=["--solver", "pbf", "--particles", "400000", "--frames", "300", "--no-viewer",
                         "--no-surface", "--metrics-every", "5", "--output-dir", str(tmp_path)])
    assert (a.solver, a.particles, a.frames, a.substeps, a.viewer) == ("pbf", 400000, 300, 4, "none")
    assert a.metrics_every == 5 and a.report_every == 10 and a.output_dir == tmp_path
    w = parse_args(argv=["--solver", "wcsph", "--wcsph-stiffness", "1e5", "--wcsph-viscosity", "0",
                         "--wcsph-smoothing-length-coff", "2.5", "--wcsph-allow-negative-pressure"])
    assert (w.wcsph_stiffness, w.wcsph_viscosity, w.wcsph_smoothing_length_coff) == (1e5, 0.0, 2.5)
    assert w.wcsph_allow_negative_pressure
    assert parse_args("dfsph", argv=[]).solver == "dfsph"  # the per-solver entry points


@pytest.mark.parametrize("argv", [
    ["--frames", "0"], ["--particles", "-3"], ["--substeps", "x"],
    ["--solver", "pbf", "--wcsph-stiffness", "1e5"],      # WCSPH options with another solver
    ["--solver", "wcsph", "--wcsph-viscosity", "-1"],
    ["--solver", "wcsph", "--wcsph-stiffness", "inf"],
    ["--water-opacity", "1.5"],
    ["--solver", "apic"], ["--viewer", "gl"], ["--usd", "out.usd"], ["--voxel-size", "0.01"],
    ["--no-projection"],
])
def test_invalid_or_unavailable_options_exit(argv):
    with pytest.raises(SystemExit):
        parse_args(argv=argv)
