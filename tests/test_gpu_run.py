"""The headless runner end to end: a few frames of each particle solver,
metrics.csv and run.json written as the reference example writes them."""

import csv
import json

import pytest

from fluid_simulation_b200.run import main

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("solver", ["wcsph", "dfsph", "pbf"])
def test_runner_writes_metrics_and_report(solver, tmp_path, cuda_device):
    report = main(solver, argv=["--particles", "10000", "--frames", "2", "--report-every", "1",
                                "--metrics-every", "1", "--device", str(cuda_device), "--output-dir", str(tmp_path)])
    assert report["completed_frames"] == 2
    rows = list(csv.DictReader((tmp_path / "metrics.csv").open()))
    assert [int(r["frame"]) for r in rows] == [0, 1, 2]
    assert all(r["finite"] == "True" for r in rows)
    run = json.loads((tmp_path / "run.json").read_text())
    assert run["scene"]["actual_count"] == 9936 and run["simulation"]["method"] == solver
    assert run["final_metrics"]["frame"] == 2 and run["surface"] == {"enabled": False}
    assert abs(run["simulation_seconds"] - 2.0 / 60.0) < 1e-9
