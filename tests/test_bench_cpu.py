"""bench.py's host-side legs on CPU: the reference arm runs and reports
exactly the warm-up and timed steps it ran."""
import json
import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_reference_arm_reports_the_steps_it_ran(monkeypatch, capsys, built):
    sys.path.insert(0, ROOT)
    import bench
    for k in ("RANK", "WORLD_SIZE", "LOCAL_RANK"):
        monkeypatch.delenv(k, raising=False)
    monkeypatch.setattr(sys, "argv", ["bench.py", "--impl", "reference", "--workload", "plain_cube",
                                      "--steps", "2", "--warmup", "1"])
    assert bench.main() == 0
    line = json.loads(capsys.readouterr().out.strip().splitlines()[-1])
    assert line["impl"] == "reference"
    assert line["steps"] == 2 and line["warmup"] == 1
    assert line["value"] > 0 and line["e2e"]["value"] == line["value"]
    assert line["cpu_baseline"]["kind"] in ("reference", "port")
    assert "1 untimed and 2 timed full steps" in line["cpu_baseline"]["sample"]
    assert line["ms_per_step"] * 2 / 1e3 <= 600.0


def test_reference_arm_stops_at_its_budget(monkeypatch, capsys, built):
    sys.path.insert(0, ROOT)
    import bench
    for k in ("RANK", "WORLD_SIZE", "LOCAL_RANK"):
        monkeypatch.delenv(k, raising=False)
    monkeypatch.setattr(bench, "REFERENCE_BUDGET_S", 0.0)
    monkeypatch.setattr(sys, "argv", ["bench.py", "--impl", "reference", "--workload", "plain_cube",
                                      "--steps", "5", "--warmup", "0"])
    assert bench.main() == 0
    line = json.loads(capsys.readouterr().out.strip().splitlines()[-1])
    assert line["steps"] == 1 and line["warmup"] == 0
    assert "stopped after 1 of 5 steps" in line["cpu_baseline"]["sample"]
