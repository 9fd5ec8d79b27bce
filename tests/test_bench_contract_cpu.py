"""The reference arm of bench.py (``--impl reference``) on the CPU: one JSON line with the
arm's metric, unit and config, a ``cpu_baseline`` describing the run and an ``e2e`` object
with no host copies; under several ranks only rank 0 runs and prints it.  The CPU oracle is
the reference arm's implementation (it times the reference algorithm on the host cores)."""
import io
import json
import os
import sys
import types
from contextlib import redirect_stdout

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

import bench  # noqa: E402


def test_reference_arm_line():
    assert bench.DEFAULT_CONFIG == "batched" and bench.WORKLOAD == bench.CONFIGS["batched"]["workload"]
    # the mid-size workload keeps this CPU test short; the default run times the batched one
    line = bench.run_reference(types.SimpleNamespace(steps=1, warmup=3, config="mid"))
    for key in ("metric", "value", "unit", "impl", "n_gpus", "steps", "warmup", "ms_per_step",
                "higher_is_better", "scaling", "vs_baseline", "dtype", "data", "config", "cpu_baseline", "e2e"):
        assert key in line, key
    assert line["impl"] == "reference" and line["metric"] == "fwd+bwd Mrays/s" and line["unit"] == "Mrays/s"
    assert line["higher_is_better"] is True and line["steps"] == 1 and line["value"] > 0
    assert line["config"]["workload"] == bench.CONFIGS["mid"]["workload"]
    cb = line["cpu_baseline"]
    assert cb["kind"] == "port" and cb["cores"] >= 1 and cb["value"] == line["value"] and cb["sample"]
    assert line["e2e"] == {"value": line["value"], "unit": "Mrays/s", "h2d_bytes_per_step": 0,
                           "d2h_bytes_per_step": 0}
    json.dumps(line)


def test_reference_arm_prints_on_rank_zero_only(monkeypatch):
    calls = []
    monkeypatch.setattr(bench, "run_reference", lambda args: calls.append(args) or {"impl": "reference"})
    for rank, expect_line in (("1", False), ("0", True)):
        monkeypatch.setenv("RANK", rank)
        monkeypatch.setenv("WORLD_SIZE", "2")
        monkeypatch.setattr(sys, "argv", ["bench.py", "--impl", "reference", "--gpus", "2"])
        buf = io.StringIO()
        with redirect_stdout(buf):
            bench.main()
        out = buf.getvalue().strip()
        assert (json.loads(out) == {"impl": "reference"}) if expect_line else out == ""
    assert len(calls) == 1
