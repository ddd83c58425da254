"""bench.py's reference arm (``--impl reference``) on CPU.

The arm times the reference's own CPU build (oracle/_ref, compiled from the
reference sources; the C restatement when that is absent) on the host cores,
for the same workload, metric and unit as the engine arm.  These tests run
the arm for the cheapest workload end to end and check the JSON line
against the bench contract, and check that every workload either names its
own configuration or reports itself unavailable.
"""
import contextlib
import io
import json
import os
import sys
import types

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

import bench  # noqa: E402


def run_ref(workload, steps=2, warmup=3):
    out = io.StringIO()
    with contextlib.redirect_stdout(out):
        rc = bench.run_reference(types.SimpleNamespace(workload=workload, steps=steps, warmup=warmup))
    lines = [ln for ln in out.getvalue().splitlines() if ln.strip()]
    assert rc == 0 and len(lines) == 1, out.getvalue()
    return json.loads(lines[0])


def test_batch_reference_line_follows_the_contract():
    line = run_ref("batch4096")
    assert line["impl"] == "reference"
    assert line["metric"].startswith("GFLOP/s") and line["unit"] == "GFLOP/s"
    assert line["higher_is_better"] is True and line["n_gpus"] == 1
    assert line["steps"] == 2 and line["warmup"] == 3 and line["value"] > 0
    assert line["config"]["workload"] == "1024 x complex DFT N=4096 c128, forward then inverse"
    cb = line["cpu_baseline"]
    assert cb["value"] == line["value"] and cb["cores"] >= 1 and cb["kind"] in ("reference", "port") and cb["sample"]
    assert line["e2e"] == {"value": line["value"], "unit": "GFLOP/s", "h2d_bytes_per_step": 0,
                           "d2h_bytes_per_step": 0}
    # 5 N log2 N per transform, 1024 transforms each way per step
    flops = 5.0 * 4096 * 12 * 1024 * 2
    assert line["value"] == pytest.approx(flops / (line["ms_per_step"] / 1e3) / 1e9, rel=1e-2)


@pytest.mark.parametrize("name", sorted(bench.WORKLOADS))
def test_every_workload_names_its_own_reference_config(name):
    W = bench.WORKLOADS[name]
    if not hasattr(W, "cpu_measure"):
        out = io.StringIO()
        with contextlib.redirect_stdout(out):
            assert bench.run_reference(types.SimpleNamespace(workload=name, steps=1, warmup=3)) == 0
        line = json.loads(out.getvalue())
        assert line["impl"] == "reference" and line["unavailable"]
        return
    cfg = bench._ref_config(W)
    others = {bench._ref_config(V)["workload"] for n, V in bench.WORKLOADS.items()
              if n != name and hasattr(V, "cpu_measure")}
    assert cfg["workload"] not in others, (name, cfg)
