"""bench.py end to end on the 64^3 uniform box (the CPU-runnable workload):
every leg of the line runs, and the line carries what it promises -- the
contract keys, a roofline below the measured peak, the drop-in and the
reference kernel beside the sweep, parity with the reference CPU direct on
the sampled cells, and one workload config shared with the reference arm."""
import json
import os
import pathlib
import subprocess
import sys

import pytest

pytestmark = pytest.mark.gpu

ROOT = pathlib.Path(__file__).resolve().parents[1]
ARGS = ["--workload", "uniform64", "--steps", "2", "--warmup", "3", "--cpu-pairs", "3e8",
        "--serve-boxes", "17,21", "--serve-requests", "150", "--precision-steps", "1"]


def _run(extra):
    env = dict(os.environ)
    env.pop("WORLD_SIZE", None)
    r = subprocess.run([sys.executable, str(ROOT / "bench.py")] + ARGS + extra, cwd=ROOT,
                       capture_output=True, text=True, timeout=900, env=env)
    assert r.returncode == 0, r.stderr[-3000:]
    lines = [ln for ln in r.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1, r.stdout[-2000:]
    return json.loads(lines[0])


def test_bench_line_contract():
    d = _run([])
    for k in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step",
              "higher_is_better", "scaling", "vs_baseline", "dtype", "data", "config",
              "roofline", "cpu_baseline", "e2e", "gpu_launches", "clocks"):
        assert k in d, k
    assert d["n_gpus"] == 1 and d["steps"] == 2 and d["warmup"] == 3
    assert d["value"] > 0 and d["higher_is_better"] is True
    assert d["config"]["workload"] == "uniform64"
    r = d["roofline"]
    assert r["unit"] == "TFLOP/s"
    if r.get("peak_clock_derived"):
        assert r["peak"] >= r["peak_clock_derived"] * 0.999
    assert 0.05 < r["frac"] <= 1.05, r["frac"]
    assert abs(r["achieved"] / r["peak"] - r["frac"]) < 1e-9
    e = d["e2e"]
    assert e["value"] > 0 and e["h2d_bytes_per_step"] > 0 and e["d2h_bytes_per_step"] > 0
    assert d["gpu_launches"] > 0
    c = d["cpu_baseline"]
    assert c["value"] > 0 and c["cores"] >= 1 and c["kind"] in ("reference", "port")
    assert set(c["cpu"]) == {"model", "host_logical_cpus", "usable_cpus"}
    assert d["parity_vs_reference"]["pass"], d["parity_vs_reference"]
    acc = d["accuracy_vs_fp64"]
    assert acc["rms_frac"] <= 2e-6 and acc["max_frac"] <= 1e-4, acc
    p = d["plain_dropin"]
    assert p["value"] > 0 and p["kernel"]["pairs"] == d["config"]["pairs_per_step_per_gpu"]
    # both forms lie within 1e-4 |a_ref| of the reference CPU direct per component
    assert p["vs_fp64"]["rms_frac"] <= 2e-6 and p["max_comp_rel_vs_batched"] <= 2e-4
    if d.get("ref_gpu_kernel") is not None and "value" in d["ref_gpu_kernel"]:
        assert d["ref_gpu_kernel"]["pairs"] == d["config"]["pairs_per_step_per_gpu"]
    s = d["serving"]
    assert s["slots"] == 2 and len(s["boxes"]) == 2
    assert [lv["load"] for lv in s["levels"]] == [0.5, 1.0, 1.5]
    for lv in s["levels"]:
        assert lv["requests"] == 150 and lv["p99_ms"] >= lv["p50_ms"] > 0
    for box, a in s["accuracy_vs_fp64"].items():
        assert a["rms_frac"] <= 2e-6, (box, a)

    ref = _run(["--impl", "reference"])
    assert ref["impl"] == "reference" and ref["config"] == d["config"]
    assert c["sample"].startswith(ref["cpu_baseline"]["sample"])  # the same cells
    assert ref["e2e"]["h2d_bytes_per_step"] == 0
