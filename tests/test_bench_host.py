"""Host-side pieces of bench.py that decide what is measured (no GPU)."""
import importlib.util
import pathlib

import numpy as np

ROOT = pathlib.Path(__file__).resolve().parents[1]


def _bench():
    spec = importlib.util.spec_from_file_location("bench_under_test", ROOT / "bench.py")
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def test_cell_pairs_sum_to_direct_total(synth, oracle):
    bench = _bench()
    box = synth.clustered_box(40000, 11, seed=3, n_clumps=20)
    cp = bench.cell_pairs(box)
    assert cp.shape == (11, 11, 11)
    assert int(cp.sum()) == oracle.pair_count(box)


def test_cpu_sample_is_fixed_and_exact(synth, oracle):
    bench = _bench()
    box = synth.clustered_box(40000, 11, seed=3, n_clumps=20)
    total = oracle.pair_count(box)
    cells, sinks, pairs, desc = bench.cpu_sample(box, 0.2 * total)
    c2, s2, p2, d2 = bench.cpu_sample(box, 0.2 * total)
    assert np.array_equal(cells, c2) and np.array_equal(sinks, s2) and p2 == pairs and d2 == desc
    assert 0.2 * total <= pairs < total
    # non-empty cells, sorted, and their exact pairs
    assert np.all(np.diff(cells) > 0) and np.all(box.counts[cells] > 0)
    assert pairs == int(bench.cell_pairs(box).ravel()[cells].sum())
    # sinks are exactly the particles of those cells, in cell order
    cs = box.cell_start
    want = np.concatenate([np.arange(cs[c], cs[c + 1]) for c in cells])
    assert np.array_equal(sinks, want)
    # a target beyond the box takes every non-empty cell
    cells_all, _, p_all, _ = bench.cpu_sample(box, 10 * total)
    assert p_all == total and cells_all.size == int((box.counts > 0).sum())


def test_parity_vs_reference_bound(synth):
    bench = _bench()
    rng = np.random.default_rng(0)
    ref = rng.normal(size=(100, 3)).astype(np.float32)
    sinks = np.arange(0, 100, 2)
    got = np.concatenate([ref, np.zeros((100, 1), np.float32)], axis=1)
    r = bench.parity_vs_reference(got, ref, sinks)
    assert r["pass"] and r["max_comp_rel"] == 0.0 and r["sinks"] == 50
    got[4, 1] += 1e-3 * np.linalg.norm(ref[4])  # a sampled sink off by 1e-3 of |a|
    r = bench.parity_vs_reference(got, ref, sinks)
    assert not r["pass"] and abs(r["max_comp_rel"] - 1e-3) < 1e-5
    got[4, 1] = ref[4, 1]
    got[5, 1] += 1.0  # an unsampled sink does not count
    assert bench.parity_vs_reference(got, ref, sinks)["pass"]


def test_both_arms_report_one_workload_config(synth):
    """The reference arm and this arm describe the same workload with the
    same config dict (a ratio of the two lines needs one workload); the L2
    note follows the box size."""
    import argparse
    bench = _bench()
    args = argparse.Namespace(workload="clustered512")
    box = synth.clustered_box(40000, 11, seed=3, n_clumps=20)
    pairs = int(bench.cell_pairs(box).sum())
    a = bench.workload_config(args, bench.WORKLOADS["clustered512"], box, pairs)
    b = bench.workload_config(args, bench.WORKLOADS["clustered512"], box, pairs, 1)
    assert a == b and a["pairs_per_step_per_gpu"] == pairs and a["particles_per_gpu"] == box.n
    assert "fit in L2" in a["l2"]  # 40,000 particles: 5.4 MB of inputs


def test_roofline_peak_is_the_larger_of_probe_and_clock():
    bench = _bench()
    peak, derived = bench.peak_from(72.0, {"sm_mhz": 1965.0}, 148)
    assert abs(derived - 148 * 128 * 2 * 1965e6 / 1e12) < 1e-9 and peak == derived
    peak, _ = bench.peak_from(80.0, {"sm_mhz": 1965.0}, 148)
    assert peak == 80.0
    peak, derived = bench.peak_from(72.0, {"sm_mhz": None}, 148)
    assert peak == 72.0 and derived is None  # JSON null, never NaN


def test_cpu_baseline_names_the_host_cpu():
    bench = _bench()
    cpu = bench.host_cpu()
    assert set(cpu) == {"model", "host_logical_cpus", "usable_cpus"}
    assert 1 <= cpu["usable_cpus"] <= cpu["host_logical_cpus"]


def test_bench_lines_are_strict_json():
    import json
    bench = _bench()
    line = bench.json_line({"a": float("nan"), "b": [1.0, float("inf")], "c": {"d": -float("inf")}})
    assert json.loads(line) == {"a": None, "b": [1.0, None], "c": {"d": None}}
