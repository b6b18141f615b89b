"""The benchmark's JSON contract on the CPU: the reference arm (the CPU restatement of eT's algorithm
timed on the host cores) prints one line with the benchmark's metric, its own cpu_baseline and an e2e
record without device copies; the roofline traffic comes from the committed launch list."""

import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _bench():
    sys.path.insert(0, ROOT)
    import bench
    return bench


def test_roofline_traffic_comes_from_the_committed_capture():
    """bytes per issued FLOP of the committed 10240^3 capture, scaled to a launch's issued FLOPs"""
    bench = _bench()
    per_10240 = bench.gemm_traffic(6.0 * 10240 ** 3)
    assert per_10240 is not None and 5e9 < per_10240 < 1e10
    assert abs(bench.gemm_traffic(3.0 * 10240 ** 3) - 0.5 * per_10240) < 1.0


def test_reference_arm_prints_one_contract_line():
    """At a small shape (the default is the benchmark's o=32, v=320, N_J=1200): one line whose steps
    are the iterations actually timed."""
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--steps", "20",
                        "--warmup", "5", "--cpu-iterations", "2", "--n-o", "4", "--n-v", "24", "--n-J", "60"],
                       capture_output=True, text=True, timeout=600, cwd=ROOT)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [ln for ln in r.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["unit"] == "s/iter" and d["higher_is_better"] is False
    assert d["metric"] == _bench().METRIC
    assert d["value"] > 0 and d["value"] == d["cpu_baseline"]["value"] == d["e2e"]["value"]
    cb = d["cpu_baseline"]
    assert cb["kind"] in ("port", "reference") and cb["cores"] >= 1 and cb["sample"] and cb["cpu_model"]
    assert d["steps"] == cb["iterations_timed"] == 2 and d["warmup"] == 0
    assert d["e2e"]["h2d_bytes_per_step"] == 0 and d["e2e"]["d2h_bytes_per_step"] == 0
    assert d["config"]["n_o"] == 4 and "workload" in d["config"]


def test_synthetic_cholesky_vectors_in_et_layout():
    """make_system gives L(J, p, q) with J fastest (eT's layout), symmetric in p, q, seeded, so the
    host arrays go to the library without a reordering copy and every run sees the same input."""
    import numpy as np
    sys.path.insert(0, ROOT)
    from et_b200.synthetic import make_system
    a, b = make_system(3, 9, 20, seed=5), make_system(3, 9, 20, seed=5)
    assert a.L_mo.flags.f_contiguous and a.L_mo.shape == (20, 12, 12)
    assert np.array_equal(a.L_mo, b.L_mo) and np.array_equal(a.h_mo, b.h_mo)
    assert np.abs(a.L_mo - a.L_mo.transpose(0, 2, 1)).max() == 0.0
    flat = a.L_mo.reshape(-1, order="F")
    assert np.shares_memory(flat, a.L_mo)


def test_cpu_baseline_is_bounded():
    """The CPU restatement runs in a child process with a wall-time bound: a sample that runs out of
    time is reported (no value, the reason in `sample`) instead of holding the benchmark."""
    import types
    bench = _bench()
    args = types.SimpleNamespace(n_o=32, n_v=320, n_J=1200, cpu_iterations=1)
    cb = bench.cpu_sample_isolated(args, timeout_s=1)
    assert cb["value"] is None and cb["iterations_timed"] == 0 and "timed out" in cb["sample"]
    assert cb["kind"] == "port" and cb["cores"] >= 1
