"""The reference arm of bench.py on the CPU: one JSON line on the same
metric, unit and workload as the GPU arm, with the keys the benchmark
contract asks for: the CPU restatement on the device arm's step window, one
replica per core (two here), and the direct-vs-iterative linear solve
sample."""
import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _last_json(out: str) -> dict:
    lines = [ln for ln in out.splitlines() if ln.startswith("{")]
    assert len(lines) == 1, out[-2000:]
    return json.loads(lines[0])


def test_reference_arm_prints_one_contract_line():
    sys.path.insert(0, ROOT)
    import bench
    p = subprocess.run([sys.executable, "bench.py", "--impl", "reference", "--steps", "1",
                        "--warmup", "1", "--cpu-procs", "2"], cwd=ROOT, capture_output=True,
                       text=True, timeout=600)
    assert p.returncode == 0, p.stderr[-2000:]
    d = _last_json(p.stdout)
    assert d["impl"] == "reference"
    assert d["metric"] == bench.METRIC and d["unit"] == "steps/s"
    assert d["higher_is_better"] is True and d["n_gpus"] == 1
    assert d["config"]["workload"] == bench.WORKLOAD_NAME
    assert d["value"] > 0 and d["steps"] == 1 and d["warmup"] == 1
    cb = d["cpu_baseline"]
    cores = min(2, len(os.sched_getaffinity(0)))
    assert cb["kind"] == "port" and cb["cores"] == cores and cb["value"] == d["value"]
    assert d["config"]["replicas"] == cores and cb["sample"]
    assert 0 < cb["per_replica_steps_per_s"] <= d["value"]
    ls = cb["linear_solve_sample"]
    assert ls["superlu_s"] > 0 and ls["gmres_ilu"]["iterations"] > 0
    e = d["e2e"]
    assert e["value"] == d["value"] and e["unit"] == d["unit"]
    assert e["h2d_bytes_per_step"] == 0 and e["d2h_bytes_per_step"] == 0
    assert d["vs_baseline"] is None


def test_reference_arm_under_torchrun_prints_once():
    """Launched like the multi-GPU arm (torchrun, two ranks here on the CPU),
    the reference arm runs on rank 0 alone: one JSON line, every rank exits
    0."""
    import socket
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    p = subprocess.run([sys.executable, "-m", "torch.distributed.run", "--nnodes=1",
                        "--nproc-per-node", "2", "--master-addr", "127.0.0.1",
                        "--master-port", str(port), "bench.py", "--impl", "reference",
                        "--gpus", "2", "--steps", "1", "--warmup", "1", "--cpu-procs", "1"],
                       cwd=ROOT, capture_output=True, text=True, timeout=600)
    assert p.returncode == 0, p.stderr[-2000:]
    d = _last_json(p.stdout)
    assert d["impl"] == "reference" and d["n_gpus"] == 2 and d["value"] > 0


def _sampler(rows):
    sys.path.insert(0, ROOT)
    import bench
    c = bench.ClockSampler()
    c.rows = [[p.strip() for p in r.split(",")] for r in rows]
    return c.summary()


def test_clock_summary_median_under_load_and_reasons():
    rows = ["0, 345, 1965, 150.0, 0x0, Not Active, Not Active, Not Active, Not Active",
            "0, 1965, 1965, 700.1, 0x0, Not Active, Not Active, Not Active, Not Active",
            "0, 1950, 1965, 990.3, 0x4, Not Active, Not Active, Not Active, Active",
            "0, 1965, 1965, 800.0, 0x0, Not Active, Not Active, Not Active, Not Active"]
    s = _sampler(rows)
    # the idle sample (below half the maximum) is left out of the median
    assert s["sm_mhz"] == 1965.0 and s["sm_max_mhz"] == 1965.0
    assert s["reasons"] == ["sw_power_cap"] and s["samples"] == 4
    json.dumps(s, allow_nan=False)


def test_clock_summary_without_values_is_valid_json():
    rows = ["0, [N/A], [N/A], [N/A], [N/A], Active, Not Active, Not Active, Not Active"]
    s = _sampler(rows)
    assert s["sm_mhz"] is None and s["sm_max_mhz"] is None
    assert s["reasons"] == ["hw_slowdown"]
    json.dumps(s, allow_nan=False)
    assert _sampler([])["reasons"] == ["unsampled"]


def test_json_lines_carry_no_nan():
    sys.path.insert(0, ROOT)
    import bench
    import numpy as np
    d = json.loads(bench.jline({"value": float("nan"), "e2e": {"value": float("inf")},
                                "rows": [1.0, np.float64("nan"), 2], "name": "x"}))
    assert d == {"value": None, "e2e": {"value": None}, "rows": [1.0, None, 2], "name": "x"}
