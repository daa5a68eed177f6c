"""bench.py's reference arm on the CPU: the oracle port timed on the host on a
small sample, one JSON line with the keys the benchmark contract names; under
torchrun only rank 0 prints."""
import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _run(extra_env=None, args=()):
    env = dict(os.environ, **(extra_env or {}))
    return subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference",
                           "--steps", "2", "--warmup", "0", "--cpu-n", "512", "--cpu-n-big",
                           "768", "--n", "1024", *args],
                          capture_output=True, text=True, timeout=300, cwd=ROOT, env=env)


def test_reference_arm_json_line():
    r = _run()
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [ln for ln in r.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    for k in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step",
              "higher_is_better", "scaling", "vs_baseline", "dtype", "data", "config",
              "cpu_baseline", "e2e"):
        assert k in d, k
    assert d["impl"] == "reference" and d["value"] > 0 and d["unit"] == "TFLOP/s"
    assert d["cpu_baseline"]["kind"] in ("port", "reference") and d["cpu_baseline"]["cores"] >= 1
    assert d["cpu_baseline"]["resid"] < 16.0
    assert d["e2e"]["h2d_bytes_per_step"] == 0 and d["e2e"]["d2h_bytes_per_step"] == 0
    # The line names the target workload; its value is extrapolated as N^3 from
    # the larger measured host point, and both measured points are listed.
    assert d["config"]["n"] == 1024 and "workload" in d["config"]
    assert d["config"]["extrapolated"] is True
    pts = d["config"]["measured_points"]
    assert [p["n"] for p in pts] == [512, 768] and pts[0]["steps"] == 2
    assert abs(d["value"] - pts[1]["tflops"]) <= 1e-9 * pts[1]["tflops"]
    host = d["cpu_baseline"]["host"]
    assert host["nproc"] == os.cpu_count() and host["ram_gb"] > 0 and host["cpu_model"]


def test_reference_arm_other_ranks_are_silent():
    r = _run({"RANK": "1", "WORLD_SIZE": "2", "LOCAL_RANK": "1"})
    assert r.returncode == 0, r.stderr[-2000:]
    assert not [ln for ln in r.stdout.splitlines() if ln.startswith("{")]
