"""bench.py's reference arm (the FP64 oracle port timed on the host cores) prints the one-line
JSON contract the benchmark driver reads: the same metric / unit / direction and the same config
object as the device arm, `impl: reference`, a measured ms_per_step (whole oracle iterations at
the sample walker counts, so steps x ms_per_step fits inside the run), a cpu_baseline describing
the run, and an e2e object with no host-device bytes. Runs a short sample on the CPU."""
import json
import os
import subprocess
import sys
import time

ROOT = os.path.abspath(os.path.join(os.path.dirname(__file__), os.pardir))


def test_reference_arm_json_line():
    t0 = time.time()
    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference",
                          "--steps", "2", "--warmup", "0", "--cpu-budget", "1"],
                         capture_output=True, text=True, timeout=600, cwd=ROOT)
    wall = time.time() - t0
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [ln for ln in out.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    for k in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step",
              "higher_is_better", "scaling", "vs_baseline", "dtype", "data", "config",
              "cpu_baseline", "e2e"):
        assert k in d, k
    assert d["impl"] == "reference" and d["metric"] == "VMC iter/s" and d["unit"] == "VMC iter/s"
    assert d["higher_is_better"] is True and d["scaling"] == "weak" and d["value"] > 0
    assert d["steps"] * d["ms_per_step"] < 1e3 * wall  # measured, not modelled
    sys.path.insert(0, ROOT)
    sys.path.insert(0, os.path.join(ROOT, "continuum-nqs_b200"))
    import bench
    from nqs.configs import config
    model, _, su = config(2)
    assert d["config"] == json.loads(json.dumps(bench.workload_config(su, model.n_params())))
    cb = d["cpu_baseline"]
    assert cb["kind"] == "port" and cb["cores"] >= 1 and cb["value"] == d["value"]
    assert cb["sample"]
    e = d["e2e"]
    assert e["value"] == d["value"] and e["unit"] == d["unit"]
    assert e["h2d_bytes_per_step"] == 0 and e["d2h_bytes_per_step"] == 0
