"""bench.py's reference arm on the host cores (no GPU): the JSON line the round's
driver reads -- metric, unit and direction of our arm, impl = "reference", a
cpu_baseline describing the run, and an e2e entry with no host-device bytes.  Each
step is one whole-circuit run from the observable, the same configuration the GPU
arm times, and the workers map no product library (only the oracle)."""
import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_reference_arm_line_chain20():
    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference",
                          "--workload", "chain20", "--steps", "2", "--warmup", "1", "--ref-workers", "2"],
                         cwd=ROOT, capture_output=True, text=True, timeout=300,
                         env=dict(os.environ, MASTER_ADDR="127.0.0.1"))
    assert out.returncode == 0, out.stderr[-2000:]
    line = json.loads(out.stdout.strip().splitlines()[-1])
    assert line["impl"] == "reference"
    assert line["metric"] == "terms/s rotate+merge+clip" and line["unit"] == "terms/s"
    assert line["higher_is_better"] is True and line["steps"] == 2 and line["warmup"] == 1
    assert line["value"] > 0
    assert line["config"]["workload"].startswith("chain20: N=20, 8 layers x 39 rotations")
    assert line["config"]["step"] == "one whole-circuit run from the observable"
    assert sum(line["config"]["runs_per_worker"]) == 2
    assert line["native_libs_loaded"] == ["oracle/_build/liborc.so"]
    cb = line["cpu_baseline"]
    assert cb["kind"] == "port" and cb["cores"] == 2 and "end to end" in cb["sample"] and cb["value"] == line["value"] and cb["sample"]
    assert line["e2e"] == {"value": line["value"], "unit": "terms/s", "h2d_bytes_per_step": 0,
                           "d2h_bytes_per_step": 0}
