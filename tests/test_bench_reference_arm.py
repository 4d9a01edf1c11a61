"""The reference arm of bench.py (--impl reference) on the CPU: it prints the benchmark line
with the same `config` dict as the GPU arm, and times the oracle alone: the product library
is never loaded into its process (inputs come from the oracle's own scene restatement)."""
import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

PROBE = r"""
import sys, json, io, contextlib
sys.argv = ["bench.py", "--impl", "reference", "--steps", "2", "--warmup", "1"]
sys.path.insert(0, ".")
import bench
buf = io.StringIO()
with contextlib.redirect_stdout(buf):
    bench.main()
maps = open("/proc/self/maps").read()
print(json.dumps({"line": buf.getvalue().strip().splitlines()[-1],
                  "product_loaded": "libcampfire_gas.so" in maps,
                  "product_imported": any(m.startswith("campfire_b200") for m in sys.modules),
                  "oracle_loaded": "liboracle_gas.so" in maps,
                  "config": bench.workload_config("plain", 1)}))
"""


def test_reference_arm_runs_the_oracle_alone():
    r = subprocess.run([sys.executable, "-c", PROBE], cwd=ROOT, capture_output=True, text=True, timeout=600,
                       env=dict(os.environ, OMP_NUM_THREADS="4"))
    assert r.returncode == 0, r.stderr
    out = json.loads(r.stdout.strip().splitlines()[-1])
    line = json.loads(out["line"])
    assert line["impl"] == "reference" and line["unit"] == line["metric"] == "cell-updates/s"
    assert line["value"] > 0 and line["higher_is_better"] is True
    assert line["config"] == out["config"]
    assert line["e2e"]["value"] == line["value"] and line["cpu_baseline"]["kind"] == "port"
    assert out["oracle_loaded"] and not out["product_loaded"] and not out["product_imported"]
