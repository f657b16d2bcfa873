"""bench.py --impl reference on the CPU: one JSON line with the bench
contract's keys, the same config dict the GPU arm prints, the reference's own
step built for the host when that build exists (kind "reference"), and no
product library loaded in the arm's own process (its initial dump comes
from a separate process)."""
import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

PROBE = r"""
import runpy, sys, os
sys.argv = ["bench.py", "--impl", "reference", "--workload", "cfg0", "--steps", "2", "--warmup", "3"]
try:
    runpy.run_path(os.path.join(sys.argv_root, "bench.py"), run_name="__main__")
finally:
    maps = open("/proc/self/maps").read()
    print("LOADED_PRODUCT=" + str("libpenguin_b200.so" in maps), file=sys.stderr)
"""


def test_reference_arm_line_and_isolation():
    code = "import sys; sys.argv_root = %r\n" % ROOT + PROBE
    env = dict(os.environ, PG_REF_BUDGET_S="2")
    r = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, cwd=ROOT, env=env,
                       timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    line = json.loads(r.stdout.strip().splitlines()[-1])
    for k in ("impl", "metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better",
              "scaling", "vs_baseline", "dtype", "data", "config", "cpu_baseline", "e2e"):
        assert k in line, k
    assert line["impl"] == "reference" and line["metric"] == "zone-updates/s" and line["value"] > 0
    assert set(line["config"]) == {"workload", "cells", "imax", "jmax", "kmax", "parallelism", "l2"}
    assert line["config"]["imax"] == 256 and line["config"]["jmax"] == 768
    assert line["e2e"] == {"value": line["value"], "unit": line["unit"], "h2d_bytes_per_step": 0,
                           "d2h_bytes_per_step": 0}
    host_build = os.path.exists(os.path.join(ROOT, "oracle", "_ref", "bench_cfg0", "penguin_ref_host"))
    assert line["cpu_baseline"]["kind"] == ("reference" if host_build else "port")
    assert "LOADED_PRODUCT=False" in r.stderr
