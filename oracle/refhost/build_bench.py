"""Build the reference's own hydro step for the host CPU on the bench
workloads (TEST INFRASTRUCTURE: bench.py's CPU baseline and reference arm).

For each workload it writes the parameters (as bench.py runs them: seed 0,
no output times inside the run), the workload's copies of the reference's
two configuration headers (oracle/ref/gen_headers.py) and the host build
(build_refhost.sh) into oracle/_ref/bench_<workload>/ (git-ignored; it
travels with the working tree to machines without the reference tree).

usage: PG_REFERENCE=<reference tree> python oracle/refhost/build_bench.py [workload ...]
"""
import json
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

# bench.py workload -> (config index, overrides)
WORKLOADS = {"cfg0": (0, {}), "cfg1": (1, {}), "cfg2_fp64": (2, {"precision": 0})}


def bench_params(which, over):
    from penguin_2_0_b200 import _lib
    import ctypes as C
    p = _lib.pg_params()
    assert _lib.lib().pg_config_params(which, C.byref(p)) == 0
    p.update(**over)
    p.precision = 0
    p.nprin = 100
    p.seed = 0
    p.endtime = 1.0e9
    p.tmovie = 1.0e9
    return p


def main(names):
    ref = os.environ["PG_REFERENCE"]
    for name in names or list(WORKLOADS):
        which, over = WORKLOADS[name]
        p = bench_params(which, over)
        case = f"bench_{name}"
        d = os.path.join(ROOT, "oracle", "_ref", case)
        os.makedirs(d, exist_ok=True)
        pj = os.path.join(d, "params.json")
        json.dump({k: (float(v).hex() if isinstance(v, float) else v) for k, v in p.as_dict().items()},
                  open(pj, "w"), indent=1)
        subprocess.check_call([sys.executable, os.path.join(ROOT, "oracle", "ref", "gen_headers.py"), pj, d, ref],
                              stdout=subprocess.DEVNULL)
        subprocess.check_call([os.path.join(HERE, "build_refhost.sh"), case], stdout=subprocess.DEVNULL)
        print(os.path.join(d, "penguin_ref_host"))


if __name__ == "__main__":
    main(sys.argv[1:])
