"""Golden values of the reference's own read/ post-processing -> post_ref.npz.

For each case: the seeded dump advanced a few steps by the CPU oracle (the
state is regenerated the same way by the tests), then the reference's own
get_torque (read/transform.cpp:386-420) and write_har_file
(read/p_output.cpp:35-55), run on the host by oracle/ref/post_harness.cpp
against the case's copy of include/post_global.h (oracle/ref/gen_headers.py).
MathGL, which read/post.cu needs for its plots, is not involved.

Needs the reference tree (PG_REFERENCE) and g++; no GPU.
usage: python tests/golden/make_post_golden.py
"""
import json
import os
import subprocess
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, HERE)

# name -> (config index, overrides, oracle steps before the post-processing)
POST_CASES = {
    "post2d": (0, dict(imax=128, jmax=384), 20),
    "post2d_moving": (0, dict(imax=136, jmax=200, plnt_flag=2, M_p=3e-4), 12),
    "post3d": (1, dict(imax=64, jmax=132, kmax=16), 3),
}
HARMONICS = (1.0, 2.0, 5.0)


def post_params(case):
    from penguin_2_0_b200 import _lib
    import ctypes as C
    base, over, _ = POST_CASES[case]
    p = _lib.pg_params()
    assert _lib.lib().pg_config_params(base, C.byref(p)) == 0
    p.update(**over)
    return p


def post_state(case):
    """The dump the post-processing reads: the seeded initial state advanced
    by the oracle (deterministic)."""
    import penguin_2_0_b200 as pg
    from oracle.pyoracle import Oracle
    p = post_params(case)
    o = Oracle(p, pg.build_ic(p))
    o.run_steps(POST_CASES[case][2])
    return p, o.save()


def main():
    from make_golden import to_json
    ref = os.environ["PG_REFERENCE"]   # the reference source tree (required)
    out = {}
    for case in POST_CASES:
        p, dump = post_state(case)
        d = os.path.join(ROOT, "oracle", "_ref", case)
        os.makedirs(d, exist_ok=True)
        pj = os.path.join(d, "params.json")
        json.dump(to_json(p), open(pj, "w"), indent=1)
        subprocess.check_call([sys.executable, os.path.join(ROOT, "oracle", "ref", "gen_headers.py"), pj, d, ref],
                              stdout=subprocess.DEVNULL)
        exe = os.path.join(d, "post_ref")
        subprocess.check_call(["g++", "-O2", "-std=c++17", "-w", f"-I{d}/include", f"-I{ref}/include", f"-I{ref}",
                               "-o", exe, os.path.join(ROOT, "oracle", "ref", "post_harness.cpp")])
        dpath = os.path.join(d, "dump.bin")
        open(dpath, "wb").write(dump)
        r = subprocess.run([exe, dpath, ",".join(repr(m) for m in HARMONICS)], capture_output=True, text=True,
                           check=True)
        os.remove(dpath)
        lines = r.stdout.splitlines()
        out[f"{case}_torque"] = np.array(float.fromhex(lines[0].split()[1]))
        cur = None
        rows = {}
        for ln in lines[1:]:
            t = ln.split()
            if t[0] == "harmonic":
                cur = float(t[1])
                rows[cur] = []
            else:
                rows[cur].append([float(x) for x in t])
        for m in HARMONICS:
            a = np.array(rows[m])
            assert a.shape == (p.imax, 3), a.shape
            out[f"{case}_m{m:g}_an"] = a[:, 1]
            out[f"{case}_m{m:g}_bn"] = a[:, 2]
        print(case, "torque", float(out[f"{case}_torque"]))
    np.savez_compressed(os.path.join(HERE, "post_ref.npz"), **out)


if __name__ == "__main__":
    main()
