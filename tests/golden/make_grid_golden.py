"""Golden vectors for the grid generator from the reference's own grid().

Builds oracle/ref/grid_harness.cu against the reference's src/shared/global.cu
(which includes grid.cu) with the configuration headers of the 2D 256x768
disk (its dx/dy/dz spacing limits), runs it on the host for every supported
grid type over the radial, azimuthal and polar ranges the tests use, and
writes tests/golden/grid_ref.npz.  Host code only: no GPU is needed.

usage: python tests/golden/make_grid_golden.py
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

# (name, grid type, zones, lower, upper)
HALF_PI = 1.570796326794896619231321691639751442
TWO_PI = 6.283185307179586476925286766559
GRID_CASES = [
    ("r_lg0", 0, 256, 0.4, 2.5), ("r_lg1", 1, 256, 0.4, 2.5), ("r_lg2", 2, 256, 0.4, 2.5),
    ("r_lg3", 3, 256, 0.4, 2.5), ("r_lg4", 4, 256, 0.4, 2.5), ("r_lg6", 6, 256, 0.4, 2.5),
    ("phi_lg0", 0, 768, 0.0, TWO_PI), ("phi_lg4", 4, 768, 0.0, TWO_PI),
    ("theta_lg0", 0, 32, HALF_PI - 0.15, HALF_PI), ("theta_lg6", 6, 32, HALF_PI - 0.15, HALF_PI),
]


def main():
    from make_golden import to_json
    from penguin_2_0_b200 import _lib
    import ctypes as C
    ref = os.environ["PG_REFERENCE"]   # the reference source tree (required)
    out = os.path.join(ROOT, "oracle", "_ref", "grid")
    os.makedirs(out, exist_ok=True)
    p = _lib.pg_params()
    assert _lib.lib().pg_config_params(0, C.byref(p)) == 0
    pj = os.path.join(out, "params.json")
    json.dump(to_json(p), open(pj, "w"))
    subprocess.check_call([sys.executable, os.path.join(ROOT, "oracle", "ref", "gen_headers.py"), pj, out, ref],
                          stdout=subprocess.DEVNULL)
    inc = ["-I" + os.path.join(out, "include"), "-I" + os.path.join(ref, "include")]
    exe = os.path.join(out, "grid_ref")
    subprocess.check_call(["nvcc", "-O2", "-w", "-rdc=true", "-gencode", "arch=compute_100a,code=sm_100a", *inc,
                           "-o", exe, os.path.join(ROOT, "oracle", "ref", "grid_harness.cu"),
                           os.path.join(ref, "src", "shared", "global.cu")])
    raw = os.path.join(out, "grid.bin")
    args = [f"{lg},{n},{float(lo).hex()},{float(hi).hex()}" for _, lg, n, lo, hi in GRID_CASES]
    subprocess.check_call([exe, raw, *args])
    data = np.fromfile(raw, dtype=np.float64)
    res, off = {}, 0
    for name, lg, n, lo, hi in GRID_CASES:
        res[name] = data[off:off + 3 * n].reshape(3, n).copy()   # xa, xc, dx
        off += 3 * n
    assert off == data.size
    np.savez_compressed(os.path.join(HERE, "grid_ref.npz"), **res)
    print("wrote", os.path.join(HERE, "grid_ref.npz"), len(res), "cases")


if __name__ == "__main__":
    main()
