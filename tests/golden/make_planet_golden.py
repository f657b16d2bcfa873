"""Golden vectors of the reference's own planet host code -> planet_ref.npz.

For each case, builds oracle/ref/planet_harness.cu with the reference's
translation units (oracle/ref/build_ref.sh, per-case configuration headers)
and runs it on the host, where it makes no CUDA call: init_planet, then
NSTEPS steps of kick (dt/2), drift (dt), kick (dt/2) (planet.cu:36-93) under
seeded disk forces, recording the body, FrRot, get_ecc, get_E and set_M_p.

Needs the reference tree (PG_REFERENCE) and nvcc; no
GPU.  usage: python tests/golden/make_planet_golden.py
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

NSTEPS = 300
DT = 0.01

# (config index, overrides): rotating and inertial frames, a mass ramp inside
# the run, softening lengths whose scale-height exponent folds or does not
PLANET_CASES = {
    "pl2d": (0, dict()),
    "pl2d_ramp": (0, dict(FrRot_flag=0, p_beta=0.5, R_p=1.3, rs_fac=0.4, t_growth=2.0)),
    "pl2d_moving": (0, dict(plnt_flag=2, p_beta=2.0, R_p=0.8, sc_h=0.03, M_p=1e-4)),
}


def planet_params(case):
    from penguin_2_0_b200 import _lib
    import ctypes as C
    base, over = PLANET_CASES[case]
    p = _lib.pg_params()
    assert _lib.lib().pg_config_params(base, C.byref(p)) == 0
    p.update(**over)
    return p


def forces(case):
    seed = sorted(PLANET_CASES).index(case)
    return np.random.default_rng(seed).normal(scale=1e-3, size=(NSTEPS, 2))


def main():
    from make_golden import to_json
    ref = os.environ["PG_REFERENCE"]   # the reference source tree (required)
    out = {"nsteps": np.array(NSTEPS), "dt": np.array(DT)}
    for case in PLANET_CASES:
        p = planet_params(case)
        d = os.path.join(ROOT, "oracle", "_ref", case)
        os.makedirs(d, exist_ok=True)
        pj = os.path.join(d, "params.json")
        json.dump(to_json(p), open(pj, "w"))
        subprocess.check_call([os.path.join(ROOT, "oracle", "ref", "build_ref.sh"), case, pj, "golden"],
                              stdout=subprocess.DEVNULL, env=dict(os.environ, PG_REFERENCE=ref))
        nv = ["nvcc", "-O3", "-gencode", "arch=compute_100a,code=sm_100a", "-w", "-maxrregcount=64"]
        inc = ["-I" + os.path.join(d, "include"), "-I" + os.path.join(ref, "include"), "-I" + ref]
        obj = os.path.join(d, "obj")
        subprocess.check_call(nv + ["--device-c", *inc, "-o", os.path.join(d, "planet_harness.o"),
                                    os.path.join(ROOT, "oracle", "ref", "planet_harness.cu")])
        objs = [os.path.join(obj, f) for f in sorted(os.listdir(obj)) if f != "harness.o"]
        exe = os.path.join(d, "planet_ref")
        subprocess.check_call(nv + ["-o", exe, os.path.join(d, "planet_harness.o"), *objs])
        F = forces(case)
        fpath, rpath = os.path.join(d, "forces.bin"), os.path.join(d, "rows.bin")
        F.astype(np.float64).tofile(fpath)
        subprocess.check_call([exe, fpath, rpath, str(NSTEPS), repr(DT)], stdout=subprocess.DEVNULL)
        rows = np.fromfile(rpath, dtype=np.float64).reshape(NSTEPS + 1, 12)
        out[f"{case}_forces"] = F
        out[f"{case}_rows"] = rows
        print(case, "x", rows[-1, 1], "FrRot", rows[-1, 8], "ecc", rows[-1, 9], "m", rows[-1, 11], flush=True)
    np.savez_compressed(os.path.join(HERE, "planet_ref.npz"), **out)
    print("wrote", os.path.join(HERE, "planet_ref.npz"))


if __name__ == "__main__":
    main()
