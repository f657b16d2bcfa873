"""Golden text of the reference's own output naming and writers -> io_ref.json.

For each case, builds oracle/ref/io_harness.cu with the reference's
translation units (oracle/ref/build_ref.sh, per-case configuration headers)
and runs it on the host, where it makes no CUDA call:

* create_label() (output.cu:57-88), for flag sets that reach each branch;
* the dump names of main.cu:124 (frame_num, global.cu) for a few frames;
* the para file of write_para_file (output.cu:90-109);
* one time-file row of ROW_VALUES through the stream append_output_file opens
  (output.cu:25-34; main.cu:417-427), two columns without a planet.

Needs the reference tree (PG_REFERENCE) and nvcc; no
GPU.  usage: python tests/golden/make_io_golden.py
"""
import json
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, HERE)

MAINP = "/data/runs/disk"

# (config index, overrides): each reaches a different branch of create_label
IO_CASES = {
    "io2d": (0, dict()),
    "io2d_eos1": (0, dict(EOS=1, gam=1.4)),
    "io3d": (1, dict(imax=64, jmax=132, kmax=16, ntop=3)),
    "io2d_moving": (0, dict(plnt_flag=2, M_p=1e-4, rs_fac=0.7)),
    "io2d_noplanet_iso": (0, dict(plnt_flag=0, p_beta=0.0, FARGO_flag=0, FrRot_flag=0, visc_flag=0)),
    "io2d_flatvor": (0, dict(p_alpha=2.5, p_beta=1.0, xmin=0.35, xmax=3.0)),
}

# simtime, mass, torque, x, y, vx, vy, fx, fy, eccentricity, semi-major axis
ROW_VALUES = [62.83185307179586, 0.001234567890123456, -1.5e-05, 1.0, 3.141592653589793,
              1e-300, -2.220446049250313e-16, 1e20, -0.0, 0.1, 1.0000000000000002]


def io_params(case):
    from penguin_2_0_b200 import _lib
    import ctypes as C
    base, over = IO_CASES[case]
    p = _lib.pg_params()
    assert _lib.lib().pg_config_params(base, C.byref(p)) == 0
    p.update(**over)
    return p


def main():
    from make_golden import to_json
    ref = os.environ["PG_REFERENCE"]   # the reference source tree (required)
    out = {"mainp": MAINP, "row_values": [v.hex() for v in ROW_VALUES], "cases": {}}
    for case in IO_CASES:
        p = io_params(case)
        d = os.path.join(ROOT, "oracle", "_ref", case)
        os.makedirs(d, exist_ok=True)
        pj = os.path.join(d, "params.json")
        json.dump(to_json(p), open(pj, "w"))
        subprocess.check_call([os.path.join(ROOT, "oracle", "ref", "build_ref.sh"), case, pj, "golden"],
                              stdout=subprocess.DEVNULL, env=dict(os.environ, PG_REFERENCE=ref))
        nv = ["nvcc", "-O3", "-gencode", "arch=compute_100a,code=sm_100a", "-w", "-maxrregcount=64"]
        inc = ["-I" + os.path.join(d, "include"), "-I" + os.path.join(ref, "include"), "-I" + ref]
        obj = os.path.join(d, "obj")
        subprocess.check_call(nv + ["--device-c", *inc, "-o", os.path.join(d, "io_harness.o"),
                                    os.path.join(ROOT, "oracle", "ref", "io_harness.cu")])
        objs = [os.path.join(obj, f) for f in sorted(os.listdir(obj)) if f != "harness.o"]
        exe = os.path.join(d, "io_ref")
        subprocess.check_call(nv + ["-o", exe, os.path.join(d, "io_harness.o"), *objs])
        time_dat = os.path.join(d, "time.dat")
        if os.path.exists(time_dat):
            os.remove(time_dat)                      # the harness appends
        subprocess.check_call([exe, d, MAINP, *[repr(v) for v in ROW_VALUES]], stdout=subprocess.DEVNULL)
        rec = {}
        for name in ("label.txt", "frames.txt", "para.dat", "time.dat"):
            with open(os.path.join(d, name)) as f:
                rec[name] = f.read()
        out["cases"][case] = rec
        print(case, rec["label.txt"], flush=True)
    with open(os.path.join(HERE, "io_ref.json"), "w") as f:
        json.dump(out, f, indent=1, sort_keys=True)
    print("wrote", os.path.join(HERE, "io_ref.json"))


if __name__ == "__main__":
    main()
