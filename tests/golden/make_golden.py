"""Golden vectors from the reference's own CUDA build.

Three stages:
  build  (CPU container): write each case's parameter JSON and build
         oracle/_ref/<case>/penguin_ref from the reference sources
         (oracle/ref/build_ref.sh).
  run    (on a B200): write each case's seeded initial dump with the library
         (pg_write_ic) and run the reference binary on it; raw output goes to
         <outdir>/<case>/ (hist.txt and state_NNNNN.bin in the dump layout).
  pack   (CPU container): turn the raw output into the compact fixtures
         committed here: <case>.npz with the per-step history (simtime, dt,
         mass, torque) and Sigma, v_r, v_phi, rot_j of the saved steps, in
         the reference's storage order.

usage: python tests/golden/make_golden.py build | run <rawdir> | pack <rawdir> [outdir [fulldir]]
"""
import ctypes as C
import json
import os
import subprocess
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
HERE = os.path.dirname(os.path.abspath(__file__))

# name -> (base workload, overrides, nsteps, steps kept in the fixture)
CASES = {
    # two radial chunks (128 = 116 + 12), two azimuthal chunks (132 = 116 + 16)
    "g128x132": (0, dict(imax=128, jmax=132), 20, (1, 2, 5, 20)),
    # the 256 x 768 disk itself; fixtures keep a strided subsample
    "cfg0": (0, dict(), 12, (1, 12)),
    # imax % 116 == 0: the last radial chunk is never updated (ppm.cu:48)
    "g232x240": (0, dict(imax=232, jmax=240), 4, (1, 4)),
    # jmax % 116 == 0: the last azimuthal chunk is never updated (ppm.cu:196)
    "g130x232": (0, dict(imax=130, jmax=232), 4, (1, 4)),
    # no planet, no viscosity, no flattening, no FARGO, no damping
    "g120x150_plain": (0, dict(imax=120, jmax=150, plnt_flag=0, visc_flag=0, flat_flag=0,
                               FARGO_flag=0, kill_rin=0.0, kill_rout=0.0), 6, (1, 6)),
}


def params_for(case):
    from penguin_2_0_b200 import _lib
    base, over, *_ = CASES[case]
    p = _lib.pg_params()
    st = _lib.lib().pg_config_params(base, C.byref(p))
    assert st == 0
    p.update(**over)
    p.nprin = 1
    return p


def to_json(p):
    return {k: (float(v).hex() if isinstance(v, float) else v) for k, v in p.as_dict().items()}


def cmd_build():
    for case in CASES:
        p = params_for(case)
        d = os.path.join(ROOT, "oracle", "_ref", case)
        os.makedirs(d, exist_ok=True)
        pj = os.path.join(d, "params.json")
        json.dump(to_json(p), open(pj, "w"), indent=1)
        subprocess.check_call([os.path.join(ROOT, "oracle", "ref", "build_ref.sh"), case, pj])


def cmd_run(rawdir):
    from penguin_2_0_b200 import _lib
    L = _lib.lib()
    for case, (_, _, nsteps, keep) in CASES.items():
        p = params_for(case)
        out = os.path.join(rawdir, case)
        os.makedirs(out, exist_ok=True)
        ic = os.path.join(out, "ic.bin")
        assert L.pg_write_ic(C.byref(p), ic.encode()) == 0
        exe = os.path.join(ROOT, "oracle", "_ref", case, "penguin_ref")
        r = subprocess.run([exe, ic, str(nsteps), out, ",".join(map(str, keep))],
                           capture_output=True, text=True)
        open(os.path.join(out, "stdout.txt"), "w").write(r.stdout + r.stderr)
        if r.returncode != 0:
            raise SystemExit(f"{case}: reference exited {r.returncode}: {r.stderr[-400:]}")
        os.remove(ic)
        print(case, r.stdout.strip())


def read_rings(path, p):
    jmax = p.jmax
    n = p.imax * p.kmax
    rb = 72 * jmax + 96
    raw = np.fromfile(path, dtype=np.uint8)
    assert raw.size == rb * n, (path, raw.size, rb * n)
    recs = raw.reshape(n, rb)
    f = recs[:, :40 * jmax].copy().view(np.float64).reshape(n, 5, jmax)
    rot_j = recs[:, 72 * jmax + 88:72 * jmax + 92].copy().view(np.int32).reshape(n)
    return f, rot_j


def cmd_pack(rawdir, outdir=HERE, full=None):
    for case, (_, _, nsteps, keep) in CASES.items():
        p = params_for(case)
        src = os.path.join(rawdir, case)
        rows = [ln.split() for ln in open(os.path.join(src, "hist.txt"))]
        hist = np.array([[float.fromhex(x) for x in r[1:]] for r in rows])
        out = {"hist": hist}
        stride = 1
        if case == "cfg0":
            stride = 7  # every 7th cell of the 196608 keeps the fixture small
        for s in keep:
            f, rot_j = read_rings(os.path.join(src, f"state_{s:05d}.bin"), p)
            sel = f[:, [0, 2, 3], :].reshape(f.shape[0], 3, -1)
            if stride > 1:
                flat = sel.transpose(1, 0, 2).reshape(3, -1)
                out[f"fields_{s}"] = flat[:, ::stride].copy()
            else:
                out[f"fields_{s}"] = sel.copy()
            out[f"rot_j_{s}"] = rot_j
        out["stride"] = np.array(stride)
        np.savez_compressed(os.path.join(outdir, f"{case}.npz"), **out)
        if full and case == "cfg0":
            f, rot_j = read_rings(os.path.join(src, f"state_{keep[0]:05d}.bin"), p)
            np.savez_compressed(os.path.join(full, "cfg0_full_step1.npz"), fields=f[:, [0, 2, 3], :], rot_j=rot_j)
        print("packed", case)


if __name__ == "__main__":
    what = sys.argv[1]
    if what == "build":
        cmd_build()
    elif what == "run":
        cmd_run(sys.argv[2])
    elif what == "pack":
        cmd_pack(sys.argv[2], *(sys.argv[3:5]))
    else:
        raise SystemExit(__doc__)
