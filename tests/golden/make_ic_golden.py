"""Golden vectors for the initial state from the reference's own set-up.

For each case below, builds the reference's translation units for that disk
(oracle/ref/build_ref.sh) and oracle/ref/ic_harness.cu, which runs the
reference's init_grid / init_den / init_speed / init_cells / init_bound on
the host (no GPU), and packs into tests/golden/ic_ref.npz, per case: the
interior rings' Sigma, p, v_r, v_phi (phi-uniform: one value per ring), the
grid arrays, and the boundary rings' fields in the order of
pg_boundary_rings (x, dx, xvol, xc, z, dz, zvol, zc, Sigma, p, v_r, v_phi,
v_theta, rot_v).

usage: python tests/golden/make_ic_golden.py
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

# name -> (base workload, overrides)
IC_CASES = {
    "ic2d": (0, dict(imax=136, jmax=136)),
    "ic2d_eos1": (0, dict(imax=136, jmax=136, EOS=1, gam=1.4)),
    "ic3d": (1, dict(imax=64, jmax=132, kmax=16, ntop=3)),
    "ic3d_eos1": (1, dict(imax=64, jmax=132, kmax=16, ntop=3, EOS=1, gam=5.0 / 3.0)),
}


def ic_params(case):
    from penguin_2_0_b200 import _lib
    import ctypes as C
    base, over = IC_CASES[case]
    p = _lib.pg_params()
    assert _lib.lib().pg_config_params(base, C.byref(p)) == 0
    p.update(**over)
    return p


def main():
    from make_golden import to_json
    ref = os.environ["PG_REFERENCE"]   # the reference source tree (required)
    out = {}
    for case in IC_CASES:
        p = ic_params(case)
        d = os.path.join(ROOT, "oracle", "_ref", case)
        os.makedirs(d, exist_ok=True)
        pj = os.path.join(d, "params.json")
        json.dump(to_json(p), open(pj, "w"))
        subprocess.check_call([os.path.join(ROOT, "oracle", "ref", "build_ref.sh"), case, pj, "golden"],
                              stdout=subprocess.DEVNULL, env=dict(os.environ, PG_REFERENCE=ref))
        nv = ["nvcc", "-O3", "-gencode", "arch=compute_100a,code=sm_100a", "-w", "-maxrregcount=64"]
        inc = ["-I" + os.path.join(d, "include"), "-I" + os.path.join(ref, "include"), "-I" + ref]
        obj = os.path.join(d, "obj")
        subprocess.check_call(nv + ["--device-c", *inc, "-o", os.path.join(d, "ic_harness.o"),
                                    os.path.join(ROOT, "oracle", "ref", "ic_harness.cu")])
        objs = [os.path.join(obj, f) for f in sorted(os.listdir(obj)) if f != "harness.o"]
        exe = os.path.join(d, "ic_ref")
        subprocess.check_call(nv + ["-o", exe, os.path.join(d, "ic_harness.o"), *objs])
        info = json.loads(subprocess.check_output([exe, d]).decode().strip().splitlines()[-1])
        rb = 72 * p.jmax + 96
        assert info["ring_bytes"] == rb, info
        raw = np.fromfile(os.path.join(d, "ic_ref.bin"), dtype=np.uint8).reshape(-1, rb)
        f = raw[:, :40 * p.jmax].copy().view(np.float64).reshape(-1, 5, p.jmax)
        xs = raw[:, 40 * p.jmax:40 * p.jmax + 32].copy().view(np.float64)
        ys = raw[0, 40 * p.jmax + 32:72 * p.jmax + 32].copy().view(np.float64).reshape(4, p.jmax)
        zs = raw[:, 72 * p.jmax + 32:72 * p.jmax + 64].copy().view(np.float64)
        tail = raw[:, 72 * p.jmax + 64:72 * p.jmax + 96].copy()     # i k rot_v res_v rot_j inc_j
        b = np.fromfile(os.path.join(d, "boundary.bin"), dtype=np.uint8).reshape(-1, rb)
        bf = b[:, :40 * p.jmax].copy().view(np.float64).reshape(-1, 5, p.jmax)[:, :, 0]
        bx = b[:, 40 * p.jmax:40 * p.jmax + 32].copy().view(np.float64)
        bz = b[:, 72 * p.jmax + 32:72 * p.jmax + 64].copy().view(np.float64)
        brot = b[:, 72 * p.jmax + 72:72 * p.jmax + 80].copy().view(np.float64)
        nrad = 6 * p.kmax
        keep = 2 * nrad + (2 * 6 * p.imax if p.ndim == 3 else 0)
        brec = np.concatenate([bx, bz, bf, brot], axis=1)[:keep]
        out[f"{case}_fields"] = f[:, :4, 0].copy()          # Sigma, p, v_r, v_phi per ring
        out[f"{case}_phi_uniform"] = np.array(bool(np.all(f == f[:, :, :1])))
        out[f"{case}_xs"] = xs
        out[f"{case}_zs"] = zs
        out[f"{case}_tail"] = tail
        out[f"{case}_ys"] = ys
        out[f"{case}_boundary"] = brec
        print(case, info, "boundary rings", brec.shape[0], flush=True)
    np.savez_compressed(os.path.join(HERE, "ic_ref.npz"), **out)
    print("wrote", os.path.join(HERE, "ic_ref.npz"))


if __name__ == "__main__":
    main()
