"""Write per-workload copies of the reference's two configuration headers.

The reference fixes grid size and physics parameters at compile time in
include/variable_types.h and include/global.h.  This script reads those two
headers from the reference tree, substitutes the values of one parameter set
(a JSON file whose floats are hex strings, produced from pg_params) and writes
the result to oracle/_ref/<name>/include/, which is git-ignored.  Nothing
else of the reference is copied: its .cu sources are compiled where they lie.

usage: python oracle/ref/gen_headers.py <params.json> <outdir> <reference_root>
"""
import json
import os
import re
import sys


def fx(v):
    """C hex-float literal for an exact double."""
    return float(v).hex()


def patch_variable_types(txt, p):
    txt = re.sub(r"#define ndim \d+", f"#define ndim {p['ndim']}", txt)
    for name in ("imax", "jmax", "kmax"):
        txt, n = re.subn(rf"const int {name} = [^;]*;", f"const int {name} = {p[name]};", txt)
        assert n == 1, name
    return txt


def patch_global(txt, p):
    def setflag(txt, name, value):
        txt, n = re.subn(rf"#define {name} [-\d]+", f"#define {name} {value}", txt)
        assert n == 1, name
        return txt

    if p["flat_flag"]:
        txt = re.sub(r"^//\s*#define flat_flag", "#define flat_flag", txt, flags=re.M)
    else:
        txt = re.sub(r"^#define flat_flag", "//#define flat_flag", txt, flags=re.M)
    for f in ("EOS", "plnt_flag", "FrRot_flag", "kill_flag", "visc_flag", "FARGO_flag", "dump_flag"):
        txt = setflag(txt, f, p[f])
    dbl = ("p_alpha", "p_beta", "ss_alpha", "sc_h", "M_p", "R_p", "t_growth", "rs_fac", "gam",
           "courant", "endtime", "tmovie", "xmin", "xmax", "ymin", "ymax", "zmin", "zmax",
           "dx_min", "dx_max", "dy_min", "dy_max", "dz_min", "dz_max")
    for name in dbl:
        txt, n = re.subn(rf"const sdp {name} = [^;]*;", f"const sdp {name} = {fx(p[name])};", txt)
        assert n == 1, name
    ints = ("nlft", "nrgh", "nudr", "ntop", "ncycend", "nprin", "ngeomx", "ngeomy", "ngeomz",
            "grspx", "grspy", "grspz")
    for name in ints:
        txt, n = re.subn(rf"const int {name} = [^;]*;", f"const int {name} = {int(p[name])};", txt)
        assert n == 1, name
    return txt


def patch_post_global(txt, p):
    """include/post_global.h (the read/ tools' configuration): dims and M_p."""
    txt = re.sub(r"#define ndim \d+", f"#define ndim {p['ndim']}", txt)
    for name in ("imax", "jmax", "kmax"):
        txt, n = re.subn(rf"const int {name} = [^;]*;", f"const int {name} = {p[name]};", txt)
        assert n == 1, name
    txt, n = re.subn(r"const sdp M_p = [^;]*;", f"const sdp M_p = {fx(p['M_p'])};", txt)
    assert n == 1
    return txt


def main():
    pjson, outdir = sys.argv[1], sys.argv[2]
    root = sys.argv[3]
    raw = json.load(open(pjson))
    p = {k: (float.fromhex(v) if isinstance(v, str) and v.startswith(("0x", "-0x")) else v)
         for k, v in raw.items()}
    inc = os.path.join(outdir, "include")
    os.makedirs(inc, exist_ok=True)
    vt = open(os.path.join(root, "include", "variable_types.h")).read()
    gl = open(os.path.join(root, "include", "global.h")).read()
    open(os.path.join(inc, "variable_types.h"), "w").write(patch_variable_types(vt, p))
    open(os.path.join(inc, "global.h"), "w").write(patch_global(gl, p))
    # read/'s configuration header: grid sizes and the planet mass
    pg_path = os.path.join(root, "include", "post_global.h")
    if os.path.exists(pg_path):
        open(os.path.join(inc, "post_global.h"), "w").write(patch_post_global(open(pg_path).read(), p))
    # harness-only constants (damping zones of the workload)
    with open(os.path.join(inc, "harness_params.h"), "w") as f:
        f.write("#pragma once\n")
        f.write(f"const double h_kill_rin = {fx(p['kill_rin'])};\n")
        f.write(f"const double h_kill_rout = {fx(p['kill_rout'])};\n")
    print("headers written to", inc)


if __name__ == "__main__":
    main()
