"""Golden vectors from the reference's own CUDA build.

Three stages (2D cases in CASES, 3D cases in CASES3D):
  build  (CPU container): write each case's parameter JSON and build
         oracle/_ref/<case>/penguin_ref from the reference sources
         (oracle/ref/build_ref.sh), and, for the per-step cases, the same
         sources for the host CPU (oracle/_ref/<case>/penguin_ref_host,
         oracle/refhost/build_refhost.sh).
  run    (on a B200): write each case's seeded initial dump with the library
         (pg_write_ic) and run the reference binary on it; raw output goes to
         <outdir>/<case>/ (hist.txt and state_NNNNN.bin in the dump layout).
  pack   (CPU container): turn the raw output into the compact fixtures
         committed here: <case>.npz with the per-step history (simtime, dt,
         mass, torque) and Sigma, v_r, v_phi, rot_j of the saved steps, in
         the reference's storage order.

usage: python tests/golden/make_golden.py [--only=case,...] build | run <rawdir> | pack <rawdir> [outdir [fulldir]]
                                          | run_long <rawdir> | pack_long <rawdir> [outdir]
(--only restricts build, run and pack to the named cases)
"""
import ctypes as C
import json
import os
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
HERE = os.path.dirname(os.path.abspath(__file__))

# name -> (base workload, overrides, nsteps, steps kept in the fixture)
#
# Every size keeps the last chunk of each pencil warp aligned: n % 116 is 0,
# 20, 52 or 84, so the chunk's lim (n % 116 + 12) is 12 (all threads active),
# 32, 64 or 96.  With any other remainder the reference's sweepx/sweepy
# (ppm.cu:50-156, 198-303) leave a warp partially inside the
# `if (i_ring < iblk+n_pad)` block that holds ~30 __syncthreads(): divergent
# barriers inside a warp, undefined since independent thread scheduling; on
# a B200 the 128x132 case (lim 24) never finished.
CASES = {
    # two radial chunks (136 = 116 + 20), two azimuthal chunks
    "g136x136": (0, dict(imax=136, jmax=136), 12, (1, 2, 5, 12)),
    # near the 256 x 768 disk: 252 = 2*116 + 20, 780 = 6*116 + 84
    "g252x780": (0, dict(imax=252, jmax=780), 8, (1, 8)),
    # imax % 116 == 0: the last radial chunk is never updated (ppm.cu:48)
    "g232x200": (0, dict(imax=232, jmax=200), 4, (1, 4)),
    # jmax % 116 == 0: the last azimuthal chunk is never updated (ppm.cu:196)
    "g168x232": (0, dict(imax=168, jmax=232), 4, (1, 4)),
    # no planet, no viscosity, no flattening, no FARGO, no damping
    "g136x200_plain": (0, dict(imax=136, jmax=200, plnt_flag=0, visc_flag=0, flat_flag=0,
                               FARGO_flag=0, kill_rin=0.0, kill_rout=0.0), 6, (1, 6)),
    # isentropic EOS 1, gam 1.4: the Newton Riemann solver (riemann.cu:75-111)
    # and p = cs2 Sigma^gam / gam at every store; planet, viscosity, damping
    "g136x200_eos1": (0, dict(imax=136, jmax=200, EOS=1, gam=1.4), 8, (1, 3, 8)),
    # FARGO_flag 2: rings shift at the solid-body rate (1 - FrRot) r; with the
    # frame rotating at the orbit of a planet at R_p = 0.3 (FrRot = 6.1) every
    # ring moves by whole cells each step
    "g136x136_fargo2": (0, dict(imax=136, jmax=136, FARGO_flag=2, R_p=0.3), 8, (1, 8)),
    # plnt_flag 2, the reference's default (global.h:20): the planet moves
    # under the disk's forces, summed by the mode 8/9 reductions
    # (device_func.cu:83-108) in planet_forces (planet.cu:54-93)
    "g136x136_moving": (0, dict(imax=136, jmax=136, plnt_flag=2), 8, (1, 4, 8)),
}

# 3D spherical disks (ndim 3, ngeom 2/4/5) on which the reference build runs
# bundle_sweep2D: the radial and azimuthal sweeps of every polar layer and
# rotate_rings, a 3D step without the polar sweep (the reference has none).
# Same tuple as CASES; the fixture keeps Sigma, v_r, v_phi and v_theta of
# every STRIDE3D-th cell.
CASES3D = {
    # the 128x1024x32 disk's physics (p_alpha 1.5, q = 3e-4, theta over 3h
    # above the midplane) on 136 x 136 x 8, damping zones r < 0.6, r > 1.8
    "g3d136x136x8": (1, dict(imax=136, jmax=136, kmax=8, kill_rin=0.6, kill_rout=1.8), 6, (1, 6)),
    # isentropic EOS 1, gam 1.4, on a polar range inside the polytrope's
    # height (theta over 1.4h above the midplane)
    "g3d136x136x8_eos1": (1, dict(imax=136, jmax=136, kmax=8, EOS=1, gam=1.4, zmin=0.5 * 3.141592653589793 - 0.07),
                          6, (1, 6)),
}
STRIDE3D = 7


# Whole runs to the end time (the workload's 10 orbits): name -> (base
# workload, overrides, step limit).  The fixture keeps the history of every
# step and the full final state.  252 x 780 is the warp-aligned size nearest
# the 256 x 768 disk (see above).
LONG_CASES = {
    "g252x780_10orbits": (0, dict(imax=252, jmax=780), 6000),
    # q = 3e-5 (q/h^3 = 0.24) opens no gap: the reference's own 1-ulp
    # sensitivity stays small, so the flat 1e-8 bound applies to the torque
    "g252x780_10orbits_q3e-5": (0, dict(imax=252, jmax=780, M_p=3e-5), 6000),
}


# Timing builds of the reference (sweeps only, no diagnostics reductions):
# name -> (base workload, overrides, nsteps).  Warp-aligned sizes near the
# 256x768 and 1024x3072 disks.
PERF_CASES = {
    "perf_g252x780": (0, dict(imax=252, jmax=780), 200),
    "perf_g1012x3100": (0, dict(imax=1012, jmax=3100), 40),
    # the 3D spherical disk's physics on the warp-aligned grid nearest
    # 128x1024x32: the reference's bundle_sweep2D (radial and azimuthal
    # sweeps of every layer) against the same two sweeps of ours
    "perf_g3d136x1012x32": (1, dict(imax=136, jmax=1012, kmax=32), 20),
}


def params_for(case):
    from penguin_2_0_b200 import _lib
    for table in (CASES, CASES3D, LONG_CASES, PERF_CASES):
        if case in table:
            base, over, *_ = table[case]
            break
    else:
        raise KeyError(case)
    p = _lib.pg_params()
    st = _lib.lib().pg_config_params(base, C.byref(p))
    assert st == 0
    p.update(**over)
    p.nprin = 1
    return p


def to_json(p):
    return {k: (float(v).hex() if isinstance(v, float) else v) for k, v in p.as_dict().items()}


ONLY = None   # --only=case,...: restrict the stages to these cases


def _cases(names):
    return [c for c in names if ONLY is None or c in ONLY]


def cmd_build():
    for case in _cases(list(CASES) + list(CASES3D) + list(PERF_CASES) + list(LONG_CASES)):
        p = params_for(case)
        d = os.path.join(ROOT, "oracle", "_ref", case)
        os.makedirs(d, exist_ok=True)
        pj = os.path.join(d, "params.json")
        json.dump(to_json(p), open(pj, "w"), indent=1)
        mode = "perf" if case in PERF_CASES else "golden"
        subprocess.check_call([os.path.join(ROOT, "oracle", "ref", "build_ref.sh"), case, pj, mode])
        if case in CASES or case in CASES3D:
            # the same sources built for the host CPU (tests/test_refhost_cpu.py)
            subprocess.check_call([os.path.join(ROOT, "oracle", "refhost", "build_refhost.sh"), case])


def cmd_perf(rawdir):
    """Time the reference's bundle_sweep2D (CUDA events around it, summed by
    the harness) on the perf builds; prints one JSON line per case."""
    from penguin_2_0_b200 import _lib
    L = _lib.lib()
    for case in _cases(PERF_CASES):
        nsteps = PERF_CASES[case][2]
        p = params_for(case)
        p.nprin = 100
        out = os.path.join(rawdir, case)
        os.makedirs(out, exist_ok=True)
        ic = os.path.join(out, "ic.bin")
        assert L.pg_write_ic(C.byref(p), ic.encode()) == 0
        write_ghost_override(p, ic)
        exe = os.path.join(ROOT, "oracle", "_ref", case, "penguin_ref")
        r = subprocess.run(["timeout", "-k", "10", "300", exe, ic, str(nsteps), out, "0", "nodiag"],
                           capture_output=True, text=True)
        os.remove(ic)
        if os.path.exists(ic + ".lft"):
            os.remove(ic + ".lft")
        if r.returncode != 0:
            raise SystemExit(f"{case}: reference exited {r.returncode}: {r.stderr[-400:]}")
        d = json.loads(r.stdout.strip().splitlines()[-1])
        cells = p.imax * p.jmax * p.kmax
        d.update(case=case, zone_updates_per_s=cells * d["steps"] / (d["sweep_ms_total"] / 1e3))
        print(json.dumps(d), flush=True)


def write_ghost_override(p, icpath):
    """<ic>.lft for a 3D case: r, p, u, v, w, rot_v of the inner radial ghost
    rings (ring i + 6 k) as the library sets them (pg_boundary_rings).  The
    reference's init_bound leaves them unset on a 3D spherical grid
    (init.cpp:289-294), so its radial sweep would fill the first rings of
    every layer with NaN; the harness loads them from this file."""
    if p.ndim != 3:
        return
    import penguin_2_0_b200 as pg
    lft = pg.host.boundary_rings(p)["lft"]
    cols = [pg.host.BOUNDARY_FIELDS.index(c) for c in ("r", "p", "u", "v", "w", "rot_v")]
    np.ascontiguousarray(lft[:, cols], dtype=np.float64).tofile(icpath + ".lft")


def cmd_run(rawdir):
    from penguin_2_0_b200 import _lib
    L = _lib.lib()
    for case in _cases(list(CASES) + list(CASES3D)):
        _, _, nsteps, keep = CASES[case] if case in CASES else CASES3D[case]
        p = params_for(case)
        out = os.path.join(rawdir, case)
        os.makedirs(out, exist_ok=True)
        ic = os.path.join(out, "ic.bin")
        assert L.pg_write_ic(C.byref(p), ic.encode()) == 0
        write_ghost_override(p, ic)
        exe = os.path.join(ROOT, "oracle", "_ref", case, "penguin_ref")
        t0 = time.time()
        try:
            r = subprocess.run(["timeout", "-k", "10", "120", exe, ic, str(nsteps), out,
                                ",".join(map(str, keep))], capture_output=True, text=True)
        except Exception as e:  # pragma: no cover
            raise SystemExit(f"{case}: {e}")
        open(os.path.join(out, "stdout.txt"), "w").write(r.stdout + r.stderr)
        if r.returncode != 0:
            raise SystemExit(f"{case}: reference exited {r.returncode}: {r.stderr[-400:]}")
        os.remove(ic)
        print(case, f"{time.time() - t0:.1f}s", r.stdout.strip(), flush=True)


PERTURB_CELL = (126, 390)   # (ring, j) of the 1-ulp change of Sigma in the perturbed run


def cmd_run_long(rawdir):
    """Runs each long case twice: from the seeded dump, and from the same dump
    with Sigma of one cell (PERTURB_CELL, a ring at the planet's radius)
    moved up by one ulp.  The second run measures how far the reference's
    own result moves under a rounding-sized change of its input."""
    from penguin_2_0_b200 import _lib
    L = _lib.lib()
    for case in _cases(LONG_CASES):
        _, _, limit = LONG_CASES[case]
        p = params_for(case)
        out = os.path.join(rawdir, case)
        pert = os.path.join(out, "pert")
        os.makedirs(pert, exist_ok=True)
        ic = os.path.join(out, "ic.bin")
        assert L.pg_write_ic(C.byref(p), ic.encode()) == 0
        raw = np.fromfile(ic, dtype=np.uint8)
        ring, j = PERTURB_CELL
        off = ring * (72 * p.jmax + 96) + 8 * j
        x = raw[off:off + 8].copy().view(np.float64)
        raw[off:off + 8] = np.nextafter(x, np.inf).view(np.uint8)
        icp = os.path.join(out, "ic_pert.bin")
        raw.tofile(icp)
        exe = os.path.join(ROOT, "oracle", "_ref", case, "penguin_ref")
        for src, dst in ((ic, out), (icp, pert)):
            t0 = time.time()
            r = subprocess.run(["timeout", "-k", "10", "600", exe, src, str(limit), dst, "end"],
                               capture_output=True, text=True)
            open(os.path.join(dst, "stdout.txt"), "w").write(r.stdout + r.stderr)
            if r.returncode != 0:
                raise SystemExit(f"{case}: reference exited {r.returncode}: {r.stderr[-400:]}")
            print(case, os.path.basename(src), f"{time.time() - t0:.1f}s", r.stdout.strip(), flush=True)
        os.remove(ic)
        os.remove(icp)


def _hist(path):
    rows = [ln.split() for ln in open(path)]
    return np.array([[float.fromhex(x) for x in r[1:]] for r in rows])


def long_errors(f_r, f_u, f_v, ref):
    """Relative L1 of Sigma, of v_r (to the L1 of v_phi) and of v_phi; ref is
    [ring, (Sigma, v_r, v_phi), jmax]."""
    l1 = lambda a, b, sc: float(np.sum(np.abs(a - b)) / np.sum(np.abs(sc)))
    return (l1(f_r, ref[:, 0], ref[:, 0]), l1(f_u, ref[:, 1], ref[:, 2]), l1(f_v, ref[:, 2], ref[:, 2]))


def cmd_pack_long(rawdir, outdir=HERE):
    for case in _cases(LONG_CASES):
        p = params_for(case)
        src = os.path.join(rawdir, case)
        hist = _hist(os.path.join(src, "hist.txt"))
        hist_p = _hist(os.path.join(src, "pert", "hist.txt"))
        f, rot_j = read_rings(os.path.join(src, "state_final.bin"), p)
        fp, _ = read_rings(os.path.join(src, "pert", "state_final.bin"), p)
        ref = f[:, [0, 2, 3], :].copy()
        pert = long_errors(fp[:, 0], fp[:, 2], fp[:, 3], ref)
        np.savez_compressed(os.path.join(outdir, f"{case}.npz"), hist=hist, fields=ref, rot_j=rot_j,
                            hist_pert=hist_p, pert_l1=np.array(pert), perturb_cell=np.array(PERTURB_CELL))
        print("packed", case, hist.shape[0], "steps; 1-ulp sensitivity L1 (Sigma, v_r, v_phi):", pert)


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


def cmd_pack3d(rawdir, outdir=HERE):
    """3D fixtures: per-step history and, at the kept steps, Sigma, v_r,
    v_phi, v_theta [4, every STRIDE3D-th cell of the rings in storage
    order] plus rot_j of every ring."""
    for case in _cases(CASES3D):
        _, _, nsteps, keep = CASES3D[case]
        p = params_for(case)
        src = os.path.join(rawdir, case)
        out = {"hist": _hist(os.path.join(src, "hist.txt")), "stride": np.array(STRIDE3D)}
        for s in keep:
            f, rot_j = read_rings(os.path.join(src, f"state_{s:05d}.bin"), p)
            sel = f[:, [0, 2, 3, 4], :].transpose(1, 0, 2).reshape(4, -1)
            out[f"fields_{s}"] = sel[:, ::STRIDE3D].copy()
            out[f"rot_j_{s}"] = rot_j
        np.savez_compressed(os.path.join(outdir, f"{case}.npz"), **out)
        print("packed", case)


def cmd_pack(rawdir, outdir=HERE, full=None):
    cmd_pack3d(rawdir, outdir)
    for case in _cases(CASES):
        _, _, nsteps, keep = CASES[case]
        p = params_for(case)
        src = os.path.join(rawdir, case)
        rows = [ln.split() for ln in open(os.path.join(src, "hist.txt"))]
        hist = np.array([[float.fromhex(x) for x in r[1:]] for r in rows])
        out = {"hist": hist}
        stride = 1
        if case == "g252x780":
            stride = 7  # every 7th cell keeps the fixture small
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
        if full and case == "g252x780":
            f, rot_j = read_rings(os.path.join(src, f"state_{keep[0]:05d}.bin"), p)
            np.savez_compressed(os.path.join(full, "g252x780_full_step1.npz"), fields=f[:, [0, 2, 3], :],
                                rot_j=rot_j)
        print("packed", case)


if __name__ == "__main__":
    if sys.argv[1].startswith("--only="):
        ONLY = set(sys.argv.pop(1).split("=", 1)[1].split(","))
    what = sys.argv[1]
    if what == "build":
        cmd_build()
    elif what == "run":
        cmd_run(sys.argv[2])
    elif what == "perf":
        cmd_perf(sys.argv[2])
    elif what == "pack":
        cmd_pack(sys.argv[2], *(sys.argv[3:5]))
    elif what == "run_long":
        cmd_run_long(sys.argv[2])
    elif what == "pack_long":
        cmd_pack_long(sys.argv[2], *(sys.argv[3:4]))
    else:
        raise SystemExit(__doc__)
