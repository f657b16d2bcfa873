"""CUDA path (through the C ABI) against the CPU oracle on the same seeded
inputs, step by step.  Tolerance: relative L-inf <= 1e-12 per step on Sigma
(to max|Sigma|) and on v_r, v_phi (to the max speed, so a near-zero v_r does
not turn rounding into a large ratio), relative 1e-12 on dt and disk mass (FP64; the two sides differ
only by FMA contraction and libm ulps).  The torque is a sum of terms that
cancel to ~1e-3 of their magnitude, so its bound is 1e-12 times the sum of
the absolute terms (a floating-point sum's rounding scale)."""
import numpy as np
import pytest

import penguin_2_0_b200 as pg
from tests._lockstep import OracleLoop, rel_linf, torque_abs_scale

TOL = 1e-12

CASES = {
    "g128x132": dict(imax=128, jmax=132),
    "g136x136": dict(imax=136, jmax=136),
    "g232x240": dict(imax=232, jmax=240),          # imax % 116 == 0: last radial chunk idle
    "g130x232": dict(imax=130, jmax=232),          # jmax % 116 == 0: last azimuthal chunk idle
    "g120x150_plain": dict(imax=120, jmax=150, plnt_flag=0, visc_flag=0, flat_flag=0, FARGO_flag=0,
                           kill_rin=0.0, kill_rout=0.0),
    "cfg0": dict(imax=256, jmax=768),
    "g136x136_moving": dict(imax=136, jmax=136, plnt_flag=2),   # the planet feels the disk (global.h default)
    # isentropic EOS 1 (Newton Riemann solver, p = cs2 Sigma^gam / gam)
    "g136x136_eos1": dict(imax=136, jmax=136, EOS=1, gam=1.4),
    "cfg0_eos1": dict(imax=256, jmax=768, EOS=1, gam=5.0 / 3.0),
    "g136x136_eos1_moving": dict(imax=136, jmax=136, EOS=1, gam=1.4, plnt_flag=2),
    # FARGO shift at the solid-body rate: whole-cell shifts in a frame
    # rotating with a planet at R_p = 0.3; the non-rotating frame (FrRot_flag
    # 0), where the planet moves through the grid, with a fixed and a moving planet
    "g136x136_fargo2": dict(imax=136, jmax=136, FARGO_flag=2, R_p=0.3),
    "g136x136_fargo2_inertial": dict(imax=136, jmax=136, FARGO_flag=2, FrRot_flag=0),
    "g256x768_fargo2_moving": dict(imax=256, jmax=768, FARGO_flag=2, FrRot_flag=0, plnt_flag=2),
}


def _params(over):
    p = pg.params(0, nprin=1)
    p.update(**over)
    return p


@pytest.mark.gpu
@pytest.mark.parametrize("case", list(CASES))
def test_host_loop_matches_oracle(gpu, case):
    p = _params(CASES[case])
    ic = pg.build_ic(p)
    ref = OracleLoop(p, ic)
    got = {}

    def rec(s, simtime, dt_used, planet, FrRot):
        mass = pg.GPU_output_reduction(run, planet, 0.0, 0)
        tq = pg.GPU_output_reduction(run, planet, 0.0, 9) / pg.torque_norm(p) if p.plnt_flag else 0.0
        got[s] = (dt_used, mass, tq, pg.dump_fields(run.save(), p))

    with pg.Run(p, 0) as run:
        run.load(ic)
        nsteps = 4
        run.kernel_loop(nsteps, record=rec)
    for s in range(nsteps):
        dt, mass, tq = ref.step()
        f = ref.fields()
        gdt, gmass, gtq, gf = got[s]
        np.testing.assert_array_equal(gf["rot_j"], f["rot_j"])
        speed = max(np.max(np.abs(f["u"])), np.max(np.abs(f["v"])))
        e = [rel_linf(gf["r"], f["r"]), np.max(np.abs(gf["u"] - f["u"])) / speed,
             np.max(np.abs(gf["v"] - f["v"])) / speed]
        assert max(e) <= TOL, (case, s, e)
        assert np.all(gf["w"] == 0.0)
        assert abs(gdt - dt) <= TOL * dt, (s, gdt, dt)
        assert abs(gmass - mass) <= TOL * abs(mass), (s, gmass, mass)
        if p.plnt_flag:
            scale = torque_abs_scale(f, p, pg.Planet(*[getattr(ref.planet, k) for k in
                                                       ("m", "x", "y", "vx", "vy", "fx", "fy", "rs")]))
            assert abs(gtq - tq) <= TOL * scale, (s, gtq, tq, scale)


@pytest.mark.gpu
@pytest.mark.parametrize("eos", [dict(), dict(EOS=1, gam=1.4)])
def test_fused_loop_equals_host_loop(gpu, eos):
    p = _params(dict(imax=256, jmax=768, **eos))
    ic = pg.build_ic(p)
    with pg.Run(p, 0) as a, pg.Run(p, 0) as b:
        a.load(ic)
        b.load(ic)
        n, simtime, dt, planet, FrRot = a.kernel_loop(6)
        b.clock_reset(0)
        assert b.advance(6) == 6
        c, pl = b.clock()
        assert c.simtime == simtime
        assert c.dt == dt
        fa, fb = pg.dump_fields(a.save(), p), pg.dump_fields(b.save(), p)
        for fld in ("r", "p", "u", "v", "rot_j", "inc_j", "res_v", "rot_v"):
            np.testing.assert_array_equal(fa[fld], fb[fld], err_msg=fld)


@pytest.mark.gpu
def test_output_times_fused_loop_equals_host_loop(gpu):
    """tmovie well below the end time (dt ~0.018 on this disk): both loops cut
    dt to land on every output time, then go back to the step before the cut
    (main.cu:361-366, 407-411).  The device loop halts at each output time for
    the host to dump, and the next pg_advance resumes from there."""
    p = _params(dict(imax=256, jmax=768))
    p.tmovie = 0.05
    ic = pg.build_ic(p)
    nsteps = 12
    with pg.Run(p, 0) as a, pg.Run(p, 0) as b:
        a.load(ic)
        b.load(ic)
        n, simtime, dt, planet, FrRot = a.kernel_loop(nsteps)
        assert n == nsteps and simtime > 2 * p.tmovie
        b.clock_reset(0)
        done, calls = 0, 0
        while done < nsteps and calls < 4 * nsteps:
            done += b.advance(nsteps - done)
            calls += 1
        assert done == nsteps and calls > 2          # it stopped at the output times
        c, pl = b.clock()
        assert c.simtime == simtime
        assert c.dt == dt
        fa, fb = pg.dump_fields(a.save(), p), pg.dump_fields(b.save(), p)
        for fld in ("r", "p", "u", "v", "rot_j", "inc_j", "res_v", "rot_v"):
            np.testing.assert_array_equal(fa[fld], fb[fld], err_msg=fld)


@pytest.mark.gpu
def test_graph_equals_stream_loop(gpu):
    p = _params(dict(imax=256, jmax=768))
    ic = pg.build_ic(p)
    with pg.Run(p, 0) as a, pg.Run(p, 0) as b:
        a.load(ic)
        b.load(ic)
        a.clock_reset(0)
        b.clock_reset(0)
        assert a.advance(9) == 9
        assert b.advance(9, graph_chunk=4) == 9
        np.testing.assert_array_equal(np.frombuffer(a.save(), np.uint8), np.frombuffer(b.save(), np.uint8))
        ha, hb = a.history(), b.history()
        np.testing.assert_array_equal(ha, hb)
        assert ha.shape[0] == 9


@pytest.mark.gpu
def test_isentropic_dump_pressure(gpu):
    # the saved p of an EOS-1 run is the store's cs2 Sigma^gam / gam
    # (ppm.cu:140-141), derived on the device from the planes
    gam = 1.4
    p = _params(dict(imax=136, jmax=136, EOS=1, gam=gam))
    with pg.Run(p, 0) as run:
        run.load(pg.build_ic(p))
        run.clock_reset(0)
        run.advance(3)
        f = pg.dump_fields(run.save(), p)
    cs2 = p.sc_h ** 2 * f["xc"][:, None] ** -p.p_beta
    # CUDA's pow is within 2 ulp, libm's within 1; the product and the
    # division add a rounding each: 6 ulp
    np.testing.assert_allclose(f["p"], cs2 * f["r"] ** gam / gam, rtol=6 * 2.0 ** -53 * 2)


@pytest.mark.gpu
def test_dump_roundtrip_bitwise(gpu):
    p = _params(dict(imax=128, jmax=132))
    ic = pg.build_ic(p)
    with pg.Run(p, 0) as run:
        run.load(ic)
        out = run.save()
    assert bytes(out) == bytes(ic)


@pytest.mark.gpu
@pytest.mark.parametrize("precision", [0, 1])
def test_moving_planet_fused_loop_matches_host_loop(gpu, precision):
    # plnt_flag 2: the device loop drifts the planet, reduces the disk's
    # forces on it (modes 8 and 9) and kicks it every step; the host-driven
    # loop does the same through pg_planet_forces.  The softening rs = rs_fac
    # h(x) uses the device pow on one side and the host pow on the other, so
    # the two agree to rounding, not bit for bit.
    p = _params(dict(imax=136, jmax=136, plnt_flag=2, precision=precision))
    ic = pg.build_ic(p)
    hist = []

    def rec(s, simtime, dt_used, planet, FrRot):
        hist.append((simtime, planet.x, planet.y, planet.vx, planet.vy))

    with pg.Run(p, 0) as a, pg.Run(p, 0) as b:
        a.load(ic)
        b.load(ic)
        a.kernel_loop(12, record=rec)
        b.clock_reset(0)
        assert b.advance(12) == 12
        c, pl = b.clock()
        t, x, y, vx, vy = hist[-1]
        assert abs(c.simtime - t) <= 1e-12 * t
        for got, want in ((pl.x, x), (pl.y, y)):
            assert abs(got - want) <= 1e-12 * abs(want), (got, want)
        for got, want in ((pl.vx, vx), (pl.vy, vy)):
            assert abs(got - want) <= 1e-12 * max(abs(vx), abs(vy), 1e-6), (got, want)
        fa, fb = pg.dump_fields(a.save(), p), pg.dump_fields(b.save(), p)
        np.testing.assert_array_equal(fa["rot_j"], fb["rot_j"])
        tol = 1e-12 if precision == 0 else 1e-6
        speed = max(np.max(np.abs(fa["u"])), np.max(np.abs(fa["v"])))
        assert rel_linf(fb["r"], fa["r"]) <= tol
        assert np.max(np.abs(fb["u"] - fa["u"])) / speed <= tol
        assert np.max(np.abs(fb["v"] - fa["v"])) / speed <= tol
