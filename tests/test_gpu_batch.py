"""Batches: runs stepped together give, bitwise, what each run gives alone.

A batch tiles the pencil chunks of every 2D member of a precision group into
one launch per phase and gives 3D members their own launches; every member
keeps its own clock and dt.  These tests build mixed batches (FP64 and FP32,
several grid sizes, planet masses and end times, one 3D disk) and compare
every member with the same run advanced alone by pg_advance, field by field
and clock by clock, bit for bit; then repeat with persistent grids and both
register budgets to show the launch shape does not enter the results."""
import numpy as np
import pytest

import penguin_2_0_b200 as pg

CASES = [
    dict(which=0, imax=128, jmax=384, M_p=1e-3),
    dict(which=0, imax=192, jmax=576, M_p=3e-4, precision=1),
    dict(which=0, imax=256, jmax=768, M_p=1e-5, sc_h=0.04),
    dict(which=0, imax=128, jmax=384, M_p=1e-4, precision=1, ss_alpha=1e-2),
    dict(which=0, imax=136, jmax=408, plnt_flag=0, precision=1),
    dict(which=1, imax=64, jmax=132, kmax=16),
    dict(which=0, imax=136, jmax=408, plnt_flag=2),             # moving planet: own launch sequence
    dict(which=0, imax=136, jmax=408, EOS=1, gam=1.4),          # isentropic: own launch sequence
]


def _params(c, **over):
    c = dict(c)
    which = c.pop("which")
    p = pg.params(which, nprin=4, **c)
    p.update(**over)
    return p


def _fields(run, p):
    f = pg.dump_fields(run.save(), p)
    return {k: f[k].copy() for k in ("r", "u", "v", "w", "rot_j")}


def _solo(p, ic, nsteps):
    with pg.Run(p, 0) as r:
        r.load(ic)
        r.clock_reset(0)
        r.advance(nsteps)
        c, _ = r.clock()
        return _fields(r, p), (c.ncycle, c.simtime, c.dt), r.history()


def _check_batch(params, nsteps, shapes=None, chunk=4):
    ics = [pg.build_ic(p) for p in params]
    want = [_solo(p, ic, nsteps) for p, ic in zip(params, ics)]
    runs = [pg.Run(p, 0).load(ic) for p, ic in zip(params, ics)]
    for r in runs:
        r.clock_reset(0)
    with pg.Batch(0) as b:
        for r in runs:
            b.add(r)
        if shapes:
            for g, sh in shapes.items():
                b.set_shape(g, **sh)
        b.advance(nsteps, chunk=chunk)
        st = b.status()
        assert b.launches() > 0
        for r in list(runs):
            b.remove(r)
    for k, (p, r, (wf, wc, wh)) in enumerate(zip(params, runs, want)):
        c, _ = r.clock()
        assert (c.ncycle, c.simtime, c.dt) == wc, (k, (c.ncycle, c.simtime, c.dt), wc)
        assert st[k]["ncycle"] == wc[0]
        gf = _fields(r, p)
        for f in ("r", "u", "v", "w", "rot_j"):
            np.testing.assert_array_equal(gf[f], wf[f], err_msg=f"member {k} field {f}")
        np.testing.assert_array_equal(r.history(), wh, err_msg=f"member {k} history")
        r.close()


@pytest.mark.gpu
def test_batch_members_equal_solo_runs(gpu):
    _check_batch([_params(c) for c in CASES], 10)


@pytest.mark.gpu
def test_batch_launch_shape_does_not_change_results(gpu):
    shapes = {0: dict(grid_x=148 * 4, grid_y=148, minb=4), 1: dict(grid_x=296, grid_y=148 * 8, minb=8)}
    _check_batch([_params(c) for c in CASES[:5]], 6, shapes=shapes, chunk=3)


@pytest.mark.gpu
def test_batch_members_halt_at_their_own_end_time(gpu):
    # a short run halts (end time) while the others keep stepping; the batch
    # stops replaying once every member has halted
    p_short = _params(CASES[0], endtime=0.05, tmovie=0.05)
    p_long = _params(CASES[1])
    ic_s, ic_l = pg.build_ic(p_short), pg.build_ic(p_long)
    rs = pg.Run(p_short, 0).load(ic_s)
    rl = pg.Run(p_long, 0).load(ic_l)
    rs.clock_reset(0)
    rl.clock_reset(0)
    with pg.Batch(0) as b:
        b.add(rs).add(rl)
        b.advance(40, chunk=8)
        st = b.status()
        assert st[0]["halted"] == 1 and st[0]["status"] == 0
        assert abs(st[0]["simtime"] - 0.05) < 1e-12
        assert st[1]["halted"] == 0 and st[1]["ncycle"] == 40
        n_short = st[0]["ncycle"]
        b.remove(rs)
        b.remove(rl)
    want, wc, _ = _solo(p_short, ic_s, 40)
    c, _ = rs.clock()
    assert c.ncycle == n_short == wc[0]
    np.testing.assert_array_equal(_fields(rs, p_short)["r"], want["r"])
    rs.close()
    rl.close()


@pytest.mark.gpu
def test_batch_tuner_keeps_results(gpu):
    params = [_params(c) for c in CASES[:4]]
    ics = [pg.build_ic(p) for p in params]
    runs = [pg.Run(p, 0).load(ic) for p, ic in zip(params, ics)]
    for r in runs:
        r.clock_reset(0)
    with pg.Batch(0) as b:
        for r in runs:
            b.add(r)
        b.tune(2)                    # 6 candidates x (1 + 2) steps per group
        steps = [s["ncycle"] for s in b.status()]
        assert all(s == 18 for s in steps), steps
        for g in (0, 1):
            sh = b.shape(g)
            assert sh["minb"] in (4, 8)
        b.advance(4, chunk=2)
        for r in list(runs):
            b.remove(r)
    for p, ic, r in zip(params, ics, runs):
        want, wc, _ = _solo(p, ic, 22)
        np.testing.assert_array_equal(_fields(r, p)["r"], want["r"])
        r.close()
