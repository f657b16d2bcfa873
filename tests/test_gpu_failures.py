"""Failure detection without a GPU fault.

Failures are made on the host (a dump with a bad density, which the host
rejects, or a bad velocity, which the device catches; parameters whose time
step collapses; calls out of order; wrong buffer sizes).  The kernels check
every stored cell and the time step and report through the run's status
word; nothing traps, faults or waits.  After each failure the context stays
usable: a fresh run on the same device steps normally."""
import struct

import numpy as np
import pytest

import penguin_2_0_b200 as pg


def _poison(ic, p, ring, j, value, field=0):
    """One cell of a dump image set to `value`; field 0 = Sigma, 2 = v_r
    (the ring record holds r, p, u, v, w arrays of jmax doubles first)."""
    b = bytearray(ic)
    struct.pack_into("<d", b, ring * (72 * p.jmax + 96) + 8 * (field * p.jmax + j), value)
    return b


def _healthy_step_works():
    p = pg.params(0, imax=128, jmax=132)
    with pg.Run(p, 0) as r:
        r.load(pg.build_ic(p))
        r.clock_reset(0)
        assert r.advance(3) == 3


@pytest.mark.gpu
@pytest.mark.parametrize("value", [float("nan"), -1.0, 0.0, float("inf")])
def test_bad_density_is_rejected_at_load(gpu, value):
    p = pg.params(0, imax=128, jmax=384)
    with pg.Run(p, 0) as r:
        with pytest.raises(pg.PenguinError) as e:
            r.load(_poison(pg.build_ic(p), p, 60, 100, value))
        assert e.value.status == 7          # PG_ERR_STATE: non-positive density in dump
    _healthy_step_works()


@pytest.mark.gpu
@pytest.mark.parametrize("value,precision", [(float("nan"), 0), (float("inf"), 0), (float("nan"), 1)])
def test_bad_velocity_is_reported_by_the_device(gpu, value, precision):
    # the dump loads (velocities are not screened on the host); the CFL and
    # the sweeps' cell checks stop the device loop with a status code
    p = pg.params(0, imax=128, jmax=384, precision=precision)
    ic = _poison(pg.build_ic(p), p, 60, 100, value, field=2)
    with pg.Run(p, 0) as r:
        r.load(ic)
        r.clock_reset(0)
        with pytest.raises(pg.PenguinError) as e:
            r.advance(20)
        assert e.value.status in (3, 4), e.value     # non-finite state or collapsed dt
        c, _ = r.clock()
        assert c.status in (3, 4) and c.ncycle < 20
    _healthy_step_works()


@pytest.mark.gpu
def test_dt_collapse_is_reported(gpu):
    # dt ~ 1e-2 against an end time of 1e15: dt / endtime < 1e-12 (timestep.cu:143)
    p = pg.params(0, imax=128, jmax=132, endtime=1e15, tmovie=1e15)
    with pg.Run(p, 0) as r:
        r.load(pg.build_ic(p))
        r.clock_reset(0)
        with pytest.raises(pg.PenguinError) as e:
            r.advance(5)
        assert e.value.status == 4
    _healthy_step_works()


@pytest.mark.gpu
def test_calls_out_of_order_and_bad_sizes(gpu):
    p = pg.params(0, imax=128, jmax=132)
    ic = pg.build_ic(p)
    with pg.Run(p, 0) as r:
        with pytest.raises(pg.PenguinError):
            r.advance(1)                      # no dump loaded, no clock
        with pytest.raises(pg.PenguinError) as e:
            r.load(ic[:-8])                   # short dump
        assert e.value.status in (6, 9)
        r.load(ic)
        with pytest.raises(pg.PenguinError) as e:
            r.advance(1)                      # clock not reset
        assert e.value.status == 7
    _healthy_step_works()


@pytest.mark.gpu
def test_run_larger_than_the_gpu_is_refused(gpu):
    # one plane of 20012 x 1200000 rings x 8 B is 192 GB, more than the GPU
    # holds: creation fails at its first allocation and reports PG_ERR_NOMEM,
    # and the allocation error it cleared does not reach the next run's
    # launch checks
    p = pg.params(0, imax=20000, jmax=1200000)
    assert pg.host.check_params(p) == 0
    assert pg.run_device_bytes(p) > 10 ** 12
    with pytest.raises(pg.PenguinError) as e:
        pg.Run(p, 0)
    assert e.value.status == 8            # PG_ERR_NOMEM
    _healthy_step_works()


@pytest.mark.gpu
def test_batch_member_failure_stays_local(gpu):
    # a member with a bad cell halts with its status; the other member steps
    # on and still equals the same run advanced alone
    p_bad = pg.params(0, imax=128, jmax=384)
    p_ok = pg.params(0, imax=192, jmax=576, precision=1)
    ic_ok = pg.build_ic(p_ok)
    bad = pg.Run(p_bad, 0).load(_poison(pg.build_ic(p_bad), p_bad, 40, 10, float("nan"), field=2))
    ok = pg.Run(p_ok, 0).load(ic_ok)
    ok.clock_reset(0)
    bad.clock_reset(0)
    with pg.Batch(0) as b:
        b.add(bad).add(ok)
        b.advance(12, chunk=4)
        st = b.status()
        b.remove(bad)
        b.remove(ok)
    assert st[0]["halted"] == 1 and st[0]["status"] in (3, 4)
    assert st[1]["halted"] == 0 and st[1]["status"] == 0 and st[1]["ncycle"] == 12
    with pg.Run(p_ok, 0) as solo:
        solo.load(ic_ok)
        solo.clock_reset(0)
        solo.advance(12)
        np.testing.assert_array_equal(pg.dump_fields(ok.save(), p_ok)["r"], pg.dump_fields(solo.save(), p_ok)["r"])
    bad.close()
    ok.close()
