"""Post-processing on the device against the reference's read/ tools.

pg_post_harmonic restates read/p_output.cpp:35-55 (write_har_file) and
pg_post_torque read/transform.cpp:386-420 (get_torque); both work on the run's
physical-order state, which read/p_init.cpp:108-133 rebuilds from a dump by
undoing each ring's rot_j.  Here the same quantities are computed with numpy
from the saved dump (de-rotated the same way) and compared to rounding: the
device sums in a tree, the reference in a sequential loop, so the bound is
1e-12 of the sum of the absolute terms."""
import numpy as np
import pytest

import penguin_2_0_b200 as pg

TOL = 1e-12


def _azimuth(buf, p):
    """yc and dy of the dump (the y arrays of ring 0; every ring holds the same)."""
    rb = 72 * p.jmax + 96
    raw = np.frombuffer(bytes(buf), dtype=np.uint8)[:rb]
    ys = raw[40 * p.jmax + 32:72 * p.jmax + 32].copy().view(np.float64).reshape(4, p.jmax)
    return ys[3], ys[1]


def _state(p, nsteps):
    r = pg.Run(p, 0).load(pg.build_ic(p))
    r.clock_reset(0)
    r.advance(nsteps)
    buf = r.save()
    f = pg.dump_fields(buf, p)
    rho = pg.to_physical(f["r"], f["rot_j"])      # update_grid's de-rotation
    assert np.any(f["rot_j"] != 0)
    yc, dy = _azimuth(buf, p)
    return r, f, rho, yc, dy


@pytest.mark.gpu
@pytest.mark.parametrize("precision", [0, 1])
def test_harmonics_match_read_tool(gpu, precision):
    p = pg.params(0, imax=128, jmax=384, precision=precision)
    r, f, rho, yc, _ = _state(p, 30)
    try:
        for m in (1.0, 2.0, 5.0):
            an, bn = r.harmonic(m)
            ta = np.sin(m * yc)[None, :] * rho
            tb = np.cos(m * yc)[None, :] * rho
            for got, terms in ((an, ta), (bn, tb)):
                want = terms.sum(axis=1)
                scale = np.abs(terms).sum(axis=1)
                assert np.all(np.abs(got - want) <= TOL * scale), (m, np.max(np.abs(got - want) / scale))
    finally:
        r.close()


def _torque_np(f, rho, yc, dy, M_p, nr, nk):
    stm = 1.0 / (1.0 + M_p)
    plm = M_p * stm
    plx, stx = 1.0 * stm, 1.0 * plm
    cosfac = np.cos(yc - np.pi)[None, :]
    sinfac = np.sin(yc - np.pi)[None, :]
    rad = f["xc"][:, None]
    z = f["zc"][:, None]
    Rp = np.sqrt(rad * rad + plx * plx - 2.0 * plx * rad * cosfac + z * z + 0.000003)
    Rs = np.sqrt(rad * rad + stx * stx + 2.0 * stx * rad * cosfac + z * z)
    terms = rho * (plm * plx * sinfac / Rp ** 3 - stm * stx * sinfac / Rs ** 3) * rad * dy[None, :] * \
        f["dx"][:, None] * f["dz"][:, None]
    return terms.sum(), np.abs(terms).sum()


@pytest.mark.gpu
@pytest.mark.parametrize("which,over", [(0, dict(imax=128, jmax=384)), (0, dict(imax=128, jmax=384, precision=1)),
                                        (1, dict(imax=64, jmax=132, kmax=16))])
def test_torque_matches_read_tool(gpu, which, over):
    p = pg.params(which, **over)
    r, f, rho, yc, dy = _state(p, 20)
    try:
        got = r.post_torque(p.M_p)
        want, scale = _torque_np(f, rho, yc, dy, p.M_p, p.imax, p.kmax)
        assert abs(got - want) <= TOL * scale, (got, want, scale)
    finally:
        r.close()
