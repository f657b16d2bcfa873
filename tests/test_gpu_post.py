"""Post-processing on the device against the reference's read/ tools.

pg_post_harmonic restates read/p_output.cpp:35-55 (write_har_file) and
pg_post_torque read/transform.cpp:386-420 (get_torque); both work on the run's
physical-order state, which read/p_init.cpp:108-133 rebuilds from a dump by
undoing each ring's rot_j.

Two pins:
* the reference's own get_torque and write_har_file, run on the host on the
  dumps of tests/golden/post_ref.npz (make_post_golden.py: the seeded dump
  advanced by the CPU oracle, regenerated here the same way), against the
  device (GPU tests) and against the numpy restatement below (CPU test);
* that numpy restatement against the device on states the library advanced
  itself, in FP64 and FP32, 2D and 3D.
All compare to rounding: the device sums in a tree, the reference in a
sequential loop, so the bound is 1e-12 of the sum of the absolute terms."""
import os
import sys

import numpy as np
import pytest

import penguin_2_0_b200 as pg

TOL = 1e-12
HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))
from make_post_golden import HARMONICS, POST_CASES, post_state  # noqa: E402


def _ref():
    return np.load(os.path.join(HERE, "golden", "post_ref.npz"))


def _harmonic_np(rho, yc, m):
    """write_har_file's sums for layer 0 (rho in physical order [i, j])."""
    ta = np.sin(m * yc)[None, :] * rho
    tb = np.cos(m * yc)[None, :] * rho
    return ta.sum(axis=1), tb.sum(axis=1), np.abs(ta).sum(axis=1), np.abs(tb).sum(axis=1)


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


def _dump_view(p, dump):
    f = pg.dump_fields(dump, p)
    rho = pg.to_physical(f["r"], f["rot_j"])
    yc, dy = _azimuth(dump, p)
    return f, rho, yc, dy


@pytest.mark.parametrize("case", list(POST_CASES))
def test_numpy_restatement_matches_reference_read_tools(case):
    """CPU: the numpy sums the GPU tests use equal the reference's own
    get_torque and write_har_file on the same dump."""
    g = _ref()
    p, dump = post_state(case)
    f, rho, yc, dy = _dump_view(p, dump)
    tq, scale = _torque_np(f, rho, yc, dy, p.M_p, p.imax, p.kmax)
    assert abs(tq - float(g[f"{case}_torque"])) <= TOL * scale
    layer0 = rho[:p.imax]            # rings i + imax k: layer 0 first
    for m in HARMONICS:
        an, bn, sa, sb = _harmonic_np(layer0, yc, m)
        assert np.all(np.abs(an - g[f"{case}_m{m:g}_an"]) <= TOL * sa)
        assert np.all(np.abs(bn - g[f"{case}_m{m:g}_bn"]) <= TOL * sb)


@pytest.mark.gpu
@pytest.mark.parametrize("case", list(POST_CASES))
def test_device_post_matches_reference_read_tools(gpu, case):
    """The device's pg_post_torque and pg_post_harmonic on the golden dump
    (loaded with pg_load_rings) against the reference's own read/ routines."""
    g = _ref()
    p, dump = post_state(case)
    f, rho, yc, dy = _dump_view(p, dump)
    _, scale = _torque_np(f, rho, yc, dy, p.M_p, p.imax, p.kmax)
    with pg.Run(p, 0) as r:
        r.load(dump)
        got = r.post_torque(p.M_p)
        assert abs(got - float(g[f"{case}_torque"])) <= TOL * scale, (got, float(g[f"{case}_torque"]), scale)
        layer0 = rho[:p.imax]
        for m in HARMONICS:
            an, bn = r.harmonic(m)
            _, _, sa, sb = _harmonic_np(layer0, yc, m)
            assert np.all(np.abs(an - g[f"{case}_m{m:g}_an"]) <= TOL * sa), m
            assert np.all(np.abs(bn - g[f"{case}_m{m:g}_bn"]) <= TOL * sb), m
