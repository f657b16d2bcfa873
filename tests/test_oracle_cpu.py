"""The CPU oracle on its own: determinism, conservation structure and the
reference behaviours it restates (chunk-edge viscosity, idle last chunk)."""
import numpy as np

import penguin_2_0_b200 as pg
from oracle.pyoracle import Oracle


def _run(p, n):
    o = Oracle(p, pg.build_ic(p))
    h = o.run_steps(n)
    return h, pg.dump_fields(o.save(), p)


def test_oracle_deterministic_and_finite():
    p = pg.params(0, imax=128, jmax=132)
    h1, f1 = _run(p, 3)
    h2, f2 = _run(p, 3)
    np.testing.assert_array_equal(h1, h2)
    for k in ("r", "u", "v"):
        np.testing.assert_array_equal(f1[k], f2[k])
        assert np.all(np.isfinite(f1[k]))
    assert np.all(f1["r"] > 0)


def test_unperturbed_disk_without_planet_stays_near_equilibrium():
    # no planet, no noise: the pressure-supported disk is close to steady
    p = pg.params(0, imax=128, jmax=132, plnt_flag=0, noise_amp=0.0, kill_rin=0.0, kill_rout=0.0)
    h, f = _run(p, 5)
    ic = pg.dump_fields(pg.build_ic(p), p)
    inner = slice(8, 120)
    rel = np.max(np.abs(f["r"][inner] / ic["r"][inner] - 1.0))
    assert rel < 1e-5, rel
    # axisymmetry is kept to rounding
    assert np.max(np.std(f["r"][inner], axis=1) / np.mean(f["r"][inner], axis=1)) < 1e-12


def test_idle_last_radial_chunk_is_reproduced():
    # imax % 116 == 0: ppm.cu:48 gives the last chunk lim = 12, so rings
    # 116..231 are never touched by the radial sweep; with no planet, no
    # viscosity and no noise the azimuthal sweep leaves an axisymmetric ring
    # unchanged too, so those rings keep their initial values.
    p = pg.params(0, imax=232, jmax=240, plnt_flag=0, noise_amp=0.0, kill_rin=0.0, kill_rout=0.0,
                  visc_flag=0, FARGO_flag=0)
    ic = pg.dump_fields(pg.build_ic(p), p)
    h, f = _run(p, 1)
    assert np.array_equal(f["u"][116:], ic["u"][116:])
    assert not np.array_equal(f["u"][:116], ic["u"][:116])


def test_output_time_cuts_agree_between_the_oracle_loops():
    """tmovie well below the end time: the C restart loop (orc_run_steps) and
    the step-by-step loop the GPU parity tests drive (tests/_lockstep.py) cut
    dt to land on every output time and return to the step before the cut
    (main.cu:361-366, 407-411); they agree bit for bit, and the output times
    are hit exactly."""
    from tests._lockstep import OracleLoop
    p = pg.params(0, imax=128, jmax=132, nprin=1)
    p.tmovie = 0.05
    n = 10
    h, f = _run(p, n)
    loop = OracleLoop(p, pg.build_ic(p))
    dts = [loop.step()[0] for _ in range(n)]
    g = loop.fields()
    np.testing.assert_array_equal(h[:, 1], dts)
    for k in ("r", "u", "v", "rot_j"):
        np.testing.assert_array_equal(f[k], g[k], err_msg=k)
    t = h[:, 0]
    k = np.floor(t / p.tmovie + 1e-9)
    cuts = np.nonzero(np.diff(k) > 0)[0] + 1          # steps that end on an output time
    assert len(cuts) >= 2
    np.testing.assert_allclose(t[cuts], k[cuts] * p.tmovie, rtol=1e-14)
    # after a cut the step returns to the uncut dt's growth path
    assert all(h[c + 1, 1] > h[c, 1] for c in cuts if c + 1 < n)


def test_oracle_struct_images_match_the_product_binding():
    """oracle/abi.py keeps its own images of pg_params and pg_body so the CPU
    baseline can run without the product library; they must be the product
    binding's layout exactly (names, types, offsets, size)."""
    import ctypes as C
    from oracle import abi
    from penguin_2_0_b200 import _lib
    for mine, theirs in ((abi.pg_params, _lib.pg_params), (abi.pg_body, _lib.pg_body)):
        assert C.sizeof(mine) == C.sizeof(theirs)
        assert [(n, t) for n, t in mine._fields_] == [(n, t) for n, t in theirs._fields_]
        for n, _ in mine._fields_:
            assert getattr(mine, n).offset == getattr(theirs, n).offset, n


def test_oracle_polar_sweep_keeps_vertical_equilibrium_to_truncation_error():
    """The restatement of the polar sweep (which has no reference kernel)
    against physics: from the vertically isothermal equilibrium of a 3D disk
    without planet, noise or viscosity, five polar sweeps move the density by
    a truncation error that falls by 4x or more per doubling of the layers."""
    import ctypes as C
    from oracle.pyoracle import lib as olib
    from oracle.abi import pg_body
    err = {}
    for kmax in (8, 16, 32):
        p = pg.params(1, imax=64, jmax=132, kmax=kmax, plnt_flag=0, noise_amp=0.0, visc_flag=0)
        ic = pg.build_ic(p)
        o = Oracle(p, ic)
        b = pg_body()
        dt = o.get_dt(p.endtime, 0.0)
        for _ in range(5):
            olib().orc_sweepz(o._h, dt, C.byref(b), 0.0)
        f1, f0 = pg.dump_fields(o.save(), p), pg.dump_fields(ic, p)
        err[kmax] = float(np.sum(np.abs(f1["r"] - f0["r"])) / np.sum(np.abs(f0["r"])))
    assert err[32] <= 1e-4, err
    assert err[8] / err[16] >= 4.0 and err[16] / err[32] >= 4.0, err
