"""Physics invariants of the CUDA path.

* Mass: the azimuthal sweep is a conservative remap on a periodic ring and
  the FARGO shift only moves cells, so every ring keeps its mass to rounding
  (the two chunks on either side of a chunk boundary compute the same face
  flux).  The reference's idle last chunk (jmax a multiple of 116, ppm.cu:196)
  is the exception: its cells are copied through while their neighbours'
  fluxes still move mass, and the CPU oracle shows the same ~1e-7.
* FARGO: advancing the disk with the orbital advection (FARGO_flag 1) or
  without it (FARGO_flag 0, about 14x more steps at the smaller CFL step)
  gives the same state to truncation error, which falls with resolution.
"""
import numpy as np
import pytest

import penguin_2_0_b200 as pg

TWO_PI = 6.283185307179586


def _ring_mass(f):
    # per ring, the cell volumes are the ring's xvol (and zvol) times a uniform
    # dphi, so the mass is proportional to the sum of Sigma over the ring
    return f["r"].sum(axis=1)


@pytest.mark.gpu
@pytest.mark.parametrize("which,over,tol", [
    (0, dict(imax=136, jmax=408), 1e-14),                  # 408 = 3*116 + 60
    (1, dict(imax=64, jmax=132, kmax=16), 1e-14),          # 3D, 132 = 116 + 16
    (0, dict(imax=136, jmax=464), None),                   # 464 = 4*116: idle last chunk
])
def test_azimuthal_sweep_conserves_ring_mass(gpu, which, over, tol):
    p = pg.params(which, nprin=1, **over)
    with pg.Run(p, 0) as run:
        run.load(pg.build_ic(p))
        planet, frrot = pg.init_planet(p)
        dt = pg.get_dt(p.endtime, run, frrot)
        pg.Index_Shift(run, dt, frrot)
        m0 = _ring_mass(pg.dump_fields(run.save(), p))
        pg.sweep_axis(run, 1, dt, planet, frrot)
        m1 = _ring_mass(pg.dump_fields(run.save(), p))
    rel = np.abs(m1 - m0) / m0
    if tol is not None:
        assert rel.max() <= tol, rel.max()
    else:
        assert rel.max() > 1e-9           # the reference's idle chunk does not conserve


def _one_orbit(ni, nj, fargo):
    p = pg.params(0, imax=ni, jmax=nj, plnt_flag=0, FARGO_flag=fargo, kill_rin=0.0, kill_rout=0.0)
    p.endtime = TWO_PI
    p.tmovie = TWO_PI
    with pg.Run(p, 0) as run:
        run.load(pg.build_ic(p))
        run.clock_reset(0)
        n = run.advance(100000, graph_chunk=64)          # halts at the end time
        c, _ = run.clock()
        assert abs(c.simtime - TWO_PI) <= 1e-12 * TWO_PI
        f = pg.dump_fields(run.save(), p)
    return n, pg.to_physical(f["r"], f["rot_j"])


@pytest.mark.gpu
def test_fargo_on_and_off_agree_to_truncation_error(gpu):
    d = {}
    for ni, nj in ((128, 384), (256, 768)):
        n1, s1 = _one_orbit(ni, nj, 1)
        n0, s0 = _one_orbit(ni, nj, 0)
        assert n0 > 5 * n1, (n0, n1)               # without FARGO the CFL step is far smaller
        d[ni] = float(np.sum(np.abs(s1 - s0)) / np.sum(np.abs(s0)))
    print(f"\nFARGO on vs off after 1 orbit, L1(Sigma): 128x384 {d[128]:.2e}, 256x768 {d[256]:.2e}")
    # measured with the CPU oracle: 1.3e-5 and 4.7e-6
    assert d[128] <= 3e-5 and d[256] <= 1e-5, d
    assert d[128] / d[256] >= 2.0, d              # falls with resolution: truncation error


@pytest.mark.gpu
def test_polar_sweep_keeps_vertical_equilibrium_to_truncation_error(gpu):
    """The polar sweep has no reference kernel, so besides the restatement it
    is held to physics: a 3D disk without planet, noise or viscosity starts in
    vertical equilibrium (the reference's own initial profile, pinned by
    tests/test_ic_reference.py), and five polar sweeps may move it only by a
    truncation error that falls fast with the number of layers over the same
    polar range (the CPU oracle: L1 3.2e-3, 4.7e-4, 4.9e-5 at 8, 16, 32)."""
    err = {}
    for kmax in (8, 16, 32):
        p = pg.params(1, imax=64, jmax=132, kmax=kmax, plnt_flag=0, noise_amp=0.0, visc_flag=0)
        with pg.Run(p, 0) as run:
            ic = pg.build_ic(p)
            run.load(ic)
            planet = pg.Planet()
            dt = pg.get_dt(p.endtime, run, 0.0)
            for _ in range(5):
                pg.sweep_axis(run, 2, dt, planet, 0.0)
            f1 = pg.dump_fields(run.save(), p)
        f0 = pg.dump_fields(ic, p)
        err[kmax] = float(np.sum(np.abs(f1["r"] - f0["r"])) / np.sum(np.abs(f0["r"])))
    print(f"\npolar sweeps from equilibrium, L1(rho): {err}")
    assert err[32] <= 1e-4, err
    assert err[8] / err[16] >= 4.0 and err[16] / err[32] >= 4.0, err
