"""The grid generator against the reference's own grid() (grid.cu:66-221).

tests/golden/grid_ref.npz holds the face, centre and width arrays that the
reference's host grid() produced for every grid type this library supports
(uniform 0; logarithmic 1, 2, 3; refined toward the centre 4; refined toward
the upper edge 6) over a radial, an azimuthal and a polar range, built with
the spacing limits of the 2D 256x768 disk (tests/golden/make_grid_golden.py).
The library writes the same arrays into the dump records of a seeded initial
condition; both sides are host code with the same libm, so they agree bit
for bit.  Type 4 takes the radial limits dx_min/dx_max and type 6 the polar
limits dz_min/dz_max on every axis, as the reference's global constants do."""
import os

import numpy as np
import pytest

import penguin_2_0_b200 as pg

G = np.load(os.path.join(os.path.dirname(__file__), "golden", "grid_ref.npz"))


def _azimuth_arrays(buf, p):
    """y, yc, dy of ring 0's record (every ring holds the same)."""
    rb = 72 * p.jmax + 96
    raw = np.frombuffer(bytes(buf), dtype=np.uint8)[:rb]
    ys = raw[40 * p.jmax + 32:72 * p.jmax + 32].copy().view(np.float64).reshape(4, p.jmax)
    return ys[0], ys[3], ys[1]


@pytest.mark.parametrize("lg", [0, 1, 2, 3, 4, 6])
def test_radial_grid_matches_reference(lg):
    p = pg.params(0, grspx=lg)
    f = pg.dump_fields(pg.build_ic(p), p)
    want = G[f"r_lg{lg}"]
    for got, w, name in ((f["x"], want[0], "xa"), (f["xc"], want[1], "xc"), (f["dx"], want[2], "dx")):
        np.testing.assert_array_equal(got[:p.imax], w, err_msg=name)


@pytest.mark.parametrize("lg", [0, 4])
def test_azimuthal_grid_matches_reference(lg):
    p = pg.params(0, grspy=lg)
    ya, yc, dy = _azimuth_arrays(pg.build_ic(p), p)
    want = G[f"phi_lg{lg}"]
    np.testing.assert_array_equal(ya, want[0])
    np.testing.assert_array_equal(yc, want[1])
    np.testing.assert_array_equal(dy, want[2])


@pytest.mark.parametrize("lg", [0, 6])
def test_polar_grid_matches_reference(lg):
    p = pg.params(1, imax=64, jmax=132, kmax=32, grspz=lg)
    f = pg.dump_fields(pg.build_ic(p), p)
    layer0 = np.arange(p.kmax) * p.imax             # ring i = 0 of every layer
    want = G[f"theta_lg{lg}"]
    np.testing.assert_array_equal(f["z"][layer0], want[0])
    np.testing.assert_array_equal(f["zc"][layer0], want[1])
    np.testing.assert_array_equal(f["dz"][layer0], want[2])
