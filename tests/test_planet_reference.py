"""The planet's host arithmetic against the reference's own planet code.

tests/golden/planet_ref.npz holds what the reference's init_planet,
kick_drift_kick, set_M_p, get_ecc and get_E (planet.cu:11-93) produced on the
host for three flag sets, under seeded disk forces
(tests/golden/make_planet_golden.py, oracle/ref/planet_harness.cu): each step
a kick over dt/2, a drift over dt and a kick over dt/2.  The library's
pg_init_planet, pg_kick_drift_kick, pg_set_M_p, pg_get_ecc and pg_get_E, and
the CPU oracle's planet functions, give the same bits at every step."""
import ctypes as C
import os

import numpy as np
import pytest

from oracle.pyoracle import lib as olib
from penguin_2_0_b200 import _lib
from tests._golden import HERE  # puts tests/golden on sys.path
from make_planet_golden import PLANET_CASES, planet_params  # noqa: E402

G = np.load(os.path.join(HERE, "golden", "planet_ref.npz"))
NSTEPS, DT = int(G["nsteps"]), float(G["dt"])


def _row(b, fr, t, ecc, E, set_m):
    return [b.m, b.x, b.y, b.vx, b.vy, b.fx, b.fy, b.rs, fr.value,
            ecc(C.byref(b), fr.value), E(C.byref(b), fr.value), set_m(t)]


def _orbit(init, kdk, ecc, E, set_m, p, F):
    b, fr = _lib.pg_body(), C.c_double(0.0)
    init(C.byref(p), C.byref(b), C.byref(fr))
    b.fx = b.fy = 0.0
    rows = [_row(b, fr, 0.0, ecc, E, set_m)]
    for n in range(NSTEPS):
        b.fx, b.fy = F[n]
        kdk(C.byref(p), C.byref(b), C.byref(fr), 0.5 * DT, 1)
        kdk(C.byref(p), C.byref(b), C.byref(fr), DT, 0)
        kdk(C.byref(p), C.byref(b), C.byref(fr), 0.5 * DT, 1)
        rows.append(_row(b, fr, (n + 1) * DT, ecc, E, set_m))
    return np.array(rows)


@pytest.mark.parametrize("case", list(PLANET_CASES))
def test_library_planet_matches_reference(case):
    L = _lib.lib()
    p = planet_params(case)
    got = _orbit(L.pg_init_planet, L.pg_kick_drift_kick, L.pg_get_ecc, L.pg_get_E,
                 lambda t: L.pg_set_M_p(C.byref(p), t), p, G[f"{case}_forces"])
    np.testing.assert_array_equal(got, G[f"{case}_rows"])


@pytest.mark.parametrize("case", list(PLANET_CASES))
def test_oracle_planet_matches_reference(case):
    O = olib()
    p = planet_params(case)
    got = _orbit(O.orc_init_planet, O.orc_kick_drift_kick, O.orc_get_ecc, O.orc_get_E,
                 lambda t: O.orc_set_M_p(C.byref(p), t), p, G[f"{case}_forces"])
    np.testing.assert_array_equal(got, G[f"{case}_rows"])
