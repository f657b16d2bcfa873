"""The planet's host arithmetic (planet.cu:11-93): library against oracle.

pg_init_planet, pg_kick_drift_kick, pg_set_M_p, pg_get_E and pg_get_ecc run
on the host in both, as in the reference.  The softening length rs follows
the disk profile's scale height, whose constant exponents the reference's
host compiler folds (pow(r, -1) into 1/r and so on); the library and the
oracle restate that folding independently.  A sequence of kicks and drifts
with set forces (the disk's share of the force needs a GPU) gives the same
bits on both sides for several disks."""
import ctypes as C

import numpy as np
import pytest

from oracle.pyoracle import lib as olib
from penguin_2_0_b200 import _lib

FIELDS = ("m", "x", "y", "vx", "vy", "fx", "fy", "rs")


def _state(b, fr):
    return [getattr(b, f) for f in FIELDS] + [fr.value]


@pytest.mark.parametrize("over", [
    dict(),
    dict(p_beta=0.5, R_p=1.3, rs_fac=0.4),
    dict(p_beta=0.0, p_alpha=0.5, sc_h=0.03, FrRot_flag=0),
    dict(p_beta=2.0, R_p=0.8, t_growth=20.0, plnt_flag=2),
])
def test_planet_host_arithmetic_matches_oracle(over):
    L, O = _lib.lib(), olib()
    p = _lib.pg_params()
    assert L.pg_config_params(0, C.byref(p)) == 0
    p.update(**over)
    a, b = _lib.pg_body(), _lib.pg_body()
    fa, fb = C.c_double(0.0), C.c_double(0.0)
    assert L.pg_init_planet(C.byref(p), C.byref(a), C.byref(fa)) == 0
    O.orc_init_planet(C.byref(p), C.byref(b), C.byref(fb))
    assert _state(a, fa) == _state(b, fb)
    rng = np.random.default_rng(7)
    dt = 0.01
    for step in range(200):
        fx, fy = rng.normal(scale=1e-3, size=2)
        for body in (a, b):
            body.fx, body.fy = fx, fy
        L.pg_kick_drift_kick(C.byref(p), C.byref(a), C.byref(fa), 0.5 * dt, 1)
        O.orc_kick_drift_kick(C.byref(p), C.byref(b), C.byref(fb), 0.5 * dt, 1)
        L.pg_kick_drift_kick(C.byref(p), C.byref(a), C.byref(fa), dt, 0)
        O.orc_kick_drift_kick(C.byref(p), C.byref(b), C.byref(fb), dt, 0)
        assert _state(a, fa) == _state(b, fb), step
        t = step * dt
        assert L.pg_set_M_p(C.byref(p), t) == O.orc_set_M_p(C.byref(p), t)
    assert L.pg_get_E(C.byref(a), fa.value) == O.orc_get_E(C.byref(b), fb.value)
    assert L.pg_get_ecc(C.byref(a), fa.value) == O.orc_get_ecc(C.byref(b), fb.value)

