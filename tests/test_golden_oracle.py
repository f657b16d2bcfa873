"""The CPU oracle against the reference's own CUDA build (golden vectors):
per step dt, disk mass and torque, and the state at the saved steps.
Bounds: relative 1e-12 on dt, mass, Sigma and the velocities (to the max
speed); torque within 1e-12 of its absolute-term scale."""
import numpy as np
import pytest

import penguin_2_0_b200 as pg
from tests._golden import CASES, CASES3D, TOL, check_planet, field_errors, field_errors3d, load, params_for
from tests._lockstep import OracleLoop, torque_abs_scale


@pytest.mark.parametrize("case", list(CASES))
def test_oracle_matches_reference_build(case):
    _, _, nsteps, keep = CASES[case]
    p = params_for(case)
    g = load(case)
    o = OracleLoop(p, pg.build_ic(p))
    for s in range(1, max(keep) + 1):
        dt, mass, tq = o.step()
        h = g["hist"][s - 1]                       # simtime dt mass torque FrRot planet.y
        assert abs(dt - h[1]) <= TOL * h[1], (s, dt, h[1])
        assert abs(mass - h[2]) <= TOL * h[2], (s, mass, h[2])
        assert abs(o.simtime - h[0]) <= TOL * h[0]
        if h.size > 6:
            check_planet(s, o.planet, o.FrRot, h)
        f = o.fields()
        if p.plnt_flag:
            pl = pg.Planet(*[getattr(o.planet, k) for k in ("m", "x", "y", "vx", "vy", "fx", "fy", "rs")])
            assert abs(tq - h[3]) <= TOL * torque_abs_scale(f, p, pl), (s, tq, h[3])
        if s in keep:
            np.testing.assert_array_equal(f["rot_j"], g[f"rot_j_{s}"])
            e = field_errors(f, g, s)
            assert max(e) <= TOL, (case, s, e)


@pytest.mark.parametrize("case", list(CASES3D))
def test_oracle_matches_reference_build_3d(case):
    """The 3D disks on which the reference build ran bundle_sweep2D (radial
    and azimuthal sweeps of every polar layer, rotate_rings): the oracle's
    orc_sweep2d on the same 3D run, per step dt and mass, and Sigma, v_r,
    v_phi, v_theta at the saved steps."""
    _, _, nsteps, keep = CASES3D[case]
    p = params_for(case)
    g = load(case)
    o = OracleLoop(p, pg.build_ic(p), sweep2d=True)
    for s in range(1, max(keep) + 1):
        dt, mass, _ = o.step()
        h = g["hist"][s - 1]
        assert abs(dt - h[1]) <= TOL * h[1], (s, dt, h[1])
        assert abs(mass - h[2]) <= TOL * h[2], (s, mass, h[2])
        assert abs(o.simtime - h[0]) <= TOL * h[0]
        if s in keep:
            f = o.fields()
            np.testing.assert_array_equal(f["rot_j"], g[f"rot_j_{s}"])
            e = field_errors3d(f, g, s)
            assert max(e) <= TOL, (case, s, e)
