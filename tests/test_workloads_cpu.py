"""The seeded workloads of the batched ensemble and the serving stream, on the
CPU: every drawn disk is a valid run (pg_check_params), its parameters stay in
the ranges the workloads specify, the FP32 policy follows the thermal mass,
and the draws are reproducible from the seed."""
import math

import numpy as np

import penguin_2_0_b200 as pg
from penguin_2_0_b200 import ensemble, serving


def _common_ranges(p):
    assert 1e-5 * (1 - 1e-12) <= p.M_p <= 3e-3 * (1 + 1e-12)
    assert 0.03 <= p.sc_h <= 0.08
    assert 1e-4 * (1 - 1e-12) <= p.ss_alpha <= 1e-2 * (1 + 1e-12)
    assert 0.5 <= p.p_alpha <= 1.5
    assert p.jmax == 3 * p.imax


def test_ensemble_disks_are_valid_and_in_range():
    disks = ensemble.draw_ensemble(64, seed=0, orbits=10)
    assert len(disks) == 64
    for p in disks:
        assert pg.host.check_params(p) == 0
        assert p.imax in ensemble.SIZES and p.kmax == 1
        _common_ranges(p)
        assert abs(p.endtime - 10 * 2 * math.pi) < 1e-12
        assert p.precision == (1 if ensemble.thermal_mass(p) <= ensemble.THERMAL_MASS_FP32 else 0)
    assert len({p.seed for p in disks}) == 64
    again = ensemble.draw_ensemble(64, seed=0, orbits=10)
    assert [(p.imax, p.M_p, p.sc_h, p.seed) for p in disks] == [(p.imax, p.M_p, p.sc_h, p.seed) for p in again]


def test_serving_requests_are_valid_and_in_range():
    reqs = serving.draw_stream(2000, seed=0)
    n3 = 0
    for p in reqs:
        assert pg.host.check_params(p) == 0
        _common_ranges(p)
        orbits = p.endtime / (2 * math.pi)
        assert 5.0 - 1e-9 <= orbits <= 50.0 + 1e-9
        if p.ndim == 3:
            n3 += 1
            assert p.imax in serving.SIZES_3D and p.kmax in serving.NTHETA_3D
            assert abs(p.zmin - (math.pi / 2 - 3 * p.sc_h)) < 1e-15
        else:
            assert p.imax in ensemble.SIZES and p.kmax == 1
    # 10 % 3D: 200 expected, binomial sd ~13
    assert 150 <= n3 <= 250, n3
    t = serving.poisson_arrivals(2000, rate_per_s=5.0, seed=0)
    assert t[0] == 0.0 and np.all(np.diff(t) >= 0.0)
