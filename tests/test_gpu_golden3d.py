"""The 3D spherical path against the reference's own CUDA build.

The reference never wrote a polar sweep (bundle_sweep3D is called at
main.cu:376 and defined nowhere), but its sweepx and sweepy run every polar
layer of a 3D build: sweepx takes the layer from blockIdx.y (ppm.cu:32-33)
and sweepy folds it into the ring index (ppm.cu:168), with the spherical
forces (forces.cu:23-110) and the axis branches of states, evolve and remap
for ngeomx 2 / ngeomy 4.  The fixtures (tests/golden/make_golden.py,
CASES3D) hold what the reference build's bundle_sweep2D gives on 3D disks
from the seeded dump: per-step dt and mass, and Sigma, v_r, v_phi, v_theta at
the saved steps.  The library runs the same host-driven loop through the C
ABI with pg_sweep2d on the 3D run (the same two sweeps of every layer and
rotate_rings).  Bound: relative 1e-12 per step, as for the 2D cases."""
import numpy as np
import pytest

import penguin_2_0_b200 as pg
from tests._golden import CASES3D, TOL, field_errors3d, load, params_for


@pytest.mark.gpu
@pytest.mark.parametrize("case", list(CASES3D))
def test_3d_radial_azimuthal_sweeps_match_reference_build(gpu, case):
    _, _, nsteps, keep = CASES3D[case]
    p = params_for(case)
    assert p.ndim == 3
    g = load(case)
    seen = {}

    def rec(s, simtime, dt_used, planet, FrRot):
        step = s + 1
        h = g["hist"][s]
        assert abs(dt_used - h[1]) <= TOL * h[1], (step, dt_used, h[1])
        assert abs(simtime - h[0]) <= TOL * h[0]
        mass = pg.GPU_output_reduction(run, planet, 0.0, 0)
        assert abs(mass - h[2]) <= TOL * h[2], (step, mass, h[2])
        if step in keep:
            f = pg.dump_fields(run.save(), p)
            np.testing.assert_array_equal(f["rot_j"], g[f"rot_j_{step}"])
            e = field_errors3d(f, g, step)
            seen[step] = e
            assert max(e) <= TOL, (case, step, e)

    with pg.Run(p, 0) as run:
        run.load(pg.build_ic(p))
        run.kernel_loop(max(keep), record=rec, sweep2d=True)
    assert sorted(seen) == sorted(keep)
