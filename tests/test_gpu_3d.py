"""3D (r-phi-theta, spherical, reflecting midplane) CUDA path against the CPU
oracle.  The reference has no 3D driver (bundle_sweep3D is called at
main.cu:376 and never defined), so 3D parity is against the restatement
only.  Same tolerances as 2D: relative L-inf 1e-12 per step on Sigma and on
the velocities (to the max speed), relative 1e-12 on dt and mass."""
import numpy as np
import pytest

import penguin_2_0_b200 as pg
from tests._lockstep import OracleLoop, rel_linf

TOL = 1e-12


def _p(**over):
    p = pg.params(1, imax=64, jmax=132, kmax=16, nprin=1)
    p.update(**over)
    return p


@pytest.mark.gpu
@pytest.mark.parametrize("over", [dict(), dict(ntop=3), dict(plnt_flag=0, visc_flag=0),
                                  dict(EOS=1, gam=5.0 / 3.0), dict(EOS=1, gam=5.0 / 3.0, ntop=3),
                                  dict(plnt_flag=2),          # moving planet (no disk force in 3D)
                                  dict(FARGO_flag=0)])
def test_3d_host_loop_matches_oracle(gpu, over):
    p = _p(**over)
    ic = pg.build_ic(p)
    ref = OracleLoop(p, ic)
    got = {}

    def rec(s, simtime, dt_used, planet, FrRot):
        got[s] = (dt_used, pg.GPU_output_reduction(run, planet, 0.0, 0), pg.dump_fields(run.save(), p))

    with pg.Run(p, 0) as run:
        run.load(ic)
        run.kernel_loop(3, record=rec)
    for s in range(3):
        dt, mass, _ = ref.step()
        f = ref.fields()
        gdt, gmass, gf = got[s]
        np.testing.assert_array_equal(gf["rot_j"], f["rot_j"])
        speed = max(np.max(np.abs(f[k])) for k in ("u", "v", "w"))
        e = [rel_linf(gf["r"], f["r"])] + [np.max(np.abs(gf[k] - f[k])) / speed for k in ("u", "v", "w")]
        assert max(e) <= TOL, (over, s, e)
        assert abs(gdt - dt) <= TOL * dt
        assert abs(gmass - mass) <= TOL * mass


@pytest.mark.gpu
@pytest.mark.parametrize("over", [dict(), dict(EOS=1, gam=5.0 / 3.0)])
def test_3d_fused_loop_equals_host_loop(gpu, over):
    p = _p(**over)
    ic = pg.build_ic(p)
    with pg.Run(p, 0) as a, pg.Run(p, 0) as b:
        a.load(ic)
        b.load(ic)
        a.kernel_loop(4)
        b.clock_reset(0)
        assert b.advance(4, graph_chunk=2) == 4
        fa, fb = pg.dump_fields(a.save(), p), pg.dump_fields(b.save(), p)
        for k in ("r", "u", "v", "w", "rot_j"):
            np.testing.assert_array_equal(fa[k], fb[k], err_msg=k)
