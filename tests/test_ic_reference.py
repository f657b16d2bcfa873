"""The initial state and the fixed boundary rings against the reference's own
set-up (init.cpp:3-543), in 2D and 3D, isothermal and isentropic.

tests/golden/ic_ref.npz holds what the reference's init_grid, init_den,
init_speed, init_cells and init_bound produced on the host for four disks
(tests/golden/make_ic_golden.py, oracle/ref/ic_harness.cu).  The library's
initial dump (pg_build_ic without noise) and its boundary rings
(pg_boundary_rings, the values a run loads into its ghost rows and polar
ghost layers) agree with them bit for bit, down to each ring record's i, k,
res_v, rot_j and inc_j, with three exceptions:

* v_r: the seeded initial state of this library starts at rest radially
  (v_r = 0); the reference's fresh start sets the viscous inflow speed
  -1.5 nu / r.  The boundary rings carry the inflow speed in both.
* the inner radial boundary rings of a 3D spherical grid: the reference's
  branch for them (init.cpp:289-294) never forms the density and pressure it
  then uses, so its Sigma, p, v_phi and rot_v there are left over from
  whatever the variables held; here they take the disk profile's values.
  Their geometry and v_r still agree.
* rot_v: the reference's fresh start leaves it 0 until its first Index_Shift
  (main.cu:330); the initial dump here is a restart file, which carries that
  Index_Shift's value because a restart skips the call.

The 3D interior state is the part of the 3D set-up that no reference run
checks otherwise (the reference has no 3D sweep)."""
import os

import numpy as np
import pytest

import penguin_2_0_b200 as pg
from penguin_2_0_b200.host import BOUNDARY_FIELDS, boundary_rings
from tests._golden import HERE  # puts tests/golden on sys.path
from make_ic_golden import IC_CASES, ic_params  # noqa: E402

G = np.load(os.path.join(HERE, "golden", "ic_ref.npz"))
COL = {name: c for c, name in enumerate(BOUNDARY_FIELDS)}


def _ys(buf, p):
    rb = 72 * p.jmax + 96
    raw = np.frombuffer(bytes(buf), dtype=np.uint8)[:rb]
    return raw[40 * p.jmax + 32:72 * p.jmax + 32].copy().view(np.float64).reshape(4, p.jmax)


@pytest.mark.parametrize("case", list(IC_CASES))
def test_initial_state_matches_reference_setup(case):
    p = ic_params(case)
    p.noise_amp = 0.0
    buf = pg.build_ic(p)
    f = pg.dump_fields(buf, p)
    assert bool(G[f"{case}_phi_uniform"])
    ref = G[f"{case}_fields"]                       # Sigma, p, v_r, v_phi per ring
    np.testing.assert_array_equal(f["r"][:, 0], ref[:, 0])
    np.testing.assert_array_equal(f["p"][:, 0], ref[:, 1])
    np.testing.assert_array_equal(f["v"][:, 0], ref[:, 3])
    assert np.all(f["u"] == 0.0)                    # starts at rest radially (see above)
    if p.visc_flag == 1:
        assert np.all(ref[:, 2] < 0.0)              # the reference's viscous inflow
    xs, zs = G[f"{case}_xs"], G[f"{case}_zs"]
    for k, name in enumerate(("x", "dx", "xvol", "xc")):
        np.testing.assert_array_equal(f[name], xs[:, k], err_msg=name)
    for k, name in enumerate(("z", "dz", "zvol", "zc")):
        np.testing.assert_array_equal(f[name], zs[:, k], err_msg=name)
    np.testing.assert_array_equal(_ys(buf, p), G[f"{case}_ys"])


@pytest.mark.parametrize("case", list(IC_CASES))
def test_boundary_rings_match_reference_setup(case):
    p = ic_params(case)
    ours = boundary_rings(p)
    ref = G[f"{case}_boundary"]
    n6k, n6i = 6 * p.kmax, 6 * p.imax
    groups = {"lft": ref[:n6k], "rgh": ref[n6k:2 * n6k]}
    if p.ndim == 3:
        groups["udr"] = ref[2 * n6k:2 * n6k + n6i]
        groups["top"] = ref[2 * n6k + n6i:2 * n6k + 2 * n6i]
    assert sum(g.shape[0] for g in groups.values()) == ref.shape[0]
    for name, want in groups.items():
        got = ours[name]
        assert got.shape == want.shape, (name, got.shape, want.shape)
        cols = list(BOUNDARY_FIELDS)
        if name == "lft" and p.ndim == 3:
            cols = [c for c in cols if c not in ("r", "p", "v", "rot_v")]
        for c in cols:
            np.testing.assert_array_equal(got[:, COL[c]], want[:, COL[c]], err_msg=f"{name}.{c}")


@pytest.mark.parametrize("case", list(IC_CASES))
def test_ring_record_tails_match_reference_setup(case):
    """The per-ring integers and FARGO scalars of the dump (variable_types.h:
    i, k, rot_v, res_v, rot_j, inc_j).  All agree bit for bit except rot_v:
    the reference's fresh start leaves it 0 for its first Index_Shift
    (main.cu:330) to fill, while this library's initial dump is the restart
    file, whose rot_v is that Index_Shift's value val.v - FrRot xc
    (orbital_advection.cu:22), because a restart skips it."""
    p = ic_params(case)
    p.noise_amp = 0.0
    buf = pg.build_ic(p)
    rb = 72 * p.jmax + 96
    ours = np.frombuffer(bytes(buf), dtype=np.uint8).reshape(-1, rb)[:, 72 * p.jmax + 64:]
    ref = G[f"{case}_tail"]
    assert ours.shape == ref.shape

    def split(t):
        t = np.ascontiguousarray(t)
        return (t[:, 0:8].copy().view(np.int32), t[:, 8:16].copy().view(np.float64)[:, 0],
                t[:, 16:24].copy().view(np.float64)[:, 0], t[:, 24:32].copy().view(np.int32))

    ik, rot_v, res_v, jj = split(ours)
    rik, rrot_v, rres_v, rjj = split(ref)
    np.testing.assert_array_equal(ik, rik)            # i, k
    np.testing.assert_array_equal(res_v, rres_v)
    np.testing.assert_array_equal(jj, rjj)            # rot_j, inc_j
    assert np.all(rrot_v == 0.0)
    f = pg.dump_fields(buf, p)
    _, frrot = pg.init_planet(p)
    np.testing.assert_array_equal(rot_v, f["v"][:, 0] - frrot * f["xc"])
