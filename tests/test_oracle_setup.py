"""The CPU oracle's own set-up against the reference's host set-up.

The oracle builds its fixed ghost rings and its damping targets itself from
the disk profile (init.cpp:92-183, 253-539), in host arithmetic: the
reference's host compiler folds pow with the constant exponents 0, 1, -1 and 2,
and the oracle restates that folding.  Both must equal what the reference's
own init_den, init_speed and init_bound produced (tests/golden/ic_ref.npz,
made by tests/golden/make_ic_golden.py) bit for bit, with the one exception
the library shares: the inner radial rings of a 3D spherical grid, whose
Sigma, p, v_phi and rot_v the reference leaves unformed (init.cpp:289-294)."""
import os

import numpy as np
import pytest

import penguin_2_0_b200 as pg
from oracle.pyoracle import Oracle
from penguin_2_0_b200.host import BOUNDARY_FIELDS
from tests._golden import HERE  # puts tests/golden on sys.path
from make_ic_golden import IC_CASES, ic_params  # noqa: E402

G = np.load(os.path.join(HERE, "golden", "ic_ref.npz"))
COL = {name: c for c, name in enumerate(BOUNDARY_FIELDS)}


def _oracle(case):
    p = ic_params(case)
    p.noise_amp = 0.0
    return p, Oracle(p, pg.build_ic(p))


def _by_position(rows):
    # ring order differs between the two; (zc, xc) names each ghost ring
    return rows[np.lexsort((rows[:, COL["xc"]], rows[:, COL["zc"]]))]


@pytest.mark.parametrize("case", list(IC_CASES))
def test_oracle_damping_targets_match_reference_setup(case):
    p, o = _oracle(case)
    try:
        t = o.targets()
    finally:
        o.close()
    ref = G[f"{case}_fields"]                       # Sigma, p, v_r, v_phi per ring
    for c, name in enumerate(("Sigma", "p", "v_r", "v_phi")):
        np.testing.assert_array_equal(t[:, c], ref[:, c], err_msg=name)
    assert np.all(t[:, 4] == 0.0)


@pytest.mark.parametrize("case", list(IC_CASES))
def test_oracle_ghost_rings_match_reference_setup(case):
    p, o = _oracle(case)
    try:
        ours = o.boundary()
    finally:
        o.close()
    ref = G[f"{case}_boundary"]
    assert ours.shape == ref.shape
    n6k, n6i = 6 * p.kmax, 6 * p.imax
    cuts = [0, n6k, 2 * n6k] + ([2 * n6k + n6i, 2 * n6k + 2 * n6i] if p.ndim == 3 else [])
    for g, name in enumerate(("lft", "rgh", "udr", "top")[:len(cuts) - 1]):
        got = _by_position(ours[cuts[g]:cuts[g + 1]])
        want = _by_position(ref[cuts[g]:cuts[g + 1]])
        cols = list(BOUNDARY_FIELDS)
        if name == "lft" and p.ndim == 3:
            cols = [c for c in cols if c not in ("r", "p", "v", "rot_v")]
        for c in cols:
            np.testing.assert_array_equal(got[:, COL[c]], want[:, COL[c]], err_msg=f"{name}.{c}")
