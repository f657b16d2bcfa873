"""Ten orbits of the 252x780 disk against the reference's own CUDA build.

The reference's CUDA step, built from its own sources for this disk (planet
q = 1e-3 on a fixed orbit, viscosity, flattening, FARGO, damping zones), ran
from the seeded dump to the end time of 10 orbits; the fixture holds the
history of every step and the whole final state (tests/golden/make_golden.py
run_long / pack_long).  The reference also ran a second time from the same
dump with Sigma of one cell next to the planet moved by one ulp: the fixture
keeps how far that run ends from the first (its own sensitivity to a
rounding-sized change of the input).

The fused device loop runs the same dump to the same end time.  Bounds:

* step count, end time and the FARGO shifts rot_j: equal;
* disk-mass history: relative L1 <= 1e-8;
* torque history over the first 4 orbits: every step within 1e-8 of the
  largest torque;
* final Sigma, v_phi and v_r (to the L1 of v_phi, since v_r is ~1e-3 of
  v_phi and changes sign): relative L1 <= 1e-8;
* the whole torque history: relative L1 <= 1e-8, or 4x the reference's own
  1-ulp divergence where that is larger.

The last bound applies to the gap-opening disk only; a disk of q = 3e-5
(q/h^3 = 0.24, no gap) holds the flat 1e-8 on everything, the torque history
included.  The relaxed bound exists because the q = 1e-3 disk amplifies rounding: a planet of
q/h^3 = 8 opens a gap whose edges grow perturbations by about e per 160
steps after the fourth orbit, so the reference itself moves by ~1e-8 in
Sigma and ~2.5e-7 in the torque history when one input cell changes by one
ulp.  The fused loop ends at ~4e-9 in Sigma and ~7e-8 in the torque history;
no build whose arithmetic differs from the reference's at the last bit (the C
oracle, which keeps the reference's operation order, included) can meet a
flat 1e-8 on the torque history there."""
import os

import numpy as np
import pytest

import penguin_2_0_b200 as pg
from tests._golden import HERE  # puts tests/golden on sys.path
from make_golden import LONG_CASES, long_errors, params_for  # noqa: E402

CASE = "g252x780_10orbits"
CASE_NOGAP = "g252x780_10orbits_q3e-5"
L1_TOL = 1e-8
SENS = 4.0


def _l1(a, b):
    return float(np.sum(np.abs(a - b)) / np.sum(np.abs(b)))


def _run_to_end(case):
    """The fused loop from the seeded dump to the fixture's end time; returns
    the fixture, the final fields and the per-step history."""
    assert case in LONG_CASES
    p = params_for(case)
    g = np.load(os.path.join(HERE, "golden", f"{case}.npz"))
    href = g["hist"]                      # simtime dt mass torque FrRot planet.y ... per step
    nref = href.shape[0]
    with pg.Run(p, 0) as run:
        run.load(pg.build_ic(p))
        run.clock_reset(0)
        n = run.advance(nref + 10, graph_chunk=64)     # the loop halts at the end time
        c, _ = run.clock()
        f = pg.dump_fields(run.save(), p)
        hist = run.history(max_rows=nref + 10)         # simtime mass torque ... per step
    assert n == nref and hist.shape[0] == nref, (n, hist.shape, nref)
    assert abs(c.simtime - href[-1, 0]) <= 1e-12 * href[-1, 0]
    np.testing.assert_array_equal(f["rot_j"], g["rot_j"])
    return g, f, hist, n


@pytest.mark.gpu
def test_ten_orbits_no_gap_flat_bound(gpu):
    """q = 3e-5 (q/h^3 = 0.24) opens no gap.  Every quantity, the whole torque
    history included, holds the flat relative L1 <= 1e-8."""
    g, f, hist, n = _run_to_end(CASE_NOGAP)
    href = g["hist"]
    e_mass = _l1(hist[:, 1], href[:, 2])
    e_tq = _l1(hist[:, 2], href[:, 3])
    e_fields = long_errors(f["r"], f["u"], f["v"], g["fields"])
    sens_tq = _l1(g["hist_pert"][:, 3], href[:, 3])
    print(f"\n10 orbits 252x780 q=3e-5, {n} steps: L1 Sigma/v_r/v_phi {e_fields[0]:.2e}/{e_fields[1]:.2e}/"
          f"{e_fields[2]:.2e}, torque {e_tq:.2e}, mass {e_mass:.2e}; reference vs itself after a 1-ulp change: "
          f"{g['pert_l1'][0]:.2e} (Sigma), torque {sens_tq:.2e}")
    assert e_mass <= L1_TOL, e_mass
    assert e_tq <= L1_TOL, e_tq
    for got, name in zip(e_fields, ("Sigma", "v_r", "v_phi")):
        assert got <= L1_TOL, (name, got)


@pytest.mark.gpu
def test_ten_orbits_match_reference_build(gpu):
    g, f, hist, n = _run_to_end(CASE)
    href = g["hist"]

    e_mass = _l1(hist[:, 1], href[:, 2])
    assert e_mass <= L1_TOL, e_mass
    early = href[:, 0] <= 4.0 * 2.0 * np.pi
    e_early = float(np.max(np.abs(hist[early, 2] - href[early, 3])) / np.max(np.abs(href[:, 3])))
    assert e_early <= L1_TOL, e_early

    e_fields = long_errors(f["r"], f["u"], f["v"], g["fields"])
    e_tq = _l1(hist[:, 2], href[:, 3])
    sens_fields = g["pert_l1"]
    sens_tq = _l1(g["hist_pert"][:, 3], href[:, 3])
    print(f"\n10 orbits 252x780, {n} steps: L1 Sigma/v_r/v_phi {e_fields[0]:.2e}/{e_fields[1]:.2e}/"
          f"{e_fields[2]:.2e}, torque {e_tq:.2e}, mass {e_mass:.2e}, torque to 4 orbits {e_early:.2e}; "
          f"reference vs itself after a 1-ulp change: {sens_fields[0]:.2e}/{sens_fields[1]:.2e}/"
          f"{sens_fields[2]:.2e}, torque {sens_tq:.2e}")
    for got, name in zip(e_fields, ("Sigma", "v_r", "v_phi")):
        assert got <= L1_TOL, (name, got)
    assert e_tq <= max(L1_TOL, SENS * sens_tq), (e_tq, sens_tq)
