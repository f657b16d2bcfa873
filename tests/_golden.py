"""Golden vectors of the reference's own CUDA build (tests/golden/*.npz,
made by tests/golden/make_golden.py on a B200) and the comparison rule."""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))
from make_golden import CASES, CASES3D, params_for  # noqa: E402

TOL = 1e-12


def load(case):
    return np.load(os.path.join(HERE, "golden", f"{case}.npz"))


def field_errors(f, g, s):
    """Relative L-inf of Sigma (to max|Sigma|) and of v_r, v_phi (to the max
    speed, so a near-zero v_r does not turn rounding into a large ratio)."""
    stride = int(g["stride"])
    ours = np.stack([f["r"], f["u"], f["v"]], axis=1)
    ref = g[f"fields_{s}"]
    if stride > 1:
        ours = ours.transpose(1, 0, 2).reshape(3, -1)[:, ::stride]
        a, b = ours, ref
    else:
        a = ours.transpose(1, 0, 2).reshape(3, -1)
        b = ref.transpose(1, 0, 2).reshape(3, -1)
    speed = max(np.max(np.abs(b[1])), np.max(np.abs(b[2])))
    e_r = np.max(np.abs(a[0] - b[0])) / np.max(np.abs(b[0]))
    e_u = np.max(np.abs(a[1] - b[1])) / speed
    e_v = np.max(np.abs(a[2] - b[2])) / speed
    return e_r, e_u, e_v


def field_errors3d(f, g, s):
    """field_errors for the 3D fixtures: Sigma, v_r, v_phi, v_theta of every
    stride-th cell; velocities relative to the largest speed of the three."""
    stride = int(g["stride"])
    ours = np.stack([f["r"], f["u"], f["v"], f["w"]], axis=0).reshape(4, -1)[:, ::stride]
    ref = g[f"fields_{s}"]
    speed = max(np.max(np.abs(ref[k])) for k in (1, 2, 3))
    e_r = np.max(np.abs(ours[0] - ref[0])) / np.max(np.abs(ref[0]))
    return (e_r,) + tuple(float(np.max(np.abs(ours[k] - ref[k])) / speed) for k in (1, 2, 3))


def check_planet(step, planet, FrRot, h):
    """The planet after a step against the reference build's history row
    (simtime dt mass torque FrRot y x vx vy m): relative 1e-12 of the
    orbit's scale (x for positions, the Keplerian speed x^-1/2 for
    velocities), so a moving planet's orbit is pinned with its forces."""
    vk = h[6] ** -0.5
    assert abs(FrRot - h[4]) <= TOL * max(abs(h[4]), vk), (step, FrRot, h[4])
    assert abs(planet.y - h[5]) <= TOL * max(abs(h[5]), 1.0), (step, planet.y, h[5])
    assert abs(planet.x - h[6]) <= TOL * h[6], (step, planet.x, h[6])
    assert abs(planet.vx - h[7]) <= TOL * vk, (step, planet.vx, h[7])
    assert abs(planet.vy - h[8]) <= TOL * vk, (step, planet.vy, h[8])
    assert planet.m == h[9], (step, planet.m, h[9])
