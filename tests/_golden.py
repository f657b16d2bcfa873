"""Golden vectors of the reference's own CUDA build (tests/golden/*.npz,
made by tests/golden/make_golden.py on a B200) and the comparison rule."""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))
from make_golden import CASES, params_for  # noqa: E402

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
