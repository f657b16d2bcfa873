"""The reference's own hydro step compiled for the host CPU against its CUDA
build (golden vectors), on the CPU.

oracle/refhost builds the reference's unmodified .cu sources with g++: each
CUDA thread is a fiber, __syncthreads() a yield to the block's next fiber,
__shared__ data per OS thread, and only the launch syntax is rewritten.  The
same driver as the CUDA golden runs (oracle/ref/ref_harness.cu) steps it from
the same seeded dump.  Its per-step dt and mass and its state at the saved
steps must match the CUDA build's at the golden tolerance: that makes it the
reference's own code on the host, which bench.py times as the CPU baseline.
Host libm and the absence of FMA contraction differ from the device in the
last bits only."""
import ctypes as C
import os
import subprocess

import numpy as np
import pytest

from tests._golden import CASES, CASES3D, TOL, check_planet, load, params_for
from make_golden import read_rings, write_ghost_override  # noqa: E402  (tests/golden is on sys.path)

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _exe(case):
    return os.path.join(ROOT, "oracle", "_ref", case, "penguin_ref_host")


def _hist(path):
    rows = [ln.split() for ln in open(path)]
    return np.array([[float.fromhex(x) for x in r[1:]] for r in rows])


# the host build is slower than the CUDA one: a few cases keep the CPU suite short
PICK = ["g136x136", "g136x200_eos1", "g136x136_moving", "g3d136x136x8"]


@pytest.mark.parametrize("case", PICK)
def test_host_built_reference_matches_cuda_build(case, tmp_path):
    exe = _exe(case)
    if not os.path.exists(exe):
        pytest.skip("host build of the reference not present (needs the reference tree at build time)")
    from penguin_2_0_b200 import _lib
    table = CASES if case in CASES else CASES3D
    _, _, nsteps, keep = table[case]
    p = params_for(case)
    g = load(case)
    ic = str(tmp_path / "ic.bin")
    assert _lib.lib().pg_write_ic(C.byref(p), ic.encode()) == 0
    write_ghost_override(p, ic)
    r = subprocess.run([exe, ic, str(max(keep)), str(tmp_path), ",".join(map(str, keep))],
                       capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-400:]
    h = _hist(tmp_path / "hist.txt")
    gh = g["hist"]
    n = max(keep)
    assert h.shape[0] == n
    np.testing.assert_allclose(h[:, 0], gh[:n, 0], rtol=TOL, atol=0)     # simtime
    np.testing.assert_allclose(h[:, 1], gh[:n, 1], rtol=TOL, atol=0)     # dt
    np.testing.assert_allclose(h[:, 2], gh[:n, 2], rtol=TOL, atol=0)     # mass
    if gh.shape[1] > 6:
        for s in range(n):
            pl = type("P", (), dict(zip(("y", "x", "vx", "vy", "m"), h[s, 5:10])))
            check_planet(s + 1, pl, h[s, 4], gh[s])
    nf = 4 if p.ndim == 3 else 3
    for s in keep:
        f, rot = read_rings(str(tmp_path / f"state_{s:05d}.bin"), p)
        np.testing.assert_array_equal(rot, g[f"rot_j_{s}"])
        cols = [0, 2, 3, 4][:nf]
        ours = f[:, cols, :].transpose(1, 0, 2).reshape(nf, -1)
        ref = g[f"fields_{s}"]
        stride = int(g["stride"])
        if ref.ndim == 3:
            ref = ref.transpose(1, 0, 2).reshape(nf, -1)
        elif stride > 1:
            ours = ours[:, ::stride]
        speed = max(np.max(np.abs(ref[k])) for k in range(1, nf))
        e = [np.max(np.abs(ours[0] - ref[0])) / np.max(np.abs(ref[0]))]
        e += [np.max(np.abs(ours[k] - ref[k])) / speed for k in range(1, nf)]
        assert max(e) <= TOL, (case, s, e)


@pytest.mark.parametrize("case", ["g136x136", "g136x136_moving", "g136x200_eos1", "g3d136x136x8"])
def test_host_built_reference_equals_oracle(case, tmp_path):
    """The C restatement (oracle/pg_oracle.c) against the reference's own
    sources built for the host: both are host code with the reference's
    operation order and no FMA contraction, on the same libm, so they agree to
    a few ulp (bitwise in most steps).  3D runs the reference's
    bundle_sweep2D step (radial and azimuthal sweeps of every layer)."""
    exe = _exe(case)
    if not os.path.exists(exe):
        pytest.skip("host build of the reference not present (needs the reference tree at build time)")
    import penguin_2_0_b200 as pg
    from penguin_2_0_b200 import _lib
    from tests._lockstep import OracleLoop
    table = CASES if case in CASES else CASES3D
    _, _, nsteps, keep = table[case]
    p = params_for(case)
    ic = str(tmp_path / "ic.bin")
    assert _lib.lib().pg_write_ic(C.byref(p), ic.encode()) == 0
    write_ghost_override(p, ic)
    n = max(keep)
    r = subprocess.run([exe, ic, str(n), str(tmp_path), ",".join(str(s) for s in range(1, n + 1))],
                       capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-400:]
    h = _hist(tmp_path / "hist.txt")
    o = OracleLoop(p, pg.build_ic(p), sweep2d=(p.ndim == 3))
    for s in range(1, n + 1):
        dt, mass, _ = o.step()
        assert abs(dt - h[s - 1, 1]) <= 1e-14 * dt, (s, dt, h[s - 1, 1])
        assert abs(mass - h[s - 1, 2]) <= 1e-14 * mass, (s, mass, h[s - 1, 2])
        f, rot = read_rings(str(tmp_path / f"state_{s:05d}.bin"), p)
        fo = o.fields()
        np.testing.assert_array_equal(rot, fo["rot_j"])
        speed = max(np.max(np.abs(fo[k])) for k in ("u", "v", "w"))
        assert np.max(np.abs(f[:, 0] - fo["r"])) <= 1e-14 * np.max(np.abs(fo["r"])), s
        for c, k in ((2, "u"), (3, "v"), (4, "w")):
            assert np.max(np.abs(f[:, c] - fo[k])) <= 1e-14 * speed, (s, k)
