"""ctypes binding of the CPU oracle (TEST INFRASTRUCTURE ONLY).

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg use this
module; the product path never imports it, and it imports nothing of the
product (its struct images are in oracle/abi.py).  The oracle is built in-tree
by build() into oracle/liboracle.so (gcc + OpenMP).
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
SO = os.path.join(HERE, "liboracle.so")


def build(force: bool = False) -> str:
    src = os.path.join(HERE, "pg_oracle.c")
    hdrs = [os.path.join(HERE, "pg_oracle.h"), os.path.join(ROOT, "include", "penguin_b200.h")]
    if (not force and os.path.exists(SO)
            and all(os.path.getmtime(f) <= os.path.getmtime(SO) for f in [src] + hdrs)):
        return SO
    subprocess.check_call(["gcc", "-O2", "-fPIC", "-shared", "-fopenmp", "-std=gnu11", "-o", SO, src, "-lm"])
    return SO


_L = None


def lib():
    global _L
    if _L is None:
        if not os.path.exists(SO):
            build()
        L = C.CDLL(SO)
        vp, dp = C.c_void_p, C.POINTER(C.c_double)
        # params and bodies go in by reference as plain pointers: the caller's
        # struct may be oracle.abi's or the product binding's (same layout)
        P, B = vp, vp
        sig = {
            "orc_create": (vp, [P, vp, C.c_size_t]),
            "orc_destroy": (None, [vp]),
            "orc_save": (C.c_int, [vp, vp, C.c_size_t]),
            "orc_get_dt": (C.c_double, [vp, C.c_double, C.c_double]),
            "orc_index_shift": (None, [vp, C.c_double, C.c_double]),
            "orc_sweepx": (None, [vp, C.c_double, B, C.c_double]),
            "orc_sweepy": (None, [vp, C.c_double, B, C.c_double]),
            "orc_sweepz": (None, [vp, C.c_double, B, C.c_double]),
            "orc_rotate": (None, [vp]),
            "orc_sweep2d": (None, [vp, C.c_double, B, C.c_double]),
            "orc_sweep3d": (None, [vp, C.c_double, B, C.c_double]),
            "orc_damp": (None, [vp, C.c_double]),
            "orc_reduce": (C.c_double, [vp, B, C.c_double, C.c_int]),
            "orc_init_planet": (None, [P, B, dp]),
            "orc_planet_forces": (None, [vp, B, C.c_double, C.c_double]),
            "orc_kick_drift_kick": (None, [P, B, dp, C.c_double, C.c_int]),
            "orc_run_steps": (C.c_int, [vp, C.c_int, C.c_int, dp]),
            "orc_threads": (C.c_int, []),
            "orc_boundary": (C.c_int, [vp, dp, C.c_size_t, C.POINTER(C.c_int)]),
            "orc_set_M_p": (C.c_double, [P, C.c_double]),
            "orc_get_E": (C.c_double, [B, C.c_double]),
            "orc_get_ecc": (C.c_double, [B, C.c_double]),
            "orc_targets": (C.c_int, [vp, dp, C.c_size_t]),
        }
        for k, (r, a) in sig.items():
            f = getattr(L, k)
            f.restype = r
            f.argtypes = a
        _L = L
    return _L


class Oracle:
    """CPU restatement of one run, loaded from a reference-layout dump."""

    def __init__(self, p, rings: bytes):
        self.p = p
        n = len(rings)
        buf = (C.c_char * n).from_buffer_copy(bytes(rings))
        self._h = lib().orc_create(C.byref(p), buf, n)
        if not self._h:
            raise RuntimeError("orc_create failed (size mismatch?)")

    def close(self):
        if self._h:
            lib().orc_destroy(self._h)
            self._h = None

    def __del__(self):
        self.close()

    def save(self) -> bytearray:
        n = 72 * self.p.jmax + 96
        n *= self.p.imax * self.p.kmax
        buf = bytearray(n)
        cbuf = (C.c_char * n).from_buffer(buf)
        assert lib().orc_save(self._h, cbuf, n) == 0
        return buf

    def run_steps(self, nsteps: int, startat: int = 0) -> np.ndarray:
        """main.cu restart loop; rows: simtime, dt, mass, torque (normalised)."""
        h = (C.c_double * (4 * nsteps))()
        n = lib().orc_run_steps(self._h, nsteps, startat, h)
        return np.frombuffer(h, dtype=np.float64)[: 4 * n].reshape(n, 4).copy()

    def boundary(self) -> np.ndarray:
        """The fixed ghost rings, one row of 14 columns (x dx xvol xc z dz
        zvol zc r p u v w rot_v) per ring: lft, rgh, then udr, top in 3D."""
        cnt = C.c_int(0)
        lib().orc_boundary(self._h, None, 0, C.byref(cnt))
        out = np.zeros((cnt.value, 14))
        assert lib().orc_boundary(self._h, out.ctypes.data_as(C.POINTER(C.c_double)), out.size, C.byref(cnt)) == 0
        return out

    def targets(self) -> np.ndarray:
        """The damping targets, r p u v w per ring i + imax k."""
        out = np.zeros((self.p.imax * self.p.kmax, 5))
        assert lib().orc_targets(self._h, out.ctypes.data_as(C.POINTER(C.c_double)), out.size) == 0
        return out

    def get_dt(self, dt, frrot):
        return lib().orc_get_dt(self._h, dt, frrot)

    def index_shift(self, dt, frrot):
        lib().orc_index_shift(self._h, dt, frrot)

    def sweep(self, dt, planet_c, frrot):
        if self.p.ndim == 2:
            lib().orc_sweep2d(self._h, dt, C.byref(planet_c), frrot)
        else:
            lib().orc_sweep3d(self._h, dt, C.byref(planet_c), frrot)

    def damp(self, dt):
        lib().orc_damp(self._h, dt)

    def reduce(self, planet_c, exclude, mode):
        return lib().orc_reduce(self._h, C.byref(planet_c), exclude, mode)

    @staticmethod
    def threads() -> int:
        return lib().orc_threads()
