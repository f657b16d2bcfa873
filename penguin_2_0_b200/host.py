"""Host-side mirror of the reference's hydro-step interface.

The reference exposes its hot path as C++ functions called from main.cu's
time loop.  This module gives the same names, argument meaning and order over
the C ABI of libpenguin_b200.so, so a caller (or a test) reads like the
reference's own driver:

    reference (file:line)                          here
    bundle_sweep2D(set, dt, planet, FrRot)         bundle_sweep2D(run, dt, planet, FrRot)
      include/ppm.h:4, src/ppm/ppm.cu:358
    get_dt(dt, set, FrRot)                         get_dt(dt, run, FrRot)
      include/timestep.h:4, timestep.cu:112
    Index_Shift(set, dt, FrRot)                    Index_Shift(run, dt, FrRot)
      include/orbital_advection.h:4, orbital_advection.cu:45
    GPU_output_reduction(set, planet, exclude, m)  GPU_output_reduction(run, planet, exclude, m)
      include/output.h:32, device_func.cu:169
    init_planet / planet_forces / kick_drift_kick  same names, planet.cu:36-93
    kernel() time loop main.cu:343-441             Run.kernel_loop(nsteps) (host-driven)
                                                   Run.advance(nsteps) (device-resident)

Errors: every call raises PenguinError carrying the C status and message
(the reference prints and exits, include/cuSafe.cu:8-47).
"""
from __future__ import annotations

import ctypes as C
import math
from dataclasses import dataclass

import numpy as np

from . import _lib
from ._lib import pg_body, pg_clock, pg_params

TWOPI = 6.283185307179586476925286766559
HIST_COLS = 11


class PenguinError(RuntimeError):
    def __init__(self, status: int, msg: str):
        super().__init__(f"{_lib.STATUS.get(status, status)}: {msg}")
        self.status = status


def _check(st: int, run=None, what: str = ""):
    if st != 0:
        msg = what
        if run is not None and getattr(run, "_h", None):
            m = _lib.lib().pg_last_error(run._h)
            msg = f"{what}: {m.decode() if m else ''}"
        raise PenguinError(st, msg)


def params(which: int | None = None, **over) -> pg_params:
    """pg_params of a named workload (0: 2D 256x768, 1: 3D 128x1024x32,
    2: 2D 1024x3072) or of the reference defaults (which=None)."""
    p = pg_params()
    L = _lib.lib()
    _check(L.pg_default_params(C.byref(p)) if which is None else L.pg_config_params(which, C.byref(p)),
           what="params")
    p.update(**over)
    return p


def check_params(p: pg_params) -> int:
    return _lib.lib().pg_check_params(C.byref(p))


def ring_bytes(jmax: int) -> int:
    return _lib.lib().pg_ring_bytes(jmax)


def build_ic(p: pg_params) -> bytearray:
    """Seeded initial condition in the reference dump layout."""
    n = ring_bytes(p.jmax) * p.imax * p.kmax
    buf = bytearray(n)
    cbuf = (C.c_char * n).from_buffer(buf)
    _check(_lib.lib().pg_build_ic(C.byref(p), cbuf, n), what="pg_build_ic")
    return buf


BOUNDARY_FIELDS = ("x", "dx", "xvol", "xc", "z", "dz", "zvol", "zc", "r", "p", "u", "v", "w", "rot_v")


def boundary_rings(p: pg_params) -> dict:
    """The fixed boundary rings of init_bound (init.cpp:253-543) on the grid of
    p (pg_boundary_rings): {"lft", "rgh", "udr", "top"} -> [rings, 14] arrays
    with the columns of BOUNDARY_FIELDS; udr and top are empty in 2D."""
    L = _lib.lib()
    cnt = C.c_int(0)
    _check(L.pg_boundary_rings(C.byref(p), None, 0, C.byref(cnt)), what="pg_boundary_rings")
    nf = len(BOUNDARY_FIELDS)
    out = np.zeros(cnt.value * nf)
    _check(L.pg_boundary_rings(C.byref(p), out.ctypes.data_as(C.POINTER(C.c_double)), out.size, C.byref(cnt)),
           what="pg_boundary_rings")
    out = out.reshape(cnt.value, nf)
    nrad = 6 * p.kmax
    npol = 6 * p.imax if p.ndim == 3 else 0
    return dict(lft=out[:nrad], rgh=out[nrad:2 * nrad], udr=out[2 * nrad:2 * nrad + npol],
                top=out[2 * nrad + npol:2 * nrad + 2 * npol])


def label(p: pg_params) -> str:
    b = C.create_string_buffer(256)
    _check(_lib.lib().pg_label(C.byref(p), b, 256), what="pg_label")
    return b.value.decode()


def dump_name(p: pg_params, directory: str, frame: int) -> str:
    """<directory>/binary_<label>_<NNNNN>, the dump name of main.cu:124."""
    b = C.create_string_buffer(4096)
    _check(_lib.lib().pg_dump_name(C.byref(p), directory.encode(), int(frame), b, 4096), what="pg_dump_name")
    return b.value.decode()


def write_para_file(p: pg_params, path: str, mainp: str) -> None:
    """read/para_<label>.dat as write_para_file (output.cu:90-109) writes it."""
    _check(_lib.lib().pg_write_para_file(C.byref(p), path.encode(), mainp.encode()), what="pg_write_para_file")


def write_time_rows(p: pg_params, path: str, rows, append: bool = False) -> None:
    """files/time_<label>.dat rows (main.cu:417-427) from rows of 11 values in
    the pg_history layout; two columns without a planet."""
    a = np.ascontiguousarray(np.asarray(rows, dtype=np.float64).reshape(-1, 11))
    _check(_lib.lib().pg_write_time_rows(C.byref(p), path.encode(), a.ctypes.data_as(C.POINTER(C.c_double)),
                                         a.shape[0], int(append)), what="pg_write_time_rows")


# ---- dump layout (variable_types.h:67-97) ---------------------------------------
def dump_fields(buf, p: pg_params) -> dict:
    """Views of a dump image: r,p,u,v,w [nring, jmax] (storage order) and the
    per-ring scalars."""
    jmax = p.jmax
    n = p.imax * p.kmax
    rb = 72 * jmax + 96
    raw = np.frombuffer(buf, dtype=np.uint8)
    assert raw.size == rb * n
    rec = raw.reshape(n, rb)
    f = rec[:, :40 * jmax].copy().view(np.float64).reshape(n, 5, jmax)
    tail = rec[:, 72 * jmax + 32:].copy()
    zs = tail[:, :32].view(np.float64)
    ik = tail[:, 32:40].view(np.int32)
    rot = tail[:, 40:56].view(np.float64)
    rj = tail[:, 56:64].view(np.int32)
    xs = rec[:, 40 * jmax:40 * jmax + 32].copy().view(np.float64)
    return dict(r=f[:, 0], p=f[:, 1], u=f[:, 2], v=f[:, 3], w=f[:, 4], x=xs[:, 0], dx=xs[:, 1],
                xvol=xs[:, 2], xc=xs[:, 3], z=zs[:, 0], dz=zs[:, 1], zvol=zs[:, 2], zc=zs[:, 3],
                i=ik[:, 0], k=ik[:, 1], rot_v=rot[:, 0], res_v=rot[:, 1], rot_j=rj[:, 0], inc_j=rj[:, 1])


def to_physical(a: np.ndarray, rot_j: np.ndarray) -> np.ndarray:
    """Storage order -> physical azimuth order (j_phys = j_store + rot_j)."""
    out = np.empty_like(a)
    for m in range(a.shape[0]):
        out[m] = np.roll(a[m], int(rot_j[m]))
    return out


@dataclass
class Planet:
    """struct body (variable_types.h:26-37)."""
    m: float = 0.0
    x: float = 0.0
    y: float = 0.0
    vx: float = 0.0
    vy: float = 0.0
    fx: float = 0.0
    fy: float = 0.0
    rs: float = 0.0

    def to_c(self) -> pg_body:
        return pg_body(self.m, self.x, self.y, self.vx, self.vy, self.fx, self.fy, self.rs)

    def set_from(self, b: pg_body):
        for k in ("m", "x", "y", "vx", "vy", "fx", "fy", "rs"):
            setattr(self, k, getattr(b, k))


class Run:
    """One disk run resident on one GPU (pg_run)."""

    def __init__(self, p: pg_params, device: int = 0):
        self.p = p
        self._h = None
        h = C.c_void_p()
        _check(_lib.lib().pg_create(C.byref(p), device, C.byref(h)), what="pg_create")
        self._h = h

    def close(self):
        if self._h:
            _lib.lib().pg_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    # ---- state I/O (copy_bfile / save_cells) ----
    def load(self, buf) -> "Run":
        n = len(buf)
        if isinstance(buf, (bytes, bytearray)):
            cbuf = (C.c_char * n).from_buffer_copy(buf)
        else:
            cbuf = buf
        _check(_lib.lib().pg_load_rings(self._h, cbuf, n), self, "pg_load_rings")
        return self

    def load_from(self, ptr: int, nbytes: int) -> "Run":
        """pg_load_rings from a raw host pointer (e.g. a pinned buffer)."""
        _check(_lib.lib().pg_load_rings(self._h, C.c_void_p(ptr), nbytes), self, "pg_load_rings")
        return self

    def save_to(self, ptr: int, nbytes: int):
        """pg_save_rings into a raw host pointer (e.g. a pinned buffer)."""
        _check(_lib.lib().pg_save_rings(self._h, C.c_void_p(ptr), nbytes), self, "pg_save_rings")

    def harmonic(self, m: float) -> tuple[np.ndarray, np.ndarray]:
        """Azimuthal harmonic m of Sigma per ring of layer 0 (read/ write_har_file)."""
        an = np.zeros(self.p.imax)
        bn = np.zeros(self.p.imax)
        dp = C.POINTER(C.c_double)
        _check(_lib.lib().pg_post_harmonic(self._h, m, an.ctypes.data_as(dp), bn.ctypes.data_as(dp)), self,
               "pg_post_harmonic")
        return an, bn

    def post_torque(self, M_p: float) -> float:
        """Disk torque on a planet at r = 1, azimuth pi (read/ get_torque)."""
        out = C.c_double(0.0)
        _check(_lib.lib().pg_post_torque(self._h, M_p, C.byref(out)), self, "pg_post_torque")
        return out.value

    def load_dump(self, path: str) -> "Run":
        _check(_lib.lib().pg_load_dump(self._h, path.encode()), self, "pg_load_dump")
        return self

    def save(self) -> bytearray:
        n = ring_bytes(self.p.jmax) * self.p.imax * self.p.kmax
        buf = bytearray(n)
        cbuf = (C.c_char * n).from_buffer(buf)
        _check(_lib.lib().pg_save_rings(self._h, cbuf, n), self, "pg_save_rings")
        return buf

    def save_dump(self, path: str):
        _check(_lib.lib().pg_save_dump(self._h, path.encode()), self, "pg_save_dump")

    def sync(self):
        _check(_lib.lib().pg_sync(self._h), self, "pg_sync")

    def launches(self) -> int:
        return _lib.lib().pg_launch_count(self._h)

    def timing(self, on: bool):
        _check(_lib.lib().pg_timing(self._h, 1 if on else 0), self, "pg_timing")

    def timing_read(self) -> tuple[list, list]:
        ms = (C.c_double * 4)()
        cnt = (C.c_int64 * 4)()
        _check(_lib.lib().pg_timing_read(self._h, ms, cnt, 4), self, "pg_timing_read")
        return list(ms), list(cnt)

    def stream_ptr(self) -> int:
        v = _lib.pg_device_view()
        _check(_lib.lib().pg_device_view_get(self._h, C.byref(v)), self, "pg_device_view_get")
        return v.stream or 0

    # ---- fused device-resident loop ----
    def clock_reset(self, startat: int = 0):
        _check(_lib.lib().pg_clock_reset(self._h, startat), self, "pg_clock_reset")

    def advance(self, nsteps: int, graph_chunk: int = 0) -> int:
        taken = C.c_int(0)
        if graph_chunk > 0:
            st = _lib.lib().pg_advance_graph(self._h, nsteps, graph_chunk, C.byref(taken))
        else:
            st = _lib.lib().pg_advance(self._h, nsteps, C.byref(taken))
        _check(st, self, "pg_advance")
        return taken.value

    def clock(self) -> tuple[pg_clock, Planet]:
        c, b = pg_clock(), pg_body()
        _check(_lib.lib().pg_clock_get(self._h, C.byref(c), C.byref(b)), self, "pg_clock_get")
        pl = Planet()
        pl.set_from(b)
        return c, pl

    def history(self, max_rows: int = 4096) -> np.ndarray:
        buf = (C.c_double * (max_rows * HIST_COLS))()
        n = C.c_int(0)
        _check(_lib.lib().pg_history(self._h, buf, max_rows, C.byref(n)), self, "pg_history")
        return np.frombuffer(buf, dtype=np.float64)[: n.value * HIST_COLS].reshape(n.value, HIST_COLS).copy()

    # ---- host-driven loop with the reference's call sequence ----
    def kernel_loop(self, nsteps: int, startat: int = 0, damping: bool = True, record=None,
                    sweep2d: bool = False):
        """main.cu:270-441 restart path, host-driven: one get_dt (host sync),
        Index_Shift, kick, bundle_sweep2D, damping, drift/forces/kick per step.
        record(step, simtime, dt_used, planet, FrRot) is called after each step.
        A 3D run steps with bundle_sweep3D, or with bundle_sweep2D (radial and
        azimuthal sweeps of every layer, no polar sweep) when sweep2d is set."""
        p = self.p
        dt = p.endtime
        simtime = p.tmovie * startat
        timem = 0.0
        old_dt = 0.0
        planet, FrRot = init_planet(p)
        planet_forces(planet, FrRot, self, simtime)
        make_pict = False
        cont = True
        ncycle = 0
        s = 0
        while s < nsteps and cont:
            dt = get_dt(dt, self, FrRot)
            if ncycle == p.ncycend:
                cont = False
            if simtime + dt >= p.endtime:
                old_dt = dt
                dt = p.endtime - simtime
                make_pict = True
                cont = False
            if timem + dt >= p.tmovie:
                old_dt = dt
                dt = p.tmovie - timem
                make_pict = True
            dt_used = dt
            Index_Shift(self, dt, FrRot)
            if p.plnt_flag > 0:
                FrRot = kick_drift_kick(p, planet, FrRot, 0.5 * dt, True)
            if p.ndim == 2 or sweep2d:
                bundle_sweep2D(self, dt, planet, FrRot)
            else:
                bundle_sweep3D(self, dt, planet, FrRot)
            if damping:
                _check(_lib.lib().pg_damp(self._h, dt), self, "pg_damp")
            simtime += dt
            timem += dt
            ncycle += 1
            if p.plnt_flag > 0:
                FrRot = kick_drift_kick(p, planet, FrRot, dt, False)
                planet_forces(planet, FrRot, self, simtime)
                FrRot = kick_drift_kick(p, planet, FrRot, 0.5 * dt, True)
            if make_pict:
                timem = 0.0
                make_pict = False
                dt = old_dt
            if record is not None:
                record(s, simtime, dt_used, planet, FrRot)
            s += 1
        return s, simtime, dt, planet, FrRot


class Batch:
    """Many runs stepped together (include/penguin_b200.h, pg_batch_*).

    Members are Run objects that are loaded and clock-reset; each keeps its own
    clock and dt.  While a run is in a batch, step it only through the batch."""

    def __init__(self, device: int = 0):
        h = C.c_void_p()
        _check(_lib.lib().pg_batch_create(device, C.byref(h)), None, "pg_batch_create")
        self._h = h
        self.members: list[Run] = []

    def _ck(self, st: int, what: str):
        if st != 0:
            msg = _lib.lib().pg_batch_last_error(self._h) or b""
            raise PenguinError(st, f"{what}: {msg.decode(errors='replace')}")

    def close(self):
        if self._h:
            _lib.lib().pg_batch_destroy(self._h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def add(self, run: Run) -> "Batch":
        self._ck(_lib.lib().pg_batch_add(self._h, run._h), "pg_batch_add")
        self.members.append(run)
        return self

    def remove(self, run: Run):
        self._ck(_lib.lib().pg_batch_remove(self._h, run._h), "pg_batch_remove")
        self.members.remove(run)

    def advance(self, nsteps: int, chunk: int = 32):
        self._ck(_lib.lib().pg_batch_advance(self._h, nsteps, chunk), "pg_batch_advance")

    def sync(self):
        self._ck(_lib.lib().pg_batch_sync(self._h), "pg_batch_sync")

    def status(self) -> list[dict]:
        n = len(self.members)
        arr = (_lib.pg_batch_member * max(n, 1))()
        self._ck(_lib.lib().pg_batch_status(self._h, arr, n), "pg_batch_status")
        return [dict(halted=arr[i].halted, status=arr[i].status, ncycle=arr[i].ncycle,
                     simtime=arr[i].simtime) for i in range(n)]

    def shape(self, group: int) -> dict:
        sh = _lib.pg_batch_shape()
        self._ck(_lib.lib().pg_batch_get_shape(self._h, group, C.byref(sh)), "pg_batch_get_shape")
        return dict(grid_x=sh.grid_x, grid_y=sh.grid_y, minb=sh.minb)

    def set_shape(self, group: int, grid_x: int = 0, grid_y: int = 0, minb: int = 8):
        sh = _lib.pg_batch_shape(grid_x, grid_y, minb, 0)
        self._ck(_lib.lib().pg_batch_set_shape(self._h, group, C.byref(sh)), "pg_batch_set_shape")

    def tune(self, trial_steps: int = 8):
        self._ck(_lib.lib().pg_batch_tune(self._h, trial_steps), "pg_batch_tune")

    def launches(self) -> int:
        return int(_lib.lib().pg_batch_launch_count(self._h))

    def stream_ptr(self) -> int:
        return _lib.lib().pg_batch_stream(self._h) or 0


class Server:
    """Continuous-batching serving loop (include/penguin_b200.h, pg_server_*)."""

    def __init__(self, device: int = 0, hbm_budget: int = 150 * 10 ** 9, max_slots: int = 64,
                 chunk: int = 32, keep_results: bool = False):
        h = C.c_void_p()
        _check(_lib.lib().pg_server_create(device, hbm_budget, max_slots, chunk, 1 if keep_results else 0,
                                           C.byref(h)), None, "pg_server_create")
        self._h = h

    def _ck(self, st: int, what: str):
        if st != 0:
            msg = _lib.lib().pg_server_last_error(self._h) or b""
            raise PenguinError(st, f"{what}: {msg.decode(errors='replace')}")

    def close(self):
        if self._h:
            _lib.lib().pg_server_destroy(self._h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def run_trace(self, reqs: list, arrival_s, ids=None) -> list[dict]:
        n = len(reqs)
        arr = (pg_params * max(n, 1))(*reqs)
        t = (C.c_double * max(n, 1))(*[float(x) for x in arrival_s])
        ids = list(range(n)) if ids is None else list(ids)
        ii = (C.c_int64 * max(n, 1))(*ids)
        out = (_lib.pg_completion * max(n, 1))()
        self._ck(_lib.lib().pg_server_run_trace(self._h, arr, t, ii, n, out), "pg_server_run_trace")
        keys = [f for f, _ in _lib.pg_completion._fields_ if f != "pad"]
        return [{k: getattr(out[i], k) for k in keys} for i in range(n)]

    def result(self, rid: int, p: pg_params) -> bytearray:
        buf = bytearray(ring_bytes(p.jmax) * p.imax * p.kmax)
        c = (C.c_char * len(buf)).from_buffer(buf)
        self._ck(_lib.lib().pg_server_result(self._h, rid, c, len(buf)), "pg_server_result")
        return buf

    def rounds(self) -> int:
        return int(_lib.lib().pg_server_rounds(self._h))


def run_device_bytes(p: pg_params) -> int:
    """Device memory pg_create allocates for these parameters."""
    return int(_lib.lib().pg_run_device_bytes(C.byref(p)))


# ---- the reference's free functions ----------------------------------------------
def get_dt(dt: float, run: Run, FrRot: float = 0.0) -> float:
    out = C.c_double(0.0)
    st = _lib.lib().pg_get_dt(run._h, dt, FrRot, C.byref(out))
    if st not in (0, 4):   # PG_ERR_DT_COLLAPSE: the reference prints and goes on
        _check(st, run, "pg_get_dt")
    return out.value


def Index_Shift(run: Run, dt: float, FrRot: float = 0.0):
    _check(_lib.lib().pg_index_shift(run._h, dt, FrRot), run, "pg_index_shift")


def bundle_sweep2D(run: Run, dt: float, planet: Planet, FrRot: float = 0.0):
    b = planet.to_c()
    _check(_lib.lib().pg_sweep2d(run._h, dt, C.byref(b), FrRot), run, "pg_sweep2d")


def bundle_sweep3D(run: Run, dt: float, planet: Planet, FrRot: float = 0.0):
    b = planet.to_c()
    _check(_lib.lib().pg_sweep3d(run._h, dt, C.byref(b), FrRot), run, "pg_sweep3d")


def sweep_axis(run: Run, axis: int, dt: float, planet: Planet, FrRot: float = 0.0):
    """One directional sweep: 0 = sweepx (ppm.cu:26), 1 = sweepy (ppm.cu:162,
    FARGO shift at the store), 2 = the polar sweep (3D)."""
    b = planet.to_c()
    _check(_lib.lib().pg_sweep_axis(run._h, axis, dt, C.byref(b), FrRot), run, "pg_sweep_axis")


def rotate_rings(run: Run):
    """rotate_rings (ppm.cu:309-322): rot_j += inc_j."""
    _check(_lib.lib().pg_rotate(run._h), run, "pg_rotate")


def GPU_output_reduction(run: Run, planet: Planet, exclude: float = 0.0, mode: int = 0) -> float:
    b = planet.to_c()
    out = C.c_double(0.0)
    _check(_lib.lib().pg_reduce(run._h, C.byref(b), exclude, mode, C.byref(out)), run, "pg_reduce")
    return out.value


def init_planet(p: pg_params) -> tuple[Planet, float]:
    b = pg_body()
    fr = C.c_double(0.0)
    _check(_lib.lib().pg_init_planet(C.byref(p), C.byref(b), C.byref(fr)), what="pg_init_planet")
    pl = Planet()
    pl.set_from(b)
    return pl, fr.value


def planet_forces(planet: Planet, FrRot: float, run: Run, simtime: float):
    b = planet.to_c()
    _check(_lib.lib().pg_planet_forces(run._h, C.byref(b), FrRot, simtime), run, "pg_planet_forces")
    planet.set_from(b)


def kick_drift_kick(p: pg_params, planet: Planet, FrRot: float, dt: float, kick: bool) -> float:
    """Returns the new FrRot (the reference passes it by reference)."""
    b = planet.to_c()
    fr = C.c_double(FrRot)
    _check(_lib.lib().pg_kick_drift_kick(C.byref(p), C.byref(b), C.byref(fr), dt, 1 if kick else 0),
           what="pg_kick_drift_kick")
    planet.set_from(b)
    return fr.value


def get_ecc(planet: Planet, FrRot: float) -> float:
    b = planet.to_c()
    return _lib.lib().pg_get_ecc(C.byref(b), FrRot)


def _pow_const(x: float, y: float) -> float:
    """pow in the form the reference's compiler gives a constant exponent:
    0, 1, -1 and 2 fold to 1, x, 1/x and x*x."""
    if y == 0.0:
        return 1.0
    if y == 1.0:
        return x
    if y == -1.0:
        return 1.0 / x
    if y == 2.0:
        return x * x
    return math.pow(x, y)


def torque_norm(p: pg_params) -> float:
    """main.cu:421 normalisation of the mode-9 torque."""
    return p.M_p * p.M_p * _pow_const(p.R_p, 1.0 - p.p_alpha + (p.p_beta - 1.0)) / (p.sc_h * p.sc_h)
