"""Drive the CUDA path and the CPU oracle through the same restart-path time
loop (main.cu:270-441), one step at a time, for parity tests."""
import ctypes as C

import numpy as np

import penguin_2_0_b200 as pg
from oracle.pyoracle import Oracle, lib as olib
from penguin_2_0_b200._lib import pg_body


def rel_linf(a, b):
    den = np.max(np.abs(b))
    if den == 0.0:
        return float(np.max(np.abs(a - b)))
    return float(np.max(np.abs(a - b)) / den)


class OracleLoop:
    """main.cu restart loop on the oracle, advanced one step per call."""

    def __init__(self, p, ic, sweep2d=False):
        self.p = p
        self.sweep2d = sweep2d        # 3D: radial + azimuthal sweeps only (bundle_sweep2D)
        self.o = Oracle(p, ic)
        self.planet = pg_body()
        fr = C.c_double(0.0)
        olib().orc_init_planet(C.byref(p), C.byref(self.planet), C.byref(fr))
        self.FrRot = fr.value
        olib().orc_planet_forces(self.o._h, C.byref(self.planet), self.FrRot, 0.0)
        self.dt = p.endtime
        self.simtime = 0.0
        self.timem = 0.0
        self.old_dt = 0.0

    def step(self):
        p, o = self.p, self.o
        fr = C.c_double(self.FrRot)
        self.dt = o.get_dt(self.dt, self.FrRot)
        make_pict = False
        if self.simtime + self.dt >= p.endtime:
            self.old_dt = self.dt
            self.dt = p.endtime - self.simtime
            make_pict = True
        if self.timem + self.dt >= p.tmovie:
            self.old_dt = self.dt
            self.dt = p.tmovie - self.timem
            make_pict = True
        dt = self.dt
        o.index_shift(dt, self.FrRot)
        if p.plnt_flag > 0:
            olib().orc_kick_drift_kick(C.byref(p), C.byref(self.planet), C.byref(fr), 0.5 * dt, 1)
            self.FrRot = fr.value
        if self.sweep2d:
            olib().orc_sweep2d(o._h, dt, C.byref(self.planet), self.FrRot)
        else:
            o.sweep(dt, self.planet, self.FrRot)
        o.damp(dt)
        self.simtime += dt
        self.timem += dt
        if p.plnt_flag > 0:
            fr = C.c_double(self.FrRot)
            olib().orc_kick_drift_kick(C.byref(p), C.byref(self.planet), C.byref(fr), dt, 0)
            olib().orc_planet_forces(o._h, C.byref(self.planet), fr.value, self.simtime)
            olib().orc_kick_drift_kick(C.byref(p), C.byref(self.planet), C.byref(fr), 0.5 * dt, 1)
            self.FrRot = fr.value
        if make_pict:
            self.timem = 0.0
            self.dt = self.old_dt
        mass = o.reduce(self.planet, 0.0, 0)
        torque = o.reduce(self.planet, 0.0, 9) / pg.torque_norm(p) if (p.plnt_flag > 0 and p.ndim == 2) else 0.0
        return dt, mass, torque

    def fields(self):
        return pg.dump_fields(self.o.save(), self.p)


def torque_abs_scale(fields, p, planet):
    """Sum over cells of |integrand| of the mode-9 torque (device_func.cu:96-108),
    normalised like main.cu:421: the scale that bounds the rounding of a sum
    whose terms cancel."""
    rot = fields["rot_j"]
    r = to_phys(fields["r"], rot)
    xc = fields["xc"][:, None]
    jmax = p.jmax
    dy = 2 * np.pi / jmax
    phi = (np.arange(jmax) + 0.5) * dy
    cosf = np.cos(phi - planet.y)[None, :]
    sinf = np.sin(phi - planet.y)[None, :]
    Rp = np.sqrt(xc * xc + planet.x ** 2 - 2 * planet.x * xc * cosf + planet.rs ** 2)
    g = -planet.m * planet.x * sinf / Rp ** 3 + planet.m * sinf / planet.x ** 2
    integ = g * xc * (r - xc ** (-p.p_alpha)) * fields["xvol"][:, None] * dy
    return float(np.sum(np.abs(integ))) / pg.torque_norm(p)


def to_phys(a, rot):
    out = np.empty_like(a)
    for m in range(a.shape[0]):
        out[m] = np.roll(a[m], int(rot[m]))
    return out
