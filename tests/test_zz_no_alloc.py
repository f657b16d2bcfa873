"""pg_reduce_noalloc: the disk mass / force / torque reduction for callers
that cannot allocate device memory, such as a process whose HBM belongs to
its own memory pool (a cudaMalloc there fails or takes memory the pool
counts on) or a time loop that allocated its buffers once at start-up and
must not allocate, or synchronise the device as cudaMalloc/cudaFree may,
inside the loop.  The entry point works on device buffers the caller owns;
its only scratch is a static device array shared by every call.

Checked here, on two calls in a row each time (the second call reuses the
scratch the first one left behind):
  * the same mass, radial force and torque as pg_reduce on the same state;
  * the reference build's own mass and torque (golden vectors of the
    136x136 disk) after the library's steps;
  * a disk of more than 1024 rings (the chunked final sum) and FARGO
    offsets outside [0, jmax), against sums formed on the host.
Inputs and outputs are buffers the test allocates with torch; the entry
point only launches into them.  This file runs last (pytest collects it
last), so a failure here leaves every other test already run."""
import ctypes as C
import math

import numpy as np
import pytest

import penguin_2_0_b200 as pg
from penguin_2_0_b200 import _lib
from tests._golden import load, params_for
from tests._lockstep import torque_abs_scale

TOL = 1e-12


def _device_inputs(run, p, dev):
    """Sigma in physical order and the per-ring / per-column geometry of a
    run's current state, as device tensors."""
    import torch
    raw = bytes(run.save())
    f = pg.dump_fields(raw, p)
    rb = 72 * p.jmax + 96
    cols = np.frombuffer(raw[:rb], dtype=np.uint8)[40 * p.jmax + 32:72 * p.jmax + 32].copy().view(np.float64)
    cols = cols.reshape(4, p.jmax)
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(dev)
    return f, dict(sigma=t(pg.to_physical(f["r"], f["rot_j"])), xc=t(f["xc"]), xvol=t(f["xvol"]),
                   rot_j=t(f["rot_j"].astype(np.int32)), yc=t(cols[3]), yvol=t(cols[2]))


def _call(d, imax, jmax, planet, mode, p_alpha, sc_h, out_ptr, stream):
    b = planet.to_c()
    return _lib.lib().pg_reduce_noalloc(d["sigma"].data_ptr(), jmax, d["xc"].data_ptr(), d["xvol"].data_ptr(),
                                        d["rot_j"].data_ptr(), d["yc"].data_ptr(), d["yvol"].data_ptr(), imax,
                                        jmax, C.byref(b), 0.0, mode, p_alpha, sc_h, out_ptr, stream)


@pytest.mark.gpu
def test_noalloc_reduction_matches_pg_reduce(gpu):
    import torch

    p = pg.params(0, imax=256, jmax=768, nprin=1)
    dev = torch.device("cuda", 0)
    with pg.Run(p, 0) as run:
        run.load(pg.build_ic(p))
        run.clock_reset(0)
        assert run.advance(3) == 3
        _, planet = run.clock()
        ref = [pg.GPU_output_reduction(run, planet, 0.0, m) for m in (0, 8, 9)]
        f, d = _device_inputs(run, p, dev)
        out = torch.zeros(3, dtype=torch.float64, device=dev)
        stream = torch.cuda.current_stream(dev).cuda_stream
        scale = torque_abs_scale(f, p, planet) * pg.torque_norm(p)
        for _ in range(2):
            out.zero_()
            for slot, mode in enumerate((0, 8, 9)):
                assert _call(d, p.imax, p.jmax, planet, mode, p.p_alpha, p.sc_h, out.data_ptr() + 8 * slot,
                             stream) == 0
            torch.cuda.synchronize()
            mass, f8, tq = out.cpu().numpy()
            assert abs(mass - ref[0]) <= TOL * abs(ref[0]), (mass, ref[0])
            # radial force: same terms as the torque without the lever arm r
            assert abs(f8 - ref[1]) <= TOL * scale, (f8, ref[1], scale)
            assert abs(tq - ref[2]) <= TOL * scale, (tq, ref[2], scale)

        # sizes beyond the static scratch are refused before any launch
        assert _call(d, 16385, p.jmax, planet, 0, p.p_alpha, p.sc_h, out.data_ptr(), stream) == 2


@pytest.mark.gpu
def test_noalloc_reduction_matches_reference_build(gpu):
    """After the library's steps on the golden 136x136 disk, the mass and
    torque of the no-allocation reduction equal the reference build's own
    (its GPU_output_reduction at every step), at the golden tolerance."""
    import torch

    case = "g136x136"
    p = params_for(case)
    g = load(case)
    dev = torch.device("cuda", 0)
    stream = torch.cuda.current_stream(dev).cuda_stream
    with pg.Run(p, 0) as run:
        run.load(pg.build_ic(p))
        run.clock_reset(0)
        for step in (2, 5):
            done = int(run.clock()[0].ncycle)
            assert run.advance(step - done) == step - done
            _, planet = run.clock()
            f, d = _device_inputs(run, p, dev)
            h = g["hist"][step - 1]
            scale = torque_abs_scale(f, p, planet)
            out = torch.zeros(2, dtype=torch.float64, device=dev)
            for _ in range(2):
                out.zero_()
                assert _call(d, p.imax, p.jmax, planet, 0, p.p_alpha, p.sc_h, out.data_ptr(), stream) == 0
                assert _call(d, p.imax, p.jmax, planet, 9, p.p_alpha, p.sc_h, out.data_ptr() + 8, stream) == 0
                torch.cuda.synchronize()
                mass, tq = out.cpu().numpy()
                tq /= pg.torque_norm(p)
                assert abs(mass - h[2]) <= TOL * h[2], (step, mass, h[2])
                assert abs(tq - h[3]) <= TOL * scale, (step, tq, h[3], scale)


@pytest.mark.gpu
def test_noalloc_reduction_many_rings_any_offset(gpu):
    """1536 rings (the ring partials summed in two 1024-wide blocks) with
    FARGO offsets drawn from [-2 jmax, 3 jmax): mass and torque against
    host sums, and bitwise the same as with the offsets reduced mod jmax."""
    import torch

    rng = np.random.default_rng(7)
    imax, jmax = 1536, 200
    dev = torch.device("cuda", 0)
    stream = torch.cuda.current_stream(dev).cuda_stream
    xa = 0.4 * (2.5 / 0.4) ** (np.arange(imax + 1) / imax)
    dx = np.diff(xa)
    xc = xa[:-1] + 0.5 * dx
    xvol = dx * xc
    dy = 2 * np.pi / jmax
    yc = (np.arange(jmax) + 0.5) * dy
    yvol = np.full(jmax, dy)
    sig = (1.0 / xc)[:, None] * (1.0 + 1e-2 * rng.uniform(-1, 1, (imax, jmax)))
    rot = rng.integers(-2 * jmax, 3 * jmax, imax).astype(np.int32)
    planet = pg.Planet(m=1e-3, x=1.0, y=np.pi, vx=0.0, vy=1.0, fx=0.0, fy=0.0, rs=0.03)
    p_alpha = 1.0
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(dev)
    d = dict(sigma=t(sig), xc=t(xc), xvol=t(xvol), rot_j=t(rot), yc=t(yc), yvol=t(yvol))
    d_mod = dict(d, rot_j=t((rot % jmax).astype(np.int32)))

    # host sums over the same cells (physical order; the offsets only permute a ring)
    mass_ref = math.fsum((sig * xvol[:, None] * yvol[None, :]).ravel())
    cosf = np.cos(yc - planet.y)[None, :]
    sinf = np.sin(yc - planet.y)[None, :]
    r = xc[:, None]
    Rp = np.sqrt(r * r + planet.x ** 2 - 2 * planet.x * r * cosf + planet.rs ** 2)
    g_azi = -planet.m * planet.x * sinf / Rp ** 3 + planet.m * sinf / planet.x ** 2
    terms = -g_azi * r * (sig - r ** (-p_alpha)) * xvol[:, None] * yvol[None, :]
    tq_ref = math.fsum(terms.ravel())
    tq_scale = float(np.sum(np.abs(terms)))

    out = torch.zeros(4, dtype=torch.float64, device=dev)
    for _ in range(2):
        out.zero_()
        for slot, (dd, mode) in enumerate(((d, 0), (d, 9), (d_mod, 0), (d_mod, 9))):
            assert _call(dd, imax, jmax, planet, mode, p_alpha, 0.05, out.data_ptr() + 8 * slot, stream) == 0
        torch.cuda.synchronize()
        mass, tq, mass_m, tq_m = out.cpu().numpy()
        assert abs(mass - mass_ref) <= TOL * mass_ref, (mass, mass_ref)
        assert abs(tq - tq_ref) <= TOL * tq_scale, (tq, tq_ref, tq_scale)
        assert mass == mass_m and tq == tq_m
