"""pg_reduce_noalloc: the reduction for callers that cannot allocate device
memory (a thread capturing a CUDA graph, a process whose HBM belongs to its
own pool, a time loop that allocated everything up front).  It must give the
same disk mass and torque as pg_reduce on the same state, on two calls in a
row (the second call reuses the static scratch the first one left behind).
Inputs and the output are buffers the test allocates; the entry point only
launches into them."""
import ctypes as C

import numpy as np
import pytest

import penguin_2_0_b200 as pg
from penguin_2_0_b200 import _lib
from tests._lockstep import torque_abs_scale

TOL = 1e-12


@pytest.mark.gpu
def test_noalloc_reduction_matches_pg_reduce(gpu):
    import torch

    p = pg.params(0, imax=256, jmax=768, nprin=1)
    with pg.Run(p, 0) as run:
        run.load(pg.build_ic(p))
        run.clock_reset(0)
        assert run.advance(3) == 3
        _, planet = run.clock()
        f = pg.dump_fields(run.save(), p)
        mass_ref = pg.GPU_output_reduction(run, planet, 0.0, 0)
        tq_ref = pg.GPU_output_reduction(run, planet, 0.0, 9)

        dev = torch.device("cuda", 0)
        sigma = torch.from_numpy(pg.to_physical(f["r"], f["rot_j"]).copy()).to(dev)
        xc = torch.from_numpy(f["xc"].copy()).to(dev)
        xvol = torch.from_numpy(f["xvol"].copy()).to(dev)
        rot_j = torch.from_numpy(f["rot_j"].astype(np.int32)).to(dev)
        raw = np.frombuffer(bytes(run.save()), dtype=np.uint8)
        rb = 72 * p.jmax + 96
        ring0 = raw[:rb]
        cols = ring0[40 * p.jmax + 32:72 * p.jmax + 32].copy().view(np.float64).reshape(4, p.jmax)
        yvol = torch.from_numpy(cols[2].copy()).to(dev)
        yc = torch.from_numpy(cols[3].copy()).to(dev)
        out = torch.zeros(2, dtype=torch.float64, device=dev)
        stream = torch.cuda.current_stream(dev)
        b = planet.to_c()
        L = _lib.lib()

        def call(mode, slot):
            st = L.pg_reduce_noalloc(sigma.data_ptr(), p.jmax, xc.data_ptr(), xvol.data_ptr(),
                                     rot_j.data_ptr(), yc.data_ptr(), yvol.data_ptr(), p.imax, p.jmax,
                                     C.byref(b), 0.0, mode, p.p_alpha, p.sc_h,
                                     out.data_ptr() + 8 * slot, stream.cuda_stream)
            assert st == 0, st

        scale = torque_abs_scale(f, p, planet) * pg.torque_norm(p)
        for _ in range(2):
            out.zero_()
            call(0, 0)
            call(9, 1)
            torch.cuda.synchronize()
            mass, tq = out.cpu().numpy()
            assert abs(mass - mass_ref) <= TOL * abs(mass_ref), (mass, mass_ref)
            assert abs(tq - tq_ref) <= TOL * scale, (tq, tq_ref, scale)

        # sizes beyond the static scratch are refused before any launch
        st = L.pg_reduce_noalloc(sigma.data_ptr(), p.jmax, xc.data_ptr(), xvol.data_ptr(), rot_j.data_ptr(),
                                 yc.data_ptr(), yvol.data_ptr(), 16385, p.jmax, C.byref(b), 0.0, 0,
                                 p.p_alpha, p.sc_h, out.data_ptr(), stream.cuda_stream)
        assert st == 2
