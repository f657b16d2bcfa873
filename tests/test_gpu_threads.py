"""Runs driven from several host threads at once.

The C ABI keeps no global state for a run: each pg_run has its own stream,
tables and clock, and error state is per run (the CUDA runtime's last error is
per host thread).  Two threads each create, load and advance their own disk
(one 2D, one 3D, through the device loop and through the reference's per-call
sequence) at the same time; ctypes releases the interpreter lock around the
calls, so they overlap.  Every result equals the same run advanced alone, bit
for bit."""
import threading

import numpy as np
import pytest

import penguin_2_0_b200 as pg

CASES = [
    (0, dict(imax=136, jmax=408), "advance"),
    (1, dict(imax=64, jmax=132, kmax=16), "advance"),
    (0, dict(imax=128, jmax=384, M_p=3e-4), "kernel_loop"),
]


def _job(which, over, how, nsteps=12):
    p = pg.params(which, **over)
    with pg.Run(p, 0) as r:
        r.load(pg.build_ic(p))
        if how == "advance":
            r.clock_reset(0)
            r.advance(nsteps, graph_chunk=4)
        else:
            r.kernel_loop(nsteps)
        return bytes(r.save())


@pytest.mark.gpu
def test_runs_on_concurrent_threads_equal_runs_alone(gpu):
    alone = [_job(*c) for c in CASES]
    out = [None] * len(CASES)
    errors = []

    def work(i):
        try:
            for _ in range(2):                 # twice: overlap in both orders
                out[i] = _job(*CASES[i])
        except Exception as e:                 # re-raised below
            errors.append(e)

    threads = [threading.Thread(target=work, args=(i,)) for i in range(len(CASES))]
    for t in threads:
        t.start()
    for t in threads:
        t.join(timeout=600)
    assert not any(t.is_alive() for t in threads)
    assert not errors, errors
    for i, (a, b) in enumerate(zip(alone, out)):
        assert np.array_equal(np.frombuffer(a, np.uint8), np.frombuffer(b, np.uint8)), f"case {i}"
