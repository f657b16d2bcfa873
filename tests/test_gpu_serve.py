"""Serving loop: continuous batching of arriving disk runs.

Requests arrive while others are on the GPU, are admitted as slots and the
HBM budget free up, and are stepped together in one batch.  Each result must
be the same alone and in the mix: the final dump of every request equals,
bit for bit, the dump of the same request advanced alone to its end time."""
import numpy as np
import pytest

import penguin_2_0_b200 as pg


def _req(which, t_end, **kw):
    p = pg.params(which, endtime=t_end, tmovie=t_end, nprin=10, **kw)
    return p


REQS = [
    _req(0, 0.30, imax=128, jmax=384, M_p=1e-3),
    _req(0, 0.20, imax=192, jmax=576, M_p=2e-5, precision=1),
    _req(1, 0.15, imax=64, jmax=192, kmax=16),
    _req(0, 0.20, imax=136, jmax=408, EOS=1, gam=1.4),       # isentropic: own step sequence
    _req(0, 0.25, imax=136, jmax=408, M_p=3e-4, sc_h=0.06, ss_alpha=1e-2),
    _req(0, 0.10, imax=256, jmax=768, M_p=1e-5, precision=1, p_alpha=0.7),
    _req(0, 0.20, imax=136, jmax=408, plnt_flag=2),          # moving planet: own step sequence
    _req(0, 0.35, imax=128, jmax=384, plnt_flag=0),
]
ARRIVALS = [0.0, 0.0, 0.02, 0.03, 0.05, 0.08, 0.10, 0.12]


def _alone(p):
    with pg.Run(p, 0) as r:
        r.load(pg.build_ic(p))
        r.clock_reset(0)
        n = r.advance(100000)
        c, _ = r.clock()
        assert c.done
        return n, bytes(r.save())


@pytest.mark.gpu
def test_server_results_equal_alone(gpu):
    with pg.Server(0, hbm_budget=8 * 10 ** 9, max_slots=4, chunk=4, keep_results=True) as s:
        done = s.run_trace(REQS, ARRIVALS, ids=[100 + i for i in range(len(REQS))])
        assert s.rounds() > 0
        got = {d["id"]: d for d in done}
        for i, p in enumerate(REQS):
            d = got[100 + i]
            assert d["status"] == 0, d
            assert d["arrival_s"] <= d["admit_s"] <= d["finish_s"]
            assert abs(d["simtime"] - p.endtime) < 1e-12
            steps, dump = _alone(p)
            assert d["steps"] == steps, (i, d["steps"], steps)
            mixed = bytes(s.result(100 + i, p))
            assert mixed == dump, f"request {i}: mixed result differs from the run alone"


@pytest.mark.gpu
def test_server_admission_respects_slots_and_budget(gpu):
    reqs = [_req(0, 0.1, imax=128, jmax=384, M_p=1e-4) for _ in range(5)]
    need = pg.run_device_bytes(reqs[0])
    # room for two runs: at most two live at any time
    with pg.Server(0, hbm_budget=2 * need + need // 2, max_slots=8, chunk=2) as s:
        done = s.run_trace(reqs, [0.0] * 5)
    assert all(d["status"] == 0 for d in done)
    events = sorted([(d["admit_s"], 1) for d in done] + [(d["finish_s"], -1) for d in done],
                    key=lambda e: (e[0], e[1]))
    live = peak = 0
    for _, dv in events:
        live += dv
        peak = max(peak, live)
    assert peak <= 2, peak
    with pg.Server(0, hbm_budget=100 * need, max_slots=3, chunk=2) as s:
        done = s.run_trace(reqs, [0.0] * 5)
    admits = sorted(d["admit_s"] for d in done)
    finishes = sorted(d["finish_s"] for d in done)
    assert admits[3] >= finishes[0]          # the fourth waits for a slot


def test_request_stream_is_valid_and_seeded():
    from penguin_2_0_b200 import serving
    a = serving.draw_stream(200, seed=3)
    b = serving.draw_stream(200, seed=3)
    assert [x.as_dict() for x in a] == [x.as_dict() for x in b]
    assert all(pg.host.check_params(p) == 0 for p in a)
    n3 = sum(p.ndim == 3 for p in a)
    assert 5 <= n3 <= 40
    t = serving.poisson_arrivals(1000, rate_per_s=10.0, seed=1)
    assert np.all(np.diff(t) >= 0) and abs(t[-1] / 999 - 0.1) < 0.02
