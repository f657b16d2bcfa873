"""The multi-GPU form of the path, replicas, on the library itself: two
processes (gloo process group, world_size 2) each advance their own disk
through the C ABI on the one GPU this run has, then take the max over ranks
of their timed regions as bench.py does.  Replicas never wait on each other
(no collective inside a step), so sharing one GPU is only slower.  Each
rank's final state must equal the same disk (its seed) advanced alone, bit
for bit, and the two disks must differ."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


P = dict(imax=128, jmax=132, nprin=1)
STEPS = 6


def _worker(rank, world, port, out):
    import datetime
    import time

    import torch.distributed as dist

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=120))
    import penguin_2_0_b200 as pg
    from penguin_2_0_b200 import replicas

    p = replicas.rank_params(pg.params(0, **P), rank)
    with pg.Run(p, 0) as r:
        r.load(pg.build_ic(p))
        r.clock_reset(0)
        dist.barrier()
        t0 = time.perf_counter()
        n = r.advance(STEPS)
        r.sync()
        el = time.perf_counter() - t0
        tmax = replicas.max_over_ranks(el, dist)
        out[rank] = (n, el, tmax, bytes(r.save()), int(p.seed))
    dist.barrier()
    dist.destroy_process_group()


@pytest.mark.gpu
def test_two_library_replicas_equal_their_solo_runs(gpu):
    import penguin_2_0_b200 as pg
    ctx = mp.get_context("spawn")
    mgr = ctx.Manager()
    out = mgr.dict()
    mp.start_processes(_worker, args=(2, _free_port(), out), nprocs=2, join=True, start_method="spawn")
    assert out[0][2] == out[1][2] == max(out[0][1], out[1][1])
    assert out[0][4] != out[1][4]
    dumps = []
    for rank in (0, 1):
        n, _, _, dump, seed = out[rank]
        assert n == STEPS
        p = pg.params(0, **P)
        p.seed = seed
        with pg.Run(p, 0) as r:
            r.load(pg.build_ic(p))
            r.clock_reset(0)
            assert r.advance(STEPS) == STEPS
            solo = bytes(r.save())
        assert dump == solo, rank
        dumps.append(dump)
    assert dumps[0] != dumps[1]
