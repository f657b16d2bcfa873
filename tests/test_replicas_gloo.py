"""The multi-GPU path is independent replicas (one disk per rank) plus a max
over ranks of the timed region.  Exercised here with world_size 2 on the
gloo backend, each rank advancing its own disk on the CPU oracle."""
import os
import socket

import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, out):
    import datetime
    import time

    import torch.distributed as dist

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    import penguin_2_0_b200 as pg
    from oracle.pyoracle import Oracle
    from penguin_2_0_b200 import replicas

    p = replicas.rank_params(pg.params(0, imax=64, jmax=132), rank)
    o = Oracle(p, pg.build_ic(p))
    t0 = time.perf_counter()
    h = o.run_steps(2)
    el = time.perf_counter() - t0 + 0.05 * rank
    tmax = replicas.max_over_ranks(el, dist)
    out[rank] = (float(h[-1, 2]), el, tmax)
    dist.barrier()
    dist.destroy_process_group()


def test_two_replicas_max_over_ranks():
    ctx = mp.get_context("spawn")
    mgr = ctx.Manager()
    out = mgr.dict()
    port = _free_port()
    mp.start_processes(_worker, args=(2, port, out), nprocs=2, join=True, start_method="spawn")
    (m0, e0, t0), (m1, e1, t1) = out[0], out[1]
    assert t0 == t1 == max(e0, e1)
    assert m0 != m1          # different seeds, different disks
    from penguin_2_0_b200 import replicas
    assert replicas.job_throughput(100, 10, 2, 2.0) == 1000.0
