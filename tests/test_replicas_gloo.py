"""Multi-process path of ``bench.py`` on CPU: two ``gloo`` ranks, each timing
its own replica; the job time is the max over ranks and the whole-job GLUPS
counts the lattice updates of both ranks."""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank(rank, ws, port, q):
    import datetime
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(ws),
                      LOCAL_RANK=str(rank))
    dist.init_process_group("gloo", rank=rank, world_size=ws, timeout=datetime.timedelta(seconds=60))
    import bench
    assert bench.dist_env() == (ws, rank, rank)
    dev, e2e = bench.replica_totals(10.0 + rank, 20.0 - rank, ws, "cpu")
    q.put((rank, dev, e2e, bench.replica_glups(1_000_000, ws, dev)))
    dist.destroy_process_group()


def test_two_gloo_ranks_take_the_max_time():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    out = sorted(q.get(timeout=10) for _ in range(2))
    for rank, dev, e2e, glups in out:
        assert dev == 11.0 and e2e == 20.0
        assert glups == pytest.approx(2 * 1_000_000 / 11e-3 / 1e9)
