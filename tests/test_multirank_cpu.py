"""The multi-rank bench path on CPU ranks (gloo, world size 2): every rank
solves its own replica of the spectrum (no data-path collective); the job's
throughput is all ranks' solves over the slowest rank's device time."""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(('127.0.0.1', 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _rank(rank, world, port, q):
    os.environ.update(MASTER_ADDR='127.0.0.1', MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    import bench
    r, w, local, pg = bench.dist_setup('gloo')
    bench.barrier(pg, local)
    # rank r "solved" 201 frequencies in (1000 + 500 r) ms of device time
    value, total, slowest = bench.job_throughput(pg, local, 201, 1000.0 + 500.0 * r)
    q.put((r, value, total, slowest))
    pg.destroy_process_group()


def test_two_rank_weak_scaling_reduction():
    ctx = mp.get_context('spawn')
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for r, value, total, slowest in out:
        assert total == 402.0 and slowest == 1500.0
        assert value == pytest.approx(402.0 / 1.5)
