"""The multi-rank paths on CPU ranks (gloo, world size 2): the spectrum split into
frequency blocks per rank with the results gathered to rank 0, and the bench's
job throughput (all ranks' solves over the slowest rank's device time)."""
import os
import socket

import numpy as np
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


class _StandInSolver:
    """Deterministic per-frequency outputs (a function of the frequency alone), so
    a block solved on any rank gives the rows one rank would give."""

    def set_frequencies(self, freqs, alpha_w=None):
        self.freqs = np.asarray(freqs, dtype=np.float64)
        self.aw = alpha_w

    def solve(self, **kw):
        w = self.freqs
        F = len(w)
        res = np.sin(np.outer(w, np.arange(1, 21)) * 7.0) * (1.0 + w[:, None])
        if self.aw is not None:
            res[:, 3] += np.asarray(self.aw)[0].real
        polar = (np.cos(np.outer(w, np.arange(9)))
                 + 1j * np.sin(np.outer(w, np.arange(9)) * 3.0)).reshape(F, 3, 3)
        status = (np.round(w * 1000).astype(np.int32) % 3 == 0).astype(np.int32) * 5
        steps = np.stack([np.round(w * 977).astype(np.int32) % 400, np.zeros(F, np.int32),
                          np.zeros(F, np.int32)], axis=1)
        return {'results': res, 'polar': polar, 'status': status, 'steps': steps, 'device_ms': 10.0 * F}


def _grid(F=23):
    freqs = np.linspace(0.08, 0.17, F)
    aw = np.vstack([freqs * 2.0 + 1j * freqs, freqs * 3.0 - 1j]).astype(np.complex128)
    return freqs, aw


def _partition_rank(rank, world, port, q):
    os.environ.update(MASTER_ADDR='127.0.0.1', MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    import bench
    from plasmonx_b200.spectrum import solve_partitioned
    r, w, local, pg = bench.dist_setup('gloo')
    freqs, aw = _grid()
    out = solve_partitioned(_StandInSolver(), freqs, aw, pg, device='cpu', precision='mixed_bf16x3')
    q.put((r, out['block'].tolist(), None if out['results'] is None else
           (out['results'], out['status'], out['steps'], out['polar'])))
    pg.destroy_process_group()


def test_partition_covers_every_frequency_once():
    from plasmonx_b200.spectrum import partition
    for F in (1, 2, 7, 201):
        for world in (1, 2, 3, 8):
            blocks = partition(F, world)
            assert len(blocks) == world
            allidx = np.sort(np.concatenate(blocks))
            assert np.array_equal(allidx, np.arange(F))
            sizes = [len(b) for b in blocks]
            assert max(sizes) - min(sizes) <= 1


def test_two_rank_spectrum_partition_and_gather_bitwise():
    """Two gloo ranks solve the two blocks of one 23-frequency spectrum; rank 0's
    gathered results, status, step counts and polarizabilities equal one rank's
    solve of the whole grid bit for bit."""
    from plasmonx_b200.spectrum import solve_partitioned
    freqs, aw = _grid()
    one = solve_partitioned(_StandInSolver(), freqs, aw, None)
    ctx = mp.get_context('spawn')
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_partition_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = dict((r, (blk, data)) for r, blk, data in [q.get(timeout=120) for _ in procs])
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert got[0][0] == list(range(0, 23, 2)) and got[1][0] == list(range(1, 23, 2))
    assert got[1][1] is None
    res, status, steps, polar = got[0][1]
    assert np.array_equal(res, one['results'])
    assert np.array_equal(status, one['status'])
    assert np.array_equal(steps, one['steps'])
    assert np.array_equal(polar, one['polar'])
