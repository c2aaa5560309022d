"""Scheduling of the serving loop (admission by footprint, resident geometries,
continuous batching -- requests joining a batch while others are in flight,
grouped steps over several geometries -- and concurrent workers), exercised with
a stand-in solver and batch on the CPU; the GPU test of the same loop is
test_gpu_serving.py."""
import threading
import time

import numpy as np

from plasmonx_b200 import configs
from plasmonx_b200.serving import build_peak, Server, ServeRequest, footprint, request_pool, run_mix


class FakeContext:
    def __init__(self, dev):
        self.closed = False

    def close(self):
        self.closed = True


class FakeSolver:
    """Returns results[:, 0] = the frequencies it was given; sleeps to simulate work."""
    log = []
    lock = threading.Lock()

    def __init__(self, problem, ctx, store_t, delay=0.05):
        self.problem, self.store_t, self.delay = problem, store_t, delay
        self.closed = False
        with FakeSolver.lock:
            FakeSolver.log.append(('build', id(problem), store_t))

    def set_frequencies(self, freqs, alpha_w=None):
        self.freqs = np.asarray(freqs)

    def solve(self, mode=None, precision=None, pol_mask=None, tol=None, freq_block=0):
        t0 = time.perf_counter()
        time.sleep(self.delay)
        F = len(self.freqs)
        res = np.zeros((F, 20))
        res[:, 0] = self.freqs
        with FakeSolver.lock:
            FakeSolver.log.append(('solve', id(self.problem), mode, F, t0, time.perf_counter(), freq_block))
        return {'results': res, 'polar': np.zeros((F, 3, 3), complex), 'status': np.zeros(F, np.int32),
                'steps': np.zeros((F, 3), np.int32)}

    def close(self):
        self.closed = True


class FakeBatch:
    """Continuous batch stand-in: a request needs 1 + (its frequency count mod 3)
    outer steps; a step sleeps `delay`; results[:, 0] = the request's frequencies."""

    def __init__(self, solver, mode, precision, delay=0.02):
        self.solver, self.mode, self.precision, self.delay = solver, mode, precision, delay
        self.left, self.freqs, self.done = {}, {}, []
        self.closed = False

    def add(self, tag, freqs, alpha_w, pol_mask, tol):
        self.freqs[tag] = np.asarray(freqs)
        self.left[tag] = 1 + len(freqs) % 3

    @property
    def active(self):
        return len(self.left)

    def _advance(self):
        for t in list(self.left):
            self.left[t] -= 1
            if self.left[t] == 0:
                del self.left[t]
                self.done.append(t)

    def step(self):
        FakeBatch.step_group([self])

    @staticmethod
    def step_group(batches):
        t0 = time.perf_counter()
        time.sleep(batches[0].delay)
        for b in batches:
            b._advance()
        with FakeSolver.lock:
            FakeSolver.log.append(('step', tuple(id(b.solver.problem) for b in batches), t0, time.perf_counter()))

    def poll(self):
        return self.done[0] if self.done else None

    def take(self, tag):
        self.done.remove(tag)
        f = self.freqs.pop(tag)
        res = np.zeros((len(f), 20))
        res[:, 0] = f
        return {'results': res, 'polar': np.zeros((len(f), 3, 3), complex), 'status': np.zeros(len(f), np.int32),
                'steps': np.zeros((len(f), 3), np.int32)}

    def close(self):
        self.closed = True


def _server(budget, workers=2):
    FakeSolver.log = []
    return Server(hbm_budget=budget, workers=workers, solver_factory=FakeSolver, context_factory=FakeContext,
                  batch_factory=FakeBatch)


def _na(radius=12.0, nf=5):
    p = configs.particle('Na', 'sphere', radius, n_freq=nf, method='iterative', tolerance=1e-9, polarization='x')
    return p


def _req(i, p, freqs=None, arrival=0.0):
    if freqs is not None:
        import copy
        q = copy.copy(p)
        q.freqs = np.asarray(freqs)
        q.geometry_key = getattr(p, 'geometry_key', id(p))
        p = q
    return ServeRequest(i, p, arrival=arrival, precision='mixed_bf16x3', pol_mask=1, tol=1.0)


def test_requests_join_a_running_batch_and_get_their_own_slice():
    p = _na()
    p.geometry_key = 'na'
    with _server(1 << 40, workers=1) as srv:
        first = srv.submit(_req(0, p, [1.0, 2.0, 3.0, 4.0, 5.0]))      # three outer steps
        time.sleep(0.03)                                              # the first batch is running
        later = [srv.submit(_req(k, p, [10.0 * k, 10.0 * k + 1, 10.0 * k + 2])) for k in (1, 2, 3)]
        for r in [first] + later:
            assert r.done.wait(5)
    for r in later:
        assert r.t_start < first.t_done                   # joined while the first was in flight
        assert r.batch_size >= 2
        np.testing.assert_array_equal(r.result['results'][:, 0], r.problem.freqs)
    builds = [e for e in FakeSolver.log if e[0] == 'build']
    assert len(builds) == 1                               # the geometry stayed resident


def test_two_geometries_on_one_worker_share_grouped_steps():
    a, b = _na(12.0), _na(13.0)
    with _server(1 << 40, workers=1) as srv:
        ra = srv.submit(_req(0, a, [1.0, 2.0, 3.0, 4.0, 5.0]))
        rb = srv.submit(_req(1, b, [6.0, 7.0, 8.0, 9.0, 10.0]))
        assert ra.done.wait(5) and rb.done.wait(5)
    grouped = [e for e in FakeSolver.log if e[0] == 'step' and len(e[1]) == 2]
    assert grouped and set(grouped[0][1]) == {id(ra.problem), id(rb.problem)}
    assert ra.geometries_shared == 2 and rb.geometries_shared == 2
    np.testing.assert_array_equal(rb.result['results'][:, 0], rb.problem.freqs)


def test_admission_picks_matrix_free_when_t_does_not_fit_and_rejects_too_large():
    # large enough that the matrix-free build's window of generated T rows (~6 GB,
    # held while the geometry is built) is smaller than T itself
    p = configs.particle('Ag', 'sphere', 33.0, n_freq=4, method='iterative', tolerance=1e-9)
    geo_mem, bat = footprint(p, 'iterative', 'mixed_bf16x3', 4)
    geo_otf, _ = footprint(p, 'iterative on the fly', 'mixed_bf16x3', 4)
    peak = build_peak(p, 'iterative on the fly', 'mixed_bf16x3')
    assert peak < geo_mem - geo_otf
    budget = geo_otf + bat + peak + (geo_mem - geo_otf - peak) // 2
    with _server(budget) as srv:
        r = srv.submit(ServeRequest(0, p, precision='mixed_bf16x3', pol_mask=1, tol=1.0))
        assert r.done.wait(5)
        assert r.error is None and r.mode == 'iterative on the fly'
    with _server(geo_otf // 2) as srv:
        r = srv.submit(ServeRequest(1, p, precision='mixed_bf16x3', pol_mask=1, tol=1.0))
        assert r.done.wait(5)
        assert isinstance(r.error, MemoryError)


def test_idle_geometry_is_evicted_for_a_new_one():
    a, b = _na(12.0), _na(14.0)
    geo, bat = footprint(b, 'iterative', 'mixed_bf16x3', 5)
    with _server(geo + bat + geo // 2, workers=1) as srv:
        ra = srv.submit(_req(0, a))
        assert ra.done.wait(5)
        rb = srv.submit(_req(1, b))
        assert rb.done.wait(5)
        assert rb.error is None
        assert srv.committed <= srv.budget
    assert [e[1] for e in FakeSolver.log if e[0] == 'build'] == [id(a), id(b)]


def test_two_workers_overlap_different_geometries():
    a, b = _na(12.0), _na(13.0)
    with _server(1 << 40, workers=2) as srv:
        ra, rb = srv.submit(_req(0, a)), srv.submit(_req(1, b))
        assert ra.done.wait(5) and rb.done.wait(5)
    assert ra.worker != rb.worker
    sa = [(e[2], e[3]) for e in FakeSolver.log if e[0] == 'step' and e[1] == (id(a),)]
    sb = [(e[2], e[3]) for e in FakeSolver.log if e[0] == 'step' and e[1] == (id(b),)]
    assert sa and sb
    # the two workers' steps ran at the same time
    assert max(sa[0][0], sb[0][0]) < min(sa[-1][1], sb[-1][1])


def test_plain_fp64_requests_are_solved_as_one_batch():
    p = _na()
    p.geometry_key = 'na64'
    with _server(1 << 40, workers=1) as srv:
        rs = [ServeRequest(k, p, precision='fp64', pol_mask=1, tol=1.0) for k in range(3)]
        for r in rs:
            srv.submit(r)
        for r in rs:
            assert r.done.wait(5) and r.error is None
    solves = [e for e in FakeSolver.log if e[0] == 'solve']
    assert 1 <= len(solves) <= 3


def test_mix_statistics_and_pool_is_seeded():
    pool1 = request_pool(n_requests=6, rate=200.0, seed=3)
    pool2 = request_pool(n_requests=6, rate=200.0, seed=3)
    assert [r.n_freq for r in pool1] == [r.n_freq for r in pool2]
    assert [r.arrival for r in pool1] == [r.arrival for r in pool2]
    with _server(1 << 44, workers=2) as srv:
        st = run_mix(srv, pool1)
    assert st['requests'] == 6 and st['errors'] == 0
    assert st['p50_ms'] <= st['p99_ms'] and st['throughput'] > 0


def test_plain_fp64_batch_runs_in_blocks_that_fit():
    """An unrestarted FP64 basis for every frequency would not fit: the plain arm
    solves the batch in frequency blocks of at most a quarter of the budget."""
    p = _na(nf=20)
    p.geometry_key = 'na64-blocks'
    geo, per_col = footprint(p, 'iterative', 'fp64', 1)
    budget = geo + 4 * 5 * per_col                    # room for blocks of about 5 columns
    block = budget // (4 * per_col)
    with _server(budget, workers=1) as srv:
        r = ServeRequest(0, p, precision='fp64', pol_mask=1, tol=1.0)
        srv.submit(r)
        assert r.done.wait(5) and r.error is None, r.error
    solves = [e for e in FakeSolver.log if e[0] == 'solve' and e[1] == id(p)]
    assert len(solves) == 1 and solves[0][6] == block < r.n_freq
    assert r.result['results'].shape[0] == r.n_freq


class StallingBatch(FakeBatch):
    """Reports every other frequency of a request as not converged (status 5)."""

    def take(self, tag):
        out = FakeBatch.take(self, tag)
        out['status'][::2] = 5
        out['results'][::2, 0] = -1.0          # what a stalled refinement leaves behind
        return out


def test_unconverged_mixed_frequencies_are_solved_again_in_fp64():
    p = _na(nf=7)
    p.geometry_key = 'na-stall'
    FakeSolver.log = []
    srv = Server(hbm_budget=1 << 40, workers=1, solver_factory=FakeSolver, context_factory=FakeContext,
                 batch_factory=StallingBatch)
    with srv:
        r = srv.submit(ServeRequest(0, p, precision='mixed_bf16x3', pol_mask=1, tol=1.0))
        assert r.done.wait(5) and r.error is None, r.error
    assert r.escalated == 4
    assert np.all(r.result['status'] == 0)
    # the follow-up solved exactly the stalled frequencies on the resident geometry
    solves = [e for e in FakeSolver.log if e[0] == 'solve']
    assert len(solves) == 1 and solves[0][3] == 4
    assert [e for e in FakeSolver.log if e[0] == 'build'] == [('build', id(p), True)]
    np.testing.assert_array_equal(r.result['results'][:, 0], p.freqs)


class OnceOutOfMemoryBatch(FakeBatch):
    """The first outer step of the run fails the way a device allocation does."""
    failed = False

    @staticmethod
    def step_group(batches):
        if not OnceOutOfMemoryBatch.failed:
            OnceOutOfMemoryBatch.failed = True
            raise MemoryError('device allocation failed')
        FakeBatch.step_group(batches)

    def step(self):
        OnceOutOfMemoryBatch.step_group([self])


def test_requests_of_a_step_that_ran_out_of_memory_run_again():
    p = _na(nf=5)
    p.geometry_key = 'na-oom'
    FakeSolver.log = []
    OnceOutOfMemoryBatch.failed = False
    srv = Server(hbm_budget=1 << 40, workers=1, solver_factory=FakeSolver, context_factory=FakeContext,
                 batch_factory=OnceOutOfMemoryBatch)
    with srv:
        rs = [srv.submit(_req(k, p, [1.0 + k, 2.0 + k, 3.0 + k])) for k in range(3)]
        for r in rs:
            assert r.done.wait(5)
    assert OnceOutOfMemoryBatch.failed
    for r in rs:
        assert r.error is None, r.error
        np.testing.assert_array_equal(r.result['results'][:, 0], r.problem.freqs)
    assert max(r.mem_retries for r in rs) == 1
    # every batch reservation was given back, only the resident geometry's remains
    assert srv.committed == footprint(p, 'iterative', 'mixed_bf16x3', 1)[0]
    builds = [e for e in FakeSolver.log if e[0] == 'build']
    assert len(builds) == 1                                   # the geometry stayed resident
