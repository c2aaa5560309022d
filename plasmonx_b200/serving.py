"""Spectrum-request serving on one GPU: admission by HBM footprint, resident
geometries, continuous batching, concurrent solves on separate CUDA streams.

A request is one spectrum: a geometry (``Problem`` or ``BemProblem``), its
frequency grid and the solve settings.  The server keeps

* **worker slots** — each worker owns a library context (its own CUDA stream),
  so solves of different geometries run concurrently on the device;
* **resident geometries** — a geometry built for one request (dense T or the
  BEM matrix, the conductance, the tensor-core operand) stays on its worker
  for the next request of the same geometry, until memory is needed;
* **admission by footprint** — before a geometry is built, its device bytes
  (on-memory if they fit, else matrix-free with only the tensor-core operand)
  plus the Krylov state of the batch are reserved against the HBM budget;
  idle resident geometries are evicted (least recently used) to make room,
  and a request that does not fit waits until running batches release memory;
* **continuous batching** -- a refinement request (mixed or FP64-refined) joins
  its geometry's open batch (``plx_batch_*``) as soon as its worker is between
  two outer steps, even while earlier requests are in flight; every step is
  one outer refinement step of all in-flight columns of all the worker's open
  batches together (``plx_batch_step_group``: every inner Arnoldi step is ONE
  grouped tensor-core launch over the geometries' operands), and a request
  leaves with its results as soon as its own columns have converged.  Plain
  FP64 requests (the reference's unrestarted GMRES) are solved as one batch
  of the queued requests of a geometry.

Latency is measured per request from its arrival to its results on the host;
``run_mix`` replays a seeded Poisson arrival stream and reports p50/p99
latency and throughput (freq-solves/s).
"""
import collections
import math
import threading
import time

import numpy as np

from .solver import Batch, Context, Solver

KRYLOV_INNER = 64
MEMORY_RETRIES = 3


def _out_of_memory(e):
    """A device allocation failure (the library's NOMEM / BUDGET statuses, or the
    loop's own refusal)."""
    return isinstance(e, MemoryError) or getattr(e, 'code', None) in (3, 4)


def _is_bem(problem):
    return getattr(problem, 'triangles', None) is not None


def geometry_key(problem):
    """Identity of a geometry: requests with the same key share a resident geometry."""
    key = getattr(problem, 'geometry_key', None)
    return key if key is not None else id(problem)


def build_peak(problem, mode, precision):
    """Device bytes held only while a geometry is built: matrix-free with the
    tensor-core operand, the window of generated T rows its fold reads (up to
    ~6 GB, freed when the operand is done)."""
    n = int(problem.n_var)
    if precision.startswith('mixed') and mode == 'iterative on the fly' and not _is_bem(problem):
        return min(int(6.0e9), 8 * n * n)
    return 0


def footprint(problem, mode, precision, n_cols):
    """Device bytes of a solve: (geometry bytes, batch bytes) for n_cols complex columns.

    Geometry: stored FP64 matrix (on-memory modes), the conductance CSR (about 540
    entries per atom, 20 bytes each), the BF16 high/low tensor-core operand (mixed).
    Batch: the Krylov slabs (FP32 basis of the inner solve for the mixed form, FP64 up
    to the GMRES dimension for the plain form), the work arrays and the k-split
    partials of the contraction."""
    n = int(problem.n_var)
    ld = (n + 63) // 64 * 64
    rows = (n + 255) // 256 * 256
    geo = 0
    if mode != 'iterative on the fly':
        geo += 8 * n * n
    if not _is_bem(problem):
        geo += 20 * 600 * int(problem.n_atoms)
    mixed = precision.startswith('mixed')
    if mixed:
        # the BF16 high/low operand and the k-split partials (at most 148 pieces of
        # 256 x 256 FP32)
        geo += 4 * rows * ld + 148 * 256 * 256 * 4
    if mixed:
        krylov = (KRYLOV_INNER + 1) * n_cols * 2 * n * 4
    else:
        m = min(int(getattr(problem, 'gmres_dim', 1000) or 1000), n)
        krylov = (m + 1) * n_cols * 2 * n * 8
    # work arrays of the outer and inner solves, and the BF16 split of the
    # contraction's input (2 real columns per complex one, 4 bytes per entry)
    work = 12 * n_cols * 2 * n * 8 + (4 * 2 * n_cols * n * 8 + 4 * 2 * n_cols * ld if mixed else 0)
    return geo, krylov + work


class ServeRequest:
    """One spectrum request."""

    def __init__(self, rid, problem, arrival=0.0, precision='mixed_bf16x3', pol_mask=1, tol=None):
        self.id = rid
        self.problem = problem
        self.arrival = float(arrival)
        self.precision = precision
        self.pol_mask = int(pol_mask)
        self.tol = problem.tol if tol is None else float(tol)
        self.key = geometry_key(problem)
        self.n_freq = len(problem.freqs)
        self.t_submit = self.t_start = self.t_done = None
        self.result = None
        self.error = None
        self.mode = None
        self.batch_size = 0
        self.escalated = 0          # frequencies solved again in plain FP64 (mixed form, unconverged)
        self.mem_retries = 0        # times put back after running out of device memory
        self.waiting_memory = False
        self.worker = None
        self.done = threading.Event()

    @property
    def settings(self):
        return (self.precision, self.pol_mask, self.tol)

    @property
    def latency(self):
        return None if self.t_done is None else self.t_done - self.t_submit


class _Resident:
    def __init__(self, solver, mode, geo_bytes):
        self.solver = solver
        self.mode = mode
        self.geo_bytes = geo_bytes
        self.busy = False
        self.last_used = time.perf_counter()


class Server:
    """Request loop over `workers` concurrent slots on one device.

    `solver_factory(problem, ctx, store_t)` builds a resident geometry (default: the
    library's Solver); `context_factory(device)` makes a worker's context.  Both are
    parameters so that the scheduling can be exercised without a GPU.

    Memory accounting: a geometry's bytes are reserved when it is admitted and
    released when its worker has freed it; a batch's Krylov bytes are reserved
    while it runs.  Device memory belongs to the worker's context, so evicted
    geometries are freed by their own worker thread."""

    def __init__(self, device=0, hbm_budget=None, workers=2, solver_factory=None, context_factory=None,
                 batch_factory=None):
        self.device = device
        self.n_workers = int(workers)
        self.solver_factory = solver_factory or (lambda p, ctx, store_t: Solver(p, ctx=ctx, store_t=store_t))
        self.context_factory = context_factory or (lambda dev: Context(dev))
        self.batch_factory = batch_factory or (lambda solver, mode, precision: Batch(solver, mode=mode,
                                                                                   precision=precision))
        self.steps = []              # (worker, geometries, requests, seconds) per batch step
        if hbm_budget is None:
            hbm_budget = self._free_bytes()
        self.budget = int(hbm_budget)
        self.committed = 0          # reserved bytes (resident geometries, running batches)
        self.freeing = 0            # bytes of evicted geometries not yet freed by their worker
        self.lock = threading.Condition()
        self.pending = collections.deque()
        self.queues = [collections.deque() for _ in range(self.n_workers)]
        self.resident = [dict() for _ in range(self.n_workers)]   # key -> _Resident
        self.evicted = [[] for _ in range(self.n_workers)]        # _Resident to free
        self.busy = [False] * self.n_workers
        self.stopping = False
        self.batches = []            # (worker, request ids, mode, seconds)
        self.threads = []
        self.errors = []
        self.min_free = None         # (device free bytes, committed bytes) at the fullest step
        self.escalate = True         # unconverged mixed-precision frequencies are solved again in FP64

    def _free_bytes(self):
        free = self._device_free()
        return 64 << 30 if free is None else int(0.75 * free)

    def _device_free(self):
        try:
            import torch
            return int(torch.cuda.mem_get_info(self.device)[0])
        except Exception:
            return None

    # ---- lifecycle ------------------------------------------------------------
    def start(self):
        for w in range(self.n_workers):
            t = threading.Thread(target=self._worker, args=(w,), daemon=True)
            t.start()
            self.threads.append(t)
        return self

    def stop(self):
        with self.lock:
            self.stopping = True
            self.lock.notify_all()
        for t in self.threads:
            t.join()
        self.threads = []

    def __enter__(self):
        return self.start()

    def __exit__(self, *a):
        self.stop()

    # ---- submission and dispatch ----------------------------------------------
    def submit(self, req):
        req.t_submit = time.perf_counter()
        with self.lock:
            self.pending.append(req)
            self._dispatch()
            self.lock.notify_all()
        return req

    def _dispatch(self):
        """Route pending requests (lock held): to the worker holding their geometry,
        else to the least-loaded worker once admitted; the rest stay pending."""
        still = collections.deque()
        while self.pending:
            req = self.pending.popleft()
            w = self._holder(req.key)
            if w is None:
                w = self._admit(req)
            if w == 'reject':
                req.error = MemoryError('request needs more device memory than the budget (%d bytes)' % self.budget)
                req.t_done = time.perf_counter()
                req.done.set()
            elif w is None:
                still.append(req)
            else:
                req.worker = w
                self.queues[w].append(req)
        self.pending = still

    def _holder(self, key):
        for w in range(self.n_workers):
            if key in self.resident[w] or any(q.key == key for q in self.queues[w]):
                return w
        return None

    def _load(self, w):
        return len(self.queues[w]) + (1 if self.busy[w] else 0)

    def _admit(self, req):
        """Pick a mode and a worker for a new geometry and reserve its bytes
        (lock held): on-memory if it fits, else matrix-free (atomistic only);
        idle resident geometries are evicted to make room."""
        p = req.problem
        modes = ['iterative'] if _is_bem(p) else ['iterative', 'iterative on the fly']
        for mode in modes:
            geo, batch = footprint(p, mode, req.precision, self._block_cols(p, mode, req.precision, self._cols(req)))
            batch += build_peak(p, mode, req.precision)      # transient, checked at admission
            short = self.committed + geo + batch - self.budget
            if short > 0 and short > self.freeing:
                self._evict(short - self.freeing)
            if self.committed + geo + batch <= self.budget:
                w = min(range(self.n_workers), key=self._load)
                self.committed += geo
                req.mode = mode
                req.geo_bytes = geo
                return w
            if self.committed + geo + batch <= self.budget + self.freeing:
                return None          # room is being freed: wait for it
        geo, batch = footprint(p, modes[-1], req.precision,
                               self._block_cols(p, modes[-1], req.precision, self._cols(req)))
        if geo + batch > self.budget:
            return 'reject'          # would not fit even on an empty device
        return None

    def _evict(self, need):
        """Evict idle resident geometries, least recently used first (lock held)."""
        idle = [(r.last_used, w, k) for w in range(self.n_workers) for k, r in self.resident[w].items()
                if not r.busy and not any(q.key == k for q in self.queues[w])]
        for _, w, k in sorted(idle):
            if need <= 0:
                break
            r = self.resident[w].pop(k)
            self.evicted[w].append(r)
            self.freeing += r.geo_bytes
            need -= r.geo_bytes
        self.lock.notify_all()

    @staticmethod
    def _cols(req):
        return req.n_freq * bin(req.pol_mask).count('1')

    def _block_cols(self, problem, mode, precision, cols):
        """Columns a batch holds on the device at once.  The mixed form keeps a
        short inner basis, so a whole batch runs as one block; the plain FP64 GMRES
        keeps its unrestarted basis (up to the GMRES dimension) per column, so a
        batch whose basis would pass a quarter of the budget runs in frequency blocks
        of that size, one after the other (the reference solves one frequency at a
        time)."""
        if precision.startswith('mixed'):
            return cols
        per_col = footprint(problem, mode, precision, 1)[1]
        return max(1, min(cols, int(self.budget // (4 * per_col))))

    # ---- workers --------------------------------------------------------------
    def _free_evicted(self, w):
        with self.lock:
            gone, self.evicted[w] = self.evicted[w], []
        for r in gone:
            r.solver.close()
        if gone:
            with self.lock:
                for r in gone:
                    self.freeing -= r.geo_bytes
                    self.committed -= r.geo_bytes
                self._dispatch()
                self.lock.notify_all()

    def _worker(self, w):
        try:
            ctx = self.context_factory(self.device)
        except Exception as e:          # device failure: report through the requests
            self.errors.append(e)
            return
        # continuous batching state of this worker: geometry key -> open batch
        self._open = getattr(self, '_open', {})
        self._open[w] = {}
        try:
            while True:
                self._free_evicted(w)
                with self.lock:
                    while (not self.queues[w] and not self.evicted[w] and not self._in_flight(w)
                           and not self.stopping):
                        self.lock.wait()
                    if self.evicted[w]:
                        continue
                    if not self.queues[w] and not self._in_flight(w):
                        break        # stopping, nothing queued or in flight
                    joining = self._take_joining(w)
                    plain = [] if joining or self._in_flight(w) else self._take_plain(w)
                    if not joining and not plain and not self._in_flight(w):
                        # queued work that waits for memory another worker holds
                        self.lock.wait(0.05)
                        continue
                if plain:
                    self._plain_batch(w, plain, ctx)
                    continue
                for r in joining:
                    self._join(w, r, ctx)
                if self._in_flight(w):
                    self._step(w)
        finally:
            with self.lock:
                left = list(self.resident[w].values()) + self.evicted[w]
                self.resident[w].clear()
                self.evicted[w] = []
                opened = list(self._open.get(w, {}).values())
                self._open[w] = {}
            for ob in opened:
                try:
                    ob['batch'].close()
                except Exception:
                    pass
            for r in left:
                try:
                    r.solver.close()
                except Exception:
                    pass
            ctx.close()

    # ---- continuous batching (refinement forms) ---------------------------------
    def _in_flight(self, w):
        return any(ob['reqs'] for ob in self._open.get(w, {}).values())

    def _take_joining(self, w):
        """Queued refinement requests that can join this worker's batches now (lock
        held): every one whose geometry has no open batch or an open batch with its
        settings; their batch bytes are reserved."""
        q = self.queues[w]
        out = []
        busy = self._in_flight(w)
        device_busy = any(self._in_flight(v) for v in range(self.n_workers))
        for r in list(q):
            if r.precision == 'fp64':
                continue
            if r.waiting_memory and busy:
                continue                  # out of memory before: waits for this worker to drain
            ob = self._open[w].get(r.key)
            if ob is not None and ob['precision'] != r.precision:
                continue                  # waits until that batch drains
            res = self.resident[w].get(r.key)
            mode = res.mode if res is not None else (r.mode or 'iterative')
            _, bb = footprint(r.problem, mode, r.precision, self._cols(r))
            short = self.committed + bb - self.budget
            if short > 0 and short > self.freeing:
                self._evict(short - self.freeing)     # idle resident geometries first
            if self.committed + bb > self.budget and (out or device_busy):
                continue                  # waits until running batches give their memory back
            r.waiting_memory = False
            r.batch_bytes = bb
            self.committed += bb
            q.remove(r)
            out.append(r)
        return out

    def _join(self, w, r, ctx):
        """Adds a request to its geometry's batch (building the geometry and
        opening the batch on first use)."""
        try:
            ob = self._open[w].get(r.key)
            if ob is None:
                with self.lock:
                    res = self.resident[w].get(r.key)
                if res is None:
                    mode = r.mode or 'iterative'
                    solver = self.solver_factory(r.problem, ctx, mode != 'iterative on the fly')
                    res = _Resident(solver, mode, getattr(r, 'geo_bytes', 0))
                    with self.lock:
                        self.resident[w][r.key] = res
                batch = self.batch_factory(res.solver, res.mode, r.precision)
                ob = {'batch': batch, 'res': res, 'precision': r.precision, 'reqs': {}}
                with self.lock:
                    res.busy = True
                    self._open[w][r.key] = ob
            res = ob['res']
            p = r.problem
            ob['batch'].add(r.id, p.freqs, getattr(p, 'alpha_w', None), r.pol_mask, r.tol)
            r.mode = res.mode
            r.t_start = time.perf_counter()
            r.worker = w
            ob['reqs'][r.id] = r
        except Exception as e:
            if _out_of_memory(e) and r.mem_retries < MEMORY_RETRIES:
                self._requeue(w, r)
            else:
                self._finish(r, error=e)

    def _step(self, w):
        """One outer step of every open batch of this worker with columns in flight:
        a grouped step (one tensor-core launch per inner Arnoldi step over all their
        geometries), then the finished requests are taken out."""
        live = [ob for ob in self._open[w].values() if ob['reqs']]
        batches = [ob['batch'] for ob in live]
        n_req = sum(len(ob['reqs']) for ob in live)
        t0 = time.perf_counter()
        try:
            if len(batches) == 1:
                batches[0].step()
            else:
                type(batches[0]).step_group(batches)
        except Exception as e:
            if _out_of_memory(e):
                # the failed step leaves its batches unusable: close them and run their
                # requests again from the start once memory is free
                for key, ob in list(self._open[w].items()):
                    if not any(ob is x for x in live):
                        continue
                    reqs = list(ob['reqs'].values())
                    ob['reqs'].clear()
                    try:
                        ob['batch'].close()
                    except Exception:
                        pass
                    with self.lock:
                        del self._open[w][key]
                        ob['res'].busy = False
                    for r in reqs:
                        if r.mem_retries < MEMORY_RETRIES:
                            self._requeue(w, r)
                        else:
                            self._finish(r, error=e)
                return
            for ob in live:
                for r in list(ob['reqs'].values()):
                    self._finish(r, error=e)
                ob['reqs'].clear()
            return
        with self.lock:
            self.steps.append((w, len(live), n_req, time.perf_counter() - t0))
            free = self._device_free()
            if free is not None and (self.min_free is None or free < self.min_free[0]):
                self.min_free = (free, self.committed)
        for ob in live:
            for r in ob['reqs'].values():
                r.batch_size = max(r.batch_size, n_req)
                r.geometries_shared = max(getattr(r, 'geometries_shared', 1), len(live))
            while True:
                tag = ob['batch'].poll()
                if tag is None:
                    break
                r = ob['reqs'].pop(tag)
                try:
                    r.result = ob['batch'].take(tag)
                    bad = np.flatnonzero(np.asarray(r.result['status']) != 0)
                    if bad.size and self.escalate and r.precision.startswith('mixed'):
                        self._escalate(w, r, bad)
                    else:
                        self._finish(r)
                except Exception as e:
                    self._finish(r, error=e)
        # drained batches close (a request with other settings may be waiting);
        # their geometries stay resident
        for key, ob in list(self._open[w].items()):
            if not ob['reqs']:
                ob['batch'].close()
                with self.lock:
                    del self._open[w][key]
                    ob['res'].busy = False
                    ob['res'].last_used = time.perf_counter()
                    self._dispatch()
                    self.lock.notify_all()

    def _requeue(self, w, r):
        """An out-of-memory failure (lock not held): the request's batch bytes are
        released and it goes back to the head of its worker's queue, held there until
        that worker has nothing in flight (the memory its running batches hold is
        then free), at most MEMORY_RETRIES times."""
        with self.lock:
            self.committed -= getattr(r, 'batch_bytes', 0)
            r.batch_bytes = 0
            r.result = None
            r.mem_retries += 1
            r.waiting_memory = True
            self.queues[w].appendleft(r)
            self.lock.notify_all()

    def _escalate(self, w, r, bad):
        """Frequencies of a mixed-precision request that did not converge (the
        refinement stalls where cond(A(w)) times the tensor-core operator's
        ~1e-5 error is near one: sodium close to w -> 0) are solved again by the
        plain FP64 GMRES on the same resident geometry; the request finishes when
        that follow-up is merged into its result."""
        import copy
        p = copy.copy(r.problem)
        F = len(r.problem.freqs)
        p.freqs = np.asarray(r.problem.freqs)[bad]
        for name in ('alpha_w', 'eps'):
            v = getattr(r.problem, name, None)
            if v is not None and np.ndim(v) >= 1 and np.shape(v)[-1] == F:
                setattr(p, name, np.asarray(v)[..., bad])
        fr = ServeRequest(-1 - r.id, p, arrival=r.arrival, precision='fp64', pol_mask=r.pol_mask, tol=r.tol)
        fr.key = r.key
        fr.mode = r.mode
        fr.worker = w
        fr.t_submit = time.perf_counter()
        fr.parent, fr.parent_idx = r, bad
        r.escalated = int(bad.size)
        with self.lock:
            self.queues[w].appendleft(fr)
            self.lock.notify_all()

    def _merge_followup(self, fr):
        r, idx = fr.parent, fr.parent_idx
        if fr.error is None and fr.result is not None:
            for k in ('results', 'polar', 'status', 'steps'):
                r.result[k][idx] = fr.result[k]
        self._finish(r, error=fr.error)

    def _finish(self, r, error=None):
        r.error = error if error is not None else r.error
        r.t_done = time.perf_counter()
        with self.lock:
            self.committed -= getattr(r, 'batch_bytes', 0)
            r.batch_bytes = 0
            self.batches.append((r.worker, [r.id], r.mode, r.t_done - (r.t_start or r.t_done)))
            self._dispatch()
            self.lock.notify_all()
        r.done.set()

    # ---- plain FP64 requests: one solve per batch of queued requests -------------
    def _take_plain(self, w):
        q = self.queues[w]
        heads = [r for r in q if r.precision == 'fp64']
        if not heads:
            return []
        head = heads[0]
        batch = [r for r in q if r.key == head.key and r.settings == head.settings]
        for r in batch:
            q.remove(r)
        return batch

    def _plain_batch(self, w, batch, ctx):
        with self.lock:
            self.busy[w] = True
            res = self.resident[w].get(batch[0].key)
            mode = res.mode if res is not None else (batch[0].mode or 'iterative')
            cols = sum(self._cols(r) for r in batch)
            _, batch_bytes = footprint(batch[0].problem, mode, batch[0].precision,
                                       self._block_cols(batch[0].problem, mode, batch[0].precision, cols))
            self.committed += batch_bytes
            if res is not None:
                res.busy = True
        self._run_batch(w, batch, res, mode, ctx)
        with self.lock:
            self.committed -= batch_bytes
            self.busy[w] = False
            r = self.resident[w].get(batch[0].key)
            if r is not None:
                r.busy = False
                r.last_used = time.perf_counter()
            self._dispatch()
            self.lock.notify_all()

    def _run_batch(self, w, batch, res, mode, ctx):
        t0 = time.perf_counter()
        head = batch[0]
        for r in batch:
            r.t_start = t0
            r.batch_size = len(batch)
        try:
            if res is None:
                solver = self.solver_factory(head.problem, ctx, mode != 'iterative on the fly')
                res = _Resident(solver, mode, getattr(head, 'geo_bytes', 0))
                res.busy = True
                with self.lock:
                    self.resident[w][head.key] = res
            freqs = np.concatenate([np.asarray(r.problem.freqs, dtype=np.float64) for r in batch])
            aw = [r.problem.alpha_w for r in batch]
            alpha_w = None if aw[0] is None else np.concatenate([np.asarray(a) for a in aw], axis=1)
            res.solver.set_frequencies(freqs, alpha_w)
            pols = bin(head.pol_mask).count('1')
            cols = len(freqs) * pols
            blk = self._block_cols(head.problem, res.mode, head.precision, cols)
            out = res.solver.solve(mode=res.mode, precision=head.precision, pol_mask=head.pol_mask, tol=head.tol,
                                   freq_block=0 if blk >= cols else max(1, blk // pols))
            if 'error' in out:
                raise out['error']
            off = 0
            for r in batch:
                sl = slice(off, off + r.n_freq)
                r.result = {'results': out['results'][sl], 'polar': out['polar'][sl],
                            'status': out['status'][sl], 'steps': out['steps'][sl]}
                r.mode = res.mode
                off += r.n_freq
        except Exception as e:
            for r in batch:
                r.error = e
        t1 = time.perf_counter()
        with self.lock:
            self.batches.append((w, [r.id for r in batch], res.mode if res is not None else None, t1 - t0))
        for r in batch:
            r.t_done = t1
            r.done.set()
            if getattr(r, 'parent', None) is not None:
                self._merge_followup(r)


def run_mix(server, requests, time_scale=1.0):
    """Replay the requests at their arrival times (seconds, scaled) and wait for all.
    Returns latency percentiles (ms), throughput and the per-request records."""
    requests = sorted(requests, key=lambda r: r.arrival)
    t0 = time.perf_counter()
    for r in requests:
        delay = t0 + r.arrival * time_scale - time.perf_counter()
        if delay > 0:
            time.sleep(delay)
        server.submit(r)
    for r in requests:
        r.done.wait()
    t1 = max(r.t_done for r in requests)
    lat = np.array([r.latency for r in requests]) * 1000.0
    solves = sum(r.n_freq * bin(r.pol_mask).count('1') for r in requests)
    return {'requests': len(requests), 'p50_ms': float(np.percentile(lat, 50)),
            'p99_ms': float(np.percentile(lat, 99)), 'mean_ms': float(lat.mean()),
            'throughput': solves / (t1 - t0), 'unit': 'freq-solves/s', 'wall_s': t1 - t0,
            'batches': len(server.batches), 'errors': sum(r.error is not None for r in requests),
            'error_kinds': dict(collections.Counter('%s: %s' % (type(r.error).__name__, str(r.error)[:80])
                                                    for r in requests if r.error is not None))}


def poisson_arrivals(n, rate, seed):
    rng = np.random.default_rng(seed)
    return np.cumsum(rng.exponential(1.0 / rate, size=n))


def request_pool(n_requests=24, rate=20.0, seed=7, scale='small', precision='mixed_bf16x3'):
    """Seeded serving mix: wFQ Na spheres, wFQFMu Ag/Au spheres and rods, BEM spheres
    and rods, each with 20-400 frequencies in its material's window (the 'full' scale:
    Na 500-20k atoms, Ag/Au 1k-30k atoms, BEM 1k-10k tesserae); 'medium' keeps the same
    kinds at up to 8k atoms, 6k tesserae and 200 frequencies; 'small' at 500-4k atoms /
    tesserae and 20-100 frequencies so a run takes seconds.
    Geometries repeat across requests (a third of the requests reuse an earlier
    geometry), which is what resident geometries and batching serve."""
    from . import configs
    from .bem import bem_surface
    rng = np.random.default_rng(seed)
    arrivals = poisson_arrivals(n_requests, rate, seed)
    if scale == 'full':
        na_r, fmu_atoms, bem_t, fr = (13.0, 46.0), (1000, 30000), (1000, 10000), (20, 400)
    elif scale == 'medium':
        na_r, fmu_atoms, bem_t, fr = (13.0, 32.0), (1000, 8000), (1000, 6000), (20, 200)
    else:
        na_r, fmu_atoms, bem_t, fr = (13.0, 22.0), (500, 4000), (500, 4000), (20, 100)
    cache = []
    reqs = []
    for i, t in enumerate(arrivals):
        nf = int(rng.integers(fr[0], fr[1] + 1))
        if cache and rng.random() < 1.0 / 3.0:
            base = cache[int(rng.integers(len(cache)))]
            prob = _with_freqs(base, nf, rng)
        else:
            kind = rng.choice(['na', 'fmu', 'bem'])
            if kind == 'na':
                prob = configs.particle('Na', 'sphere', float(rng.uniform(*na_r)), n_freq=nf, method='iterative',
                                        tolerance=1e-9, polarization='x')
            elif kind == 'fmu':
                metal = str(rng.choice(['Ag', 'Au']))
                shape = str(rng.choice(['sphere', 'rod']))
                atoms = float(rng.uniform(*fmu_atoms))
                dens = 4.0 / {'Ag': 4.086, 'Au': 4.08}[metal] ** 3
                if shape == 'sphere':
                    r = (3.0 * atoms / (4.0 * math.pi * dens)) ** (1.0 / 3.0)
                    prob = configs.particle(metal, 'sphere', r, n_freq=nf, method='iterative', tolerance=1e-9,
                                            polarization='x')
                else:
                    r = (atoms / (dens * math.pi * (4.0 - 2.0 / 3.0))) ** (1.0 / 3.0)
                    prob = configs.particle(metal, 'rod', r, length=4.0 * r, n_freq=nf, method='iterative',
                                            tolerance=1e-9, polarization='x')
            else:
                shape = str(rng.choice(['sphere', 'rod']))
                prob = bem_surface(int(rng.integers(*bem_t)), shape=shape, n_freq=nf, method='iterative',
                                   tolerance=1e-9, polarization='x', seed=int(rng.integers(1 << 30)))
            prob.geometry_key = ('g', i)
            cache.append(prob)
        reqs.append(ServeRequest(i, prob, arrival=float(t), precision=precision, pol_mask=1,
                                 tol=_tol(prob)))
    return reqs


def _tol(prob):
    # the metric's accuracy: 1e-12 input tolerance (absolute, times sqrt(n)) as in the bench
    return 1e-12 * math.sqrt(prob.n_var)


def _with_freqs(base, nf, rng):
    """A new request on an existing geometry: same object identity key, a new grid
    (a random sub-window of the material's window)."""
    import copy
    prob = copy.copy(base)
    lo, hi = float(base.freqs[0]), float(base.freqs[-1])
    a = rng.uniform(lo, lo + 0.5 * (hi - lo))
    prob.freqs = np.linspace(a, hi, nf)
    if _is_bem(base):
        from .bem import drude_lorentz
        prob.eps = drude_lorentz(prob.freqs)
    elif getattr(base, 'alpha_w', None) is not None:
        from . import materials as M
        names = {'Ag': 'silver etchegoin', 'Au': 'gold etchegoin'}
        prob.alpha_w = np.array([M.fitted(names[t], prob.freqs, 'polar') for t in base.type_names])
    return prob
