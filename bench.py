"""Benchmark of the per-frequency response solve on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--config ag_sphere|na_sphere|bowtie|bem_sphere|bem_rod|fq_water|fqfmu_water|field_grid]
                    [--precision fp64|mixed_bf16x3] [--n-tess 2000] [--bem-variant dpcm|iefpcm]

Workload (default): the wFQFMu silver sphere -- fcc a = 4.086 A cut to a 35 A
sphere, 10,473 atoms, 41,892 complex unknowns -- with the reference's default
Ag parameters, 201 frequencies over 3.0-4.5 eV, x polarisation, on-memory
mode.  Synthetic, seeded geometry; the dense T (14.0 GB FP64) is far larger
than L2, so every step streams it from HBM (no L2 flush needed).

Accuracy: the metric is quoted at <= 1e-6 relative error of sigma_abs.  The
reference's default input tolerance (1e-9, i.e. ||b - A x|| < 1e-9 sqrt(n_var),
a relative residual of ~2e-5 here) leaves sigma_abs errors of ~3e-5, so the
benchmark uses an input tolerance of 1e-12 (same absolute test, 1000x
tighter) for both forms; each line reports the measured sigma_abs error of
five frequencies against an FP64 refinement solved to a 1e-11 relative
residual.  The headline form is the mixed-precision refinement
(--precision mixed_bf16x3); the plain FP64 GMRES of the reference's
algorithm is timed on the same spectrum in the same run.

One step = one spectrum: every frequency solved (201 freq-solves).  `value`
is freq-solves/s over all ranks from the library's own CUDA-event timing of
each solve (max over ranks); `e2e` is the same metric through the public
Python API with host buffers: geometry upload and build, frequency tables,
solve, results back to the host.  Under torchrun (N ranks, one per GPU) the
spectrum has N times the frequencies over the same window, dealt round-robin
into one block of the workload's frequency count per rank
(plasmonx_b200.spectrum): every rank keeps its own resident geometry and
Krylov state and the results rows are gathered to rank 0, the only
collective on the data path (weak scaling: fixed work per rank).

Serving leg (`serving` in the line): a seeded Poisson stream of spectrum
requests (wFQ Na spheres, wFQFMu Ag/Au spheres and rods, BEM spheres and
rods; `--serving-scale small` keeps them at 500-4k atoms or tesserae and
20-100 frequencies) through plasmonx_b200.serving (admission by HBM
footprint, resident geometries, batching, two concurrent workers), reported as
p50/p99 request latency and freq-solves/s.

`--impl reference` times the reference's algorithm on the host CPU, per part:
the product of the workload's mode (on-memory: zgemv of the stored complex
matrix, timed on a row slab and scaled; on the fly: the threaded C port of the
reference's pair loops, oracle/pairs.c; BEM: dense D x) over at least 20
products per run, and the CGS2 orthogonalisation at the mean basis size, then
composes them into freq-solves/s with the Arnoldi step count per
frequency-solve (marked extrapolated: a whole spectrum takes hours).

Static workloads (--config fq_water / fqfmu_water): the static FQ / FQFMu solve
(ground state: charges and energy) of a seeded cluster of --waters rigid water
molecules (default 3000 FQ, 9,000 atoms and 12,000 unknowns; FQFMu 1000,
13,000 unknowns) with the reference test's water parameters.  One step = one
solve: the static matrix built on the device, the charge constraints
eliminated, the Cholesky factorisation, the energy.  The CPU arm times the
oracle's NumPy restatement (threaded LAPACK LU of the full system).  A step
takes milliseconds: run --steps 100 so that the clock sampler sees the timed
region.

Analysis workload (--config field_grid): |E|/E0 and the plasmon density of a
wFQFMu solution (seeded synthetic charges and dipoles; the cost does not depend
on their values) of a 20 A silver sphere (1,961 atoms) on a --grid^3 cubic
grid (default 100^3 = 1e6 points, the atoms' box widened by 10 A), the
reference analysis program's field / density step.  One step = the whole grid.
`value` is grid points/s from the kernel's CUDA-event time, `e2e` the same
through Solver.field_at_points with host points in and host field and density
out.  The line also times the device neighbour counts (plx_neighbour_counts)
of the default 10,473-atom silver sphere against the host all-pairs count.

BEM workloads (--config bem_sphere / bem_rod): a 10 nm sphere or a 40 x 10 nm
prolate rod meshed into --n-tess tesserae (20 nu^2; 2000, 8000, 20480) with a
seeded 2% radial jitter, Drude-Lorentz eps(w) in vacuum, 301 frequencies over
1.5-4.5 eV, x polarisation, on-memory GMRES.  The CPU arm there times the
reference's on-memory product, the dense D x of the oracle (threaded BLAS).
"""
import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = 'freq-solves/s at <=1e-6 rel sigma_abs err'
PEAKS_FALLBACK = {'hbm_gbs': 6650.0, 'bf16_tflops': 1590.0, 'bf16_tflops_sustained': 1400.0}
# Arnoldi steps per frequency-solve of the reference's GMRES (the plain FP64
# form) at the bench's input tolerance 1e-12, mean over each workload's
# spectrum, measured on B200; used to turn the CPU arm's timed products and
# orthogonalisations into freq-solves/s.
STEPS_PER_SOLVE = {'ag_sphere': 335.6, 'na_sphere': 60.0, 'bowtie': 600.0, 'bem_sphere': 60.0, 'bem_rod': 60.0}
# measured DRAM bytes / operand bytes of the tensor-core contraction: ncu of the first two
# launches of a 21,560-unknown sphere at 402 columns (two column tiles that share each
# operand tile through L2): 1.972 GB read + 0.065 GB written per launch, operand 1.877 GB
TRAFFIC_RATIO = (1.972 + 0.065) / 1.877


def contraction_bound(roof, hbm_gbs):
    """The tensor-core launch's own bound, the slower of streaming its operand once
    at the measured copy bandwidth and issuing its products at the tensor peak; when
    the operand stream binds (the one-product form, few columns) the roofline is
    stated in GB/s against the copy bandwidth, the algorithmic TFLOP/s kept beside."""
    avg_ms = roof['avg_launch_ms']
    t_hbm = roof['bytes_per_launch'] / (hbm_gbs * 1e9) * 1e3
    t_mma = roof['issued_tensor_tflops'] * avg_ms / roof['peak']
    roof.update({'hbm_bound_ms': t_hbm, 'tensor_issue_bound_ms': t_mma, 'bound_frac': max(t_hbm, t_mma) / avg_ms,
                 'binding': 'hbm' if t_hbm > t_mma else 'tensor issue'})
    if t_hbm > t_mma:
        roof.update({'bound': 'hbm', 'achieved_algorithmic_tflops': roof['achieved'],
                     'tensor_peak_tflops': roof['peak'], 'achieved': roof['achieved_hbm_gbs'], 'peak': hbm_gbs,
                     'unit': 'GB/s', 'frac': roof['achieved_hbm_gbs'] / hbm_gbs})
    return roof


def peaks():
    p = os.path.join(ROOT, 'MEASURED_PEAKS.json')
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return d, 'measured'
    return PEAKS_FALLBACK, 'fallback'


def make_problem(name, n_freq=None, method='iterative', polarization='x', radius=None, n_tess=2000,
                 bem_variant='dpcm', bowtie_edge=80.0, bem_green='approximate'):
    from plasmonx_b200 import configs
    if name in ('bem_sphere', 'bem_rod'):
        from plasmonx_b200.bem import bem_surface
        return bem_surface(n_tess, variant=bem_variant, shape=name[4:], n_freq=n_freq or 301, method=method,
                           tolerance=1e-9, polarization=polarization, gmres_dim=1000, green=bem_green)
    if name == 'ag_sphere':
        return configs.ag_sphere(radius=radius or 35.0, n_freq=n_freq or 201, method=method, tolerance=1e-9,
                                 polarization=polarization, gmres_dim=1000)
    if name == 'na_sphere':
        return configs.na_sphere(radius=20.0, n_freq=n_freq or 61, method=method, tolerance=1e-8,
                                 polarization=polarization)
    if name == 'bowtie':
        return configs.agau_bowtie(edge=bowtie_edge, n_freq=n_freq or 201, method='iterative on the fly',
                                   tolerance=1e-9, polarization=polarization)
    raise ValueError(name)


def is_bem(prob):
    return getattr(prob, 'triangles', None) is not None


def oracle_fixture(args, prob):
    """The oracle's solutions of this workload at five frequencies, when
    tests/golden/large holds them (default silver sphere, 80 A bow-tie), checked
    against the geometry before use; None otherwise."""
    name = {'ag_sphere': 'ag_sphere_r35', 'bowtie': 'agau_bowtie_e80'}.get(args.config)
    if name is None or (args.config == 'ag_sphere' and args.radius not in (None, 35.0)) or \
            (args.config == 'bowtie' and args.bowtie_edge != 80.0) or len(prob.freqs) != 201:
        return None
    path = os.path.join(ROOT, 'tests', 'golden', 'large', name + '.json')
    if not os.path.exists(path):
        return None
    with open(path) as f:
        fx = json.load(f)
    c = np.asarray(prob.coord, dtype=np.float64)
    if int(prob.n_atoms) != fx['geometry']['n_atoms'] or \
            abs(float(np.sum(c)) - fx['geometry']['coord_sum']) > 1e-9 * max(1.0, fx['geometry']['coord_abs_sum']):
        return None
    fx['reference'] = ("oracle fixture tests/golden/large/%s.json: the reference GMRES restated on the CPU "
                       "(C port of the on-the-fly product), refined in FP64 to a relative residual of at most %.1e"
                       % (name, max(fx['true_rel_residual'])))
    return fx


def workload_desc(name, prob):
    if is_bem(prob):
        return {'workload': 'BEM %s %s, %s Green function' % (prob.variant.upper(),
                                                               {'bem_sphere': 'sphere R=10 nm',
                                                                'bem_rod': 'prolate rod 40 x 10 nm'}[name],
                                                               prob.green),
                'n_tess': int(prob.n_tess), 'n_var': int(prob.n_var), 'n_freq': int(len(prob.freqs)),
                'polarization': prob.polarization, 'mode': prob.method, 'tolerance': prob.tolerance_input,
                'l2': 'inputs larger than L2 (stored D %.2f GB)' % (8.0 * prob.n_var ** 2 / 1e9)
                if 8.0 * prob.n_var ** 2 > 126e6 else 'stored D %.0f MB fits in L2 (not flushed)'
                % (8.0 * prob.n_var ** 2 / 1e6)}
    return {'workload': {'ag_sphere': 'wFQFMu Ag fcc sphere R=35 A',
                         'na_sphere': 'wFQ Na bcc sphere R=20 A',
                         'bowtie': 'wFQFMu Ag-Au bow-tie'}[name],
            'n_atoms': int(prob.n_atoms), 'n_var': int(prob.n_var), 'n_freq': int(len(prob.freqs)),
            'polarization': prob.polarization, 'mode': prob.method, 'tolerance': prob.tolerance_input,
            'l2': ('inputs larger than L2 (stored T %.1f GB)' % (8.0 * prob.n_var ** 2 / 1e9))
            if 8.0 * prob.n_var ** 2 > 126e6 else
            'stored T %.1f MB fits in L2 (not flushed between steps)' % (8.0 * prob.n_var ** 2 / 1e6)}


class Clocks:
    """nvidia-smi sampler running during the timed region."""

    def __init__(self, device):
        self.device = device
        self.proc = None
        self.lines = []

    def __enter__(self):
        q = ('clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,'
             'clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,'
             'clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap')
        try:
            self.proc = subprocess.Popen(['nvidia-smi', '-i', str(self.device), '--query-gpu=' + q,
                                          '--format=csv,noheader,nounits', '-lms', '200'],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            self.proc.wait()
            self.t.join(timeout=2)

    def summary(self):
        sm, mx, reasons = [], [], set()
        names = ['hw_slowdown', 'hw_thermal_slowdown', 'sw_thermal_slowdown', 'sw_power_cap']
        for ln in self.lines:
            p = [x.strip() for x in ln.split(',')]
            if len(p) < 8:
                continue
            try:
                sm.append(float(p[0]))
                mx.append(float(p[1]))
            except ValueError:
                continue
            for nm, v in zip(names, p[4:8]):
                if v.lower().startswith('active'):
                    reasons.add(nm)
        if not sm:
            return {'sm_mhz': None, 'sm_max_mhz': None, 'reasons': ['no samples']}
        return {'sm_mhz': float(np.median(sm)), 'sm_max_mhz': float(max(mx)), 'reasons': sorted(reasons),
                'samples': len(sm)}


def dist_setup(backend=None):
    """One process per GPU (torchrun); NCCL on GPUs, gloo when there is no GPU."""
    world = int(os.environ.get('WORLD_SIZE', '1'))
    rank = int(os.environ.get('RANK', '0'))
    local = int(os.environ.get('LOCAL_RANK', '0'))
    pg = None
    if world > 1:
        import datetime
        import torch
        import torch.distributed as dist
        backend = backend or ('nccl' if torch.cuda.is_available() else 'gloo')
        kw = {}
        if backend == 'nccl':
            torch.cuda.set_device(local)
            kw['device_id'] = torch.device('cuda', local)
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=600), **kw)
        pg = dist
    return rank, world, local, pg


def _dev(pg, local):
    return 'cuda:%d' % local if pg.get_backend() == 'nccl' else 'cpu'


def allmax(pg, v, local):
    if pg is None:
        return v
    import torch
    t = torch.tensor([v], dtype=torch.float64, device=_dev(pg, local))
    pg.all_reduce(t, op=pg.ReduceOp.MAX)
    return float(t.item())


def allsum(pg, v, local):
    if pg is None:
        return v
    import torch
    t = torch.tensor([v], dtype=torch.float64, device=_dev(pg, local))
    pg.all_reduce(t, op=pg.ReduceOp.SUM)
    return float(t.item())


def barrier(pg, local):
    if pg is not None:
        import torch
        if pg.get_backend() == 'nccl':
            torch.cuda.synchronize(local)
        pg.barrier()


def job_throughput(pg, local, solves, device_ms):
    """Whole-job freq-solves/s: all ranks' solves over the slowest rank's device time."""
    total = allsum(pg, float(solves), local)
    slowest = allmax(pg, float(device_ms), local)
    return total / (slowest / 1000.0), total, slowest


def _blas_threads():
    try:
        from threadpoolctl import threadpool_info
        return max([d.get('num_threads', 1) for d in threadpool_info() if d.get('user_api') == 'blas'] or [1])
    except Exception:
        return os.cpu_count() or 1


def _time_products(matvec, x, n_min, budget_s):
    """Mean seconds per product over at least n_min products (more while the budget lasts)."""
    matvec(0, x)
    done, t0 = 0, time.perf_counter()
    while done < n_min or (time.perf_counter() - t0 < budget_s and done < 200):
        x = matvec(done, x)
        x /= np.linalg.norm(x)
        done += 1
    return (time.perf_counter() - t0) / done, done


def _time_orthogonalisation(n, j, reps=5):
    """Seconds of one Arnoldi orthogonalisation of the reference at basis size j:
    classical Gram-Schmidt with one re-orthogonalisation, four zgemv over the
    n x j basis (gmres_module.f90:123-142; modified Gram-Schmidt below j = 25
    moves the same bytes as 2 j vector operations)."""
    rng = np.random.default_rng(1)
    V = np.full((n, max(j, 1)), 0.5 + 0.25j)
    V[:, 0] = rng.standard_normal(n)
    w = rng.standard_normal(n) + 1j * rng.standard_normal(n)
    t0 = time.perf_counter()
    for _ in range(reps):
        h = V.conj().T @ w
        w = w - V @ h
        t = V.conj().T @ w
        w = w - V @ t
        w /= np.linalg.norm(w)
    return (time.perf_counter() - t0) / reps


def _lu_reference(prob, n, budget_s):
    """The reference's inversion mode on the host cores: per frequency a complex LU
    of the n x n matrix and the solves for the three field directions (zgetrf +
    zgetrs, algorithm_module.f90:510-541), threaded LAPACK.  Timed at n when the
    factorisation is short, else on a 4,000-unknown matrix scaled by (n / 4000)^3."""
    from scipy.linalg import lu_factor, lu_solve
    ns = min(n, 4000)
    rng = np.random.default_rng(3)
    A = rng.standard_normal((ns, ns)) + 1j * rng.standard_normal((ns, ns)) + ns * np.eye(ns)
    B = rng.standard_normal((ns, 3)) + 0j
    lu_solve(lu_factor(A), B)
    done, t0 = 0, time.perf_counter()
    while done < 1 or (time.perf_counter() - t0 < budget_s and done < 20):
        lu_solve(lu_factor(A, overwrite_a=False, check_finite=False), B, check_finite=False)
        done += 1
    t = (time.perf_counter() - t0) / done * (n / ns) ** 3
    scaled = '' if ns == n else ', scaled by (%d / %d)^3' % (n, ns)
    return {'value': 1.0 / t, 'unit': 'freq-solves/s', 'cores': int(_blas_threads()), 'kind': 'port',
            'extrapolated': ns != n,
            'sample': 'complex LU + 3 solves (zgetrf/zgetrs, threaded LAPACK) of a %d x %d matrix, %d timed%s'
                      % (ns, ns, done, scaled),
            'product_s': None, 'orthogonalisation_s': None, 'steps_per_solve': None}


def cpu_reference(prob, steps_per_solve, n_min=20, budget_s=8.0):
    """The reference's per-frequency GMRES on the host cores, timed per part and
    composed into freq-solves/s (extrapolated: a whole spectrum takes hours).

    Per Arnoldi step the reference does one product and one orthogonalisation;
    a freq-solve of s steps does s products plus one for the true residual, and
    s orthogonalisations whose mean basis size is (s + 1) / 2.  The product is
      on-memory atomistic: zgemv of the stored complex n x n matrix
        (gmres_module.f90:111-119 on matrix_iterative, algorithm_module.f90:356-358),
        timed on a row slab of that matrix and scaled to n rows;
      on-the-fly atomistic: the C port of product_q_block_x / product_mu_block_x
        and the conductance rows (oracle/pairs.c);
      BEM: the dense complex D x of the oracle (threaded BLAS).
    """
    s_steps = float(steps_per_solve)
    n = int(prob.n_var)
    if prob.method == 'inversion':
        return _lu_reference(prob, n, budget_s)
    if is_bem(prob):
        import tempfile
        from oracle import bem as obem
        with tempfile.TemporaryDirectory() as d:
            o = obem.Bem(prob.write_keyword_files(d, 'bench'))
        D = np.ascontiguousarray(o.D).astype(np.complex128)

        def matvec(i, v):
            return D @ v + o.z(i % len(o.freqs)) * v
        x = np.random.default_rng(0).standard_normal(n) + 0j
        t_mv, done = _time_products(matvec, x, n_min, budget_s)
        what = 'dense complex D x (zgemv, threaded BLAS) of the %d-tessera operator' % n
        cores = _blas_threads()
    elif prob.method == 'iterative':
        rows = min(n, max(1024, int(2.0e9 // (16 * n))))
        A = np.full((rows, n), 0.5 + 0.25j)
        A[:, 0] = 1.0

        def matvec(i, v):
            y = v.copy()
            y[:rows] = A @ v
            return y
        x = np.random.default_rng(0).standard_normal(n) + 0j
        t_slab, done = _time_products(matvec, x, n_min, budget_s)
        t_mv = t_slab * n / rows
        what = ('zgemv of the stored complex matrix (on-memory mode), a %d-row slab of the %d x %d matrix timed and '
                'scaled to %d rows' % (rows, n, n, n))
        cores = _blas_threads()
        del A
    else:
        from oracle import keywords, model
        from oracle.cpu_baseline import CpuOperator
        s = model.System.from_keywords(keywords.read_keyword_text(prob.to_keyword_text()))
        op = CpuOperator(s)
        x = np.random.default_rng(0).standard_normal(n) + 1j * np.random.default_rng(1).standard_normal(n)
        t_mv, done = _time_products(lambda i, v: op.matvec(i % len(s.freqs), v), x, min(n_min, 5), budget_s)
        what = "on-the-fly A x of the C port of the reference's pair loops"
        cores = op.n_threads
    j_mid = max(1, int(round((s_steps + 1) / 2)))
    t_orth = _time_orthogonalisation(n, j_mid)
    t_solve = (s_steps + 1) * t_mv + s_steps * t_orth
    return {'value': 1.0 / t_solve, 'unit': 'freq-solves/s', 'cores': int(cores), 'kind': 'port',
            'extrapolated': True,
            'sample': '%s: %d products timed, %.4f s each; CGS2 orthogonalisation at basis size %d: %.4f s; '
                      'x %.1f Arnoldi steps per freq-solve' % (what, done, t_mv, j_mid, t_orth, s_steps),
            'product_s': t_mv, 'orthogonalisation_s': t_orth, 'steps_per_solve': s_steps}


STATIC_METRIC = 'static solves/s (ground state: charges and energy, FP64)'


def static_problem(args):
    from plasmonx_b200.static import water_cluster
    ff = 'fq' if args.config == 'fq_water' else 'fqfmu'
    n_mol = args.waters or (3000 if ff == 'fq' else 1000)
    return water_cluster(n_mol, ff, what='energy', seed=11)


def static_desc(prob):
    return {'workload': '%s water cluster, %d molecules, %s kernel, ground state'
                        % (prob.forcefield.upper(), prob.n_mol, prob.kernel),
            'n_atoms': int(prob.n_atoms), 'n_var': int(prob.n_var),
            'l2': 'inputs larger than L2 (static matrix %.2f GB)' % (8.0 * prob.n_var ** 2 / 1e9)}


def static_cpu(prob):
    """One solve of the oracle's restatement (threaded LAPACK) -> (solves/s, seconds)."""
    from oracle import static as ost
    o = ost.Static(prob.forcefield, prob.kernel, prob.coord, prob.atom_types, prob.apm, prob.chi, prob.eta,
                   prob.alpha, prob.r_q, prob.r_mu, prob.rhs_form, prob.e0)
    t0 = time.perf_counter()
    o.solve('energy')
    dt = time.perf_counter() - t0
    return 1.0 / dt, dt


def run_static(args):
    rank, world, local, pg = dist_setup()
    from plasmonx_b200.solver import Context
    from plasmonx_b200.static import StaticSolver
    prob = static_problem(args)
    ctx = Context(local)
    solver = StaticSolver(prob, ctx=ctx)
    for _ in range(args.warmup):
        solver.solve()
    barrier(pg, local)
    ctx.profile(True)
    launches0 = ctx.launches
    with Clocks(local) as clk:
        barrier(pg, local)
        t0 = time.perf_counter()
        for _ in range(args.steps):
            out = solver.solve()
        barrier(pg, local)
        wall = time.perf_counter() - t0
    launches = ctx.launches - launches0
    asm, fac = ctx.profile_read(5), ctx.profile_read(6)
    ctx.profile(False)
    dev_ms = asm['ms'] + fac['ms']
    value, solves, total_ms = job_throughput(pg, local, args.steps, dev_ms)
    # end to end through the public API: host geometry in, variables and energy out
    e2e = []
    for _ in range(max(1, args.e2e_steps)):
        barrier(pg, local)
        t0 = time.perf_counter()
        o2 = StaticSolver(prob, ctx=ctx).solve()
        barrier(pg, local)
        e2e.append(time.perf_counter() - t0)
    e2e_s = allmax(pg, float(np.mean(e2e)), local)
    h2d = prob.coord.nbytes + prob.atom_types.nbytes + prob.apm.nbytes + 5 * prob.chi.nbytes
    pk, pk_kind = peaks()
    asm_ms = asm['ms'] / max(1, asm['launches'])
    asm_bytes = asm['bytes'] / max(1, asm['launches'])
    fac_ms = fac['ms'] / max(1, fac['launches'])
    roof = {'kernel': 'static assembly: static_matrix_kernel, Householder reflections, gather of the reduced '
                      'matrix (bytes: the matrix written once and the reduced matrix once)', 'bound': 'hbm',
            'achieved': asm_bytes / (asm_ms / 1000.0) / 1e9, 'peak': pk['hbm_gbs'], 'unit': 'GB/s',
            'peak_kind': pk_kind, 'bytes_per_launch': asm_bytes, 'avg_launch_ms': asm_ms, 'traffic': None,
            'note': 'the dense factorisation (cuSOLVER dpotrf/dpotrs of the constraint-eliminated system, or '
                    'dgetrf/dgetrs of the full one; a library) takes the rest of the step: %.2f ms, %.1f FP64 TFLOP/s'
                    % (fac_ms, fac['flops'] / max(1, fac['launches']) / (fac_ms / 1e3) / 1e12)}
    roof['frac'] = roof['achieved'] / roof['peak']
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        v, dt = static_cpu(prob)
        cpu = {'value': v, 'unit': 'solves/s', 'cores': os.cpu_count(), 'kind': 'port',
               'sample': 'one full solve of the NumPy restatement (threaded LAPACK LU), %.2f s' % dt}
    if rank == 0:
        line = {'metric': STATIC_METRIC, 'value': value, 'unit': 'solves/s', 'n_gpus': world, 'steps': args.steps,
                'warmup': args.warmup, 'ms_per_step': total_ms / args.steps, 'higher_is_better': True,
                'scaling': 'weak', 'vs_baseline': None, 'dtype': 'f64',
                'data': 'synthetic (seeded water cluster, reference test parameters)', 'config': static_desc(prob),
                'e2e': {'value': 1.0 / e2e_s, 'unit': 'solves/s', 'h2d_bytes_per_step': int(h2d),
                        'd2h_bytes_per_step': int(prob.n_var * 8 + 8)},
                'gpu_launches': int(launches), 'gpu_launches_note': 'library kernels; cuSOLVER launches not counted',
                'roofline': roof, 'cpu_baseline': cpu, 'clocks': clk.summary(), 'wall_s_timed': wall,
                'device_ms_breakdown': {'static_assembly': asm['ms'], 'static_factor': fac['ms']},
                'energy': out['energy'], 'energy_e2e': o2['energy']}
        print(json.dumps(line), flush=True)
    ctx.close()
    if pg is not None:
        pg.destroy_process_group()


POINTS_METRIC = 'grid points/s (|E|/E0 and density of a wFQFMu solution)'
# FP64 operations per (point, atom) pair of field_points on the wFQFMu path
# (adds, multiplies and divisions, each exp / erf / sqrt counted once): a lower
# bound on the issued FP64 work, as the transcendentals cost several operations
POINT_PAIR_OPS = 200.0
FP64_NOMINAL_TFLOPS = 37.0


def points_problem(args):
    from plasmonx_b200 import configs
    prob = configs.particle('Ag', 'sphere', args.radius or 20.0, n_freq=1, method='iterative')
    n = args.grid
    return prob, n


def _points_chunk(job):
    """One worker's share of the CPU arm: the oracle's field and density at its points."""
    from oracle.analysis import field_and_density
    coord, rq, rmu, x, e0, pts = job
    field_and_density(coord, rq, rmu, x, e0, 0, pts, True)
    return len(pts)


def points_cpu(prob, x, pts, n_sample=4000, workers=0):
    """The oracle's NumPy restatement on a bounded sample of the grid, split over
    `workers` spawned processes (0: every host core) -> (points/s, points, seconds,
    workers).  The workers are started and warmed before the timed region."""
    import multiprocessing as mp
    workers = workers or os.cpu_count() or 1
    rng = np.random.default_rng(3)
    sample = pts[rng.choice(len(pts), size=min(n_sample, len(pts)), replace=False)]
    rq, rmu = prob.r_q[prob.atom_types], prob.r_mu[prob.atom_types]
    jobs = [(prob.coord, rq, rmu, x, prob.e0, c) for c in np.array_split(sample, workers) if len(c)]
    with mp.get_context('spawn').Pool(len(jobs)) as pool:
        pool.map(_points_chunk, [(prob.coord, rq, rmu, x, prob.e0, sample[:1])] * (2 * len(jobs)), chunksize=1)
        t0 = time.perf_counter()
        pool.map(_points_chunk, jobs, chunksize=1)
        dt = time.perf_counter() - t0
    return len(sample) / dt, len(sample), dt, len(jobs)


def run_points(args):
    rank, world, local, pg = dist_setup()
    from plasmonx_b200 import analysis as A
    from plasmonx_b200 import _lib
    from plasmonx_b200.inputs import neighbour_counts
    from plasmonx_b200.solver import Context, Solver
    prob, n = points_problem(args)
    ctx = Context(local)
    sv = Solver(prob, ctx=ctx, store_t=False)
    x = np.random.default_rng(5).standard_normal((sv.n_var, 2)) @ np.array([1.0, 1j])
    grid = A.cubic_grid(prob.coord_ang, (n, n, n), 10.0)
    pts = A._points_bohr(grid)
    P = len(pts)
    for _ in range(args.warmup):
        sv.field_at_points(0, x, pts)
    barrier(pg, local)
    ctx.profile(True)
    launches0 = ctx.launches
    with Clocks(local) as clk:
        barrier(pg, local)
        t0 = time.perf_counter()
        for _ in range(args.steps):
            field, dens = sv.field_at_points(0, x, pts)
        barrier(pg, local)
        wall = time.perf_counter() - t0
    launches = ctx.launches - launches0
    prof = ctx.profile_read(7)
    ctx.profile(False)
    value, total_pts, dev_ms = job_throughput(pg, local, P * args.steps, prof['ms'])
    e2e_s = allmax(pg, wall, local)
    avg_ms = prof['ms'] / max(1, prof['launches'])
    achieved = POINT_PAIR_OPS * P * prob.n_atoms / (avg_ms / 1e3) / 1e12
    roof = {'kernel': 'field_points (one thread per point, atoms staged in shared memory)', 'bound': 'fp64',
            'achieved': achieved, 'peak': FP64_NOMINAL_TFLOPS, 'unit': 'TFLOP/s', 'frac': achieved / FP64_NOMINAL_TFLOPS,
            'peak_kind': 'nominal FP64 (no measured FP64 peak available)',
            'ops_per_pair': POINT_PAIR_OPS, 'pairs_per_launch': float(P) * prob.n_atoms, 'avg_launch_ms': avg_ms,
            'bytes_per_launch': prof['bytes'] / max(1, prof['launches']), 'traffic': None}
    # device neighbour counts of the default silver sphere against the host all-pairs count
    big = make_problem('ag_sphere', n_freq=1)
    nt = len(big.type_names)
    nb = np.zeros((big.n_atoms, nt), dtype=np.int32)
    nnb = np.zeros(big.n_atoms, dtype=np.int32)
    ang = np.ascontiguousarray(big.coord_ang, dtype=np.float64)
    types = np.ascontiguousarray(big.atom_types, dtype=np.int32)
    r0 = np.asfortranarray(big.r0).ravel(order='F')
    ctx.profile(True)
    for _ in range(3):
        ctx.check(ctx.lib.plx_neighbour_counts(ctx.h, big.n_atoms, nt, _lib.ptr(ang), _lib.ptr(types, _lib._ip),
                                               _lib.ptr(big.type_z, _lib._ip), _lib.ptr(r0), _lib.ptr(nb, _lib._ip),
                                               _lib.ptr(nnb, _lib._ip)))
    nprof = ctx.profile_read(8)
    ctx.profile(False)
    neigh = {'n_atoms': int(big.n_atoms), 'kernel_ms': nprof['ms'] / max(1, nprof['launches'])}
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        v, ns, dt, nw = points_cpu(prob, x, pts)
        cpu = {'value': v, 'unit': 'points/s', 'cores': nw, 'kind': 'port',
               'sample': '%d random points of the grid through the NumPy restatement in %d processes, %.1f s'
                         % (ns, nw, dt)}
        t0 = time.perf_counter()
        nb_h, nn_h = neighbour_counts(big.coord_ang, big.atom_types, big.znum, nt)
        neigh['host_all_pairs_s'] = time.perf_counter() - t0
        neigh['identical'] = bool(np.array_equal(nn_h, nnb) and np.array_equal(nb_h, nb.T))
    if rank == 0:
        line = {'metric': POINTS_METRIC, 'value': value, 'unit': 'points/s', 'n_gpus': world, 'steps': args.steps,
                'warmup': args.warmup, 'ms_per_step': dev_ms / args.steps, 'higher_is_better': True,
                'scaling': 'weak', 'vs_baseline': None, 'dtype': 'f64',
                'data': 'synthetic (seeded silver sphere, seeded solution vector)',
                'config': {'workload': 'field and density of a wFQFMu Ag sphere R=%g A on a %d^3 grid'
                                       % (args.radius or 20.0, n),
                           'n_atoms': int(prob.n_atoms), 'n_points': int(P),
                           'l2': 'each step writes %.0f MB of results (larger than L2)' % (P * 64 / 1e6)},
                'e2e': {'value': total_pts / e2e_s, 'unit': 'points/s', 'h2d_bytes_per_step': int(pts.nbytes),
                        'd2h_bytes_per_step': int(field.nbytes + dens.nbytes)},
                'gpu_launches': int(launches), 'roofline': roof, 'cpu_baseline': cpu, 'clocks': clk.summary(),
                'wall_s_timed': wall, 'neighbours': neigh}
        print(json.dumps(line), flush=True)
    sv.close()
    ctx.close()
    if pg is not None:
        pg.destroy_process_group()


def run_reference(args):
    rank, world, local, pg = dist_setup()
    if rank != 0:
        return
    if args.config == 'serving':
        print(json.dumps({'impl': 'reference', 'unavailable': 'the reference has no request loop; its per-request '
                                                             'cost is the ag_sphere / na_sphere / bem lines'}))
        return
    if args.config == 'field_grid':
        from plasmonx_b200 import analysis as A
        prob, n = points_problem(args)
        x = np.random.default_rng(5).standard_normal((prob.n_var, 2)) @ np.array([1.0, 1j])
        pts = A._points_bohr(A.cubic_grid(prob.coord_ang, (n, n, n), 10.0))
        for _ in range(args.warmup):
            points_cpu(prob, x, pts, 100)
        runs = [points_cpu(prob, x, pts, 4000 * (os.cpu_count() or 1)) for _ in range(args.steps)]
        v = float(np.mean([r[0] for r in runs]))
        line = {'metric': POINTS_METRIC, 'value': v, 'unit': 'points/s', 'n_gpus': world, 'steps': args.steps,
                'warmup': args.warmup, 'ms_per_step': 1000.0 * len(pts) / v, 'higher_is_better': True,
                'scaling': 'weak', 'vs_baseline': None, 'dtype': 'f64',
                'data': 'synthetic (seeded silver sphere, seeded solution vector)',
                'config': {'workload': 'field and density of a wFQFMu Ag sphere R=%g A on a %d^3 grid'
                                       % (args.radius or 20.0, n), 'n_atoms': int(prob.n_atoms),
                           'n_points': int(len(pts))}, 'impl': 'reference',
                'cpu_baseline': {'value': v, 'unit': 'points/s', 'cores': runs[0][3], 'kind': 'port',
                                 'sample': '%d random grid points per step through the NumPy restatement in %d '
                                           'processes' % (runs[0][1], runs[0][3])},
                'e2e': {'value': v, 'unit': 'points/s', 'h2d_bytes_per_step': 0, 'd2h_bytes_per_step': 0}}
        print(json.dumps(line), flush=True)
        return
    if args.config in ('fq_water', 'fqfmu_water'):
        prob = static_problem(args)
        for _ in range(args.warmup):
            static_cpu(prob)
        vals = [static_cpu(prob)[0] for _ in range(args.steps)]
        v = float(np.mean(vals))
        line = {'metric': STATIC_METRIC, 'value': v, 'unit': 'solves/s', 'n_gpus': world, 'steps': args.steps,
                'warmup': args.warmup, 'ms_per_step': 1000.0 / v, 'higher_is_better': True, 'scaling': 'weak',
                'vs_baseline': None, 'dtype': 'f64', 'data': 'synthetic (seeded water cluster)',
                'config': static_desc(prob), 'impl': 'reference',
                'cpu_baseline': {'value': v, 'unit': 'solves/s', 'cores': os.cpu_count(), 'kind': 'port',
                                 'sample': 'one full solve of the NumPy restatement per step'},
                'e2e': {'value': v, 'unit': 'solves/s', 'h2d_bytes_per_step': 0, 'd2h_bytes_per_step': 0}}
        print(json.dumps(line), flush=True)
        return
    prob = make_problem(args.config, n_tess=args.n_tess, bem_variant=args.bem_variant, bowtie_edge=args.bowtie_edge)
    prob.tolerance_input = args.tolerance
    if args.mode:
        prob.method = args.mode
    sps = args.steps_per_solve or STEPS_PER_SOLVE[args.config]
    per_step = max(2, -(-20 // max(1, args.steps)))      # at least 20 products over the run
    for _ in range(args.warmup):
        cpu_reference(prob, sps, n_min=1, budget_s=0.0)
    runs = [cpu_reference(prob, sps, n_min=per_step, budget_s=2.0) for _ in range(args.steps)]
    v = float(np.mean([r['value'] for r in runs]))
    cpu = dict(runs[-1], value=v)
    cpu['sample'] = ('%d timed steps; last: ' % len(runs)) + runs[-1]['sample']
    line = {'metric': METRIC, 'value': v, 'unit': 'freq-solves/s', 'n_gpus': world, 'steps': args.steps,
            'warmup': args.warmup, 'ms_per_step': 1000.0 / v * len(prob.freqs), 'ms_per_step_extrapolated': True,
            'higher_is_better': True, 'scaling': 'weak', 'vs_baseline': None, 'dtype': 'f64', 'data': 'synthetic',
            'config': dict(workload_desc(args.config, prob), precision='fp64 (the reference algorithm)'),
            'impl': 'reference', 'cpu_baseline': cpu,
            'note': ('one step = one spectrum; ms_per_step is extrapolated from the LU factorisation timed in '
                     'each step' if prob.method == 'inversion' else
                     'one step = one spectrum; ms_per_step is extrapolated from the products and '
                     'orthogonalisations timed in each step (a whole spectrum takes hours on the host)'),
            'e2e': {'value': v, 'unit': 'freq-solves/s', 'h2d_bytes_per_step': 0, 'd2h_bytes_per_step': 0}}
    print(json.dumps(line), flush=True)


SERVING_METRIC = 'freq-solves/s of a seeded Poisson request mix (p50/p99 latency), batched mixed vs plain FP64'


def run_serving(args):
    """Config 5: the seeded Poisson mix (wFQ Na, wFQFMu Ag/Au spheres and rods, BEM
    spheres and rods, 20-400 frequencies each) through the serving loop, once with
    the batched mixed-precision form and once with the plain FP64 GMRES, the same
    requests in the same order; per-request sigma_abs of the two arms compared."""
    from plasmonx_b200.serving import Server, request_pool, run_mix
    n = max(1, args.serving_requests)
    # warm-up: CUDA context, kernel attributes, allocator pools
    with Server(device=0, workers=args.serving_workers) as srv:
        run_mix(srv, request_pool(n_requests=4, rate=args.serving_rate, seed=99, scale='small'))
    arms, results = {}, {}
    for prec in (('mixed_bf16x3', 'fp64') if args.serving_arms == 'both' else ('mixed_bf16x3',)):
        pool = request_pool(n_requests=n, rate=args.serving_rate, seed=7, scale=args.serving_scale, precision=prec)
        with Clocks(0) as clk:
            with Server(device=0, workers=args.serving_workers) as srv:
                st = run_mix(srv, pool)
        steps = srv.steps
        st.update({'clocks': clk.summary(), 'outer_steps': len(steps), 'budget_bytes': srv.budget,
                   'min_device_free_bytes': None if srv.min_free is None else srv.min_free[0],
                   'committed_at_min_free': None if srv.min_free is None else srv.min_free[1],
                   'grouped_steps': sum(1 for s in steps if s[1] > 1),
                   'max_geometries_per_step': max([s[1] for s in steps] or [0]),
                   'mean_requests_per_step': float(np.mean([s[2] for s in steps])) if steps else 0.0,
                   'mean_requests_sharing': float(np.mean([r.batch_size for r in pool])),
                   'modes': sorted({str(r.mode) for r in pool})})
        # a request counts as solved when every one of its frequencies converged
        ok = [r.result is not None and bool(np.all(r.result['status'] == 0)) for r in pool]
        st['unconverged'] = int(sum(1 for r, g in zip(pool, ok) if r.result is not None and not g))
        st['escalated_requests'] = int(sum(1 for r in pool if getattr(r, 'escalated', 0)))
        st['escalated_freqs'] = int(sum(getattr(r, 'escalated', 0) for r in pool))
        st['unconverged_requests'] = [
            {'id': r.id, 'n_var': int(r.problem.n_var), 'n_freq': r.n_freq, 'tol': r.tol,
             'kind': type(r.problem).__name__ + ('/' + str(getattr(r.problem, 'model', '')) if hasattr(r.problem, 'model') else ''),
             'mode': str(r.mode), 'statuses': sorted({int(v) for v in np.asarray(r.result['status']).ravel()})}
            for r, g in zip(pool, ok) if r.result is not None and not g][:20]
        arms[prec] = st
        results[prec] = [r.result['results'][:, 9] if g else None for r, g in zip(pool, ok)]
    errs = [float(np.max(np.abs(a - b) / np.abs(b))) for a, b in zip(results['mixed_bf16x3'], results['fp64'])
            if a is not None and b is not None] if 'fp64' in results else []
    mixed = arms['mixed_bf16x3']
    line = {'metric': SERVING_METRIC, 'value': mixed['throughput'], 'unit': 'freq-solves/s', 'n_gpus': 1,
            'steps': 1, 'warmup': 1, 'ms_per_step': mixed['wall_s'] * 1000.0, 'higher_is_better': True,
            'scaling': 'weak', 'vs_baseline': None, 'dtype': 'bf16x3 (fp32 acc) + f64 refinement',
            'data': 'synthetic (seeded request pool, reference default parameters)',
            'config': {'workload': 'serving mix, %d requests at %g req/s, %s scale' % (n, args.serving_rate,
                                                                                     args.serving_scale),
                       'workers': args.serving_workers},
            'p50_ms': mixed['p50_ms'], 'p99_ms': mixed['p99_ms'],
            'fp64_plain': arms.get('fp64', 'not run (--serving-arms mixed): the unrestarted FP64 GMRES of '
                                           'the 30k-atom requests takes hours per request'),
            'mixed': mixed,
            'speedup_vs_fp64_plain': mixed['throughput'] / arms['fp64']['throughput'] if 'fp64' in arms else None,
            'sigma_abs_max_rel_err_vs_fp64_plain': max(errs) if errs else None,
            'requests_compared': len(errs)}
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument('--gpus', type=int, default=1)
    ap.add_argument('--steps', type=int, default=2)
    ap.add_argument('--warmup', type=int, default=3)
    ap.add_argument('--impl', default='ours', choices=['ours', 'reference'])
    ap.add_argument('--config', default='ag_sphere',
                    choices=['ag_sphere', 'na_sphere', 'bowtie', 'bem_sphere', 'bem_rod', 'fq_water', 'fqfmu_water',
                             'field_grid', 'serving'])
    ap.add_argument('--grid', type=int, default=100, help='grid points per axis of field_grid')
    ap.add_argument('--waters', type=int, default=0, help='water molecules of fq_water / fqfmu_water')
    ap.add_argument('--n-tess', type=int, default=2000, help='BEM tesserae (20 nu^2)')
    ap.add_argument('--bowtie-edge', type=float, default=80.0, help='prism edge (A): 80 gives 5,850 atoms, 180 ~30k')
    ap.add_argument('--bem-variant', default='dpcm', choices=['dpcm', 'iefpcm'])
    ap.add_argument('--bem-green', default='approximate', choices=['approximate', 'accurate'])
    ap.add_argument('--precision', default='mixed_bf16x3')
    ap.add_argument('--tolerance', type=float, default=1e-12, help='input tolerance (times sqrt(n_var))')
    ap.add_argument('--no-fp64-compare', action='store_true')
    ap.add_argument('--fp64-freqs', type=int, default=0, help='time the plain FP64 form on this many frequencies')
    ap.add_argument('--fp64-krylov', type=int, default=0, help='Krylov dimension of the plain FP64 arm (0: input)')
    ap.add_argument('--mode', default=None,
                    choices=[None, 'inversion', 'iterative', 'iterative on the fly', 'iterative_on_the_fly'],
                    help="solver mode (default: the workload's)")
    ap.add_argument('--inner-krylov', type=int, default=0)
    ap.add_argument('--ref-rel', type=float, default=1e-11)
    ap.add_argument('--inner-tol', type=float, default=0.0)
    ap.add_argument('--e2e-steps', type=int, default=1)
    ap.add_argument('--cpu-matvecs', type=int, default=2)
    ap.add_argument('--steps-per-solve', type=float, default=None,
                    help="Arnoldi steps per freq-solve of the reference's algorithm (CPU arm)")
    ap.add_argument('--no-cpu', action='store_true')
    ap.add_argument('--accuracy-freqs', type=int, default=5)
    ap.add_argument('--radius', type=float, default=None, help='sphere radius in A: a smaller ag_sphere (profiling runs only), or the field_grid sphere (default 20)')
    ap.add_argument('--n-freq', type=int, default=None, help='fewer frequencies (profiling runs only)')
    ap.add_argument('--serving-requests', type=int, default=24, help='requests in the serving leg (0: skip)')
    ap.add_argument('--serving-arms', default='both', choices=['both', 'mixed'],
                    help='config serving: run the plain FP64 arm too (both) or the mixed arm alone')
    ap.add_argument('--serving-rate', type=float, default=20.0, help='Poisson arrival rate, requests/s')
    ap.add_argument('--serving-scale', default='small', choices=['small', 'medium', 'full'])
    ap.add_argument('--serving-workers', type=int, default=2)
    args = ap.parse_args()
    if args.mode == 'iterative_on_the_fly':
        args.mode = 'iterative on the fly'      # the same mode, spelt without spaces for shell variables
    if args.impl == 'reference':
        return run_reference(args)
    if args.config in ('fq_water', 'fqfmu_water'):
        return run_static(args)
    if args.config == 'field_grid':
        return run_points(args)
    if args.config == 'serving':
        return run_serving(args)

    rank, world, local, pg = dist_setup()
    from plasmonx_b200.solver import Context, Solver
    from plasmonx_b200.spectrum import solve_partitioned
    # N ranks: one spectrum of N times the frequencies over the same window, dealt
    # out in blocks of one workload's frequencies per rank, results gathered to rank 0
    base_f = args.n_freq or {'ag_sphere': 201, 'na_sphere': 61, 'bowtie': 201}.get(args.config, 301)
    prob = make_problem(args.config, n_freq=base_f * world, radius=args.radius, n_tess=args.n_tess,
                        bem_variant=args.bem_variant, bowtie_edge=args.bowtie_edge, bem_green=args.bem_green)
    prob.tolerance_input = args.tolerance
    prob.tol = args.tolerance * np.sqrt(prob.n_var)
    if args.mode:
        prob.method = args.mode
    ctx = Context(local)
    solver = Solver(prob, ctx=ctx, store_t=prob.method != 'iterative on the fly')
    gather_dev = 'cuda:%d' % local if pg is not None and pg.get_backend() == 'nccl' else 'cpu'
    full_freqs, full_aw = prob.freqs, prob.alpha_w
    tuning = None
    requested_precision = args.precision          # the serving leg's requests keep it
    if args.inner_krylov == 0 and args.precision.startswith('mixed'):
        # the inner basis length from a short sweep on a few of the grid's frequencies
        # (plasmonx_b200.tuning), cached per geometry; not part of the timed region
        from plasmonx_b200.tuning import Tuner
        # the probe is the whole grid (up to 256 frequencies): the balance between the
        # contraction (cheaper per column as columns grow) and the orthogonalisation
        # (linear in columns and basis length) depends on the column count
        tuner = Tuner(n_probe=min(256, len(full_freqs)))
        chosen = tuner.settings(solver, args.config, full_freqs, full_aw, precision=args.precision,
                                mode=prob.method, tol=prob.tol)
        args.inner_krylov = chosen['inner_krylov']
        if not args.inner_tol:
            args.inner_tol = chosen['inner_tol']
        args.precision = chosen.get('precision', args.precision)
        tuning = tuner.records[args.config]
    gathered = {}

    def step():
        part = solve_partitioned(solver, full_freqs, full_aw, pg, device=gather_dev, precision=args.precision,
                                 inner_krylov=args.inner_krylov, inner_tol=args.inner_tol)
        out = part['local']
        if 'error' in out:
            raise out['error']
        if part['status'] is not None:
            gathered.update(n_freq=int(len(part['status'])), status_ok=bool(np.all(part['status'] == 0)))
        return out

    step_out = step()
    F = len(step_out['results'])          # this rank's block (the whole grid on one rank)
    if world > 1:
        # the single-rank legs below (plain FP64 arm, accuracy, CPU, serving) use the rank's block
        blk = np.arange(rank, len(prob.freqs), world)
        prob.freqs = prob.freqs[blk]
        if prob.alpha_w is not None:
            prob.alpha_w = prob.alpha_w[:, blk]
        args.no_fp64_compare, args.accuracy_freqs, args.serving_requests = True, 0, 0

    for _ in range(max(0, args.warmup - 1)):
        step()
    barrier(pg, local)
    ctx.profile(True)
    dev_ms = []
    launches = 0
    steps_hist = []
    unconverged_hist = []
    with Clocks(local) as clk:
        barrier(pg, local)
        t0 = time.perf_counter()
        for _ in range(args.steps):
            out = step()
            dev_ms.append(out['device_ms'])
            launches += out['launches']
            steps_hist.append(out['steps'][:, 0].copy())
            unconverged_hist.append(int(np.sum(out['status'] != 0)))
        barrier(pg, local)
        wall = time.perf_counter() - t0
    breakdown = ctx.profile_breakdown()
    prof = breakdown['tc_contraction'] if args.precision.startswith('mixed') else breakdown['fp64_contraction']
    ctx.profile(False)
    value, solves, total_ms = job_throughput(pg, local, F * args.steps, float(np.sum(dev_ms)))

    # plain FP64 GMRES (the reference's algorithm) on the same spectrum, for the
    # speed-up of the headline form over it on the same GPU
    fp64 = None
    sub = None
    if not args.no_fp64_compare and args.precision != 'fp64':
        if args.fp64_freqs and args.fp64_freqs < F:
            # a spread subset solved as one batch (large geometries whose unrestarted
            # FP64 Krylov basis for all frequencies would not fit); throughput per frequency
            sub = np.linspace(0, F - 1, args.fp64_freqs).round().astype(int)
            solver.set_frequencies(prob.freqs[sub], None if prob.alpha_w is None else prob.alpha_w[:, sub])
        if not args.fp64_krylov and args.config == 'bowtie':
            # the gap-coupled alloy needs up to ~1,500 Arnoldi steps at this tolerance;
            # the input's dimension (1,000) leaves frequencies unconverged
            args.fp64_krylov = 2500
        o64 = solver.solve(precision='fp64', max_krylov=args.fp64_krylov or None)
        if sub is not None:
            solver.set_frequencies(prob.freqs, prob.alpha_w)
        nf64 = F if sub is None else len(sub)
        t64 = allmax(pg, o64['device_ms'], local)
        fp64 = {'value': allsum(pg, float(nf64), local) / (t64 / 1000.0), 'ms_per_step': t64 * F / nf64,
                'arnoldi_steps_mean': float(np.mean(o64['steps'][:, 0])), 'status_ok': bool((o64['status'] == 0).all()),
                'frequencies_timed': int(nf64), 'max_krylov': int(args.fp64_krylov or prob.gmres_dim or 1000)}
        if sub is not None and fp64['status_ok']:
            # the headline form against the converged plain FP64 GMRES on the subset
            s64 = o64['results'][:, 9]
            fp64['headline_vs_fp64_max_rel_err'] = float(np.max(np.abs(out['results'][sub, 9] - s64) / np.abs(s64)))

    # accuracy: sigma_abs against the oracle's fixtures of this workload (the
    # reference GMRES restated on the CPU, refined in FP64) when there are
    # some, else against an FP64 refinement on the device, on a subset of frequencies
    acc = None
    fixture = oracle_fixture(args, prob) if world == 1 else None
    if fixture is not None and args.accuracy_freqs > 0:
        idx = np.asarray(fixture['freq_index'])
        sref = np.array(fixture['results'])[:, 9]
        acc = {'freqs': [int(i) for i in idx], 'reference': fixture['reference'],
               'headline_max_rel_err': float(np.max(np.abs(out['results'][idx, 9] - sref) / np.abs(sref)))}
        if fp64 is not None and sub is None:
            fp64['sigma_abs_max_rel_err'] = float(np.max(np.abs(o64['results'][idx, 9] - sref) / np.abs(sref)))
    elif args.accuracy_freqs > 0:
        idx = np.linspace(0, F - 1, min(args.accuracy_freqs, F)).round().astype(int)
        b = solver.rhs(int(idx[0]), prob.pol_mask)
        sref, ref_status = [], []
        for i in idx:
            solver.set_frequencies(prob.freqs[[i]], None if prob.alpha_w is None else prob.alpha_w[:, [i]])
            bi = solver.rhs(0, prob.pol_mask)
            tight = solver.solve(precision='fp64_refined', tol=args.ref_rel * np.linalg.norm(bi), max_outer=30,
                                 inner_krylov=1000, inner_tol=args.ref_rel)
            ref_status.append(int(tight['status'][0]))
            sref.append(tight['results'][0, 9] if (tight['status'] == 0).all() else np.nan)
        solver.set_frequencies(prob.freqs, prob.alpha_w)
        sref = np.array(sref)
        acc = {'freqs': [int(i) for i in idx], 'reference': 'FP64 refinement to %g relative residual' % args.ref_rel,
               'reference_status': ref_status,
               'headline_max_rel_err': float(np.max(np.abs(out['results'][idx, 9] - sref) / np.abs(sref)))}
        if fp64 is not None and sub is None:
            fp64['sigma_abs_max_rel_err'] = float(np.max(np.abs(o64['results'][idx, 9] - sref) / np.abs(sref)))
        del b

    # end to end through the public API: build + upload + solve + results to host
    e2e_times = []
    h2d = 0
    for _ in range(args.e2e_steps):
        barrier(pg, local)
        t0 = time.perf_counter()
        with Solver(prob, ctx=ctx) as s2:
            o2 = s2.solve(precision=args.precision, inner_krylov=args.inner_krylov, inner_tol=args.inner_tol)
        barrier(pg, local)
        e2e_times.append(time.perf_counter() - t0)
        k = s2._keep
        h2d = sum(v.nbytes for v in k.values()) + s2.freqs.nbytes + (0 if s2._aw is None else s2._aw.nbytes)
    e2e_s = allmax(pg, float(np.mean(e2e_times)), local) if e2e_times else float('nan')
    e2e_val = solves / args.steps / e2e_s if e2e_times else None

    pk, pk_kind = peaks()
    n = prob.n_var
    tc_operand = (2.0 if args.precision == 'mixed_bf16' else 4.0) * (-(-n // 256) * 256) * (-(-n // 64) * 64)
    avg_ms = prof['ms'] / max(1, prof['launches'])
    bytes_per = prof['bytes'] / max(1, prof['launches'])
    flops_per = prof['flops'] / max(1, prof['launches'])
    if prof['launches'] == 0:
        # direct inversion: no contraction to bound (the shifted Hessenberg solves are
        # latency-bound per CTA; the LU path is cuSOLVER's)
        roof = {'kernel': 'none timed (direct inversion mode)', 'bound': None, 'achieved': None, 'peak': None,
                'unit': None, 'frac': None, 'traffic': None}
    elif args.precision == 'fp64':
        roof = {'kernel': 'T contraction (FP64, CUDA cores)', 'bound': 'hbm',
                'achieved': bytes_per / (avg_ms / 1000.0) / 1e9, 'peak': pk['hbm_gbs'], 'unit': 'GB/s',
                'peak_kind': pk_kind, 'flops_per_launch': flops_per, 'bytes_per_launch': bytes_per,
                'avg_launch_ms': avg_ms, 'achieved_fp64_tflops': flops_per / (avg_ms / 1000.0) / 1e12,
                'traffic': None}
    else:
        nprod = 3 if args.precision == 'mixed_bf16x3' else 1
        roof = {'kernel': 'T contraction (tcgen05, BF16 split, %d products)' % nprod, 'bound': 'tensor',
                # the contraction runs inside a seconds-long step: the sustained (power-capped) peak
                'achieved': flops_per / (avg_ms / 1000.0) / 1e12,
                'peak': pk.get('bf16_tflops_sustained', pk['bf16_tflops']), 'unit': 'TFLOP/s',
                'peak_kind': pk_kind, 'flops_per_launch': flops_per, 'bytes_per_launch': bytes_per,
                'avg_launch_ms': avg_ms, 'issued_tensor_tflops': nprod * flops_per / (avg_ms / 1000.0) / 1e12,
                'achieved_hbm_gbs': bytes_per / (avg_ms / 1000.0) / 1e9,
                # DRAM bytes per launch: the ncu capture of the 7,844-unknown case read its
                # operand 1.004 times (X tiles come from L2); traffic grows with the operand
                'traffic': tc_operand * TRAFFIC_RATIO, 'traffic_unit': 'bytes per launch',
                'traffic_source': 'ncu dram__bytes (read + write) of a 21,560-unknown, 402-column capture per '
                                  'operand byte (1.086), times this launch\'s operand bytes (BF16 high + low, '
                                  'padded tiles)',
                'note': 'achieved counts one product (algorithmic); the tensor pipe executes %d' % nprod}
    if roof['achieved'] is not None:
        roof['frac'] = roof['achieved'] / roof['peak']
        if 'issued_tensor_tflops' in roof:
            # the BF16 products the tensor pipe executes (3 per algorithmic product for bf16x3)
            roof['issued_frac'] = roof['issued_tensor_tflops'] / roof['peak']
            contraction_bound(roof, pk['hbm_gbs'])

    # serving leg: a seeded Poisson mix of spectrum requests through the request loop
    serving = None
    if args.serving_requests > 0 and args.impl == 'ours':
        from plasmonx_b200.serving import Server, request_pool, run_mix
        pool = request_pool(n_requests=args.serving_requests, rate=args.serving_rate, seed=7 + rank,
                            scale=args.serving_scale, precision=requested_precision)
        with Server(device=local, workers=args.serving_workers) as srv:
            serving = run_mix(srv, pool)
        steps = srv.steps
        serving.update({'rate_per_s': args.serving_rate, 'scale': args.serving_scale,
                        'workers': args.serving_workers, 'precision': requested_precision,
                        'modes': sorted({str(r.mode) for r in pool}),
                        'mean_requests_sharing_a_step': float(np.mean([r.batch_size for r in pool])),
                        'outer_steps': len(steps),
                        'grouped_steps': sum(1 for st_ in steps if st_[1] > 1),
                        'max_geometries_per_step': max([st_[1] for st_ in steps] or [0]),
                        'p99_ms_max_over_ranks': allmax(pg, serving['p99_ms'], local)})

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        # the CPU baseline runs the reference's algorithm: its step count is the plain
        # FP64 GMRES's of this run when measured
        sps = fp64['arnoldi_steps_mean'] if fp64 is not None and sub is None else \
            (args.steps_per_solve or STEPS_PER_SOLVE[args.config])
        cpu = cpu_reference(prob, sps)
    if rank == 0:
        line = {'metric': METRIC, 'value': value, 'unit': 'freq-solves/s', 'n_gpus': world,
                'steps': args.steps, 'warmup': args.warmup, 'ms_per_step': total_ms / args.steps,
                'higher_is_better': True, 'scaling': 'weak', 'vs_baseline': None,
                'dtype': {'fp64': 'f64', 'mixed_bf16x3': 'bf16x3 (fp32 acc) + f64 refinement',
                          'mixed_bf16': 'bf16 (fp32 acc) + f64 refinement', 'fp64_refined': 'f64'}[args.precision],
                'data': ('synthetic (seeded geodesic surface, Drude-Lorentz eps)' if is_bem(prob) else
                         'synthetic (seeded fcc lattice, reference default parameters)'),
                'config': dict(workload_desc(args.config, prob), precision=args.precision,
                               inner_krylov=args.inner_krylov or 64, inner_tol=args.inner_tol or 1e-4,
                               **({'partition': 'one spectrum of %d frequencies over the window, dealt round-robin '
                                                '(%d per rank), results gathered to rank 0' % (len(full_freqs), F),
                                   'gathered': gathered} if world > 1 else {})),
                'e2e': {'value': e2e_val, 'unit': 'freq-solves/s', 'h2d_bytes_per_step': int(h2d),
                        'd2h_bytes_per_step': int(F * (20 * 8 + 9 * 16 + 4 + 12))},
                'gpu_launches': int(launches), 'roofline': roof, 'cpu_baseline': cpu,
                'clocks': clk.summary(), 'wall_s_timed': wall,
                'device_ms_breakdown': {k: round(v['ms'], 3) for k, v in breakdown.items()},
                'sigma_abs_max_rel_err': None if acc is None else acc['headline_max_rel_err'],
                'status_ok': not any(unconverged_hist), 'unconverged_freq_solves': int(sum(unconverged_hist)),
                'accuracy': acc, 'fp64_plain_gmres': fp64,
                'speedup_vs_fp64_plain': None if fp64 is None else value / fp64['value'],
                'tuning': tuning,
                'arnoldi_steps': {'mean': float(np.mean(np.concatenate(steps_hist))),
                                  'max': int(np.max(np.concatenate(steps_hist)))},
                'serving': serving}
        print(json.dumps(line), flush=True)
    solver.close()
    ctx.close()
    if pg is not None:
        pg.destroy_process_group()


if __name__ == '__main__':
    main()
