"""Oracle fixtures at the benchmark sizes (test infrastructure).

    python tests/golden/make_large.py [case ...] [--threads N]

Solves, on the CPU, five frequencies of two benchmark systems with products
from the C port of the reference's on-the-fly matrix-vector product
(``oracle/pairs.c``, ``src/matrix/matrix_module.f90:727-1125`` plus
``new_gmres_diagonal_shift``):

  ag_sphere_r35    wFQFMu silver sphere, fcc a = 4.086 A, R = 35 A:
                   10,473 atoms, 41,892 unknowns, 201 frequencies 3.0-4.5 eV
  agau_bowtie_e80  wFQFMu Ag-Au bow-tie, two fcc (a = 4.08 A) prisms of edge
                   80 A and thickness 20 A, gap 10 A: 5,850 atoms, 23,400
                   unknowns, 201 frequencies 2.0-4.5 eV

at frequency indices 0, 50, 100, 150 and 200, x polarisation.  The reference
GMRES alone (unrestarted, ``oracle/gmres.py``) does not reach a relative
residual of 1e-12 within 4,000 Krylov vectors on these systems, so the solution
is refined in FP64: x = 0, r = b; repeat { solve A d = r with the reference
GMRES to 1e-5 ||r|| (at most 1,500 vectors); x += d; r = b - A x by the FP64
product } until ||r|| <= 1e-12 ||b|| or a pass gains less than a factor of two
(the floor of the FP64 residual, 1.7e-12 to 5.5e-12 of ||b|| here).  Every
residual is an explicit product of the C port, so the fixture is the solution
of the same FP64 system the reference assembles, to the attained residual,
which is stored with the sigma_abs of every refinement pass (the change
between the last two passes bounds how far the stored value can still move).
The geometry is the seeded generator the benchmark uses
(``plasmonx_b200.configs``); it reaches the oracle through the keyword file,
as every other oracle fixture does.  For each frequency the fixture stores the
20 results of the reference's results row (``target_module.f90:1989-2054``),
alpha_xx, the Krylov vectors used, and the refinement history.

Output: ``tests/golden/large/<case>.json``, written after every frequency.
Run time on 8 cores: about 1.5 s per product for the sphere, 0.5 s for the
bow-tie, a few hundred to a few thousand products per frequency.
"""
import argparse
import json
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

from oracle import keywords, model  # noqa: E402
from oracle.cpu_baseline import CpuOperator  # noqa: E402
from oracle.gmres import gmres  # noqa: E402
from plasmonx_b200 import configs  # noqa: E402

FREQ_INDEX = [0, 50, 100, 150, 200]
REL_TOL = 1e-12          # target relative residual of the refinement
INNER_REL = 1e-5         # inner GMRES: relative to the current residual
INNER_DIM = 1500
MAX_OUTER = 8


def build(case):
    """The benchmark problem of a case (keyword text and the oracle's system)."""
    if case == 'ag_sphere_r35':
        p = configs.ag_sphere(radius=35.0, n_freq=201, method='iterative', tolerance=1e-9, polarization='x')
    elif case == 'agau_bowtie_e80':
        p = configs.agau_bowtie(n_freq=201, method='iterative on the fly', tolerance=1e-9, polarization='x')
    else:
        raise ValueError(case)
    text = p.to_keyword_text()
    return text, model.System.from_keywords(keywords.read_keyword_text(text))


def signature(s):
    """Numbers that identify the geometry (checked by the tests before comparing)."""
    return {'n_atoms': int(s.n_atoms), 'n_var': int(s.n_var), 'coord_sum': float(np.sum(s.coord)),
            'coord_abs_sum': float(np.sum(np.abs(s.coord)))}


def refine(matvec, b, log=None):
    """FP64 iterative refinement around the reference GMRES (module docstring).

    Returns (x, its relative residual, history): per pass the Krylov vectors
    used and the relative residual ||b - A x|| / ||b|| after it."""
    nb = float(np.linalg.norm(b))
    x = np.zeros_like(b)
    r = b.copy()
    hist = []
    best = (np.inf, x)
    for _ in range(MAX_OUTER):
        nr = float(np.linalg.norm(r))
        d, steps = gmres(matvec, r, INNER_REL * nr, INNER_DIM, best_effort=True)
        x_new = x + d
        r_new = b - matvec(x_new)
        rel = float(np.linalg.norm(r_new)) / nb
        hist.append({'krylov': int(steps), 'rel_residual': rel})
        if log is not None:
            log(hist[-1], x_new)
        if rel >= best[0]:
            break                       # the residual stopped falling: keep the best pass
        gain = best[0] / rel
        x, r = x_new, r_new
        best = (rel, x)
        if rel <= REL_TOL or gain < 2.0:
            break                       # at the target, or at the FP64 floor of the residual
    return best[1], best[0], hist


def _sigma(s, x, i):
    X = np.zeros((s.n_var, 3), dtype=np.complex128)
    X[:, 0] = x
    P = model.polar(s, X)
    return P, model.results_row(P, s.freqs[i])


def run(case, threads):
    text, s = build(case)
    out_dir = os.path.join(HERE, 'large')
    os.makedirs(out_dir, exist_ok=True)
    path = os.path.join(out_dir, case + '.json')
    op = CpuOperator(s, n_threads=threads)
    K = model.k_matrix(s)
    Kbar = K - np.diag(K.sum(axis=1))
    rec = {'case': case, 'geometry': signature(s), 'freq_index': [], 'omega': [], 'results': [],
           'alpha_xx': [], 'krylov_total': [], 'true_rel_residual': [], 'rel_tol': REL_TOL,
           'method': 'FP64 refinement around the reference GMRES (inner 1e-5, explicit FP64 residuals)',
           'refinement': [], 'seconds': [], 'threads': op.n_threads}
    if os.path.exists(path):
        # resume: keep the frequencies already solved for this geometry
        with open(path) as f:
            old = json.load(f)
        if old.get('geometry') == rec['geometry'] and old.get('method') == rec['method']:
            rec = old
    for i in FREQ_INDEX:
        if i in rec['freq_index']:
            continue
        t0 = time.time()
        b = model.rhs(s, i, Kbar=Kbar, K=K)[:, 0]

        def log(h, xp):
            h['sigma_abs'] = float(_sigma(s, xp, i)[1][9])
            print('  %s freq %d pass: %d vectors, residual %.2e, sigma_abs %.12e (%.0f s)' %
                  (case, i, h['krylov'], h['rel_residual'], h['sigma_abs'], time.time() - t0), flush=True)
        x, res, hist = refine(lambda v: op.matvec(i, v), b, log)
        P, row = _sigma(s, x, i)
        rec['freq_index'].append(i)
        rec['omega'].append(float(s.freqs[i]))
        rec['results'].append([float(v) for v in row])
        rec['alpha_xx'].append([float(P[0, 0].real), float(P[0, 0].imag)])
        rec['krylov_total'].append(int(sum(h['krylov'] for h in hist)))
        rec['true_rel_residual'].append(res)
        rec['refinement'].append(hist)
        rec['seconds'].append(round(time.time() - t0, 1))
        with open(path, 'w') as f:
            json.dump(rec, f, indent=1)
        print('%s freq %d: residual %.2e, sigma_abs %.12e, %.0f s' % (case, i, res, row[9], time.time() - t0),
              flush=True)


if __name__ == '__main__':
    ap = argparse.ArgumentParser()
    ap.add_argument('cases', nargs='*', default=['ag_sphere_r35', 'agau_bowtie_e80'])
    ap.add_argument('--threads', type=int, default=0)
    a = ap.parse_args()
    for c in a.cases:
        run(c, a.threads)
