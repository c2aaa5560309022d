"""The reference's three per-frequency solver modes, restated (test oracle).

TEST INFRASTRUCTURE ONLY (see ``oracle/__init__.py``).

``solve`` follows ``src/solvers/algorithm_module.f90``:
  inversion         -> solve_w_inversion (:189-327) + complex_inversion (:510-541)
  iterative         -> solve_w_iter_mem (:334-410) + complex_gmres_iterative (:548-587)
  iterative on the fly -> solve_w_iter_on_the_fly (:417-465)
The GMRES columns are skipped, as in the reference, when no real part of the
right-hand side column exceeds 1e-15 (:568-585); a skipped column keeps the
right-hand side values.  On-memory and on-the-fly differ in the reference only
in how A x is formed; the oracle forms it densely for both.
"""
import numpy as np

from . import model
from .gmres import gmres


def solve(s, method=None, tol=None, freqs=None, traces=None):
    """Returns dict with 'x' (F, n_var, 3), 'polar' (F, 3, 3), 'results' (F, 20), 'steps'."""
    method = method or s.method
    op = model.Operator(s)
    tol = s.tol if tol is None else tol
    idx = range(len(s.freqs)) if freqs is None else freqs
    X, P, R, steps = [], [], [], []
    for i in idx:
        b = op.rhs(i)
        x = b.copy()
        st = [0, 0, 0]
        if method == 'inversion':
            A = op.matrix(i)
            x = np.linalg.solve(A, b)
        else:
            for c in range(3):
                if s.polarization not in ('all', 'xyz'[c]):
                    continue
                if not np.any(b[:, c].real > 1.0e-15):
                    continue
                tr = [] if traces is not None else None
                x[:, c], st[c] = gmres(lambda v: op.matvec(i, v), b[:, c], tol,
                                       s.n_dim_gmres, s.n_iter, trace=tr)
                if traces is not None:
                    traces.append((i, c, tr))
        Pw = model.polar(s, x)
        X.append(x)
        P.append(Pw)
        R.append(model.results_row(Pw, s.freqs[i]))
        steps.append(st)
    return {'x': np.array(X), 'polar': np.array(P), 'results': np.array(R), 'steps': steps}
