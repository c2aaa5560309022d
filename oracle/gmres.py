"""Restatement of the reference GMRES (test oracle).

TEST INFRASTRUCTURE ONLY (see ``oracle/__init__.py``).

Follows ``src/solvers/gmres_module.f90:30-228`` step by step:
x0 = 0; V(:,1) = b/||b||; Arnoldi with modified Gram-Schmidt for j < 25 and
classical Gram-Schmidt with one re-orthogonalisation (two zgemv pairs) for
j >= 25; Givens rotations with reference-BLAS zrotg/zrot semantics; the
residual estimate |g_{j+1}| is compared with the *absolute* tolerance; when
it passes, the upper-triangular system is solved, x += V y, and the true
residual ||b - A x|| decides convergence (the reference keeps iterating with
the already-updated x when that check fails).  There is no restart: running
out of Krylov dimension is an error.
"""
import math

import numpy as np
from scipy.linalg import solve_triangular


class GmresNotConverged(RuntimeError):
    pass


def zrotg(ca, cb):
    """Reference BLAS zrotg: returns (c, s, r)."""
    if abs(ca) == 0.0:
        return 0.0, complex(1.0, 0.0), cb
    scale = abs(ca) + abs(cb)
    norm = scale * math.sqrt(abs(ca / scale) ** 2 + abs(cb / scale) ** 2)
    alpha = ca / abs(ca)
    c = abs(ca) / norm
    s = alpha * np.conj(cb) / norm
    return c, s, alpha * norm


def zrot(x, y, c, s):
    return c * x + s * y, c * y - np.conj(s) * x


def gmres(matvec, b, tol, restart, max_iter=1, trace=None, snapshots=None, best_effort=False):
    """Solve A x = b.  ``matvec(v)`` returns A v (including the diagonal shift).

    Returns (x, n_steps).  ``trace`` (a list) receives the logged residuals.
    ``best_effort``: return the least-squares iterate as soon as the logged
    residual passes (no true-residual product), or when the Krylov dimension
    runs out instead of raising: the inner solve of an iterative refinement,
    which computes the true residual itself (the reference raises).
    ``snapshots`` (a dict {level: None}) receives, for every absolute residual
    level, the least-squares iterate of the first step whose logged residual is
    below it (no true-residual check): the convergence history that shows how
    far a solution at ``tol`` is from the ones before it.
    """
    n = b.shape[0]
    m = min(restart, n)
    r = b.astype(np.complex128).copy()
    x = np.zeros(n, dtype=np.complex128)
    normb = np.linalg.norm(r)
    if normb == 0.0:
        return x, 0
    V = np.zeros((n, m + 1), dtype=np.complex128)
    H = np.zeros((m + 1, m + 1), dtype=np.complex128)
    cs = np.zeros(m)
    sn = np.zeros(m, dtype=np.complex128)
    beta = normb
    V[:, 0] = r / beta
    H[0, m] = beta
    for j in range(m):           # reference j = 1..m is j+1 here
        w = matvec(V[:, j])
        if j + 1 < 25:
            for i in range(j + 1):
                H[i, j] = np.vdot(V[:, i], w)
                w = w - H[i, j] * V[:, i]
        else:
            # V^H w as conj(w^H V): the same sums without copying the conjugated basis
            Vj = V[:, :j + 1]
            h = (w.conj() @ Vj).conj()
            w = w - Vj @ h
            t = (w.conj() @ Vj).conj()
            w = w - Vj @ t
            H[:j + 1, j] = h + t
        H[j + 1, j] = np.linalg.norm(w)
        if H[j + 1, j] != 0.0:
            V[:, j + 1] = w / H[j + 1, j]
        for i in range(j):
            H[i, j], H[i + 1, j] = zrot(H[i, j], H[i + 1, j], cs[i], sn[i])
        cs[j], sn[j], _ = zrotg(H[j, j], H[j + 1, j])
        H[j, m], H[j + 1, m] = zrot(H[j, m], H[j + 1, m], cs[j], sn[j])
        H[j, j], H[j + 1, j] = zrot(H[j, j], H[j + 1, j], cs[j], sn[j])
        H[j + 1, j] = 0.0
        resid = abs(H[j + 1, m])
        if trace is not None:
            trace.append(resid)
        if snapshots is not None:
            for level in snapshots:
                if snapshots[level] is None and resid < level:
                    y = solve_triangular(H[:j + 1, :j + 1], H[:j + 1, m], lower=False)
                    snapshots[level] = x + V[:, :j + 1] @ y
        if resid < tol:
            y = solve_triangular(H[:j + 1, :j + 1], H[:j + 1, m], lower=False)
            x = x + V[:, :j + 1] @ y
            if best_effort:
                return x, j + 1          # the refinement computes the true residual itself
            true_res = np.linalg.norm(b - matvec(x))
            if true_res < tol:
                return x, j + 1
    if best_effort:
        y = solve_triangular(H[:m, :m], H[:m, m], lower=False)
        return x + V[:, :m] @ y, m
    raise GmresNotConverged('GMRES not converged and restart GMRES NYI.')
