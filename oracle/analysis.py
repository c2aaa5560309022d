"""Induced field and plasmon density at points (test oracle).

TEST INFRASTRUCTURE ONLY (see ``oracle/__init__.py``).

Follows the analysis step of the reference:
  calculate_induced_field_at_point_wfq / calculate_density_at_point_wfq
      src/wfq/wfq_module.f90:590-650
  calculate_induced_field_at_point_wfqfmu / calculate_density_at_point_wfqfmu
      src/wfq/wfqfmu_module.f90:975-1040
  kernels calculate_induced_field_q / _mu, calculate_density_q / _mu
      src/matrix/matrix_module.f90:1140-1322
Everything in bohr and atomic units; d = r_atom - r_point.
"""
import math

import numpy as np


def field_and_density(coord, rq, rmu, x, e0, i_pol, points, fmu):
    """coord (N, 3) bohr, rq / rmu per atom (N,), x complex (n_var,), points (P, 3) bohr.
    Returns field (P, 3) complex (external field e0 along i_pol included) and
    density (P,) complex."""
    N = coord.shape[0]
    d = coord[None, :, :] - points[:, None, :]                       # (P, N, 3)
    r2 = np.einsum('pnk,pnk->pn', d, d)
    r = np.sqrt(r2)
    far = r > 1.0e-1
    rs = np.where(far, r, 1.0)
    q = x[:N]
    E = np.zeros((points.shape[0], 3), dtype=np.complex128)
    E[:, i_pol] = e0
    R = rq[None, :]
    fac = np.array([[math.erf(v) for v in row] for row in (rs / R)]) - \
        (2.0 / (math.sqrt(math.pi) * R)) * rs * np.exp(-(rs * rs) / (R * R))
    E -= np.einsum('pn,pnk->pk', np.where(far, fac / rs ** 3, 0.0) * q[None, :], d)
    dens = (np.exp(-r2 / (R * R)) / (math.pi ** 1.5 * R ** 3)) @ q
    if fmu:
        mu = x[N:].reshape(N, 3)
        Rm = rmu[None, :]
        em = np.exp(-(rs * rs) / (Rm * Rm))
        fd1 = np.array([[math.erf(v) for v in row] for row in (rs / Rm)]) - \
            ((2.0 * rs) / (math.sqrt(math.pi) * Rm)) * em
        fd2 = (4.0 / (math.sqrt(math.pi) * Rm ** 3)) * em
        dd = np.einsum('pna,pnb->pnab', d, d)
        T = (-3.0 * dd / rs[..., None, None] ** 5 + np.eye(3) / rs[..., None, None] ** 3) * fd1[..., None, None] + \
            fd2[..., None, None] * dd / rs[..., None, None] ** 2
        T = np.where(far[..., None, None], T, 0.0)
        E += np.einsum('pnab,nb->pa', T, mu)
        g = np.exp(-r2 / (Rm * Rm)) / (math.pi ** 1.5 * Rm ** 3)
        dens -= np.einsum('pn,pn->p', 2.0 * g / (Rm * Rm), np.einsum('pnk,nk->pn', d, mu))
    return E, dens
