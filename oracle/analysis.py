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


def bem_field(centres, q, e0, i_pol, points):
    """calculate_induced_field_at_point_bem (src/bem/bem_module.f90:1152-1222) with
    calculate_induced_field_q_bem (src/matrix/matrix_module.f90:1444-1464): centres
    (n, 3) and points (P, 3) in bohr, q the (area-weighted) complex charges.  A point
    is outside when it lies farther from the centre of mass (mean of the centres)
    than its nearest tessera plus 0.5 Angstrom; inside, the field is zero; outside,
    E0 along i_pol minus sum q d / |d|^3 (d = centre - point, |d| > 0.1 bohr)."""
    com = centres.mean(axis=0)
    out = np.zeros((points.shape[0], 3), dtype=np.complex128)
    margin = 0.5 * 1.8897261254578281
    for p, pt in enumerate(points):
        d = centres - pt[None, :]
        r = np.sqrt((d ** 2).sum(axis=1))
        l = int(np.argmin(r))                    # the first nearest tessera
        if np.sqrt(((pt - com) ** 2).sum()) <= np.sqrt(((centres[l] - com) ** 2).sum()) + margin:
            continue
        out[p, i_pol] = e0
        far = r > 1.0e-1
        out[p] -= ((d[far] * (q[far] / r[far] ** 3)[:, None])).sum(axis=0)
    return out
