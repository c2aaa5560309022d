"""BEM (DPCM / IEFPCM) restatement of the reference (test oracle).

TEST INFRASTRUCTURE ONLY (see ``oracle/__init__.py``).

Follows src/bem/bem_module.f90 and src/bem/accurate_green_function.f90:
  read_gmsh_file / read_faces (:224-415)   GMSH 2.2 ASCII, vertices in Angstrom
  create_tesserae (:420-491)               centroids, normals, tangents, areas (bohr)
  construct_constant_matrix_bem (:678-782) D (approximate or accurate Green function),
                                           S A^-1 and -(2 pi I + D) for IEFPCM
  accurate_green_function.f90              polar Gauss-Lobatto diagonal integrals,
                                           28-point Strang-Fix near off-diagonals,
                                           near-element selection, -2 pi closure
  construct_dynamic_field_rhs_bem (:788-873), construct_dynamic_matrix_bem (:881-933),
  new_gmres_diagonal_shift_bem (:977-997), calculate_dynamic_polar_bem (:1051-1142)
"""
import math
import os

import numpy as np

from . import model
from .keywords import read_keyword_file, TO_BOHR
from .gmres import gmres

DIAG_PARAM = 1.0694

# Strang & Fix, "An Analysis of the Finite Element Method" (1973): 28-point
# rule on the unit triangle (barycentric x, y; weights sum to 1), the table of
# accurate_green_function.f90:138-238.
_SF_A = (0.9480217181434233, 0.02598914092828833)
_SF_B = (0.8114249947041546, 0.09428750264792270)
_SF_C = (0.01072644996557060, 0.4946367750172147)
_SF_D = (0.5853132347709715, 0.2073433826145142)
_SF_E = (0.1221843885990187, 0.4389078057004907)
SF_X = [0.3333333333333333,
        _SF_A[0], _SF_A[1], _SF_A[1], _SF_B[0], _SF_B[1], _SF_B[1], _SF_C[0], _SF_C[1], _SF_C[1],
        _SF_D[0], _SF_D[1], _SF_D[1], _SF_E[0], _SF_E[1], _SF_E[1],
        0.6779376548825902, 0.6779376548825902, 0.04484167758913055, 0.04484167758913055,
        0.27722066752827925, 0.27722066752827925,
        0.8588702812826364, 0.8588702812826364, 0.0, 0.0, 0.1411297187173636, 0.1411297187173636]
SF_Y = [0.3333333333333333,
        _SF_A[1], _SF_A[0], _SF_A[1], _SF_B[1], _SF_B[0], _SF_B[1], _SF_C[1], _SF_C[0], _SF_C[1],
        _SF_D[1], _SF_D[0], _SF_D[1], _SF_E[1], _SF_E[0], _SF_E[1],
        0.04484167758913055, 0.27722066752827925, 0.6779376548825902, 0.27722066752827925,
        0.6779376548825902, 0.04484167758913055,
        0.0, 0.1411297187173636, 0.8588702812826364, 0.1411297187173636, 0.8588702812826364, 0.0]
SF_W = [0.08797730116222190] + [0.008744311553736190] * 3 + [0.03808157199393533] * 3 + \
    [0.01885544805613125] * 3 + [0.07215969754474100] * 3 + [0.06932913870553720] * 3 + \
    [0.04105631542928860] * 6 + [0.007362383783300573] * 6


def read_msh(path):
    """Vertices (index -> xyz, Angstrom) and triangles (elements with >= 8 integers)."""
    with open(path) as f:
        lines = f.read().replace('\t', ' ').splitlines()
    low = [l.strip().lower() for l in lines]
    i0 = low.index('$nodes')
    i1 = low.index('$endnodes')
    idx, xyz = [], []
    for l in lines[i0 + 2:i1]:
        p = l.split()
        idx.append(int(p[0]))
        xyz.append([float(p[1]), float(p[2]), float(p[3])])
    e0 = low.index('$elements')
    ne = int(lines[e0 + 1].split()[0])
    faces = []
    for l in lines[e0 + 2:e0 + 2 + ne]:
        p = l.split()
        if len(p) >= 8:
            faces.append([int(p[5]), int(p[6]), int(p[7])])
    return np.array(idx), np.array(xyz), np.array(faces)


def tesserae(idx, xyz, faces, normal_factor):
    """create_tesserae: everything in bohr (bem_module.f90:420-491)."""
    pos = {k: v * TO_BOHR for k, v in zip(idx, xyz)}
    n = len(faces)
    tri = np.array([[pos[f[0]], pos[f[1]], pos[f[2]]] for f in faces])    # (n, 3 verts, 3)
    c = tri.sum(axis=1) / 3.0
    a = tri[:, 1] - tri[:, 0]
    b = tri[:, 2] - tri[:, 0]
    t1 = -a / np.linalg.norm(a, axis=1)[:, None]
    cr = np.cross(a, b)
    nc = np.linalg.norm(cr, axis=1)
    area = nc / 2.0
    nrm = normal_factor * cr / nc[:, None]
    t2 = np.cross(nrm, t1)
    return dict(n=n, tri=tri, coord=c, normal=nrm, t1=t1, t2=t2, area=area)


def lgl(npol):
    """legendre_gauss_lobatto_integration (accurate_green_function.f90:361-434)."""
    x = np.cos(math.pi * np.arange(npol) / (npol - 1))
    xold = np.full(npol, 2.0)
    P = np.zeros((npol, npol))
    check = np.max(np.abs(x - xold))
    # the convergence test sees the change of the previous sweep, so one more
    # Newton update follows it, and the weights use the last Vandermonde matrix
    while check > 2.2204e-16:
        check = np.max(np.abs(x - xold))
        xold = x.copy()
        P[:, 0] = 1.0
        P[:, 1] = x
        for j in range(2, npol):
            P[:, j] = ((2 * j - 1) * x * P[:, j - 1] - (j - 1) * P[:, j - 2]) / j
        x = xold - (x * P[:, npol - 1] - P[:, npol - 2]) / (npol * P[:, npol - 1])
    w = 2.0 / (npol * (npol - 1) * P[:, npol - 1] ** 2)
    return x, w


def polar_rule(npol1=8, npol2=6):
    """tesserae_integration_polar_coordinates (accurate_green_function.f90:245-356)."""
    p1, w1 = lgl(npol1)
    p2, w2 = lgl(npol2)
    rho = 0.5 * (p1 + 1.0 + 1.0e-06)
    phi = math.pi * (270.0 + 60.0 * p2) / 180.0
    tphi = np.repeat(phi, npol1)
    trho = np.tile(rho, npol2)
    phi0 = (120.0 / 180.0) * math.pi
    s = np.abs(2.0 * np.sin(tphi))
    tx = np.concatenate([np.cos(tphi + k * phi0) * trho / s for k in range(3)])
    ty = np.concatenate([np.sin(tphi + k * phi0) * trho / s for k in range(3)])
    ix = (1.0 - math.sqrt(3.0) * tx - ty) / 3.0
    iy = (1.0 + math.sqrt(3.0) * tx - ty) / 3.0
    tw = np.outer(w2, w1).ravel()          # w1(i) w2(j) at i + npol1 j
    w = np.tile(tw * trho * (np.abs(1.0 / s)) ** 2, 3)
    return ix, iy, w / w.sum()


class Bem:
    """A BEM system built from a reference keyword file."""

    def __init__(self, kwpath):
        base = os.path.dirname(os.path.abspath(kwpath))
        kw = read_keyword_file(kwpath)[0]
        self.variant = kw.get('bem variant', 'dpcm').strip()
        self.green = kw.get('bem green function', 'approximate').strip()
        self.sphere_r = float(kw.get('bem sphere radius', '0').replace('d', 'e'))
        self.eps_s = float(kw.get('bem epsilon solvent', '1').replace('d', 'e'))
        nf = float(kw.get('bem normal scalar factor', '1').replace('d', 'e'))
        msh = kw['bem mesh file'].strip()
        idx, xyz, faces = read_msh(msh if os.path.isabs(msh) else os.path.join(base, msh))
        self.t = tesserae(idx, xyz, faces, nf)
        self.n_var = self.t['n']
        self.e0 = float(kw.get('field field intensity', 1e-4))
        self.polarization = kw.get('field polarization', 'all')
        self.method = kw.get('algorithm method', 'inversion')
        n = int(float(kw['field nfreq']))
        fmin, fmax = float(kw['field min freq']), float(kw['field max freq'])
        if fmin == 0.0 and fmax == 0.0:
            self.freqs = np.array([float(x) for x in kw['field external freq'].replace(',', ' ').split()][:n])
        else:
            st = float(kw['field step freq'])
            self.freqs = np.array([fmin + st * i for i in range(n)])
        perm = kw.get('bem permittivity', 'none').strip()
        pfile = kw.get('bem permittivity file', 'none').strip()
        if perm == 'silver etchegoin':
            self.eps = model.silver_etchegoin(self.freqs, 'epsilon')
        elif perm == 'gold etchegoin':
            self.eps = model.gold_etchegoin(self.freqs, 'epsilon')
        else:
            self.eps = model.read_permittivity_file(pfile if os.path.isabs(pfile) else os.path.join(base, pfile),
                                                    self.freqs)
        self.tol = float(kw.get('algorithm tolerance', 0.0)) * math.sqrt(self.n_var)
        self.n_dim_gmres = int(float(kw.get('algorithm gmres dimension', 0)))
        self.D = self.green_derivative()
        if self.variant == 'iefpcm':
            c = self.t['coord']
            r = np.linalg.norm(c[:, None, :] - c[None, :, :], axis=2)
            a = self.t['area']
            with np.errstate(divide='ignore'):
                M = 1.0 / r
            M[np.diag_indices(self.n_var)] = DIAG_PARAM * np.sqrt(4.0 * math.pi * a) / a
            self.M = M
            # the IEF right-hand side uses -(2 pi I + D) as written before the
            # accurate refinement of the diagonal (bem_module.f90:747-755)
            self.G = self._d_pre_refinement - 2.0 * math.pi * np.eye(self.n_var)

    def green_derivative(self):
        t = self.t
        c, nrm, a = t['coord'], t['normal'], t['area']
        n = self.n_var
        d = c[:, None, :] - c[None, :, :]
        r = np.linalg.norm(d, axis=2)
        with np.errstate(divide='ignore', invalid='ignore'):
            D = a[None, :] * np.einsum('ijk,ik->ij', d, nrm) / r ** 3
        if self.green != 'accurate':
            D[np.diag_indices(n)] = DIAG_PARAM * np.sqrt(4.0 * math.pi * a) / (2.0 * self.sphere_r)
            self._d_pre_refinement = D.copy()
            return D
        tri = t['tri']
        # diagonal: polar rule around each centroid
        ix, iy, w = polar_rule()
        bary = np.stack([ix, iy, 1.0 - ix - iy], axis=1)               # (144, 3)
        pts = np.einsum('pk,ikx->ipx', bary, tri)                       # (n, 144, 3)
        v = c[:, None, :] - pts
        dist = np.linalg.norm(v, axis=2)
        gn = -np.sum(w[None, :] * a[:, None] * np.einsum('ipx,ix->ip', v, nrm) / dist ** 3, axis=1)
        dist2 = np.where(dist < 1.0e-4, dist.max() * 1.0e-4, dist)
        g1 = -np.sum(w[None, :] * a[:, None] * np.einsum('ipx,ix->ip', v, t['t1']) / dist2 ** 3, axis=1)
        g2 = -np.sum(w[None, :] * a[:, None] * np.einsum('ipx,ix->ip', v, t['t2']) / dist2 ** 3, axis=1)
        gvec = nrm * gn[:, None] + t['t1'] * g1[:, None] + t['t2'] * g2[:, None]
        # near elements: centroid distance below the circumradius of tessera j
        rad = np.max(np.linalg.norm(c[:, None, :] - tri, axis=2), axis=1)
        norm2 = np.sum(c ** 2, axis=1)
        tmp = norm2[:, None] + norm2[None, :] - 2.0 * (c @ c.T)
        tmp[tmp < 1.0e-10] = 0.0
        sel = np.sqrt(tmp) - rad[None, :]
        sf = np.stack([np.array(SF_X), np.array(SF_Y), 1.0 - np.array(SF_X) - np.array(SF_Y)], axis=1)
        qp = np.einsum('pk,jkx->jpx', sf, tri)                          # (n, 28, 3)
        sw = np.array(SF_W)
        for i, j in zip(*np.nonzero(sel < 0.0)):
            if i == j:
                D[i, i] = -np.dot(gvec[i], nrm[i])
            else:
                vv = c[i][None, :] - qp[j]
                nn = np.linalg.norm(vv, axis=1)
                off = -np.sum((sw * a[j])[:, None] * vv / nn[:, None] ** 3, axis=0)
                D[i, j] = -np.dot(off, nrm[i])
        self._d_pre_refinement = D.copy()
        # final refinement (accurate_green_function.f90:796-838)
        tmp2 = D / a[None, :] * a[:, None]
        colsum = tmp2.sum(axis=0)
        gvec = gvec + nrm * (-2.0 * math.pi + colsum)[:, None]
        D[np.diag_indices(n)] = -np.sum(gvec * nrm, axis=1)
        return D

    def z(self, i):
        e = self.eps[i]
        return 2.0 * math.pi * (self.eps_s + e) / (self.eps_s - e)

    def matrix(self, i):
        A = self.D.astype(np.complex128)
        A[np.diag_indices(self.n_var)] += self.z(i)
        if self.variant == 'iefpcm':
            A = -(A @ self.M)
        return A

    def matvec(self, i, x):
        """The GMRES operator of the reference: D x + z x (no S A^-1 factor)."""
        return self.D @ x + self.z(i) * x

    def rhs(self, i=0):
        n = self.n_var
        b = np.zeros((n, 3), dtype=np.complex128)
        cols = [0, 1, 2] if self.polarization == 'all' else [{'x': 0, 'y': 1, 'z': 2}[self.polarization]]
        for p in cols:
            if self.variant == 'iefpcm':
                b[:, p] = self.G @ (-self.e0 * self.t['coord'][:, p])
            else:
                b[:, p] = -self.e0 * self.t['normal'][:, p]
        return b

    def polar(self, x):
        c = self.t['coord']
        wts = np.ones(self.n_var) if self.variant == 'iefpcm' else self.t['area']
        return (c.T @ (wts[:, None] * x)) / self.e0

    def solve(self, method=None, traces=None, tol=None):
        method = method or ('inversion' if self.method == 'inversion' else 'gmres')
        tol = self.tol if tol is None else tol
        X, R, steps = [], [], []
        for i in range(len(self.freqs)):
            b = self.rhs(i)
            x = b.copy()
            st = [0, 0, 0]
            if method == 'inversion':
                x = np.linalg.solve(self.matrix(i), b)
            else:
                for c in range(3):
                    if not np.any(b[:, c].real > 1.0e-15):
                        continue
                    tr = [] if traces is not None else None
                    x[:, c], st[c] = gmres(lambda v: self.matvec(i, v), b[:, c], tol, self.n_dim_gmres,
                                           trace=tr)
                    if traces is not None:
                        traces.append((i, c, tr))
            X.append(x)
            R.append(model.results_row(self.polar(x), self.freqs[i]))
            steps.append(st)
        return {'x': np.array(X), 'results': np.array(R), 'steps': steps}
