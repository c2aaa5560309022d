"""Static FQ / FQFMu solves and the principal-axis rotation (test oracle).

TEST INFRASTRUCTURE ONLY (see ``oracle/__init__.py``).

Follows the reference's static and ground-state path:
  * interaction blocks construct_static_t_qq (Coulomb / Ohno / Gaussian kernel),
    construct_static_t_qmu, construct_static_t_mumu (diagonal 1/alpha for the
    static models)                    src/matrix/matrix_module.f90:58-345
  * charge-constraint rows and columns add_lagrangian_blocks
                                      src/matrix/matrix_module.f90:351-382
  * matrix layout: FQ [T_qq L; L^T 0] (construct_static_matrix_fq,
    src/forcefield/fq_module.f90:179-207); FQFMu [T_qq L T_qmu; L^T 0 0;
    T_qmu^T 0 T_mumu] (construct_static_matrix_fqfmu,
    src/forcefield/fqfmu_module.f90:81-132)
  * right-hand sides: ground state -chi per atom (fq_module.f90:212-242);
    static field construct_static_field_rhs_q / _mu
                                      src/rhs/rhs_module.f90:43-127
  * solve: dsysv on the upper triangle (real_inversion,
    src/solvers/algorithm_module.f90:469-504); the energy -1/2 x.b
    (calculate_energy_fq, fq_module.f90:358-374); the static polarizability
    R^T J^-1 R - (1^T J^-1 R)^T (1^T J^-1 1)^-1 (1^T J^-1 R) with J the charge
    block (calculate_static_polar_fq, fq_module.f90:379-595)
  * molecules: n_atoms_per_molecule from runs of equal molecule index
    (create_n_atoms_per_molecule, src/input_output/input_module.f90:1007-1030)
  * principal axes: centre of mass, inertia tensor, eigenvectors in ascending
    order of the eigenvalues, coordinates r' = V^T r (rotate_principal_axis,
    src/target/target_module.f90:684-835; masses mass_atom :233-289).
Everything in bohr and atomic units.
"""
import math

import numpy as np
from scipy.special import erf

TO_BOHR = 1.8897261254578281

# atom names the reference maps to atomic numbers (assign_atomic_number,
# src/target/target_module.f90:315-378); unknown names map to 0
ATOM_NAMES = {'h': 1, 'hw': 1, 'h-hw': 1, 'he': 2, 'li': 3, 'be': 4, 'b': 5, 'c': 6, 'n': 7, 'o': 8,
              'ow': 8, 'o-ow': 8, 'f': 9, 'ne': 10, 'na': 11, 'mg': 12, 'al': 13, 'si': 14, 'p': 15,
              's': 16, 'cl': 17, 'ar': 18, 'ag': 47, 'cu': 29, 'au': 79}

# standard atomic masses (mass_atom, src/target/target_module.f90:233-289)
MASS = {1: 1.00794, 2: 4.00260, 3: 6.941, 4: 9.01218, 5: 10.81, 6: 12.0107, 7: 14.0067, 8: 15.9990,
        9: 18.998403, 10: 20.179, 11: 22.989770, 12: 24.305, 13: 26.98154, 14: 28.0855, 15: 30.97376,
        16: 32.06, 17: 35.453, 18: 39.948, 29: 63.546, 47: 107.8682, 79: 196.9665}


def atoms_per_molecule(imol):
    """create_n_atoms_per_molecule: a new molecule starts where the index changes."""
    n_mol = len(set(int(i) for i in imol))
    if n_mol == 1:
        return [len(imol)]
    apm = [1] * n_mol
    k = 0
    for i in range(len(imol) - 1):
        if imol[i] == imol[i + 1]:
            apm[k] += 1
        else:
            k += 1
    return apm


def t_qq(coord, types, eta, r_q, kernel):
    """construct_static_t_qq (matrix_module.f90:58-115)."""
    d = np.sqrt(((coord[:, None, :] - coord[None, :, :]) ** 2).sum(-1))
    e = eta[types]
    ea = 0.5 * (e[:, None] + e[None, :])
    if kernel == 'ohno':
        return ea / np.sqrt(1.0 + ea ** 2 * d ** 2)
    with np.errstate(divide='ignore', invalid='ignore'):
        if kernel == 'coulomb':
            T = 1.0 / d
        elif kernel == 'gaussian':
            rq = r_q[types]
            T = erf(d / np.sqrt(rq[:, None] ** 2 + rq[None, :] ** 2)) / d
        else:
            raise ValueError('unknown kernel %r' % kernel)
    T[np.diag_indices(len(types))] = (e + e) / 2.0
    return T


def _screen(d, R):
    return erf(d / R) - ((2.0 * d) / (math.sqrt(math.pi) * R)) * np.exp(-d ** 2 / R ** 2)


def t_qmu(coord, types, r_q, r_mu):
    """construct_static_t_qmu (matrix_module.f90:120-167): T(i, 3j + k) = r_ij,k / r^3 * f."""
    n = len(types)
    r = coord[:, None, :] - coord[None, :, :]
    d = np.sqrt((r ** 2).sum(-1))
    R = np.sqrt(r_q[types][:, None] ** 2 + r_mu[types][None, :] ** 2)
    with np.errstate(divide='ignore', invalid='ignore'):
        f = _screen(d, R) / d ** 3
    np.fill_diagonal(f, 0.0)
    return (r * f[:, :, None]).reshape(n, 3 * n)


def t_mumu(coord, types, r_mu, alpha):
    """construct_static_t_mumu (matrix_module.f90:240-345), 1/alpha on the diagonal blocks."""
    n = len(types)
    r = coord[:, None, :] - coord[None, :, :]
    d = np.sqrt((r ** 2).sum(-1))
    R = np.sqrt(r_mu[types][:, None] ** 2 + r_mu[types][None, :] ** 2)
    with np.errstate(divide='ignore', invalid='ignore'):
        fd1 = _screen(d, R)
        fd2 = (4.0 / (math.sqrt(math.pi) * R ** 3)) * np.exp(-d ** 2 / R ** 2)
        rr = r[:, :, :, None] * r[:, :, None, :]
        B = (-3.0 * rr / d[:, :, None, None] ** 5 + np.eye(3) / d[:, :, None, None] ** 3) * fd1[:, :, None, None] \
            + fd2[:, :, None, None] * rr / d[:, :, None, None] ** 2
    idx = np.arange(n)
    B[idx, idx] = np.eye(3)[None, :, :] / alpha[types][:, None, None]
    return B.transpose(0, 2, 1, 3).reshape(3 * n, 3 * n)


def lagrangian_rows(n_q, apm):
    """add_lagrangian_blocks (matrix_module.f90:351-382): the atoms of molecule k are
    rows apm[k-1]*k .. apm[k-1]*k + apm[k] - 1 (0-based), as the reference indexes them
    (exact for molecules of equal size)."""
    L = np.zeros((n_q, len(apm)))
    for k in range(len(apm)):
        lo = 0 if k == 0 else apm[k - 1] * k
        hi = apm[0] if k == 0 else apm[k - 1] * k + apm[k]
        if hi > n_q:
            raise ValueError('molecule %d: the constraint rows run past the atoms' % (k + 1))
        L[lo:hi, k] = 1.0
    return L


class Static:
    """A static FQ / FQFMu problem (bohr, a.u.)."""

    def __init__(self, forcefield, kernel, coord, types, apm, chi, eta, alpha, r_q, r_mu,
                 rhs_form='field', e0=0.0):
        self.ff, self.kernel = forcefield, kernel
        self.coord = np.asarray(coord, dtype=np.float64).reshape(-1, 3)
        self.types = np.asarray(types, dtype=np.int64)
        self.apm = list(apm)
        self.chi, self.eta, self.alpha, self.r_q, self.r_mu = (np.asarray(v, dtype=np.float64)
                                                                 for v in (chi, eta, alpha, r_q, r_mu))
        self.rhs_form, self.e0 = rhs_form, float(e0)
        self.n = len(self.types)
        self.n_mol = len(self.apm)
        self.n_fq = self.n + self.n_mol
        self.n_var = self.n_fq if forcefield == 'fq' else 4 * self.n + self.n_mol

    def matrix(self):
        n, nfq = self.n, self.n_fq
        A = np.zeros((self.n_var, self.n_var))
        A[:n, :n] = t_qq(self.coord, self.types, self.eta, self.r_q, self.kernel)
        L = lagrangian_rows(n, self.apm)
        A[:n, n:nfq] = L
        A[n:nfq, :n] = L.T
        if self.ff == 'fqfmu':
            Tqm = t_qmu(self.coord, self.types, self.r_q, self.r_mu)
            A[:n, nfq:] = Tqm
            A[nfq:, :n] = Tqm.T
            A[nfq:, nfq:] = t_mumu(self.coord, self.types, self.r_mu, self.alpha)
        return A

    def rhs_ground_state(self):
        b = np.zeros((self.n_var, 1))
        b[:self.n, 0] = -self.chi[self.types]
        return b

    def rhs_static_field(self):
        """construct_static_field_rhs_q / _mu (rhs_module.f90:43-127)."""
        b = np.zeros((self.n_var, 3))
        c = self.coord
        if self.rhs_form == 'potential':
            b[:self.n] = -self.e0 * np.abs(c - c.min(axis=0))
        elif self.rhs_form == 'field':
            b[:self.n] = -self.e0 * c
        if self.ff == 'fqfmu':
            # the reference writes e0 when e0 == 0 (|e0| <= 1e-14) and 1 otherwise
            v = self.e0 if abs(self.e0) <= 1.0e-14 else 1.0
            for k in range(3):
                b[self.n_fq + k::3, k] = v
        return b

    def solve(self, what='energy'):
        A = self.matrix()
        U = np.triu(A)
        S = U + np.triu(A, 1).T          # dsysv('U') reads the upper triangle
        b = self.rhs_ground_state() if what == 'energy' else self.rhs_static_field()
        x = np.linalg.solve(S, b)
        out = {'variables': x, 'rhs': b, 'charges': x[:self.n], 'charge_sum': x[:self.n].sum(axis=0)}
        if self.ff == 'fqfmu':
            out['dipoles'] = x[self.n_fq:]
        if what == 'energy':
            out['energy'] = -0.5 * float(x[:, 0] @ b[:, 0])
        elif self.ff == 'fq':
            out.update(self.static_polar(A))
        return out

    def static_polar(self, A):
        n, nfq = self.n, self.n_fq
        J = A[:n, :n]
        Ji = np.linalg.inv(J)
        R = self.coord
        X = Ji @ R
        pol = R.T @ X
        L = A[:n, n:nfq]
        J11 = L.T @ Ji @ L
        J1R = L.T @ X
        J11i = np.linalg.inv(J11)
        pol = pol - J1R.T @ J11i @ J1R
        # the reference prints J_1_1 after inverting it in place
        return {'polar': pol, 'polar_iso': float(np.trace(pol) / 3.0), 'j_inverse': Ji, 'j_1_1': J11i}


def principal_axes(coord, znum):
    """rotate_principal_axis (target_module.f90:684-835).  Returns (rotated coordinates,
    eigenvalues, eigenvectors as columns).  LAPACK leaves each eigenvector's sign to the
    implementation; the sign here makes the last nonzero component of each positive,
    which reproduces the reference log's rotated geometry."""
    c = np.asarray(coord, dtype=np.float64).reshape(-1, 3)
    m = np.array([MASS[int(z)] for z in znum])
    com = (m[:, None] * c / m.sum()).sum(axis=0)
    c = c - com
    x, y, z = c[:, 0], c[:, 1], c[:, 2]
    I = np.array([[(m * (y ** 2 + z ** 2)).sum(), -(m * x * y).sum(), -(m * x * z).sum()],
                  [0.0, (m * (x ** 2 + z ** 2)).sum(), -(m * y * z).sum()],
                  [0.0, 0.0, (m * (y ** 2 + x ** 2)).sum()]])
    I = np.triu(I) + np.triu(I, 1).T
    w, V = np.linalg.eigh(I)
    for k in range(3):
        nz = np.nonzero(V[:, k])[0]
        if len(nz) and V[nz[-1], k] < 0:
            V[:, k] = -V[:, k]
    return c @ V, w, V


def static_from_keyword_file(path):
    """The static problem of a reference keyword file (the front end's output)."""
    from .keywords import read_keyword_file
    kw, types, _, _, _ = read_keyword_file(path)
    with open(path) as f:
        lines = f.read().splitlines()
    g0 = next(i for i, l in enumerate(lines) if l.startswith('input_geometry'))
    n = int(float(kw['number of atoms']))
    names = [t['name'] for t in types]
    geo = [l.split() for l in lines[g0 + 1:g0 + 1 + n]]
    tix = [names.index(g[0]) for g in geo]
    imol = [int(g[1]) for g in geo]
    coord = np.array([[float(v) for v in g[2:5]] for g in geo]) * TO_BOHR
    getv = lambda k: [float(t.get(k, 0.0)) for t in types]  # noqa: E731
    # the solve follows the field type (src/plasmonX.f90:40-46): a static field
    # solves the three field right-hand sides, no field the ground state
    what = 'static' if kw.get('field type', 'none').strip().lower() == 'static' else 'energy'
    st = Static(kw['forcefield static'].lower(), kw['forcefield kernel'].lower(), coord, tix,
                atoms_per_molecule(imol), getv('chi'), getv('eta'), getv('alpha'), getv('rq'), getv('rmu'),
                rhs_form=kw.get('field rhs type', 'field'), e0=float(kw.get('field field intensity', 0.0)))
    rotated = None
    if kw.get('control principal axes', 'False').strip().lower() == 'true':
        z = [ATOM_NAMES.get(g[0].lower(), 0) for g in geo]
        st.coord, _, _ = principal_axes(st.coord, z)
        rotated = st.coord / TO_BOHR
    return st, what, rotated
