"""Static FQ / FQFMu problems: the ground state and the static-field response.

Host side of ``plx_static_solve`` and ``plx_principal_axes``.  The reference's
static path (src/plasmonX.f90:37-46) rotates the geometry onto its principal
axes when asked (rotate_principal_axis, src/target/target_module.f90:684-835),
then either solves the static field (solve_static_field,
src/solvers/algorithm_module.f90:120-145: three right-hand sides, charges and
dipoles, the FQ static polarizability) or the ground state (solve_ground_state,
:91-115: right-hand side -chi, the energy).  Both are direct solves; the
reference stops with 'Iterative not implemented ...' otherwise, and so does
``StaticSolver``.

``StaticProblem.from_keyword_file`` reads the keyword file of the reference's
Python front end for a static run (``forcefield static``, ``forcefield
kernel``, ``field type``, ``field rhs type``, ``field field intensity``,
``control principal axes``, the atom types' chi / eta / alpha / rq / rmu and the
geometry with its molecule indices), following
src/input_output/input_module.f90:156-258 and :680-1030; molecules are runs of
equal molecule index (create_n_atoms_per_molecule, :1007-1030).
"""
import ctypes as C

import numpy as np

from . import _lib
from . import materials as M
from .inputs import read_keywords
from .outputs import fortran_f
from .solver import Context


FACTORIZATION = {'auto': 0, 'lu': 1, 'cholesky_mixed': 2, 'cholesky_blocked': 3}


def atoms_per_molecule(mol_index):
    """Number of atoms of each molecule: a molecule starts where the index changes."""
    mol_index = [int(v) for v in mol_index]
    n_mol = len(set(mol_index))
    if n_mol == 1:
        return [len(mol_index)]
    apm = [1] * n_mol
    k = 0
    for a, b in zip(mol_index[:-1], mol_index[1:]):
        if a == b:
            apm[k] += 1
        else:
            k += 1
    return apm


def rotate_principal_axes(coord_bohr, atomic_numbers):
    """Rotated copy of coord (N x 3, bohr) and (eigenvalues, axes) of the inertia tensor."""
    lib = _lib.load()
    c = np.ascontiguousarray(coord_bohr, dtype=np.float64).reshape(-1, 3).copy()
    z = np.ascontiguousarray(atomic_numbers, dtype=np.int32)
    w = np.zeros(3)
    v = np.zeros(9)
    st = lib.plx_principal_axes(len(z), _lib.ptr(z, _lib._ip), _lib.ptr(c), _lib.ptr(w), _lib.ptr(v))
    if st != _lib.PLX_OK:
        raise _lib.PlxError(st, 'principal axes: an atomic number without a mass (%s)' %
                            sorted(set(int(x) for x in z)))
    return c, w, v.reshape(3, 3).T


class StaticProblem:
    """Geometry and parameters of a static FQ / FQFMu calculation (bohr, a.u.)."""

    def __init__(self, forcefield, kernel, coord_ang, type_names, atom_types, mol_index, chi, eta, alpha=None,
                 r_q=None, r_mu=None, what='energy', rhs_form='field', e0=0.0, principal_axes=False,
                 atom_names=None, method='inversion', factorization='auto'):
        self.forcefield = forcefield.lower()
        self.kernel = kernel.lower()
        if self.forcefield not in _lib.STATIC_FF:
            raise ValueError('static forcefield must be fq or fqfmu, got %r' % forcefield)
        if self.kernel not in _lib.KERNEL:
            raise ValueError('kernel must be coulomb, ohno or gaussian, got %r' % kernel)
        if what not in _lib.STATIC_WHAT:
            raise ValueError("what must be 'energy' (ground state) or 'static' (static field)")
        self.what = what
        self.method = method
        if factorization not in FACTORIZATION:
            raise ValueError("factorization must be 'auto', 'lu', 'cholesky_mixed' or 'cholesky_blocked'")
        # 'auto': charge constraints eliminated, the rest factored by a double-precision
        # Cholesky (LU of the full system where that does not apply); 'cholesky_mixed':
        # the same with a single-precision factor refined in double; 'lu': LU of the
        # full system, the reference's form
        self.factorization = factorization
        self.type_names = list(type_names)
        nt = len(self.type_names)
        self.atom_types = np.ascontiguousarray(atom_types, dtype=np.int32)
        self.n_atoms = len(self.atom_types)
        self.mol_index = np.asarray(mol_index, dtype=np.int64)
        self.apm = np.ascontiguousarray(atoms_per_molecule(self.mol_index), dtype=np.int32)
        self.n_mol = len(self.apm)
        z = lambda v: np.zeros(nt) if v is None else np.ascontiguousarray(v, dtype=np.float64)  # noqa: E731
        self.chi, self.eta, self.alpha, self.r_q, self.r_mu = z(chi), z(eta), z(alpha), z(r_q), z(r_mu)
        self.rhs_form = rhs_form
        self.e0 = float(e0)
        names = atom_names if atom_names is not None else [self.type_names[t] for t in self.atom_types]
        self.znum = np.array([M.atom_name_number(n) for n in names], dtype=np.int32)
        self.coord_ang = np.ascontiguousarray(coord_ang, dtype=np.float64).reshape(-1, 3)
        self.coord = self.coord_ang * M.TO_BOHR
        self.rotated = bool(principal_axes)
        self.inertia = None
        if self.rotated:
            self.coord, w, v = rotate_principal_axes(self.coord, self.znum)
            self.inertia = {'eigenvalues': w, 'axes': v}

    @property
    def n_var(self):
        return self.n_atoms + self.n_mol if self.forcefield == 'fq' else 4 * self.n_atoms + self.n_mol

    def desc(self):
        """plx_static_desc over this problem's arrays (kept alive by the problem)."""
        self._coord_c = np.ascontiguousarray(self.coord, dtype=np.float64)
        d = _lib.StaticDesc()
        d.forcefield = _lib.STATIC_FF[self.forcefield]
        d.kernel = _lib.KERNEL[self.kernel]
        d.n_atoms, d.n_types, d.n_mol = self.n_atoms, len(self.type_names), self.n_mol
        d.rhs_potential = 1 if self.rhs_form == 'potential' else 0
        d.coord = _lib.ptr(self._coord_c)
        d.atom_type = _lib.ptr(self.atom_types, _lib._ip)
        d.atoms_per_molecule = _lib.ptr(self.apm, _lib._ip)
        d.chi, d.eta, d.alpha = _lib.ptr(self.chi), _lib.ptr(self.eta), _lib.ptr(self.alpha)
        d.r_q, d.r_mu = _lib.ptr(self.r_q), _lib.ptr(self.r_mu)
        d.e0 = self.e0
        d.factorization = FACTORIZATION[self.factorization]
        return d

    @classmethod
    def from_keyword_text(cls, text):
        kw, types, _, _, _ = read_keywords(text)
        lines = text.splitlines()
        g0 = next(i for i, l in enumerate(lines) if l.startswith('input_geometry'))
        n = int(float(kw['number of atoms']))
        geo = [l.split() for l in lines[g0 + 1:g0 + 1 + n]]
        names = [t['name'] for t in types]
        get = lambda k: [float(t.get(k, 0.0)) for t in types]  # noqa: E731
        # the solve follows the field type (src/plasmonX.f90:40-46)
        what = 'static' if kw.get('field type', 'none').strip().lower() == 'static' else 'energy'
        return cls(kw['forcefield static'], kw.get('forcefield kernel', 'none'),
                   np.array([[float(v) for v in g[2:5]] for g in geo]), names, [names.index(g[0]) for g in geo],
                   [int(g[1]) for g in geo], get('chi'), get('eta'), get('alpha'), get('rq'), get('rmu'),
                   what=what, rhs_form=kw.get('field rhs type', 'field'),
                   e0=float(kw.get('field field intensity', 0.0)),
                   principal_axes=kw.get('control principal axes', 'False').strip().lower() == 'true',
                   atom_names=[g[0] for g in geo], method=kw.get('algorithm method', 'inversion'))

    @classmethod
    def from_keyword_file(cls, path):
        with open(path) as f:
            return cls.from_keyword_text(f.read())


class StaticSolver:
    """Direct solve of a StaticProblem on one device."""

    def __init__(self, problem, ctx=None, device=0):
        self.prob = problem
        self.own_ctx = ctx is None
        self.ctx = Context(device) if ctx is None else ctx
        self.lib = self.ctx.lib

    def close(self):
        if self.own_ctx and self.ctx is not None:
            self.ctx.close()
        self.ctx = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def solve(self, polarizability=True):
        """Returns variables (n_var x n_rhs), charges (N x n_rhs), constraint
        multipliers, dipoles (FQFMu: 3N x n_rhs), the charge sums, and the energy
        (ground state) or the static polarizability (static field, FQ)."""
        p = self.prob
        if p.method != 'inversion':
            raise ValueError('Iterative not implemented for %s' %
                             ('static field' if p.what == 'static' else 'ground state'))
        nrhs = 3 if p.what == 'static' else 1
        x = np.zeros((nrhs, p.n_var))          # column-major n_var x n_rhs
        energy = C.c_double()
        want_polar = p.what == 'static' and p.forcefield == 'fq' and polarizability
        polar = np.zeros(9)
        d = p.desc()
        self.ctx.check(self.lib.plx_static_solve(self.ctx.h, C.byref(d), _lib.STATIC_WHAT[p.what], _lib.ptr(x),
                                                 C.byref(energy) if p.what == 'energy' else None,
                                                 _lib.ptr(polar) if want_polar else None))
        X = x.T.copy()
        n, nfq = p.n_atoms, p.n_atoms + p.n_mol
        out = {'variables': X, 'charges': X[:n], 'constraints': X[n:nfq], 'charge_sum': X[:n].sum(axis=0)}
        if p.forcefield == 'fqfmu':
            out['dipoles'] = X[nfq:]
        if p.what == 'energy':
            out['energy'] = energy.value
        if want_polar:
            P = polar.reshape(3, 3).T
            out['polar'] = P
            out['polar_iso'] = float((P[0, 0] + P[1, 1] + P[2, 2]) / 3.0)
        if p.rotated:
            out['rotated_ang'] = p.coord / M.TO_BOHR
        return out


def energy_line(e):
    """The reference's log line (calculate_energy_fq, fq_module.f90:358-374)."""
    return ' Energy = %s a.u.' % fortran_f(e, 14, 8)


def polar_iso_line(v):
    """The reference's log line (calculate_static_polar_fq, fq_module.f90:379-595)."""
    return ' Polar Iso  = %s a.u.' % fortran_f(v, 19, 10)


# FQ / FQFMu water parameters of the reference's static tests (a.u.):
# tests/fq_energy (Ohno kernel) and tests/fqfmu_energy (Gaussian kernel)
WATER_FQ = {'O-OW': dict(chi=0.11685879436, eta=0.58485173233), 'H-HW': dict(chi=1.0e-11, eta=0.62501048888)}
WATER_FQFMU = {'O-OW': dict(chi=0.290842985, eta=0.582518114, alpha=2.218798372),
               'H-HW': dict(chi=0.167571197, eta=0.629326577, alpha=1.190641609)}


def water_cluster(n_mol, forcefield='fq', kernel=None, what='energy', rhs_form='field', e0=0.0, seed=0,
                  spacing=3.1, principal_axes=False, factorization='auto'):
    """A seeded synthetic water cluster: n_mol rigid waters (O-H 0.9572 A, H-O-H
    104.52 deg) with random orientations on a jittered cubic lattice of `spacing`
    Angstrom, one molecule index per water, typed O-OW / H-HW.  Gaussian widths
    follow the front end's defaults (r_q = sqrt(2/pi) / eta, r_mu = (alpha /
    (3 sqrt(pi/2)))^(1/3), python/input_/validation.py:1081-1090)."""
    import math
    rng = np.random.default_rng(seed)
    side = int(math.ceil(n_mol ** (1.0 / 3.0)))
    cells = np.array([(i, j, k) for i in range(side) for j in range(side) for k in range(side)][:n_mol], float)
    centres = cells * spacing + rng.uniform(-0.25, 0.25, size=(n_mol, 3))
    half = math.radians(104.52) / 2.0
    local = np.array([[0.0, 0.0, 0.0], [0.9572 * math.sin(half), 0.0, 0.9572 * math.cos(half)],
                      [-0.9572 * math.sin(half), 0.0, 0.9572 * math.cos(half)]])
    coords, mol = [], []
    for m in range(n_mol):
        q, _ = np.linalg.qr(rng.standard_normal((3, 3)))
        coords.append(centres[m] + local @ q.T)
        mol += [m + 1] * 3
    params = WATER_FQ if forcefield == 'fq' else WATER_FQFMU
    kernel = kernel or ('ohno' if forcefield == 'fq' else 'gaussian')
    names = ['H-HW', 'O-OW']     # the front end orders atom types by name
    eta = np.array([params[n]['eta'] for n in names])
    alpha = np.array([params[n].get('alpha', 0.0) for n in names])
    r_q = np.sqrt(2.0 / math.pi) / eta
    r_mu = (alpha / (3.0 * math.sqrt(math.pi / 2.0))) ** (1.0 / 3.0)
    types = [1, 0, 0] * n_mol
    return StaticProblem(forcefield, kernel, np.concatenate(coords), names, types, mol,
                         [params[n]['chi'] for n in names], eta, alpha, r_q, r_mu, what=what, rhs_form=rhs_form,
                         e0=e0, principal_axes=principal_axes, factorization=factorization)
