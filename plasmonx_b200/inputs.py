"""Problem description of the per-frequency response solve.

``read_keywords`` reads the keyword file that the reference's Python front end
writes and its Fortran executable reads (``key: value`` lines, atom-type and
parameter blocks, ``parameters interaction name: A->B`` entries, geometry in
Angstrom after ``input_geometry``), following
src/input_output/input_module.f90:156-258 and :680-1000.  ``Problem`` holds
what the solve needs in the reference's units (bohr, a.u.), with the same
derived quantities the reference computes at input time:
  * density n = sigma0 / tau, then sigma0 and tau divided by the scaling
    factor (assign_model_parameters_wfq, src/wfq/wfq_module.f90:96-127);
  * neighbour counts per atom type (get_neighbours,
    src/target/target_module.f90:417-464), evaluated on the Angstrom
    coordinates times ToBohr exactly as the reference does (here on the host,
    on demand; the solver counts on the device, plx_neighbour_counts);
  * coordinates scaled to bohr (input_module.f90:238);
  * the GMRES tolerance multiplied by sqrt(n_var) (input_module.f90:250-251);
  * alpha_t(w) per atom type from the Etchegoin fits or a CSV table
    (read_alpha, src/wfq/wfqfmu_module.f90:97-166).
"""
import math
import os

import numpy as np

from . import materials as M


def _num(v):
    try:
        return float(str(v).strip().replace('d', 'e').replace('D', 'e'))
    except ValueError:
        return str(v).strip()


def read_keywords(text):
    kw, types, params, inter, geom = {}, [], [], [], []
    lines = text.splitlines()
    g0 = None
    for idx, line in enumerate(lines):
        if line.startswith('input_geometry'):
            g0 = idx
            break
        s = line.strip()
        if not s or s.startswith('#'):
            continue
        key, _, value = line.partition(':')
        key, value = key.strip(), value.strip()
        if key == 'atom_types name':
            types.append({'name': value})
        elif key.startswith('atom_types ') and key != 'atom_types number':
            types[-1][key[11:]] = _num(value)
        elif key == 'parameters atomtype name':
            params.append({'name': value})
        elif key.startswith('parameters atomtype '):
            params[-1][key[20:]] = _num(value)
        elif key == 'parameters interaction name':
            a, b = value.split('->')
            inter.append({'pair': (a.strip(), b.strip())})
        elif key.startswith('parameters interaction '):
            inter[-1][key[23:]] = _num(value)
        else:
            kw[key] = value
    if g0 is not None:
        n = int(float(kw.get('number of atoms', 0)))
        for line in lines[g0 + 1:g0 + 1 + n]:
            p = line.split()
            geom.append((p[0], float(p[-3]), float(p[-2]), float(p[-1]), int(p[1]) if len(p) > 4 else 1))
    return kw, types, params, inter, geom


def neighbour_counts(coord_ang, types, znum, n_types):
    """Per-atom counts of neighbours by atom type within the nearest-neighbour distance.

    Same test as the reference: sqrt(dx^2 + dy^2 + dz^2) * ToBohr <= r0(Z_i, Z_j) on
    the Angstrom coordinates; the atom itself counts once for its own type.
    """
    from scipy.spatial import cKDTree
    N = len(types)
    nb = np.zeros((n_types, N), dtype=np.int32)
    nb[types, np.arange(N)] = 1
    nn = np.ones(N, dtype=np.int32)
    zs = sorted(set(int(z) for z in znum))
    rmax = max(M.nearest_distance(a, b) for a in zs for b in zs) / M.TO_BOHR * 1.001
    pairs = cKDTree(coord_ang).query_pairs(rmax, output_type='ndarray')
    if len(pairs) == 0:
        return nb, nn
    i, j = pairs[:, 0], pairs[:, 1]
    d = np.sqrt((coord_ang[j, 0] - coord_ang[i, 0]) ** 2 + (coord_ang[j, 1] - coord_ang[i, 1]) ** 2
                + (coord_ang[j, 2] - coord_ang[i, 2]) ** 2) * M.TO_BOHR
    r0 = np.empty(len(i))
    for a in zs:
        for b in zs:
            sel = (znum[i] == a) & (znum[j] == b)
            r0[sel] = M.nearest_distance(a, b)
    hit = d <= r0
    i, j = i[hit], j[hit]
    for a, b in ((i, j), (j, i)):
        np.add.at(nn, a, 1)
        same = znum[a] == znum[b]
        np.add.at(nb, (types[a][same], a[same]), 1)
        np.add.at(nb, (types[b][~same], a[~same]), 1)
    return nb, nn


class Problem:
    """Geometry, model parameters and frequency grid of one response calculation."""

    def __init__(self, model, coord_ang, type_names, atom_types, eta, r_q, r_mu, tau, sigma0, scaling,
                 a_ij, fermi_d, fermi_s, freqs, e0=1e-4, alpha_w=None, rhs_form='field',
                 polarization='all', method='inversion', tolerance=1e-9, gmres_dim=1000, n_iter=1000,
                 fermi_energy=None, atom_names=None, permittivity=None, kernel='gaussian', chi=None, alpha=None,
                 mol_index=None, principal_axes=False):
        self.raw = dict(tau=list(map(float, tau)), sigma0=list(map(float, sigma0)),
                        scaling=list(map(float, scaling)), permittivity=permittivity,
                        fermi_energy=None if fermi_energy is None else list(map(float, fermi_energy)))
        self.model = model.lower()
        if self.model not in ('wfq', 'wfqfmu'):
            raise ValueError('dynamic forcefield must be wfq or wfqfmu, got %r' % model)
        self.type_names = list(type_names)
        nt = len(self.type_names)
        self.coord_ang = np.ascontiguousarray(coord_ang, dtype=np.float64).reshape(-1, 3)
        self.atom_types = np.ascontiguousarray(atom_types, dtype=np.int32)
        names = atom_names if atom_names is not None else [self.type_names[t] for t in self.atom_types]
        self.znum = np.array([M.atomic_number(n) for n in names], dtype=np.int64)
        self.n_atoms = len(self.atom_types)
        self.heterogeneous = nt > 1
        self.eta, self.r_q, self.r_mu = (np.asarray(v, dtype=np.float64) for v in (eta, r_q, r_mu))
        self.a_ij = np.asarray(a_ij, dtype=np.float64)
        self.fermi_d = np.asarray(fermi_d, dtype=np.float64).reshape(nt, nt)
        self.fermi_s = np.asarray(fermi_s, dtype=np.float64).reshape(nt, nt)
        tau = np.array(tau, dtype=np.float64)
        sigma0 = np.array(sigma0, dtype=np.float64)
        scaling = np.array(scaling, dtype=np.float64)
        fe = np.zeros(nt) if fermi_energy is None else np.asarray(fermi_energy, dtype=np.float64)
        dens = np.zeros(nt)
        for t in range(nt):
            # the reference tests atomic_number(t) with the atom-type index t
            # (wfq_module.f90:107): graphene density from the Fermi energy
            if self.n_atoms > t and self.znum[t] == 6:
                dens[t] = fe[t] / (math.pi * M.AU_TO_EV)
            else:
                dens[t] = sigma0[t] / tau[t]
            if abs(scaling[t] - 1.0) > 1e-14:
                sigma0[t] /= scaling[t]
                tau[t] /= scaling[t]
        self.tau, self.sigma0, self.density = tau, sigma0, dens
        self.r0 = np.array([[M.nearest_distance(int(self._type_z(a)), int(self._type_z(b)))
                             for b in range(nt)] for a in range(nt)])
        self._nb = None
        self.coord = self.coord_ang * M.TO_BOHR
        # carried for the .info file: charge kernel, the static force field the
        # w-model extends, chi / alpha per type, molecule index per atom
        self.kernel = kernel
        self.forcefield = 'fq' if self.model == 'wfq' else 'fqfmu'
        self.chi = np.zeros(nt) if chi is None else np.asarray(chi, dtype=np.float64)
        self.alpha = np.zeros(nt) if alpha is None else np.asarray(alpha, dtype=np.float64)
        self.mol_index = (np.ones(self.n_atoms, dtype=np.int64) if mol_index is None
                          else np.asarray(mol_index, dtype=np.int64))
        from .static import atoms_per_molecule, rotate_principal_axes
        self.apm = atoms_per_molecule(self.mol_index)
        self.n_mol = len(self.apm)
        # rotate_principal_axis runs after the input (and its neighbour counts),
        # before any solve (src/plasmonX.f90:37-38)
        self.principal_axes = bool(principal_axes)
        self.inertia = None
        if self.principal_axes:
            self.coord, w, v = rotate_principal_axes(self.coord, self.znum)
            self.inertia = {'eigenvalues': w, 'axes': v}
        self.freqs = np.asarray(freqs, dtype=np.float64)
        self.e0 = float(e0)
        self.rhs_form = rhs_form
        self.polarization = polarization
        self.method = method
        self.n_var = self.n_atoms if self.model == 'wfq' else 4 * self.n_atoms
        self.tolerance_input = float(tolerance)
        self.tol = self.tolerance_input * math.sqrt(self.n_var)
        self.gmres_dim = int(gmres_dim)
        self.n_iter = int(n_iter)
        if self.model == 'wfqfmu':
            if alpha_w is None:
                raise ValueError('wFQFMu needs alpha(w) per atom type')
            self.alpha_w = np.ascontiguousarray(alpha_w, dtype=np.complex128).reshape(nt, len(self.freqs))
        else:
            self.alpha_w = None

    def _counts(self):
        if self._nb is None:
            self._nb = neighbour_counts(self.coord_ang, self.atom_types, self.znum, len(self.type_names))
        return self._nb

    @property
    def neighbours(self):
        """Per-type neighbour counts (n_types x N), on the host; the solver counts on the
        device (plx_neighbour_counts) with the same test."""
        return self._counts()[0]

    @property
    def n_neighbours(self):
        return self._counts()[1]

    @property
    def type_z(self):
        return np.array([self._type_z(t) for t in range(len(self.type_names))], dtype=np.int32)

    def _type_z(self, t):
        hit = np.nonzero(self.atom_types == t)[0]
        if len(hit):
            return self.znum[hit[0]]
        return M.atomic_number(self.type_names[t])

    def to_keyword_text(self):
        """The problem as a reference keyword file (the format read_keywords parses)."""
        nt = len(self.type_names)
        L = ['forcefield dynamic: %s' % self.model,
             'algorithm method: %s' % self.method,
             'algorithm tolerance: %r' % self.tolerance_input,
             'algorithm gmres dimension: %d' % self.gmres_dim,
             'algorithm number of iterations: %d' % self.n_iter,
             'field rhs type: %s' % self.rhs_form,
             'field field intensity: %r' % self.e0,
             'field nfreq: %d' % len(self.freqs),
             'field min freq: 0.0', 'field max freq: 0.0', 'field step freq: 0.0',
             'field external freq: ' + ' '.join(repr(float(w)) for w in self.freqs),
             'field polarization: %s' % self.polarization,
             'atom_types number: %d' % nt]
        for t, n in enumerate(self.type_names):
            L += ['atom_types name: %s' % n, 'atom_types eta: %r' % float(self.eta[t]),
                  'atom_types rq: %r' % float(self.r_q[t]), 'atom_types rmu: %r' % float(self.r_mu[t])]
        perm = self.raw['permittivity'] or [None] * nt
        for t, n in enumerate(self.type_names):
            L += ['parameters atomtype name: %s' % n, 'parameters atomtype tau: %r' % self.raw['tau'][t],
                  'parameters atomtype sigma0: %r' % self.raw['sigma0'][t],
                  'parameters atomtype scaling sigma0-tau: %r' % self.raw['scaling'][t],
                  'parameters atomtype a_ij: %r' % float(self.a_ij[t]),
                  'parameters atomtype fermi function d: %r' % float(self.fermi_d[t, t]),
                  'parameters atomtype fermi function s: %r' % float(self.fermi_s[t, t]),
                  'parameters atomtype permittivity: %s' % (perm[t] or 'none')]
        for a in range(nt):
            for b in range(nt):
                if a != b:
                    L += ['parameters interaction name: %s->%s' % (self.type_names[a], self.type_names[b]),
                          'parameters interaction fermi function d: %r' % float(self.fermi_d[a, b]),
                          'parameters interaction fermi function s: %r' % float(self.fermi_s[a, b])]
        L += ['number of atoms: %d' % self.n_atoms, 'input_geometry: read from yaml file']
        names = {t: n for t, n in enumerate(self.type_names)}
        for t, (x, y, z) in zip(self.atom_types, self.coord_ang):
            L.append('%-6s %10d %25.16f %25.16f %25.16f' % (names[int(t)], 1, x, y, z))
        return '\n'.join(L) + '\n'

    @property
    def pol_mask(self):
        return {'all': 7, 'x': 1, 'y': 2, 'z': 4}[self.polarization]

    @classmethod
    def from_keyword_text(cls, text, base_dir='.'):
        kw, types, params, inter, geom = read_keywords(text)
        names = [t['name'] for t in types]
        idx = {n: i for i, n in enumerate(names)}
        nt = len(names)
        get = lambda lst, k: [float(x.get(k, 0.0)) for x in lst]  # noqa: E731
        par = {p['name']: p for p in params}
        plist = [par.get(n, {}) for n in names]
        fd = np.zeros((nt, nt))
        fs = np.zeros((nt, nt))
        for t, p in enumerate(plist):
            fd[t, t] = float(p.get('fermi function d', 0.0))
            fs[t, t] = float(p.get('fermi function s', 0.0))
        for it in inter:
            a, b = idx[it['pair'][0]], idx[it['pair'][1]]
            fd[a, b] = float(it.get('fermi function d', 0.0))
            fs[a, b] = float(it.get('fermi function s', 0.0))
        nf = int(float(kw['field nfreq']))
        fmin, fmax, fstep = (float(kw['field min freq']), float(kw['field max freq']),
                             float(kw['field step freq']))
        if fmin == 0.0 and fmax == 0.0:
            freqs = [float(x) for x in kw['field external freq'].replace(',', ' ').split()][:nf]
        else:
            freqs = [fmin + fstep * i for i in range(nf)]
        model = kw['forcefield dynamic'].lower()
        alpha_w = None
        if model == 'wfqfmu':
            alpha_w = np.zeros((nt, nf), dtype=np.complex128)
            for t, p in enumerate(plist):
                perm = str(p.get('permittivity', 'none'))
                fn = str(p.get('wfqfmu file', 'none'))
                if perm != 'none':
                    alpha_w[t] = M.fitted(perm, freqs, 'polar')
                elif fn != 'none':
                    alpha_w[t] = M.read_table(fn if os.path.isabs(fn) else os.path.join(base_dir, fn), freqs)
        atom_names = [g[0] for g in geom]
        return cls(model, np.array([g[1:4] for g in geom]), names, [idx[n] for n in atom_names],
                   get(types, 'eta'), get(types, 'rq'), get(types, 'rmu'), get(plist, 'tau'),
                   get(plist, 'sigma0'), get(plist, 'scaling sigma0-tau'), get(plist, 'a_ij'), fd, fs,
                   freqs, e0=float(kw.get('field field intensity', 1e-4)), alpha_w=alpha_w,
                   rhs_form=kw.get('field rhs type', 'field'), polarization=kw.get('field polarization', 'all'),
                   method=kw.get('algorithm method', 'inversion'),
                   tolerance=float(kw.get('algorithm tolerance', 0.0)),
                   gmres_dim=int(float(kw.get('algorithm gmres dimension', 1000))),
                   n_iter=int(float(kw.get('algorithm number of iterations', 1000))),
                   fermi_energy=get(plist, 'fermi energy'), atom_names=atom_names,
                   kernel=kw.get('forcefield kernel', 'gaussian').strip().lower(), chi=get(types, 'chi'),
                   alpha=get(types, 'alpha'), mol_index=[g[4] for g in geom],
                   principal_axes=kw.get('control principal axes', 'False').strip().lower() == 'true')

    @classmethod
    def from_keyword_file(cls, path):
        with open(path) as f:
            return cls.from_keyword_text(f.read(), base_dir=os.path.dirname(os.path.abspath(path)))
