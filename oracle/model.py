"""FP64 NumPy restatement of the wFQ / wFQFMu frequency-domain model (oracle).

TEST INFRASTRUCTURE ONLY (see ``oracle/__init__.py``).  Every function cites
the reference routine it restates; paths are relative to the plasmonX tree.

Ordering of unknowns follows the reference: charges q_1..q_N, then dipoles
mu_1x, mu_1y, mu_1z, ..., mu_Nz (``src/wfq/wfqfmu_module.f90:79-90``).
"""
import math
import os

import numpy as np
from scipy.special import erf

from .keywords import read_keyword_file, TO_BOHR, AU_TO_EV

# src/parameters/parameters_module.f90:38-62
AU_TO_CM = 219474.63136320
LIGHT = 137.035227
R_AG0 = 2.885 * TO_BOHR
R_AU0 = 2.885 * TO_BOHR
R_NA0 = 6.9226100144600462
R_C0 = 1.418 * TO_BOHR
R_OH0 = 1.65
R_AL0 = 2.861 * TO_BOHR
R_CU0 = 2.543463 * TO_BOHR

# atomic numbers used by nearest_distance (src/target/target_module.f90:243-310)
ATOMIC_NUMBER = {'h': 1, 'he': 2, 'li': 3, 'be': 4, 'b': 5, 'c': 6, 'n': 7, 'o': 8,
                 'f': 9, 'ne': 10, 'na': 11, 'mg': 12, 'al': 13, 'si': 14, 'p': 15,
                 's': 16, 'cl': 17, 'ar': 18, 'cu': 29, 'ag': 47, 'au': 79}


def nearest_distance(zi, zj):
    """src/target/target_module.f90:472-518 (bohr)."""
    pair = {zi, zj}
    if pair <= {1, 8}:
        return R_OH0
    if zi == zj == 47:
        return R_AG0
    if zi == zj == 79:
        return R_AU0
    if zi == zj == 11:
        return R_NA0
    if zi == zj == 6:
        return R_C0
    if zi == zj == 13:
        return R_AL0
    if zi == zj == 29:
        return R_CU0
    if pair == {47, 79}:
        return (R_AG0 + R_AU0) / 2.0
    raise ValueError('I do not recognize atomic couples in nearest distance')


def freq_au_to_nm(w):
    """src/parameters/parameters_module.f90:552-562."""
    return 10000000.0 / (w * AU_TO_CM)


def silver_etchegoin(freqs, what):
    """src/parameters/parameters_module.f90:107-194."""
    bsline = complex(1.469322, 0.2450325)
    aj = [0.1632212, 0.9672775, 0.6150938]
    pij = [complex(0, -1.709221), complex(0, 0.1546664), complex(0, -1.782307)]
    lam = 137.9643
    gammap = 1.0 / 74484.21
    lamj = [1.0 / 307.9550, 1.0 / 260.7301, 1.0 / 236.2128]
    gamj = [1.0 / 4277.721, 1.0 / 1051.474, 1.0 / 1008.622]
    n0 = 10.49 / 107.8682 * 6.022e23 / ((1.0e8 * TO_BOHR) ** 3)
    wp = math.sqrt(4.0 * math.pi * n0)
    out = []
    for w in freqs:
        f3 = 1.0 / freq_au_to_nm(w)
        lor = 0j
        for a, l, g, p in zip(aj, lamj, gamj, pij):
            lor += a * l * (np.exp(p) / complex(l - f3, -g) + np.exp(-p) / complex(l + f3, g))
        if what == 'epsilon':
            out.append(bsline - 1.0 / (lam ** 2 * f3 * complex(f3, gammap)) + lor)
        else:
            out.append((bsline - bsline.real + lor) / wp ** 2)
    return np.array(out, dtype=np.complex128)


def gold_etchegoin(freqs, what):
    """src/parameters/parameters_module.f90:295-375 (incl. the Im >= 1e-10 clamp)."""
    bsline = complex(1.54, 0.0)
    aj = [1.27, 1.10]
    pij = [complex(0, -math.pi / 4.0), complex(0, -math.pi / 4.0)]
    lam = 143.0
    gammap = 1.0 / 14500.0
    lamj = [1.0 / 470.0, 1.0 / 325.0]
    gamj = [1.0 / 1900.0, 1.0 / 1060.0]
    n0 = 19.320 / 196.96657 * 6.022e23 / ((1.0e8 * TO_BOHR) ** 3)
    wp = math.sqrt(4.0 * math.pi * n0)
    out = []
    for w in freqs:
        f3 = 1.0 / freq_au_to_nm(w)
        lor = 0j
        for a, l, g, p in zip(aj, lamj, gamj, pij):
            lor += a * l * (np.exp(p) / complex(l - f3, -g) + np.exp(-p) / complex(l + f3, g))
        if what == 'epsilon':
            out.append(bsline - 1.0 / (lam ** 2 * f3 * complex(f3, gammap)) + lor)
        else:
            v = lor / wp ** 2
            if v.imag <= 0.0:
                v = complex(v.real, 1.0e-10)
            out.append(v)
    return np.array(out, dtype=np.complex128)


def read_permittivity_file(path, freqs):
    """src/parameters/parameters_module.f90:384-462: rows 'eV Re Im', match within 1e-8 eV."""
    rows = []
    with open(path) as f:
        for line in f:
            if '#' in line or not line.strip():
                continue
            p = line.replace(',', ' ').split()
            rows.append((float(p[0]), float(p[1]), float(p[2])))
    tab = np.array(rows)
    out = []
    for w in freqs:
        ev = w * AU_TO_EV
        hit = np.nonzero(np.abs(ev - tab[:, 0]) <= 1.0e-8)[0]
        if len(hit) == 0:
            raise ValueError('I did not find data for freq = %6.2f' % ev)
        out.append(complex(tab[hit[0], 1], tab[hit[0], 2]))
    return np.array(out, dtype=np.complex128)


class System:
    """Everything the per-frequency solve needs, in the reference's units (a.u., bohr).

    Built from a reference keyword file by ``from_keywords`` (following
    ``src/input_output/input_module.f90:156-258`` and
    ``src/wfq/wfq_module.f90:96-127``) or directly by ``from_arrays``.
    """

    def __init__(self):
        pass

    @classmethod
    def from_keywords(cls, path_or_tuple, base_dir=None):
        if isinstance(path_or_tuple, (str, os.PathLike)):
            base_dir = base_dir or os.path.dirname(os.path.abspath(path_or_tuple))
            kw, ats, prs, inter, geom = read_keyword_file(path_or_tuple)
        else:
            kw, ats, prs, inter, geom = path_or_tuple
        s = cls()
        s.model = kw['forcefield dynamic'].lower()
        s.method = kw.get('algorithm method', 'inversion')
        s.tol_input = float(kw.get('algorithm tolerance', 0.0))
        s.n_dim_gmres = int(float(kw.get('algorithm gmres dimension', 0)))
        s.n_iter = int(float(kw.get('algorithm number of iterations', 0)))
        s.e0 = float(kw.get('field field intensity', 0.0))
        s.rhs_form = kw.get('field rhs type', 'field')
        s.polarization = kw.get('field polarization', 'all')
        nfreq = int(float(kw['field nfreq']))
        fmin, fmax = float(kw['field min freq']), float(kw['field max freq'])
        fstep = float(kw['field step freq'])
        if fmin == 0.0 and fmax == 0.0:
            s.freqs = np.array([float(x) for x in kw['field external freq'].replace(',', ' ').split()][:nfreq])
        else:
            s.freqs = np.array([fmin + fstep * i for i in range(nfreq)])
        s.type_names = [a['name'] for a in ats]
        nt = len(ats)
        s.eta = np.array([a.get('eta', 0.0) for a in ats])
        s.alpha = np.array([a.get('alpha', 0.0) for a in ats])
        s.rq = np.array([a.get('rq', 0.0) for a in ats])
        s.rmu = np.array([a.get('rmu', 0.0) for a in ats])
        idx = {n: i for i, n in enumerate(s.type_names)}
        s.tau = np.zeros(nt)
        s.sigma0 = np.zeros(nt)
        s.scaling = np.zeros(nt)
        s.a_ij = np.zeros(nt)
        s.fermi_energy = np.zeros(nt)
        s.fermi_d = np.zeros((nt, nt))
        s.fermi_s = np.zeros((nt, nt))
        s.wfqfmu_file = ['none'] * nt
        s.permittivity = ['none'] * nt
        for p in prs:
            t = idx[p['name']]
            s.tau[t] = p.get('tau', 0.0)
            s.sigma0[t] = p.get('sigma0', 0.0)
            s.scaling[t] = p.get('scaling sigma0-tau', 0.0)
            s.a_ij[t] = p.get('a_ij', 0.0)
            s.fermi_energy[t] = p.get('fermi energy', 0.0)
            s.fermi_d[t, t] = p.get('fermi function d', 0.0)
            s.fermi_s[t, t] = p.get('fermi function s', 0.0)
            s.wfqfmu_file[t] = str(p.get('wfqfmu file', 'none'))
            s.permittivity[t] = str(p.get('permittivity', 'none'))
        for it in inter:
            a, b = idx[it['pair'][0]], idx[it['pair'][1]]
            s.fermi_d[a, b] = it.get('fermi function d', 0.0)
            s.fermi_s[a, b] = it.get('fermi function s', 0.0)
        names = [g[0] for g in geom]
        coord_ang = np.array([[g[1], g[2], g[3]] for g in geom], dtype=np.float64)
        s.types = np.array([idx[n] for n in names], dtype=np.int64)
        s.znum = np.array([ATOMIC_NUMBER[n.lower()] for n in names], dtype=np.int64)
        s._finish(coord_ang, base_dir)
        return s

    def _finish(self, coord_ang, base_dir):
        s = self
        s.heterogeneous = len(s.type_names) > 1
        s.n_atoms = len(s.types)
        s.neighbours, s.n_neighbours = get_neighbours(coord_ang, s.types, s.znum, len(s.type_names))
        # src/wfq/wfq_module.f90:96-127 (the atomic_number(i) lookup uses the
        # atom-type index i on the per-atom array, as the reference does)
        nt = len(s.type_names)
        s.density = np.zeros(nt)
        for t in range(nt):
            if s.znum[t] == 6:
                s.density[t] = s.fermi_energy[t] / (math.pi * AU_TO_EV)
            else:
                s.density[t] = s.sigma0[t] / s.tau[t]
            if abs(s.scaling[t] - 1.0) > 1e-14:
                s.sigma0[t] = s.sigma0[t] / s.scaling[t]
                s.tau[t] = s.tau[t] / s.scaling[t]
        s.coord = coord_ang * TO_BOHR          # src/input_output/input_module.f90:238
        s.n_q = s.n_atoms
        s.n_var = s.n_atoms if s.model == 'wfq' else 4 * s.n_atoms
        s.tol = s.tol_input * math.sqrt(s.n_var)  # input_module.f90:250-251
        s.alpha_w = None
        if s.model == 'wfqfmu':
            s.alpha_w = np.zeros((nt, len(s.freqs)), dtype=np.complex128)
            for t in range(nt):
                if s.permittivity[t] != 'none':
                    if s.permittivity[t] == 'silver etchegoin':
                        s.alpha_w[t] = silver_etchegoin(s.freqs, 'polar')
                    elif s.permittivity[t] == 'gold etchegoin':
                        s.alpha_w[t] = gold_etchegoin(s.freqs, 'polar')
                    else:
                        raise ValueError('Fitted permittivity not implemented: ' + s.permittivity[t])
                elif s.wfqfmu_file[t] != 'none':
                    path = s.wfqfmu_file[t]
                    if base_dir and not os.path.isabs(path):
                        path = os.path.join(base_dir, path)
                    s.alpha_w[t] = read_permittivity_file(path, s.freqs)

    @property
    def pol_index(self):
        return {'x': 0, 'y': 1, 'z': 2}.get(self.polarization)


def get_neighbours(coord_ang, types, znum, ntypes):
    """src/target/target_module.f90:417-464 (distances in Angstrom * ToBohr)."""
    n = len(types)
    nb = np.zeros((ntypes, n), dtype=np.int64)
    nn = np.zeros(n, dtype=np.int64)
    r0cache = {}
    for i in range(n):
        d = np.sqrt((coord_ang[:, 0] - coord_ang[i, 0]) ** 2 + (coord_ang[:, 1] - coord_ang[i, 1]) ** 2
                    + (coord_ang[:, 2] - coord_ang[i, 2]) ** 2) * TO_BOHR
        factor = np.zeros(ntypes, dtype=np.int64)
        factor[types[i]] = 1
        ntot = 1
        for j in np.nonzero(d <= 20.0)[0]:
            if j == i:
                continue
            key = (znum[i], znum[j])
            if key not in r0cache:
                r0cache[key] = nearest_distance(*key)
            if d[j] <= r0cache[key]:
                ntot += 1
                if znum[i] == znum[j]:
                    factor[types[i]] += 1
                else:
                    factor[types[j]] += 1
        nb[:, i] = factor
        nn[i] = ntot
    return nb, nn


# ----------------------------------------------------------------------------
# interaction tiles (src/matrix/matrix_module.f90:58-345)
# ----------------------------------------------------------------------------

def _pair_geometry(s):
    c = s.coord
    dx = c[:, None, 0] - c[None, :, 0]
    dy = c[:, None, 1] - c[None, :, 1]
    dz = c[:, None, 2] - c[None, :, 2]
    r = np.sqrt(dx ** 2 + dy ** 2 + dz ** 2)
    return dx, dy, dz, r


def t_qq(s):
    """construct_static_t_qq, Gaussian kernel (matrix_module.f90:58-115)."""
    _, _, _, r = _pair_geometry(s)
    rq = s.rq[s.types]
    R = np.sqrt(rq[:, None] ** 2 + rq[None, :] ** 2)
    with np.errstate(divide='ignore', invalid='ignore'):
        T = erf(r / R) / r
    eta = s.eta[s.types]
    T[np.diag_indices(s.n_atoms)] = (eta + eta) / 2.0
    return T


def _fqmu(r, R):
    return erf(r / R) - ((2.0 * r) / (math.sqrt(math.pi) * R)) * np.exp(-r ** 2 / R ** 2)


def t_qmu(s):
    """construct_static_t_qmu / t_muq (matrix_module.f90:120-234): T_qmu(i, 3j+k)."""
    dx, dy, dz, r = _pair_geometry(s)
    R = np.sqrt(s.rq[s.types][:, None] ** 2 + s.rmu[s.types][None, :] ** 2)
    with np.errstate(divide='ignore', invalid='ignore'):
        f = _fqmu(r, R) / r ** 3
    np.fill_diagonal(f, 0.0)
    N = s.n_atoms
    T = np.zeros((N, 3 * N))
    T[:, 0::3] = dx * f
    T[:, 1::3] = dy * f
    T[:, 2::3] = dz * f
    return T


def t_mumu(s):
    """construct_static_t_mumu for w-models (diagonal blocks zero), matrix_module.f90:240-345."""
    dx, dy, dz, r = _pair_geometry(s)
    rm = s.rmu[s.types]
    R = np.sqrt(rm[:, None] ** 2 + rm[None, :] ** 2)
    with np.errstate(divide='ignore', invalid='ignore'):
        fD1 = _fqmu(r, R)
        fD2 = (4.0 / (math.sqrt(math.pi) * R ** 3)) * np.exp(-r ** 2 / R ** 2)
        r2, r3, r5 = r ** 2, r ** 3, r ** 5
        comps = (dx, dy, dz)
        N = s.n_atoms
        T = np.zeros((3 * N, 3 * N))
        for a in range(3):
            for b in range(3):
                blk = (-3.0 * comps[a] * comps[b] / r5 + (1.0 / r3 if a == b else 0.0)) * fD1 \
                    + fD2 * comps[a] * comps[b] / r2
                np.fill_diagonal(blk, 0.0)
                T[a::3, b::3] = blk
    return T


def t_full(s):
    if s.model == 'wfq':
        return t_qq(s)
    Tqq, Tqmu, Tmm = t_qq(s), t_qmu(s), t_mumu(s)
    return np.block([[Tqq, Tqmu], [Tqmu.T, Tmm]])


# ----------------------------------------------------------------------------
# Drude / Fermi conductance (matrix_module.f90:393-482, 694-715)
# ----------------------------------------------------------------------------

def fermi_matrix(s):
    _, _, _, r = _pair_geometry(s)
    ti, zi = s.types, s.znum
    d = s.fermi_d[ti[:, None], ti[None, :]]
    sij = s.fermi_s[ti[:, None], ti[None, :]]
    r0 = np.zeros_like(r)
    for a in np.unique(zi):
        for b in np.unique(zi):
            r0[np.ix_(zi == a, zi == b)] = nearest_distance(int(a), int(b))
    with np.errstate(over='ignore'):
        f = 1.0 / (1.0 + np.exp(-d * ((r / (sij * r0)) - 1.0)))
    return f, r


def k_matrix(s):
    """Off-diagonal K_ij = (1 - f_ij) A_type(i) / r_ij, zero diagonal."""
    f, r = fermi_matrix(s)
    with np.errstate(divide='ignore', invalid='ignore'):
        K = (1.0 - f) * s.a_ij[s.types][:, None] / r
    np.fill_diagonal(K, 0.0)
    return K


def k_minus_p(s):
    """construct_K_minus_P_matrix (matrix_module.f90:393-426)."""
    K = k_matrix(s)
    return K - np.diag(K.sum(axis=1))


def drude_w(s, omega):
    """w_i = 2 n_i / (1/tau_i - i w) per atom type (matrix_module.f90:435-482)."""
    return 2.0 * s.density / (1.0 / s.tau - 1j * omega)


def h_minus_l(s, omega, K=None):
    """construct_H_minus_L_matrix: H_ij = (w_j/w_i) K_ji, diagonal -row sum."""
    if K is None:
        K = k_matrix(s)
    w = drude_w(s, omega)[s.types]
    H = (w[None, :] / w[:, None]) * K.T
    np.fill_diagonal(H, 0.0)
    return H - np.diag(H.sum(axis=1))


# ----------------------------------------------------------------------------
# frequency diagonals (wfq_module.f90:398-424, wfqfmu_module.f90:698-746)
# ----------------------------------------------------------------------------

def z_q(s, omega):
    """z_i(w) = w (-w tau - i) / (2 n tau), per atom."""
    tau = s.tau[s.types]
    n = s.density[s.types]
    return omega * (-omega * tau - 1j) / (2.0 * n * tau)


def z_mu(s, i_freq):
    """sum_t (nb_t,i / nn_i) / alpha_t(w), per atom."""
    frac = s.neighbours.astype(np.float64) / s.n_neighbours.astype(np.float64)[None, :]
    return (frac / s.alpha_w[:, i_freq][:, None]).sum(axis=0)


def diagonal(s, i_freq):
    """The diagonal D(w) that new_gmres_diagonal_shift adds: w += D * r."""
    omega = s.freqs[i_freq]
    dq = -z_q(s, omega)
    if s.model == 'wfq':
        return dq.astype(np.complex128)
    dm = np.repeat(z_mu(s, i_freq), 3)
    return np.concatenate([dq, dm]).astype(np.complex128)


# ----------------------------------------------------------------------------
# right-hand sides (src/rhs/rhs_module.f90:43-430)
# ----------------------------------------------------------------------------

def static_potential(s):
    """construct_static_field_rhs_q: V(i,k) = -E0 * r_ik (or |r - r_min|)."""
    if s.rhs_form == 'potential':
        return -s.e0 * np.abs(s.coord - s.coord.min(axis=0))
    return -s.e0 * s.coord


def pol_columns(s):
    return [0, 1, 2] if s.polarization == 'all' else [s.pol_index]


def rhs(s, i_freq, Kbar=None, K=None):
    """Dynamic RHS (n_var x 3): q rows -(K-P)V (homo) or -1/2 (K+H)(w) V (hetero); mu rows E0."""
    n = s.n_var
    b = np.zeros((n, 3), dtype=np.complex128)
    V = static_potential(s)
    cols = pol_columns(s)
    if not s.heterogeneous:
        Kbar = k_minus_p(s) if Kbar is None else Kbar
        bq = -(Kbar @ V)
    else:
        K = k_matrix(s) if K is None else K
        Kbar = K - np.diag(K.sum(axis=1))
        KH = h_minus_l(s, s.freqs[i_freq], K) + Kbar
        bq = -0.5 * (KH @ V.astype(np.complex128))
    for c in cols:
        b[:s.n_q, c] = bq[:, c]
    if s.model == 'wfqfmu':
        N = s.n_atoms
        for c in cols:
            b[N + np.arange(N) * 3 + c, c] = s.e0
    return b


# ----------------------------------------------------------------------------
# dense operators
# ----------------------------------------------------------------------------

class Operator:
    """A(w) = blockdiag(Kbar(w), I) T + D(w), formed densely (small systems only)."""

    def __init__(self, s):
        self.s = s
        self.T = t_full(s)
        self.K = k_matrix(s)
        self.Kbar = self.K - np.diag(self.K.sum(axis=1))

    def q_block(self, i_freq):
        s = self.s
        if not s.heterogeneous:
            return self.Kbar.astype(np.complex128)
        return 0.5 * (h_minus_l(s, s.freqs[i_freq], self.K) + self.Kbar)

    def constant_matrix(self):
        """construct_constant_matrix_{wfq,wfqfmu} for homogeneous systems (real)."""
        s = self.s
        A = self.T.copy()
        N = s.n_q
        A[:N, :] = self.Kbar @ self.T[:N, :]
        return A

    def matrix(self, i_freq):
        """Full complex A(w) (construct_dynamic_matrix_*)."""
        s = self.s
        N = s.n_q
        A = self.T.astype(np.complex128)
        A[:N, :] = self.q_block(i_freq) @ self.T[:N, :]
        A[np.diag_indices(s.n_var)] += diagonal(s, i_freq)
        return A

    def matvec(self, i_freq, x):
        """Same product as product_matrix_vector + new_gmres_diagonal_shift."""
        s = self.s
        N = s.n_q
        y = self.T @ x
        y[:N] = self.q_block(i_freq) @ y[:N]
        return y + diagonal(s, i_freq) * x

    def rhs(self, i_freq):
        return rhs(self.s, i_freq, Kbar=self.Kbar, K=self.K)


# ----------------------------------------------------------------------------
# observables (wfq_module.f90:523-583, wfqfmu_module.f90:879-964,
#              target_module.f90:1989-2054)
# ----------------------------------------------------------------------------

def polar(s, x):
    """alpha(a, b) = sum_i q_i^(b) r_ia / E0 (+ sum_i mu_ia^(b) / E0)."""
    N = s.n_atoms
    P = (s.coord.T @ x[:N, :]) / s.e0
    if s.model == 'wfqfmu':
        for a in range(3):
            P[a, :] += x[N + a::3, :][:N].sum(axis=0) / s.e0
    return P


def results_row(P, omega):
    """results(1..20) for one frequency."""
    r = np.zeros(20)
    r[0] = (P[0, 0].real + P[1, 1].real + P[2, 2].real) / 3
    r[1] = (P[0, 0].imag + P[1, 1].imag + P[2, 2].imag) / 3
    r[2:5] = [P[0, 0].real, P[1, 1].real, P[2, 2].real]
    r[5:8] = [P[0, 0].imag, P[1, 1].imag, P[2, 2].imag]
    m_iso = r[0] ** 2 + r[1] ** 2
    m = [r[2] ** 2 + r[5] ** 2, r[3] ** 2 + r[6] ** 2, r[4] ** 2 + r[7] ** 2]
    r[8] = 4.0 * math.pi * omega * r[1] / LIGHT
    r[9:12] = [4.0 * math.pi * omega * r[5 + k] / LIGHT for k in range(3)]
    c4 = 3.0 * LIGHT ** 4
    r[12] = (8.0 * math.pi * omega ** 4) * m_iso / c4
    r[13:16] = [(8.0 * math.pi * omega ** 4) * mk / c4 for mk in m]
    r[16] = r[8] + r[12]
    r[17:20] = [r[9 + k] + r[13 + k] for k in range(3)]
    return r
