"""Benchmark configurations: seeded synthetic geometries with the reference's
default material parameters.

Defaults are the predefined atom types and Drude/Fermi parameters of the
reference front end (python/input_/validation.py:952-977, :1125-1153,
:1420-1423): Na (eta 0.292, tau 1323, sigma0 2.39494681e7 S/m, scaling 10,
A_ij 12.07910025, d 12, s 1.1), Ag (eta 0.4829838, alpha 49.9843,
R_q 3.3775793621738925, R_mu 2.368922250085755, tau 1633.608,
sigma0 6.5313e7 S/m, A_ij 9.61, d 12, s 1.1, silver Etchegoin), Au (eta
0.52685, alpha 39.5297, R_q 3.4996572071713126, R_mu 3.0710227258450864,
tau 318.018, sigma0 11834849.81 S/m, A_ij 9.61, d 12, s 1.1, gold
Etchegoin) and the Ag<->Au interaction d 12, s 0.95.  Unset Gaussian widths
follow validation.py:1084-1090: R_q = sqrt(2/pi)/eta.  Field intensity 1e-4 a.u.
Frequencies are uniform in eV and converted with 1/27.211386245981.
"""
import math

import numpy as np

from . import geometry as G
from . import materials as M
from .inputs import Problem

TYPES = {
    'Na': dict(eta=0.292, alpha=0.0, rq=math.sqrt(2 / math.pi) / 0.292, rmu=0.0, tau=1323.0,
               sigma0=2.39494681e7 * M.FSM_AU, scaling=10.0, a_ij=12.07910025, d=12.0, s=1.1, perm=None),
    'Ag': dict(eta=0.4829838, alpha=49.9843, rq=3.3775793621738925, rmu=2.368922250085755, tau=1633.608,
               sigma0=6.5313e7 * M.FSM_AU, scaling=1.0, a_ij=9.61, d=12.0, s=1.1, perm='silver etchegoin'),
    'Au': dict(eta=0.52685, alpha=39.5297, rq=3.4996572071713126, rmu=3.0710227258450864, tau=318.018,
               sigma0=11834849.81 * M.FSM_AU, scaling=1.0, a_ij=9.61, d=12.0, s=1.1, perm='gold etchegoin'),
}
INTERACTION = {('Ag', 'Au'): (12.0, 0.95), ('Au', 'Ag'): (12.0, 0.95)}


def ev_grid(lo, hi, n):
    return np.array([(lo + (hi - lo) * i / (n - 1)) / M.AU_TO_EV for i in range(n)]) if n > 1 \
        else np.array([lo / M.AU_TO_EV])


def build(model, coords, type_names, atom_types, freqs, **kw):
    nt = len(type_names)
    P = [TYPES[t] for t in type_names]
    fd = np.zeros((nt, nt))
    fs = np.zeros((nt, nt))
    for a, ta in enumerate(type_names):
        for b, tb in enumerate(type_names):
            if a == b:
                fd[a, a], fs[a, a] = P[a]['d'], P[a]['s']
            else:
                fd[a, b], fs[a, b] = INTERACTION[(ta, tb)]
    alpha_w = None
    if model == 'wfqfmu':
        alpha_w = np.array([M.fitted(p['perm'], freqs, 'polar') for p in P])
    return Problem(model, coords, type_names, atom_types, [p['eta'] for p in P], [p['rq'] for p in P],
                   [p['rmu'] for p in P], [p['tau'] for p in P], [p['sigma0'] for p in P],
                   [p['scaling'] for p in P], [p['a_ij'] for p in P], fd, fs, freqs, alpha_w=alpha_w,
                   permittivity=[p['perm'] for p in P], **kw)


def na_sphere(radius=20.0, n_freq=61, seed=1, jitter=0.01, **kw):
    """wFQ sodium: bcc a = 4.225 A cut to a sphere (893 sites at 20 A), 2.0-4.0 eV."""
    pts = G.sphere('bcc', 4.225, radius, jitter, seed)
    return build('wfq', pts, ['Na'], np.zeros(len(pts), np.int32), ev_grid(2.0, 4.0, n_freq), **kw)


def ag_sphere(radius=35.0, n_freq=201, seed=1, jitter=0.0, lo=3.0, hi=4.5, **kw):
    """wFQFMu silver: fcc a = 4.086 A cut to a sphere (10,473 sites at 35 A), 3.0-4.5 eV."""
    pts = G.sphere('fcc', 4.086, radius, jitter, seed)
    return build('wfqfmu', pts, ['Ag'], np.zeros(len(pts), np.int32), ev_grid(lo, hi, n_freq), **kw)


LATTICE = {'Na': ('bcc', 4.225), 'Ag': ('fcc', 4.086), 'Au': ('fcc', 4.08)}
WINDOW = {'Na': (2.0, 4.0), 'Ag': (3.0, 4.5), 'Au': (2.0, 3.0)}


def particle(metal, shape='sphere', radius=20.0, length=None, n_freq=61, seed=1, jitter=0.0, **kw):
    """A single-metal sphere or rod (cylinder with hemispherical caps along z) of the
    metal's lattice, in its frequency window: wFQ for Na, wFQFMu for Ag and Au."""
    kind, a = LATTICE[metal]
    if shape == 'sphere':
        pts = G.sphere(kind, a, radius, jitter, seed)
    elif shape == 'rod':
        pts = G.rod(kind, a, length if length is not None else 4.0 * radius, radius, jitter, seed)
    else:
        raise ValueError(shape)
    lo, hi = WINDOW[metal]
    model = 'wfq' if metal == 'Na' else 'wfqfmu'
    return build(model, pts, [metal], np.zeros(len(pts), np.int32), ev_grid(lo, hi, n_freq), **kw)


def agau_bowtie(edge=80.0, thickness=20.0, gap=10.0, n_freq=201, seed=1, jitter=0.0, **kw):
    """wFQFMu Ag-Au bow-tie: two fcc (a = 4.08 A) prisms tip to tip along x, 2.0-4.5 eV."""
    pts, sp = G.bowtie(4.08, edge, thickness, gap, jitter, seed)
    return build('wfqfmu', pts, ['Ag', 'Au'], sp, ev_grid(2.0, 4.5, n_freq), **kw)
