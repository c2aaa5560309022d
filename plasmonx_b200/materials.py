"""Constants, unit conversions and frequency-dependent material tables.

Restates src/parameters/parameters_module.f90: the constants (:13-62), the
Etchegoin fits of the silver and gold permittivity / interband
polarizability (:107-194, :295-375, including the Im >= 1e-10 floor of the
gold polarizability at :365-366) and the CSV reader that matches tabulated
frequencies within 1e-8 eV (:384-462).  The Brendel-Bormann model is not
implemented in the reference either (:205-284 stops), so it raises here.
"""
import cmath
import math

import numpy as np

TO_BOHR = 1.8897261254578281
AU_TO_EV = 27.211386245981
AU_TO_CM = 219474.63136320
LIGHT = 137.035227
FSM_AU = 0.00000021739

# nearest-neighbour distances (bohr)
R_AG0 = 2.885 * TO_BOHR
R_AU0 = 2.885 * TO_BOHR
R_NA0 = 6.9226100144600462
R_C0 = 1.418 * TO_BOHR
R_OH0 = 1.65
R_AL0 = 2.861 * TO_BOHR
R_CU0 = 2.543463 * TO_BOHR

ELEMENTS = {'h': 1, 'he': 2, 'li': 3, 'be': 4, 'b': 5, 'c': 6, 'n': 7, 'o': 8, 'f': 9, 'ne': 10,
            'na': 11, 'mg': 12, 'al': 13, 'si': 14, 'p': 15, 's': 16, 'cl': 17, 'ar': 18, 'cu': 29,
            'ag': 47, 'au': 79}


def atomic_number(name):
    z = ELEMENTS.get(name.strip().lower())
    if z is None:
        raise ValueError('unknown element %r' % name)
    return z


# atom names the reference also accepts (assign_atomic_number,
# src/target/target_module.f90:315-400)
NAME_ALIASES = {'hw': 1, 'h-hw': 1, 'ow': 8, 'o-ow': 8}


def atom_name_number(name):
    """Atomic number of an atom name as the reference assigns it: element symbols and
    the water names (HW, H-HW, OW, O-OW), case-insensitive; 0 when not recognised."""
    key = name.strip().lower()
    return ELEMENTS.get(key, NAME_ALIASES.get(key, 0))


def nearest_distance(zi, zj):
    """Nearest-neighbour distance of an element pair (target_module.f90:472-518)."""
    if {zi, zj} <= {1, 8}:
        return R_OH0
    same = {47: R_AG0, 79: R_AU0, 11: R_NA0, 6: R_C0, 13: R_AL0, 29: R_CU0}
    if zi == zj and zi in same:
        return same[zi]
    if {zi, zj} == {47, 79}:
        return (R_AG0 + R_AU0) / 2.0
    raise ValueError('I do not recognize atomic couples in nearest distance')


def au_to_nm(w):
    return 10000000.0 / (w * AU_TO_CM)


def _lorentz(f3, aj, lamj, gamj, pij):
    s = 0j
    for a, l, g, p in zip(aj, lamj, gamj, pij):
        s += a * l * (cmath.exp(p) / complex(l - f3, -g) + cmath.exp(-p) / complex(l + f3, g))
    return s


def silver_etchegoin(freqs, what='polar'):
    bsline = complex(1.469322, 0.2450325)
    aj = (0.1632212, 0.9672775, 0.6150938)
    pij = (complex(0, -1.709221), complex(0, 0.1546664), complex(0, -1.782307))
    lam, gammap = 137.9643, 1.0 / 74484.21
    lamj = (1.0 / 307.9550, 1.0 / 260.7301, 1.0 / 236.2128)
    gamj = (1.0 / 4277.721, 1.0 / 1051.474, 1.0 / 1008.622)
    wp = math.sqrt(4.0 * math.pi * (10.49 / 107.8682 * 6.022e23 / ((1.0e8 * TO_BOHR) ** 3)))
    out = np.empty(len(freqs), dtype=np.complex128)
    for i, w in enumerate(freqs):
        f3 = 1.0 / au_to_nm(w)
        lor = _lorentz(f3, aj, lamj, gamj, pij)
        if what == 'epsilon':
            out[i] = bsline - 1.0 / (lam ** 2 * f3 * complex(f3, gammap)) + lor
        else:
            out[i] = (bsline - bsline.real + lor) / wp ** 2
    return out


def gold_etchegoin(freqs, what='polar'):
    bsline = complex(1.54, 0.0)
    aj = (1.27, 1.10)
    pij = (complex(0, -math.pi / 4.0), complex(0, -math.pi / 4.0))
    lam, gammap = 143.0, 1.0 / 14500.0
    lamj = (1.0 / 470.0, 1.0 / 325.0)
    gamj = (1.0 / 1900.0, 1.0 / 1060.0)
    wp = math.sqrt(4.0 * math.pi * (19.320 / 196.96657 * 6.022e23 / ((1.0e8 * TO_BOHR) ** 3)))
    out = np.empty(len(freqs), dtype=np.complex128)
    for i, w in enumerate(freqs):
        f3 = 1.0 / au_to_nm(w)
        lor = _lorentz(f3, aj, lamj, gamj, pij)
        if what == 'epsilon':
            out[i] = bsline - 1.0 / (lam ** 2 * f3 * complex(f3, gammap)) + lor
        else:
            v = lor / wp ** 2
            out[i] = complex(v.real, 1.0e-10) if v.imag <= 0.0 else v
    return out


FITTED = {'silver etchegoin': silver_etchegoin, 'gold etchegoin': gold_etchegoin}


def fitted(name, freqs, what='polar'):
    if name not in FITTED:
        raise ValueError('Fitted permittivity for material: %s not yet implemented' % name)
    return FITTED[name](freqs, what)


def read_table(path, freqs):
    """Rows 'freq(eV) Re Im' after leading '#' comment lines; exact 1e-8 eV match."""
    rows = []
    with open(path) as f:
        lines = f.readlines()
    k = 0
    while k < len(lines) and '#' in lines[k]:
        k += 1
    for line in lines[k:]:
        p = line.replace(',', ' ').split()
        if len(p) >= 3:
            rows.append((float(p[0]), float(p[1]), float(p[2])))
    tab = np.array(rows, dtype=np.float64).reshape(-1, 3)
    out = np.empty(len(freqs), dtype=np.complex128)
    for i, w in enumerate(freqs):
        ev = w * AU_TO_EV
        hit = np.nonzero(np.abs(ev - tab[:, 0]) <= 1.0e-8)[0]
        if len(hit) == 0:
            raise ValueError('I did not find data for freq = %6.2f' % ev)
        out[i] = complex(tab[hit[0], 1], tab[hit[0], 2])
    return out
