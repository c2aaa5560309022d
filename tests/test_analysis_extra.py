"""The reference's grid analysis tests -- planes (one or several, user-bounded),
slabs with their effective volume, the binary .plt format, wFQFMu densities,
BEM planes -- through the oracle and the product's grids and writers
(plasmonx_b200/analysis.py); the checks are in tests/analysis_grid_cases.py and
the device kernels are held to the same files in test_gpu_analysis.py.  The .pqr
and .xyz writers are compared with the reference's lines character for
character (``make_golden.py --pqr-xyz`` samples)."""
import json
import os

import numpy as np
import pytest

from oracle.analysis import bem_field, field_and_density
from tests import analysis_grid_cases as G
from tests.conftest import GOLDEN

EXTRA = os.path.join(GOLDEN, 'analysis_extra')


def oracle_fns(a):
    from plasmonx_b200 import analysis as A
    pos = G.positions(a) * G.TO_BOHR
    N = len(pos)

    def field(x, i_pol, g, third):
        pts = A._points_bohr(g, third)
        if a['model'] == 'bem':
            E = bem_field(pos, x, a['e0'], i_pol, pts)
        else:
            E, _ = field_and_density(pos, np.full(N, a['rq']), np.full(N, a['rmu']), x, a['e0'], i_pol, pts,
                                     a['model'] == 'wfqfmu')
        nx, ny, nz = g.shape()
        return (np.sqrt((np.abs(E) ** 2).sum(axis=1)) / a['e0']).reshape(nz, ny, nx).transpose(2, 1, 0)

    def density(x, g, third):
        _, rho = field_and_density(pos, np.full(N, a['rq']), np.full(N, a['rmu']), x, a['e0'], 0,
                                   A._points_bohr(g, third), a['model'] == 'wfqfmu')
        nx, ny, nz = g.shape()
        return rho.reshape(nz, ny, nx).transpose(2, 1, 0)
    return field, density


@pytest.mark.parametrize('name', G.GRIDS)
def test_oracle_through_writers_reproduces_reference(name):
    a = G.load(name)
    g = G.grid_for(a)
    f, d = oracle_fns(a)
    G.check(a, g, G.outputs(a, g, f, d))


def _pqr_xyz_cases():
    with open(os.path.join(EXTRA, 'pqr_xyz.json')) as f:
        return json.load(f)


@pytest.mark.parametrize('case', range(6))
def test_pqr_and_xyz_lines_match_reference(case):
    """write_pqr_file / plot_xyz: the reference's .pqr (atoms and tesserae, real and
    imaginary charges) and .xyz lines, character for character."""
    from plasmonx_b200 import analysis as A
    c = _pqr_xyz_cases()[case]
    if c['kind'] == 'pqr':
        # a charge the .freq file prints as -0.0000000000000000 comes out of the
        # reference's reader as +0 or -0 (its .pqr shows both for the same text):
        # the sign of a zero charge is not compared
        same_zero = lambda t: t.replace('-0.000E+00', ' 0.000E+00')  # noqa: E731
        for k, line, pos, v, z in zip(c['index'], c['lines'], c['pos'], c['value'], c['z']):
            name = '' if c['bem'] else A.element_symbol(z)
            mine = A.pqr_line(k + 1, name, pos, v, A.VDW_RADIUS.get(name, 0.0), c['bem'])
            assert same_zero(mine) == same_zero(line)
    else:
        info = {'model': 'bem' if c['bem'] else 'wfq', 'z': c['z'],
                ('centres_ang' if c['bem'] else 'coord_ang'): np.array(c['pos'])}
        text = A.xyz_text(info).splitlines()
        assert text[2:] == c['lines']
        assert A.xyz_text(dict(info, **{('centres_ang' if c['bem'] else 'coord_ang'):
                                        np.zeros((c['n'], 3))}, z=[0] * c['n'])).splitlines()[:2] == c['head']
