"""Planes, effective volume and the binary .plt format of the analysis step against
four more of the reference's analysis tests (inputs and sampled outputs extracted
by ``make_golden.py --analysis-extra``): the oracle's field / density through the
product's grids and writers (plasmonx_b200/analysis.py) reproduce the reference's
grid block, the plane .csv lines (coordinates to every printed digit, values to
1e-10), the .plt header and values (float32, to one unit in the last place) and
the effective volume and area lines; the .pqr and .xyz writers reproduce the
reference's lines character for character (``--pqr-xyz`` samples).  The device kernel is held to the same files
in test_gpu_analysis.py."""
import json
import os
import struct

import numpy as np
import pytest

from oracle.analysis import field_and_density
from tests.conftest import GOLDEN

TO_BOHR = 1.8897261254578281
EXTRA = os.path.join(GOLDEN, 'analysis_extra')
NAMES = ['analysis_field_2d_x_yz_wfq_sodium', 'analysis_density_2d_x_wfq_sodium',
         'analysis_field_volume_x_wfq_sodium', 'analysis_field_3d_x_wfq_sodium_plt']


def load(name):
    with open(os.path.join(EXTRA, name + '.json')) as f:
        return json.load(f)


def grid_of(a):
    from plasmonx_b200 import analysis as A
    n = [int(a['log_grid'][k].split()[-1]) for k in (4, 6, 8)]
    coords = np.array(a['coords_ang'])
    if a['kind'] == 'plane':
        axes = {'xy': (0, 1), 'xz': (0, 2), 'yz': (1, 2)}[a['options']['plane']]
        return A.plane_grid(coords, a['options']['plane'], tuple(n[k] for k in axes), 10.0)
    if a['kind'] == 'volume':
        return A.cubic_grid(coords, n, lo=np.array(a['options']['lo']), hi=np.array(a['options']['hi']))
    return A.cubic_grid(coords, n, 10.0)


def values_by(a, g, field_fn, density_fn):
    """The quantities the test wrote: [(suffix or kind, (nx, ny, nz) values)]."""
    third = a['options'].get('third', 0.0)
    if 'density' in a['name']:
        rho = density_fn(g, third)
        return [('-densityRe', rho.real), ('-densityIm', rho.imag)]
    return [('field', field_fn(g, third))]


def oracle_fns(a):
    from plasmonx_b200 import analysis as A
    coords = np.array(a['coords_ang']) * TO_BOHR
    N = len(coords)
    x = np.array(a['x'])[:, 0] + 1j * np.array(a['x'])[:, 1]

    def run(g, third):
        E, rho = field_and_density(coords, np.full(N, a['rq']), np.zeros(N), x, a['e0'], a['pol'],
                                   A._points_bohr(g, third), False)
        nx, ny, nz = g.shape()
        return E, rho, (nx, ny, nz)

    def field(g, third):
        E, _, (nx, ny, nz) = run(g, third)
        return (np.sqrt((np.abs(E) ** 2).sum(axis=1)) / a['e0']).reshape(nz, ny, nx).transpose(2, 1, 0)

    def density(g, third):
        _, rho, (nx, ny, nz) = run(g, third)
        return rho.reshape(nz, ny, nx).transpose(2, 1, 0)
    return field, density


def check_outputs(a, g, vals):
    """Compare the writers' output for `vals` with the reference's sampled files."""
    from plasmonx_b200 import analysis as A
    assert [l.rstrip() for l in g.info_text().splitlines()] == [l.rstrip() for l in a['log_grid']]
    if a['kind'] == 'plane':
        for suffix, v in vals:
            key = [f for f in a['options']['files'] if f.endswith(suffix + '.csv') or suffix == 'field'][0]
            ref = a['csv'][key]
            mine = A.plane_csv_text(g, A.on_plane(g, v)).splitlines()
            assert len(mine) == ref['n_lines']
            for i, line in zip(ref['index'], ref['lines']):
                m, r = mine[i].split(), line.split()
                assert m[:2] == r[:2] and len(mine[i]) == len(line), (i, mine[i], line)
                if r:
                    a_, b_ = float(m[2]), float(r[2])
                    assert abs(a_ - b_) <= 1e-10 * abs(b_) + 1e-300, (i, mine[i], line)
    elif a['kind'] == 'volume':
        v = vals[0][1]
        assert A.effective_volume_lines('Ex', g, v).splitlines() == a['volume_lines']
        assert A.maximum_lines('Field', 'Ex', g, v).splitlines() == a['log_max']
    else:
        data = A.plt_bytes(g, vals[0][1])
        ref = a['plt']
        assert len(data) == ref['bytes']
        assert list(struct.unpack('<5i', data[:20])) == ref['head_i']
        assert list(struct.unpack('<6f', data[20:44])) == ref['head_f']
        mine = np.frombuffer(data[44:], dtype='<f4')[np.array(ref['index'])]
        theirs = np.array(ref['values'], dtype=np.float32)
        assert np.all(np.abs(mine - theirs) <= np.spacing(np.abs(theirs)))


@pytest.mark.parametrize('name', NAMES)
def test_oracle_through_writers_reproduces_reference(name):
    a = load(name)
    g = grid_of(a)
    f, d = oracle_fns(a)
    check_outputs(a, g, values_by(a, g, f, d))


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
