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


class _OracleFieldSolver:
    """field_at_points answered by the oracle (the host logic of the analysis flow
    runs on the CPU; the device kernel is checked in test_gpu_analysis.py)."""

    def __init__(self, prob):
        self.p = prob

    def field_at_points(self, i_pol, x, points):
        p = self.p
        return field_and_density(p.coord, p.r_q[p.atom_types], p.r_mu[p.atom_types], x, p.e0, i_pol, points,
                                 p.model == 'wfqfmu')


def test_archive_to_cubes_on_the_host(tmp_path):
    """A spectrum packed with save_info / save_freq, read back by read_archive, turned
    into a problem by problem_from_info and into cube files by write_cubes: names,
    headers and values as the reference's analysis program writes them."""
    from plasmonx_b200 import analysis as A
    from plasmonx_b200 import configs
    from plasmonx_b200 import outputs as O
    from tests.test_outputs import OracleSolver
    p = configs.particle('Na', 'sphere', 7.0, n_freq=2, method='inversion')
    stem = str(tmp_path / 'na')
    kw = stem + '.kw'
    with open(kw, 'w') as f:
        f.write(p.to_keyword_text())
    run = O.solve_spectrum(OracleSolver(p, kw), stem, save_freq=True, save_info=True)
    info, sols = A.read_archive(run['paths']['tar'])
    q = A.problem_from_info(info)
    assert q.n_atoms == p.n_atoms and np.allclose(q.coord, p.coord, rtol=1e-15, atol=1e-13)
    label = sorted(sols)[0]
    grid, files = A.write_cubes(run['paths']['tar'], _OracleFieldSolver(q), info, sols[label], pols=('x', 'z'),
                                n=(8, 7, 6), offset=4.0)
    assert [os.path.basename(f) for f in files] == ['na-Ex-%s.cube' % label, 'na-Ez-%s.cube' % label]
    with open(files[0]) as f:
        lines = f.read().splitlines()
    assert lines[0] == 'Generated by plasmonX analysis' and lines[1] == ''
    assert int(lines[2].split()[0]) == p.n_atoms and int(lines[3].split()[0]) == 8
    vals = np.array([float(v) for l in lines[6 + p.n_atoms:] for v in l.split()])
    direct = A.field_on_grid(_OracleFieldSolver(q), sols[label][2]['x'], 0, grid, info['e0'])
    assert vals.size == 8 * 7 * 6
    assert np.allclose(vals, direct.ravel(), rtol=5.01e-6, atol=0)
    # densities: real and imaginary cubes
    _, dfiles = A.write_cubes(run['paths']['tar'], _OracleFieldSolver(q), info, sols[label], pols=('y',),
                              what='density', n=(5, 5, 5), offset=3.0)
    assert [os.path.basename(f)[-15:] for f in dfiles] == ['-densityRe.cube', '-densityIm.cube']


def test_plane_and_plt_writers_name_files_as_the_reference(tmp_path):
    """write_planes / write_cubes(fmt='plt') write the files the reference's analysis
    program writes for the same options (names from its plane and .plt tests)."""
    from plasmonx_b200 import analysis as A
    from plasmonx_b200 import configs
    from plasmonx_b200 import outputs as O
    from tests.test_outputs import OracleSolver
    p = configs.particle('Na', 'sphere', 7.0, n_freq=1, method='inversion')
    stem = str(tmp_path / 'na')
    with open(stem + '.kw', 'w') as f:
        f.write(p.to_keyword_text())
    run = O.solve_spectrum(OracleSolver(p, stem + '.kw'), stem, save_freq=True, save_info=True)
    info, sols = A.read_archive(run['paths']['tar'])
    sv = _OracleFieldSolver(A.problem_from_info(info))
    label = sorted(sols)[0]
    g, files = A.write_planes(run['paths']['tar'], sv, info, sols[label], 'xy', 6.35, n_plane=3, step=0.5,
                              pols=('x',), what='density', n=(6, 5))
    names = [os.path.basename(f) for f in files]
    assert names == ['na-Ex-%s-p-%s-density%s.csv' % (label, c, part) for c in ('6.35', '6.85', '7.35')
                     for part in ('Re', 'Im')]
    with open(files[0]) as f:
        lines = f.read().splitlines()
    assert len(lines) == 6 * 5 + 6 and lines[5] == ''
    g3, pl = A.write_cubes(run['paths']['tar'], sv, info, sols[label], pols=('x',), n=(4, 4, 4), fmt='plt')
    assert [os.path.basename(f) for f in pl] == ['na-Ex-%s.plt' % label]
    assert os.path.getsize(pl[0]) == 44 + 4 * 64
