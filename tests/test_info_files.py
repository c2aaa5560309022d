"""The .info / .tar.gz / .freq files the reference's analysis tool reads, against the
reference's own files (three .info files and one .freq file from the tarballs of its
analysis tests, copied by ``make_golden.py --info``).

Those tarballs were written by an earlier release of the reference, whose closing
line names the program 'nanoFQ'; that line is left out of the comparison, every
other character is compared.
"""
import os
import re
import tarfile

import numpy as np
import pytest

from plasmonx_b200 import materials as M
from plasmonx_b200 import outputs as O
from tests.conftest import GOLDEN

INFO = os.path.join(GOLDEN, 'info')
NUM = re.compile(r'^[-+]?\d*\.\d+(?:[EeDd][-+]?\d+)?$')


def _text(name):
    with open(os.path.join(INFO, name)) as f:
        return f.read()


def _body(text):
    """Lines before the closing block that make_targz appends."""
    lines = text.splitlines()
    return lines[:-3] if lines[-2].strip().startswith('Normal termination') else lines


def assert_same_layout(mine, ref):
    """Same lines, same columns; numbers equal to the last printed digit or within
    1 ulp of a round trip (Angstrom -> bohr -> Angstrom, eV -> a.u. -> eV)."""
    assert len(mine) == len(ref)
    for a, b in zip(mine, ref):
        assert len(a) == len(b), (a, b)
        ta, tb = a.split(), b.split()
        assert len(ta) == len(tb), (a, b)
        for x, y in zip(ta, tb):
            if NUM.match(y):
                assert abs(float(x) - float(y)) <= 4e-16 * max(1.0, abs(float(y))), (a, b)
            else:
                assert x == y, (a, b)


@pytest.mark.parametrize('name', ['analysis_field_3d_x_wfq_sodium.info', 'analysis_field_3d_x_y_z_wfqfmu_ag.info',
                                  'analysis_pqr_bem.info'])
def test_reader_parses_reference_info(name):
    d = O.read_info(_text(name))
    assert d['terminated']
    if d['model'] == 'bem':
        assert d['centres_ang'].shape == (d['n_var'], 3) and d['n_atoms'] == 0
    else:
        assert d['coord_ang'].shape == (d['n_atoms'], 3)
        assert sum(d['atoms_per_molecule']) == d['n_atoms']
        assert len(d['dynamic']) == len(d['types'])
    assert len(d['freqs_ev']) == d['n_freq']


def _problem_from_info(d):
    """The dynamic problem a reference run with this .info described."""
    from plasmonx_b200.inputs import Problem
    names = [t[0] for t in d['types']]
    model = d['model']
    par = [t[1] for t in d['types']]
    nt = len(names)
    dyn = np.array(d['dynamic'])
    if model == 'wfq':
        chi, eta, rq = [p[0] for p in par], [p[1] for p in par], [p[2] for p in par]
        alpha, rmu = [0.0] * nt, [0.0] * nt
    else:
        chi, eta, alpha, rq, rmu = ([p[k] for p in par] for k in range(5))
    freqs = d['freqs_ev'] / M.AU_TO_EV
    return Problem(model, d['coord_ang'], names, [0] * d['n_atoms'], eta, rq, rmu, dyn[:, 0], dyn[:, 1],
                   [1.0] * nt, dyn[:, 2], np.diag(dyn[:, 3]), np.diag(dyn[:, 4]), freqs, e0=d['e0'],
                   alpha_w=None if model == 'wfq' else np.zeros((nt, len(freqs)), complex),
                   fermi_energy=dyn[:, 5], kernel=d['kernel'], chi=chi, alpha=alpha, mol_index=d['mol_index'])


@pytest.mark.parametrize('name', ['analysis_field_3d_x_wfq_sodium.info', 'analysis_field_3d_x_y_z_wfqfmu_ag.info'])
def test_writer_reproduces_reference_info(name):
    ref = _text(name)
    prob = _problem_from_info(O.read_info(ref))
    assert_same_layout(O.info_text(prob).splitlines(), _body(ref))


def test_bem_info_layout_and_round_trip():
    from plasmonx_b200.bem import bem_surface
    ref = _body(_text('analysis_pqr_bem.info'))
    d = O.read_info('\n'.join(ref))
    # the reference's geometry lines re-printed from their values with this writer's format
    lines = ['%8d' % (i + 1) + ''.join(' ' + O.fortran_f(v, 25, 16) for v in c) for i, c in enumerate(d['centres_ang'])]
    g0 = ref.index('Input Geometry (angstrom)') + 1
    assert lines == ref[g0:g0 + d['n_var']]
    p = bem_surface(80, n_freq=3)
    mine = O.read_info(O.info_text(p))
    t = p.triangles
    assert mine['model'] == 'bem' and mine['n_var'] == 80 and mine['n_freq'] == 3
    assert np.allclose(mine['centres_ang'], (t[:, 0] + t[:, 1] + t[:, 2]) / 3.0 / M.TO_BOHR, rtol=0, atol=1e-15)
    # header block line for line against the reference's BEM file (sizes and frequencies differ)
    head = O.info_text(p).splitlines()
    for k in (3, 4, 5, 8, 9, 10):
        assert head[k] == ref[k]


def test_freq_writer_reproduces_reference_file():
    text = _text('analysis_field_3d_x_y_z_wfqfmu_ag-3.0000000000.freq')
    name, ev, blocks = O.read_freq(text)
    assert name == 'Charges/Dipoles' and ev == 3.0
    X = np.stack([blocks['x'], blocks['y'], blocks['z']], axis=1)
    mine = O.freq_text(ev / M.AU_TO_EV, X, name)
    assert mine == text


def test_make_targz(tmp_path):
    stem = str(tmp_path / 'run')
    for ext, body in (('.info', 'NAtoms     :          1\n'), ('.csv', '# csv\n')):
        with open(stem + ext, 'w') as f:
            f.write(body)
    freqs = [stem + '-1.0000000000.freq', stem + '-2.0000000000.freq']
    for p in freqs:
        with open(p, 'w') as f:
            f.write('complex Charges: x. freq = 1.0\n')
    path = O.make_targz(stem, freqs)
    with tarfile.open(path) as tf:
        names = sorted(tf.getnames())
        info = tf.extractfile('run.info').read().decode()
    assert names == sorted(['run.info', 'run.csv', 'run-1.0000000000.freq', 'run-2.0000000000.freq'])
    assert info.splitlines()[-2] == ' ' * 24 + 'Normal termination of plasmonX'
    assert info.splitlines()[-1] == O.STICKS
    assert not os.path.exists(stem + '.info') and not any(os.path.exists(p) for p in freqs)
    assert os.path.exists(stem + '.csv')


def test_static_info_with_rotated_geometry():
    from plasmonx_b200.static import StaticProblem
    p = StaticProblem.from_keyword_file(os.path.join(GOLDEN, 'fq_principal_axis_energy', 'input.kw'))
    text = O.info_text(p)
    lines = text.splitlines()
    assert lines[3] == 'Field      :     absent' and lines[4] == 'Kernel     :       ohno'
    assert lines[5] == 'Model      :         fq' and lines[8] == 'PrincAxes  :          T'
    d = O.read_info(text)
    assert d['n_var'] == 8 and d['atoms_per_molecule'] == [3, 3]
    assert [t[0] for t in d['types']] == ['H-', 'O-'] and len(d['types'][0][1]) == 2
    assert 'freqs_ev' not in d
    assert np.allclose(d['rotated_ang'], p.coord / M.TO_BOHR, atol=1e-15)
    assert np.allclose(d['coord_ang'], p.coord_ang, atol=1e-15)


def test_dynamic_problem_principal_axes():
    """A dynamic run with `control principal axes` is rotated after the input (and
    its neighbour counts), as rotate_principal_axis does before any solve."""
    from oracle import static as ost
    from plasmonx_b200.inputs import Problem
    base = os.path.join(GOLDEN, 'wfqfmu_hetero_agau_inversion')     # three distinct principal moments
    text = _kw('wfqfmu_hetero_agau_inversion')
    plain = Problem.from_keyword_text(text, base_dir=base)
    rot = Problem.from_keyword_text(text.replace('control principal axes: False', 'control principal axes: True'),
                                    base_dir=base)
    assert rot.principal_axes and not plain.principal_axes
    ref, w, _ = ost.principal_axes(plain.coord, plain.znum)
    assert np.allclose(rot.coord, ref, atol=1e-10)
    assert np.array_equal(rot.neighbours, plain.neighbours)
    d0 = np.linalg.norm(plain.coord[:, None] - plain.coord[None], axis=-1)
    d1 = np.linalg.norm(rot.coord[:, None] - rot.coord[None], axis=-1)
    assert np.allclose(d0, d1, atol=1e-10)
    assert O.read_info(O.info_text(rot))['principal_axes']


def _kw(name):
    with open(os.path.join(GOLDEN, name, 'input.kw')) as f:
        return f.read()
