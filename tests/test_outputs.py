"""Output and restart files (plasmonx_b200/outputs.py) against the reference's
own restart tests: the backup files they ship are reproduced byte for byte, a
restarted spectrum recovers exactly the frequencies whose backup exists, and
the maxima analysis prints what the reference log printed.  The spectrum
itself comes from the oracle here (a stand-in solver on the CPU); the GPU
version of the same check is test_gpu_outputs.py."""
import glob
import json
import os
import shutil

import numpy as np
import pytest

from oracle import bem as obem, model, solve as osolve
from plasmonx_b200 import outputs as O
from plasmonx_b200.inputs import Problem
from tests.conftest import GOLDEN, golden_dirs
from tests.printed import agrees

RESTART = ['wfq_sodium_restart', 'wfqfmu_ag_restart']


def _load(name):
    d = os.path.join(GOLDEN, name)
    with open(os.path.join(d, 'expected.json')) as f:
        exp = json.load(f)
    return d, exp, Problem.from_keyword_file(os.path.join(d, 'input.kw'))


class OracleSolver:
    """The solver interface solve_spectrum drives, answered by the oracle."""

    def __init__(self, prob, path):
        self.prob = prob
        self.system = model.System.from_keywords(path)
        self.freqs = np.asarray(prob.freqs)
        self.all_freqs = self.freqs.copy()
        self.calls = []

    def set_frequencies(self, freqs, alpha_w=None):
        self.freqs = np.asarray(freqs)

    def solve(self, want_x=False, **kw):
        idx = [int(np.argmin(np.abs(self.all_freqs - w))) for w in self.freqs]
        self.calls.append(idx)
        out = osolve.solve(self.system, method='inversion', freqs=idx)
        res = {'results': out['results']}
        if want_x:
            res['x'] = out['x']
        return res


@pytest.mark.parametrize('name', RESTART)
def test_backup_file_is_reproduced(name):
    d, exp, p = _load(name)
    bk = glob.glob(os.path.join(d, 'bk', '*.plasmonX.bk'))[0]
    row = O.read_backup(bk)
    w = [f for f in p.freqs if abs(O.freq_ev(f) - exp['recovered_ev'][0]) < 1e-9][0]
    with open(bk) as f:
        assert O.backup_text(w, row) == f.read()
    assert os.path.basename(O.backup_path(name, w)) == os.path.basename(bk)


@pytest.mark.parametrize('name', RESTART)
def test_restart_recovers_backups_and_prints_the_maxima(name, tmp_path):
    d, exp, p = _load(name)
    for f in glob.glob(os.path.join(d, 'bk', '*.plasmonX.bk')):
        shutil.copy(f, tmp_path)
    stem = str(tmp_path / name)
    sv = OracleSolver(p, os.path.join(d, 'input.kw'))
    out = O.solve_spectrum(sv, stem, save_freq=True, block=4)
    rec_ev = [round(O.freq_ev(p.freqs[i]), 5) for i in out['recovered']]
    assert rec_ev == exp['recovered_ev']
    solved = sorted(i for c in sv.calls for i in c)
    assert solved == [i for i in range(len(p.freqs)) if i not in out['recovered']]
    # maxima: same states, frequencies and printed values as the reference log
    assert len(out['maxima']) == len(exp['maxima']['rows'])
    for (_, ev, v), (pev, pv) in zip(out['maxima'], exp['maxima']['rows']):
        assert O.fortran_f(ev, 10, 3).strip() == '%.3f' % pev
        assert float(O.fortran_e(v, 12, 5)) == pytest.approx(pv, rel=0, abs=0)
    # the backups of the run are removed; the CSV and .freq files are written
    assert not glob.glob(stem + '-*.plasmonX.bk')
    tab = np.loadtxt(stem + '.csv', comments='#')
    assert tab.shape == (len(p.freqs), 21)
    np.testing.assert_allclose(tab[:, 1:], out["results"], rtol=5.01e-6, atol=0)      # E14.6
    assert len(glob.glob(stem + '-*.freq')) == len(p.freqs) - len(out['recovered'])


def _maxima_cases():
    out = []
    for name in golden_dirs():
        with open(os.path.join(GOLDEN, name, 'expected.json')) as f:
            if 'maxima' in json.load(f) and name not in RESTART:
                out.append(name)
    return out


@pytest.mark.parametrize('name', _maxima_cases())
def test_maxima_of_every_printed_spectrum(name):
    """print_maxima (algorithm_module.f90:907-978) over the oracle's spectrum: the
    states, frequencies (F10.3 eV) and values (E12.5) of every fixture whose log
    prints a maxima block (the restart cases above go through solve_spectrum)."""
    d = os.path.join(GOLDEN, name)
    with open(os.path.join(d, 'expected.json')) as f:
        exp = json.load(f)
    kw = os.path.join(d, 'input.kw')
    with open(kw) as f:
        kind = dict(l.split(':', 1) for l in f.read().splitlines()
                    if ':' in l and not l.startswith('#'))['output maxima analysis'].strip()
    if name.startswith('bem_'):
        b = obem.Bem(kw)
        freqs, results = b.freqs, b.solve()['results']
    else:
        s = model.System.from_keywords(kw)
        freqs = s.freqs
        results = osolve.solve(s, method='inversion' if s.method == 'inversion' else 'gmres')['results']
    peaks = O.maxima(freqs, np.asarray(results), kind)
    assert exp['maxima']['n_freq'] == len(freqs)
    assert len(peaks) == len(exp['maxima']['rows'])
    for (state, ev, v), (pev, pv), k in zip(peaks, exp['maxima']['rows'], range(len(peaks))):
        assert state == k + 1
        assert O.fortran_f(ev, 10, 3).strip() == '%.3f' % pev
        assert agrees(v, pv, 5), (ev, v, pv)


def test_fortran_edit_descriptors():
    assert O.fortran_e(-18646.1234, 14, 6) == ' -0.186461E+05'
    assert O.fortran_e(0.0735, 9, 3) == '0.735E-01'
    assert O.fortran_e(-0.0735, 9, 3) == '-.735E-01'
    assert O.fortran_e(0.0, 14, 6) == '  0.000000E+00'
    assert O.fortran_e(10.671, 12, 5) == ' 0.10671E+02'
    assert O.fortran_f(2.0, 7, 5) == '2.00000'


def test_spectrum_packed_with_its_info(tmp_path):
    """save_info: the run's .info is written first and packed at the end with the CSV
    and the .freq files into <stem>.tar.gz (make_targz); what the analysis step reads
    comes back out of the archive."""
    import tarfile
    name = 'wfq_sodium_inversion'
    d, exp, p = _load(name)
    stem = str(tmp_path / name)
    sv = OracleSolver(p, os.path.join(d, 'input.kw'))
    out = O.solve_spectrum(sv, stem, save_freq=True, save_info=True)
    with tarfile.open(out['paths']['tar']) as tf:
        names = sorted(tf.getnames())
        info = O.read_info(tf.extractfile(name + '.info').read().decode())
        fname = os.path.basename(O.freq_path(stem, p.freqs[0]))
        _, ev, blocks = O.read_freq(tf.extractfile(fname).read().decode())
    assert name + '.info' in names and name + '.csv' in names
    assert len([n for n in names if n.endswith('.freq')]) == len(p.freqs)
    assert info['terminated'] and info['model'] == 'wfq' and info['n_atoms'] == p.n_atoms
    np.testing.assert_allclose(info['coord_ang'], p.coord_ang, rtol=1e-15, atol=1e-14)
    np.testing.assert_allclose(info['freqs_ev'], p.freqs * O.M.AU_TO_EV, rtol=1e-15)
    assert ev == pytest.approx(O.freq_ev(p.freqs[0]), rel=1e-15)
    assert not glob.glob(stem + '*.freq') and not os.path.exists(stem + '.info')
