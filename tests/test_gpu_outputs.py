"""A restarted spectrum on the GPU: the reference's restart tests (a backup file for
one frequency, the rest solved) give the frequencies recovered and the maxima
analysis the reference log printed."""
import glob
import os
import shutil

import pytest

from plasmonx_b200 import outputs as O
from plasmonx_b200.solver import Context, Solver
from tests.test_outputs import RESTART, _load

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize('name', RESTART)
def test_restarted_spectrum_on_gpu(name, tmp_path):
    d, exp, p = _load(name)
    for f in glob.glob(os.path.join(d, 'bk', '*.plasmonX.bk')):
        shutil.copy(f, tmp_path)
    stem = str(tmp_path / name)
    ctx = Context(0)
    try:
        with Solver(p, ctx=ctx) as sv:
            out = O.solve_spectrum(sv, stem)
    finally:
        ctx.close()
    assert [round(O.freq_ev(p.freqs[i]), 5) for i in out['recovered']] == exp['recovered_ev']
    assert len(out['maxima']) == len(exp['maxima']['rows'])
    for (_, ev, v), (pev, pv) in zip(out['maxima'], exp['maxima']['rows']):
        assert O.fortran_f(ev, 10, 3).strip() == '%.3f' % pev
        assert float(O.fortran_e(v, 12, 5)) == pv
    for i, blk in enumerate(exp['results']):
        for v, pv in zip(out['results'][i], blk['values']):
            assert abs(v - pv) <= 5.01e-6 * abs(pv) + 1e-30
