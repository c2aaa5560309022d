"""GPU parity of the boundary-element (DPCM / IEFPCM) path against the oracle.

The oracle (oracle/bem.py) is pinned to the reference's four BEM regression
logs; here the CUDA path is compared with it on those inputs and on seeded
synthetic surfaces written out as the reference's own input files.

Tolerances (FP64):
  * Green-function derivative applied to vectors (the GMRES operator D + z I)
    and the right-hand sides: relative 1e-12, norm-wise
  * direct inversion (DPCM D + z I; IEFPCM -(D + z I) S A^-1): relative 1e-10
  * GMRES at the input tolerance: the oracle's step counts, iterates relative 1e-9
  * FP64 refinement at a residual of 1e-12 E0 sqrt(n): results relative 1e-10;
    BF16x3 tensor-core contraction with refinement at 1e-9 E0 sqrt(n): relative 1e-6
IEFPCM with the accurate Green function is the one exception: its right-hand
side carries the diagonal of D before the closure, analytically zero for flat
tesserae and rounding noise of the polar quadrature in every implementation.
There the library's right-hand side is checked to differ from the oracle's by
a diagonal alone, the solves are compared on the same right-hand side, and the
end results within relative 1e-4 (the reference test's own tolerance is 5e-3).
"""
import os

import numpy as np
import pytest

from oracle import bem as obem
from oracle import model
from oracle.gmres import gmres
from plasmonx_b200.bem import BemProblem, bem_surface
from plasmonx_b200.solver import Context, Solver
from tests.conftest import GOLDEN, golden_dirs

pytestmark = pytest.mark.gpu

GOLDEN_BEM = golden_dirs('bem')


@pytest.fixture(scope='module')
def ctx():
    c = Context(0)
    yield c
    c.close()


def _rel(a, b):
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


def _noisy_rhs(p):
    return p.variant == 'iefpcm' and p.accurate


SYNTH = [('sphere', 'dpcm', 'approximate'), ('sphere', 'iefpcm', 'accurate'),
         ('rod', 'dpcm', 'accurate'), ('rod', 'iefpcm', 'approximate')]


@pytest.fixture(scope='module', params=SYNTH, ids=lambda p: '-'.join(p))
def synth(request, tmp_path_factory):
    shape, variant, green = request.param
    p = bem_surface(320, variant=variant, shape=shape, n_freq=4, green=green, method='iterative',
                    tolerance=1e-10, seed=3)
    kw = p.write_keyword_files(str(tmp_path_factory.mktemp('bem')), 'surf')
    return BemProblem.from_keyword_file(kw), obem.Bem(kw)


def _gmres_operator(o, i):
    A = o.D.astype(np.complex128)
    A[np.diag_indices(o.n_var)] += o.z(i)
    return A


@pytest.mark.parametrize('name', GOLDEN_BEM)
def test_golden_bem_matches_oracle(ctx, name):
    path = os.path.join(GOLDEN, name, 'input.kw')
    p, o = BemProblem.from_keyword_file(path), obem.Bem(path)
    ref = o.solve()
    with Solver(p, ctx=ctx) as sv:
        out = sv.solve(want_x=True)
        assert 'error' not in out
        if _noisy_rhs(p):
            assert _rel(out['results'], ref['results']) < 1e-4
            x = sv.complex_inversion(0, o.rhs(0))
            assert _rel(x, ref['x'][0]) < 1e-10
        elif p.method == 'inversion':
            assert _rel(out['results'], ref['results']) < 1e-10
            assert _rel(out['x'], ref['x']) < 1e-10
        else:
            assert [list(s) for s in out['steps']] == [list(s) for s in ref['steps']]
            assert _rel(out['results'], ref['results']) < 1e-9


def test_matvec_and_rhs_match_oracle(ctx, synth):
    p, o = synth
    rng = np.random.default_rng(11)
    with Solver(p, ctx=ctx) as sv:
        for i in (0, len(p.freqs) - 1):
            x = rng.standard_normal(p.n_var) + 1j * rng.standard_normal(p.n_var)
            assert _rel(sv.matvec(i, x), o.matvec(i, x)) < 1e-12
        b, ref = sv.rhs(0), o.rhs(0)
    if not _noisy_rhs(p):
        assert _rel(b, ref) < 1e-12
        return
    # the two differ by a diagonal only: (b - ref)_i = delta_i v_i with v = -E0 r,
    # the same delta_i for every polarisation, |delta_i| at the noise level
    v = -p.e0 * o.t['coord']
    delta = ((b - ref) / v).real
    assert np.max(np.abs((b - ref).imag)) == 0.0
    assert np.max(np.abs(delta[:, 0] - delta[:, 1])) < 1e-8
    assert np.max(np.abs(delta[:, 0] - delta[:, 2])) < 1e-8
    assert np.max(np.abs(delta)) < 1e-2


def test_inversion_matches_oracle(ctx, synth):
    p, o = synth
    ref = o.solve('inversion')
    with Solver(p, ctx=ctx) as sv:
        out = sv.solve(mode='inversion', want_x=True)
        for i in (0, len(p.freqs) - 1):
            b = sv.rhs(i)
            x = sv.complex_inversion(i, b)
            assert _rel(x, np.linalg.solve(o.matrix(i), b)) < 1e-10
    assert _rel(out['results'], ref['results']) < (1e-4 if _noisy_rhs(p) else 1e-10)
    if not _noisy_rhs(p):
        assert _rel(out['x'], ref['x']) < 1e-10


def test_gmres_matches_oracle(ctx, synth):
    """The reference's GMRES on the same right-hand side: same Arnoldi steps, same iterate."""
    p, o = synth
    with Solver(p, ctx=ctx) as sv:
        for i in (0, len(p.freqs) - 1):
            b = sv.rhs(i)
            for c in range(3):
                x, steps, _ = sv.gmres(i, b[:, c], p.tol, p.gmres_dim)
                xr, sr = gmres(lambda v: o.matvec(i, v), b[:, c], p.tol, p.gmres_dim)
                assert steps == sr
                assert _rel(x, xr) < 1e-9
        if not _noisy_rhs(p):
            ref = o.solve('gmres')
            out = sv.solve(mode='iterative')
            assert [list(s) for s in out['steps']] == [list(s) for s in ref['steps']]
            assert _rel(out['results'], ref['results']) < 1e-9


def _exact_results(sv, o):
    """results rows of the exact solution of the GMRES operator (D + z I) for the
    library's own right-hand sides."""
    rows = []
    for i in range(len(o.freqs)):
        x = np.linalg.solve(_gmres_operator(o, i), sv.rhs(i))
        rows.append(model.results_row(o.polar(x), o.freqs[i]))
    return np.array(rows)


@pytest.mark.parametrize('precision,rel,bar', [('fp64_refined', 1e-12, 1e-10), ('mixed_bf16x3', 1e-9, 1e-6)])
def test_refined_forms_reach_the_fp64_answer(ctx, synth, precision, rel, bar):
    """The refined forms solve the reference's GMRES operator (D + z I; for IEFPCM too,
    as the reference's iterative path does) to the accuracy of an FP64 LU solve.  The
    BEM right-hand sides scale with E0 (|b| ~ E0 sqrt(n)), so the absolute tolerance is
    set to rel * E0 * sqrt(n)."""
    p, o = synth
    with Solver(p, ctx=ctx) as sv:
        exact = _exact_results(sv, o)
        out = sv.solve(mode='iterative', precision=precision, tol=rel * p.e0 * np.sqrt(p.n_var))
    assert 'error' not in out, out.get('error')
    assert np.all(out['status'] == 0)
    assert _rel(out['results'], exact) < bar


def test_bem_on_the_fly_is_refused(ctx, synth):
    p, _ = synth
    with Solver(p, ctx=ctx) as sv:
        out = sv.solve(mode='iterative on the fly')
        assert 'error' in out and 'on the fly' in str(out['error'])
        with pytest.raises(Exception, match='on the fly'):
            sv.matvec(0, np.ones(p.n_var, dtype=np.complex128), on_the_fly=True)
