"""GPU parity: the CUDA path, called through the C ABI, against the oracle and
against the numbers the reference printed in its own regression logs.

Tolerances (FP64 throughout):
  * operator application and right-hand sides: relative 1e-12 (norm-wise)
  * direct inversion: results relative 1e-10 against the oracle's LU
  * GMRES at the input tolerance: same Arnoldi step counts as the reference
    log (up to the near-breakdown cases the oracle test documents) and the
    printed digits of the results, charges and dipoles
  * FP64 refinement at a tight tolerance against the oracle's LU: sigma_abs
    relative 1e-10 (the reference's unrestarted GMRES at 1e-11: 1e-9)
"""
import os

import numpy as np
import pytest

from oracle import keywords, model, solve as osolve
from plasmonx_b200 import configs
from plasmonx_b200.inputs import Problem
from plasmonx_b200.solver import Context, Solver
from tests.conftest import GOLDEN, golden_dirs
from tests.test_oracle_golden import Pin, geometry_spread, load as load_golden, printed_geometry
from tests.printed import agrees

pytestmark = pytest.mark.gpu

CASES = golden_dirs('atomistic')


@pytest.fixture(scope='module')
def ctx():
    c = Context(0)
    yield c
    c.close()


def _pair(name):
    path = os.path.join(GOLDEN, name, 'input.kw')
    return Problem.from_keyword_file(path), model.System.from_keywords(path)


def _rel(a, b):
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


@pytest.mark.parametrize('name', CASES)
@pytest.mark.parametrize('otf', [False, True])
def test_matvec_matches_oracle(ctx, name, otf):
    p, s = _pair(name)
    op = model.Operator(s)
    rng = np.random.default_rng(7)
    with Solver(p, ctx=ctx, store_t=True) as sv:
        for i in sorted({0, len(p.freqs) - 1}):
            x = rng.standard_normal(p.n_var) + 1j * rng.standard_normal(p.n_var)
            y = sv.matvec(i, x, on_the_fly=otf)
            assert _rel(y, op.matvec(i, x)) < 1e-12


@pytest.mark.parametrize('name', CASES)
def test_rhs_matches_oracle(ctx, name):
    p, s = _pair(name)
    op = model.Operator(s)
    with Solver(p, ctx=ctx, store_t=False) as sv:
        for i in sorted({0, len(p.freqs) - 1}):
            b = sv.rhs(i, p.pol_mask)
            ref = op.rhs(i)
            assert _rel(b, ref) < 1e-13


@pytest.mark.parametrize('name', CASES)
def test_solve_matches_reference_log(ctx, name):
    p, _ = _pair(name)
    s, exp = load_golden(name)
    with Solver(p, ctx=ctx) as sv:
        out = sv.solve(want_x=True, trace=True)
    assert 'error' not in out, out.get('error')
    pin = Pin(exp)
    for i, blk in enumerate(exp['results']):
        for k, (v, pv) in enumerate(zip(out['results'][i], blk['values'])):
            pin.check(v, pv, 6, ('results', i, k + 1))
    per_freq = 2 if p.model == 'wfqfmu' else 1
    for t, tab in enumerate(exp['tables']):
        x = out['x'][t // per_freq]
        off = 0 if tab['kind'] == 'wFQ Charges' else p.n_atoms
        for r, row in enumerate(tab['rows']):
            vals = []
            for c in range(3):
                vals += [x[off + r, c].real, x[off + r, c].imag]
            for v, pv in zip(vals, row):
                pin.check(v, pv, 3, (tab['kind'], t, r), abs_floor=1e-12)
    if pin.bad and printed_geometry(name):
        pin.excuse_input_rounding(geometry_spread(s, 'inversion' if p.method == 'inversion' else 'gmres'))
    pin.verify()
    # Arnoldi step counts against the reference log (same rule as the oracle test)
    if exp['gmres']:
        steps = out['steps']
        ev = p.freqs * 27.211386245981
        off = 0
        for tr in exp['gmres']:
            i = int(np.argmin(np.abs(ev - tr['freq_ev'])))
            c = 'XYZ'.index(tr['pol'])
            if steps[i, c] != len(tr['residuals']):
                assert abs(int(steps[i, c]) - len(tr['residuals'])) == 1
                off += 1
            assert agrees(out['trace'][i, c, 0], tr['residuals'][0], 5)
        # the symmetric 37-atom cluster is a near-breakdown Krylov sequence (see the
        # oracle test): one solve in a log may end one step apart
        assert off <= max(1, 0.01 * len(exp['gmres']))


@pytest.mark.parametrize('name', CASES)
def test_solve_matches_oracle(ctx, name):
    p, s = _pair(name)
    method = 'inversion' if p.method == 'inversion' else 'gmres'
    ref = osolve.solve(s, method=method)
    with Solver(p, ctx=ctx) as sv:
        out = sv.solve(want_x=True)
    scale = np.abs(ref['results']).max(axis=0) + 1e-300
    err = np.abs(out['results'] - ref['results']) / scale
    if method == 'inversion':
        # two backward-stable FP64 solves of the same A(w) (the oracle's LU; here LU,
        # or for one-type wFQ and BEM DPCM the shifted Hessenberg solve) agree to
        # ~cond(A) eps in the solution (held to 50 eps cond per frequency); the
        # results are held to 1e-10 of their column scale, or where cond(A(w)) makes
        # that unattainable (graphene at its lowest frequency, cond 1.4e4) to
        # 100 eps cond(A(w)) at that frequency
        x, xr = out['x'], np.asarray(ref['x'])
        dx = np.linalg.norm((x - xr).reshape(len(x), -1), axis=1) / np.linalg.norm(xr.reshape(len(x), -1), axis=1)
        op = model.Operator(s)
        cond = np.array([np.linalg.cond(op.matrix(i)) for i in range(len(x))])
        assert np.all(dx <= 50 * 2.22e-16 * cond)
        bar = np.maximum(1e-10, 100 * 2.22e-16 * cond)[:, None]
        assert np.all(err <= bar), (err.max(axis=1), bar[:, 0])
    else:
        # same algorithm at the same (loose) tolerance; differences are round-off
        # amplified by the Krylov recurrence, bounded by the tolerance itself.
        # A step-count difference of one happens where the last residual lands
        # next to the tolerance (the reference log itself differs from the
        # oracle in 1 of the 1350 sodium solves); two rounding variants may
        # differ in up to 2% of the solves.
        assert err.max() < 1e-5
        st_ref = np.array(ref['steps'])
        differ = np.sum(out['steps'] != st_ref)
        assert differ <= max(1, 0.02 * np.count_nonzero(st_ref))
        assert np.all(np.abs(out['steps'] - st_ref) <= 1)


@pytest.mark.parametrize('name', ['wfqfmu_ag_inversion', 'wfqfmu_hetero_agau_inversion', 'wfq_sodium_inversion'])
@pytest.mark.parametrize('mode', ['iterative', 'iterative on the fly'])
def test_tight_gmres_matches_lu(ctx, name, mode):
    """sigma_abs of the FP64 GPU solves at tight tolerances against the oracle LU:
    the reference's (unrestarted) GMRES and the FP64 refinement (restarted,
    explicit FP64 residuals), both at a 1e-12 relative residual, within 1e-10.
    (The explicit FP64 residual of the sodium operator bottoms out near 1e-13 of |b|,
    since the charge rows difference neighbouring potentials: 1e-13 is not reliably
    attainable there, while the answer is already accurate to ~2e-13.  The
    unrestarted GMRES on the sodium operator assembled on the fly stalls just above
    1e-12 of |b| -- its true residual is summed in another order than the Krylov
    recurrence -- so that arm runs at 1e-11, and a 1e-11 residual bounds the
    forward error by cond(A(w)) x 1e-11 only: cond is 66-717 at the five
    frequencies tested (oracle, numpy), and the measured error reached 1.1e-10 at
    one of them, so that arm is held per frequency to max(1e-10, cond x 1e-11).)"""
    p, s = _pair(name)
    F = len(p.freqs)
    freqs = list(range(F // 2, F, max(1, F // 10)))      # away from the w -> 0 singularity
    ref = osolve.solve(s, method='inversion', freqs=freqs)
    sref = ref['results'][:, 9:12]
    mask = np.abs(sref) > 1e-30
    with Solver(p, ctx=ctx, store_t=True) as sv:
        sv.set_frequencies(p.freqs[freqs], None if p.alpha_w is None else p.alpha_w[:, freqs])
        nb = np.linalg.norm(sv.rhs(0, 7)[:, 0])
        plain_tol = 1e-11 if ('sodium' in name and 'fly' in mode) else 1e-12
        plain = sv.solve(mode=mode, tol=plain_tol * nb, max_krylov=p.n_var)
        refined = sv.solve(mode=mode, precision='fp64_refined', tol=1e-12 * nb, inner_krylov=p.n_var,
                           inner_tol=1e-13, max_outer=10)
    bar_plain = np.full(len(freqs), 1e-10)
    if plain_tol > 1e-12:
        op = model.Operator(s)
        bar_plain = np.maximum(bar_plain, [np.linalg.cond(op.matrix(i)) * plain_tol for i in freqs])
    for out, bar in ((plain, bar_plain[:, None]), (refined, 1e-10)):
        assert (out['status'] == 0).all(), out['status']
        sig = out['results'][:, 9:12]
        err = np.where(mask, np.abs(sig - sref) / np.where(mask, np.abs(sref), 1.0), 0.0)
        assert np.all(err < bar), (err.max(axis=1), bar)


def _na_problem(n_freq=4, method='inversion', radius=20.0):
    p0 = configs.na_sphere(radius=radius, n_freq=n_freq, method=method, tolerance=1e-8)
    text = p0.to_keyword_text()
    return Problem.from_keyword_text(text), model.System.from_keywords(keywords.read_keyword_text(text))


def test_sodium_sphere_893_inversion_and_gmres(ctx):
    """The 893-atom sodium sphere: inversion vs the oracle LU (1e-10), tight GMRES vs LU
    (1e-10), charge conservation to round-off."""
    p, s = _na_problem(n_freq=3)
    ref = osolve.solve(s, method='inversion')
    with Solver(p, ctx=ctx) as sv:
        inv = sv.solve(mode='inversion', want_x=True)
        b = sv.rhs(0, 7)
        it = sv.solve(mode='iterative', tol=1e-12 * np.linalg.norm(b[:, 0]), max_krylov=p.n_var, want_x=True)
    assert (inv['status'] == 0).all() and (it['status'] == 0).all()
    for out in (inv, it):
        sig, sref = out['results'][:, 9], ref['results'][:, 9]
        assert np.max(np.abs(sig - sref) / np.abs(sref)) < 1e-10
        q = out['x'][:, :p.n_atoms, :]
        assert np.all(np.abs(q.sum(axis=1)) <= 1e-12 * np.abs(q).sum(axis=1) + 1e-30)


def test_batched_columns_equal_single_columns(ctx):
    """Each frequency gives the same answer solved alone and in a batch with the others."""
    p, _ = _na_problem(n_freq=12, method='iterative', radius=12.0)
    with Solver(p, ctx=ctx) as sv:
        alone = sv.solve(freq_block=1)
        mixed = sv.solve(freq_block=12)
    # the contraction accumulates every column in the same order whatever the
    # batch, so the answers are identical, not just close
    np.testing.assert_array_equal(alone['steps'], mixed['steps'])
    np.testing.assert_array_equal(alone['results'], mixed['results'])


def test_gmres_dimension_exhausted_reports_status(ctx):
    p, _ = _na_problem(n_freq=2, method='iterative', radius=12.0)
    with Solver(p, ctx=ctx) as sv:
        out = sv.solve(max_krylov=3)
    assert (out['status'] == 5).all()        # PLX_ERR_NOT_CONVERGED
    assert 'error' in out and 'GMRES not converged' in str(out['error'])


def test_zero_field_gives_zero_solution(ctx):
    p0 = configs.na_sphere(radius=10.0, n_freq=2, method='iterative', e0=0.0)
    p = Problem.from_keyword_text(p0.to_keyword_text())
    with Solver(p, ctx=ctx) as sv:
        out = sv.solve(want_x=True)
    assert (out['status'] == 0).all()
    assert not np.any(out['x'])


def test_single_polarisation(ctx):
    p, s = _na_problem(n_freq=2, method='inversion', radius=12.0)
    p.polarization = s.polarization = 'y'
    ref = osolve.solve(s, method='inversion')
    with Solver(p, ctx=ctx) as sv:
        out = sv.solve(want_x=True)
    assert not np.any(out['x'][:, :, 0]) and not np.any(out['x'][:, :, 2])
    assert np.max(np.abs(out['results'] - ref['results']) / (np.abs(ref['results']).max(axis=0) + 1e-300)) < 1e-10
