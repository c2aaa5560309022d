"""Parity at the benchmark sizes, against the oracle's fixtures.

``tests/golden/large/*.json`` holds the oracle's solutions of five
frequencies of two benchmark systems, made by ``tests/golden/make_large.py``
(the reference GMRES restated, products by the C port of the on-the-fly pair
loops, refined in FP64 with explicit residuals to a relative residual near
1e-12 -- the attained value is in the fixture):

  ag_sphere_r35    wFQFMu silver sphere, 10,473 atoms, 41,892 unknowns, on-memory
  agau_bowtie_e80  wFQFMu Ag-Au bow-tie, 5,850 atoms, 23,400 unknowns, matrix-free

The device solves the same frequencies, x polarisation:
  * plain FP64 GMRES (the drop-in: unrestarted, the reference's algorithm) at
    3e-11 of ||b||: sigma_abs within 1e-10 (relative) of the oracle.  Near its
    attainable accuracy the reference's recurrence is erratic: its logged
    residual passes the tolerance while the true residual does not, and it then
    goes on from the updated iterate (gmres_module.f90:174-209) and never
    recovers.  On the sphere, frequency 50 does so at 3e-11 and 5e-11 but
    converges at 1e-10 (sigma_abs error 1.3e-11); on the bow-tie, frequency 150
    does so at 5e-11 but not at 3e-11.  A frequency that stalls at 3e-11 is
    solved again at 1e-10 (at most one may) and held to the same 1e-10 bar; at
    1e-10 for all of them one sphere frequency lands at 1.06e-10;
  * the FP64 refinement (restarted FP64 GMRES, explicit FP64 residuals) at
    1e-11 of ||b||: within 1e-10;
  * mixed BF16x3 tensor-core refinement at the workload's own tolerance
    (1e-12 sqrt(n), absolute, as the reference reads it): within 1e-6.
The geometry is rebuilt here with the same seeded generator and checked against
the fixture's signature before anything is compared.
"""
import importlib.util
import json
import os

import numpy as np
import pytest

from plasmonx_b200.inputs import Problem
from plasmonx_b200.solver import Context, Solver

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
LARGE = os.path.join(HERE, 'golden', 'large')


def _builder():
    spec = importlib.util.spec_from_file_location('make_large', os.path.join(HERE, 'golden', 'make_large.py'))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def _case(name):
    path = os.path.join(LARGE, name + '.json')
    if not os.path.exists(path):
        pytest.skip('fixture %s not generated' % name)
    with open(path) as f:
        fx = json.load(f)
    ml = _builder()
    text, s = ml.build(name)
    sig = ml.signature(s)
    for k, v in fx['geometry'].items():
        assert sig[k] == pytest.approx(v, rel=1e-12, abs=0.0), k
    return fx, Problem.from_keyword_text(text)


@pytest.fixture(scope='module')
def ctx():
    c = Context(0)
    yield c
    c.close()


PLAIN_REL = 3e-11        # the tight plain arm
PLAIN_FLOOR_REL = 1e-10  # frequencies whose unrestarted recurrence stalls above 3e-11


@pytest.mark.parametrize('name', ['ag_sphere_r35', 'agau_bowtie_e80'])
def test_benchmark_size_matches_oracle(ctx, name):
    fx, p = _case(name)
    idx = np.asarray(fx['freq_index'])
    sref = np.array(fx['results'])[:, 9]
    assert max(fx['true_rel_residual']) < 1e-11
    on_the_fly = p.method == 'iterative on the fly'
    with Solver(p, ctx=ctx, store_t=not on_the_fly) as sv:
        sv.set_frequencies(p.freqs[idx], None if p.alpha_w is None else p.alpha_w[:, idx])
        nb = min(np.linalg.norm(sv.rhs(k, 1)[:, 0]) for k in range(len(idx)))
        plain = sv.solve(mode=p.method, precision='fp64', pol_mask=1, tol=PLAIN_REL * nb, max_krylov=2000)
        stalled = np.flatnonzero(plain['status'] != 0)
        if stalled.size:
            # the reference's GMRES at its attainable floor for these: 1e-10 of ||b||
            sel = idx[stalled]
            sv.set_frequencies(p.freqs[sel], None if p.alpha_w is None else p.alpha_w[:, sel])
            again = sv.solve(mode=p.method, precision='fp64', pol_mask=1, tol=PLAIN_FLOOR_REL * nb,
                             max_krylov=2000)
            sv.set_frequencies(p.freqs[idx], None if p.alpha_w is None else p.alpha_w[:, idx])
            for key in ('results', 'status'):
                plain[key][stalled] = again[key]
        assert (plain['status'] == 0).all(), plain['status']
        assert stalled.size <= 1, stalled
        refined = sv.solve(mode=p.method, precision='fp64_refined', pol_mask=1, tol=1e-11 * nb, inner_krylov=1000,
                           inner_tol=1e-11, max_outer=30)
        assert (refined['status'] == 0).all(), refined['status']
        mixed = sv.solve(mode=p.method, precision='mixed_bf16x3', pol_mask=1, tol=1e-12 * np.sqrt(p.n_var),
                         inner_krylov=256 if 'bowtie' in name else 0)
        assert (mixed['status'] == 0).all(), mixed['status']
    err = {k: np.abs(o['results'][:, 9] - sref) / np.abs(sref)
           for k, o in (('plain', plain), ('refined', refined), ('mixed', mixed))}
    assert err['plain'].max() <= 1e-10, err
    assert err['refined'].max() <= 1e-10, err
    assert err['mixed'].max() <= 1e-6, err
