"""Parity at the benchmark sizes, against the oracle's fixtures.

``tests/golden/large/*.json`` holds the oracle's solutions (the reference
GMRES restated, C port of the on-the-fly product, relative residual 1e-12) of
five frequencies of two benchmark systems, made by
``tests/golden/make_large.py``:

  ag_sphere_r35    wFQFMu silver sphere, 10,473 atoms, 41,892 unknowns, on-memory
  agau_bowtie_e80  wFQFMu Ag-Au bow-tie, 5,850 atoms, 23,400 unknowns, matrix-free

The device solves the same frequencies, x polarisation:
  * plain FP64 GMRES (the drop-in), absolute tolerance 1e-12 ||b||:
    sigma_abs within 1e-10 (relative) of the oracle;
  * mixed BF16x3 tensor-core refinement, same tolerance: within 1e-6.
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


@pytest.mark.parametrize('name', ['ag_sphere_r35', 'agau_bowtie_e80'])
def test_benchmark_size_matches_oracle(ctx, name):
    fx, p = _case(name)
    idx = np.asarray(fx['freq_index'])
    sref = np.array(fx['results'])[:, 9]
    on_the_fly = p.method == 'iterative on the fly'
    with Solver(p, ctx=ctx, store_t=not on_the_fly) as sv:
        sv.set_frequencies(p.freqs[idx], None if p.alpha_w is None else p.alpha_w[:, idx])
        nb = min(np.linalg.norm(sv.rhs(k, 1)[:, 0]) for k in range(len(idx)))
        tol = 1e-12 * nb
        plain = sv.solve(mode=p.method, precision='fp64', pol_mask=1, tol=tol, max_krylov=4000)
        assert (plain['status'] == 0).all(), plain['status']
        mixed = sv.solve(mode=p.method, precision='mixed_bf16x3', pol_mask=1, tol=tol,
                         inner_krylov=256 if 'bowtie' in name else 0)
        assert (mixed['status'] == 0).all(), mixed['status']
    e_plain = np.abs(plain['results'][:, 9] - sref) / np.abs(sref)
    e_mixed = np.abs(mixed['results'][:, 9] - sref) / np.abs(sref)
    assert e_plain.max() <= 1e-10, e_plain
    assert e_mixed.max() <= 1e-6, e_mixed
