"""GPU parity of the static FQ / FQFMu solves (plx_static_solve) with the oracle.

The oracle (oracle/static.py) is pinned to the reference's five static logs
(test_static_golden.py).  Here the device path -- matrix and right-hand sides
built by the library's kernels, the charge constraints eliminated and the rest
factored by Cholesky (or the full system by LU), the energy and the FQ static
polarizability -- is compared with it:
  * the reference's five inputs: energy, charges, dipoles and polarizability
    relative 1e-11 to the oracle, and the logs' printed numbers at their printed
    precision -- with the default factorisation (charge constraints eliminated,
    Cholesky) and with LU of the full system (the reference's form);
  * seeded water clusters over the three charge kernels, both force fields,
    ground state and static field ('field' and 'potential' right-hand sides):
    variables relative 1e-10 (norm-wise), energy and polarizability 1e-11;
  * at sizes the oracle does not reach, size-independent properties: every
    molecule's charges sum to zero, the polarizability is symmetric, and the
    energy and the polarizability's isotropic value do not change under a rigid
    rotation of the cluster.
"""
import json
import os

import numpy as np
import pytest

from oracle import static as ost
from plasmonx_b200 import _lib
from plasmonx_b200.solver import Context
from plasmonx_b200.static import StaticProblem, StaticSolver, water_cluster
from tests.conftest import GOLDEN, golden_dirs
from tests.test_static_golden import check_printed_matrix, e_tol

pytestmark = pytest.mark.gpu

CASES = golden_dirs('static')


@pytest.fixture(scope='module')
def ctx():
    c = Context(0)
    yield c
    c.close()


def _rel(a, b):
    return np.linalg.norm(np.asarray(a) - np.asarray(b)) / max(np.linalg.norm(b), 1e-300)


def _oracle(p):
    return ost.Static(p.forcefield, p.kernel, p.coord, p.atom_types, p.apm, p.chi, p.eta, p.alpha, p.r_q, p.r_mu,
                      p.rhs_form, p.e0)


@pytest.mark.parametrize('factorization', ['auto', 'cholesky_mixed', 'cholesky_blocked', 'lu'])
@pytest.mark.parametrize('name', CASES)
def test_golden_static_matches_oracle_and_log(ctx, name, factorization):
    p = StaticProblem.from_keyword_file(os.path.join(GOLDEN, name, 'input.kw'))
    p.factorization = factorization
    with open(os.path.join(GOLDEN, name, 'expected.json')) as f:
        exp = json.load(f)
    out = StaticSolver(p, ctx=ctx).solve()
    ref = _oracle(p).solve(p.what)
    assert _rel(out['variables'], ref['variables']) < 1e-11
    for a, b in zip(out['charges'].ravel(), np.array(exp['charges']).ravel()):
        assert abs(a - b) <= e_tol(b, 6) * 1.0001 + 1e-300
    if 'dipoles' in exp:
        for a, b in zip(out['dipoles'].ravel(), np.array(exp['dipoles']).ravel()):
            assert abs(a - b) <= e_tol(b, 6) * 1.0001 + 1e-15
    if 'energy' in exp:
        assert abs(out['energy'] - ref['energy']) <= 1e-11 * abs(ref['energy'])
        assert abs(out['energy'] - exp['energy']) <= 0.5e-8 * 1.0001
    if 'polar' in exp:
        assert _rel(out['polar'], ref['polar']) < 1e-11
        check_printed_matrix(exp['polar'], out['polar'], 4, floor=1e-12)
        assert abs(out['polar_iso'] - exp['polar_iso']) <= 0.5e-10 * 1.0001
    if 'rotated' in exp:
        assert np.max(np.abs(out['rotated_ang'] - np.array(exp['rotated']))) <= 0.5e-6 * 1.0001


SYNTH = [(ff, kernel, what, form, e0)
         for ff in ('fq', 'fqfmu')
         for kernel in ('coulomb', 'ohno', 'gaussian')
         for what, form, e0 in (('energy', 'field', 0.0), ('static', 'field', 1e-3), ('static', 'potential', 2e-3))]


@pytest.mark.parametrize('factorization', ['auto', 'cholesky_mixed', 'cholesky_blocked', 'lu'])
@pytest.mark.parametrize('ff,kernel,what,form,e0', SYNTH, ids=lambda v: str(v))
def test_water_clusters_match_oracle(ctx, ff, kernel, what, form, e0, factorization):
    p = water_cluster(40, ff, kernel, what=what, rhs_form=form, e0=e0, seed=7, factorization=factorization)
    out = StaticSolver(p, ctx=ctx).solve()
    ref = _oracle(p).solve(what)
    assert _rel(out['variables'], ref['variables']) < 1e-10
    if what == 'energy':
        assert abs(out['energy'] - ref['energy']) <= 1e-11 * abs(ref['energy'])
    elif ff == 'fq':
        assert _rel(out['polar'], ref['polar']) < 1e-11


@pytest.mark.parametrize('factorization', ['auto', 'cholesky_mixed'])
@pytest.mark.parametrize('ff,what', [('fq', 'energy'), ('fq', 'static'), ('fqfmu', 'energy')])
def test_elimination_is_the_default_path(ctx, ff, what, factorization):
    """With positive definite blocks (Ohno, Gaussian) the reduced system is factored
    by Cholesky -- in double precision by default, in single precision with
    double-precision refinement on request: the profiled flops are those of a
    reduced Cholesky (plus the corrections), not of the full LU, and the answers
    agree with the LU form."""
    p = water_cluster(40, ff, what=what, e0=1e-3, seed=7, factorization=factorization)
    ctx.profile(True)
    auto = StaticSolver(p, ctx=ctx).solve()
    fl = ctx.profile_read(6)['flops']
    ctx.profile(False)
    n, m = p.n_atoms, p.n_mol
    nr = (n if ff == 'fq' else 4 * n) - m
    ncols = (1 if what == 'energy' else 3) + (3 if (ff == 'fq' and what == 'static') else 0)
    chol = nr ** 3 / 3.0
    if factorization == 'auto':
        assert abs(fl - (chol + 2.0 * nr * nr * ncols)) <= 1e-9 * fl
    else:
        iters = (fl - chol) / (4.0 * nr * nr * ncols)
        assert 1 <= round(iters) <= 31 and abs(iters - round(iters)) < 1e-6
    p.factorization = 'lu'
    lu = StaticSolver(p, ctx=ctx).solve()
    assert _rel(auto['variables'], lu['variables']) < 1e-11
    if what == 'energy':
        assert abs(auto['energy'] - lu['energy']) <= 1e-12 * abs(lu['energy'])
    if 'polar' in lu:
        assert _rel(auto['polar'], lu['polar']) < 1e-11


@pytest.mark.parametrize('apm', [[2, 4], [3, 1, 2]])
def test_ragged_molecules_follow_the_reference_rows(ctx, apm):
    """Molecule sizes that differ: the constraint rows are the reference's
    (disjoint for [2, 4]: eliminated; overlapping for [3, 1, 2]: LU)."""
    for what in ('energy', 'static'):
        p = water_cluster(2, 'fq', what=what, e0=1e-3, seed=5)
        p.apm = np.array(apm, dtype=np.int32)
        p.n_mol = len(apm)
        out = StaticSolver(p, ctx=ctx).solve()
        ref = _oracle(p).solve(what)
        assert _rel(out['variables'], ref['variables']) < 1e-11
        if what == 'static':
            assert _rel(out['polar'], ref['polar']) < 1e-11


def test_medium_fqfmu_cluster_matches_oracle(ctx):
    p = water_cluster(300, 'fqfmu', what='energy', seed=3)
    out = StaticSolver(p, ctx=ctx).solve()
    ref = _oracle(p).solve('energy')
    assert _rel(out['variables'], ref['variables']) < 1e-10
    assert abs(out['energy'] - ref['energy']) <= 1e-11 * abs(ref['energy'])


def _rotation(seed):
    q, _ = np.linalg.qr(np.random.default_rng(seed).standard_normal((3, 3)))
    return q


@pytest.mark.parametrize('ff,n_mol', [('fq', 3000), ('fqfmu', 1000)])
def test_large_cluster_properties(ctx, ff, n_mol):
    p = water_cluster(n_mol, ff, what='energy', seed=11)
    out = StaticSolver(p, ctx=ctx).solve()
    q = out['charges'][:, 0].reshape(n_mol, 3)
    assert np.max(np.abs(q.sum(axis=1))) < 1e-10 * max(1.0, np.max(np.abs(q)))
    # a rigid rotation of the whole cluster leaves the energy unchanged
    R = _rotation(2)
    p2 = water_cluster(n_mol, ff, what='energy', seed=11)
    p2.coord = p.coord @ R.T
    e2 = StaticSolver(p2, ctx=ctx).solve()['energy']
    assert abs(e2 - out['energy']) <= 1e-10 * abs(out['energy'])
    if ff == 'fq':
        s = water_cluster(n_mol, ff, what='static', e0=1e-3, seed=11)
        o = StaticSolver(s, ctx=ctx).solve()
        P = o['polar']
        assert np.linalg.norm(P - P.T) <= 1e-10 * np.linalg.norm(P)
        qs = o['charges'].reshape(n_mol, 3, 3)
        assert np.max(np.abs(qs.sum(axis=1))) < 1e-10 * max(1.0, np.max(np.abs(qs)))
        s.coord = s.coord @ R.T
        P2 = StaticSolver(s, ctx=ctx).solve()['polar']
        # the tensor rotates with the cluster: R P R^T
        assert np.linalg.norm(P2 - R @ P @ R.T) <= 1e-9 * np.linalg.norm(P)


def test_refusals(ctx):
    import ctypes as C
    lib = ctx.lib
    # FQFMu static polarizability: the reference stops with "not yet implemented"
    p = water_cluster(4, 'fqfmu', what='static', e0=1e-3)
    polar = np.zeros(9)
    d = p.desc()
    st = lib.plx_static_solve(ctx.h, C.byref(d), 1, None, None, _lib.ptr(polar))
    assert st == 8 and 'not yet implemented' in lib.plx_last_error(ctx.h).decode()
    # molecules whose constraint rows, indexed as the reference does, run past the atoms
    p = water_cluster(3, 'fq')
    p.apm = np.array([1, 4, 4], dtype=np.int32)
    d = p.desc()
    assert lib.plx_static_solve(ctx.h, C.byref(d), 0, None, None, None) == 1
    assert 'run past the atoms' in lib.plx_last_error(ctx.h).decode()
    # the reference has no iterative static solve
    p = water_cluster(3, 'fq')
    p.method = 'iterative'
    with pytest.raises(ValueError, match='Iterative not implemented'):
        StaticSolver(p, ctx=ctx).solve()


def test_budget_is_enforced():
    c = Context(0, hbm_budget=64 << 20)
    try:
        p = water_cluster(1500, 'fq')          # 6000 unknowns: a 288 MB matrix
        with pytest.raises(_lib.PlxError) as e:
            StaticSolver(p, ctx=c).solve()
        assert e.value.code == 4
        assert c.bytes_in_use == 0
    finally:
        c.close()
