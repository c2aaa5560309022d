"""Failure paths, made on the host (nothing here faults, traps or hangs the GPU):
  * a non-finite permittivity at one frequency of a batched spectrum: that
    frequency reports PLX_ERR_NAN, the others solve as in a clean batch, in the
    plain FP64 GMRES and in the mixed form;
  * a non-finite right-hand side handed to the reference-shaped GMRES;
  * a geometry larger than the context's HBM budget is refused with
    PLX_ERR_BUDGET and leaves nothing allocated;
  * the tensor-core kernel's bounded waits: with the wait limit set to one poll
    every pipeline wait runs out; the kernel lets its copies and products finish,
    frees its tensor memory and returns, and the call reports PLX_ERR_CUDA;
  * after each failure the same context solves a clean problem.
"""
import numpy as np
import pytest

from plasmonx_b200 import _lib, configs
from plasmonx_b200.solver import Context, Solver

pytestmark = pytest.mark.gpu


@pytest.fixture(scope='module')
def ctx():
    c = Context(0)
    yield c
    c.close()


def _ag(n_freq=4):
    return configs.particle('Ag', 'sphere', 8.0, n_freq=n_freq, method='iterative', tolerance=1e-10)


@pytest.mark.parametrize('precision', ['fp64', 'mixed_bf16x3'])
def test_nan_frequency_is_isolated(ctx, precision):
    p = _ag()
    bad = p.alpha_w.copy()
    bad[:, 1] = np.nan
    with Solver(p, ctx=ctx) as sv:
        clean = sv.solve(precision=precision)
        sv.set_frequencies(p.freqs, bad)
        out = sv.solve(precision=precision)
        assert out['status'][1] == 6                  # PLX_ERR_NAN
        assert isinstance(out.get('error'), _lib.PlxError) and out['error'].code == 6
        ok = [0, 2, 3]
        assert np.all(out['status'][ok] == 0)
        rel = np.abs(out['results'][ok] - clean['results'][ok]) / np.abs(clean['results'][ok]).max(axis=0)
        assert rel.max() < (1e-12 if precision == 'fp64' else 1e-6)
        # the context and geometry stay usable
        sv.set_frequencies(p.freqs, p.alpha_w)
        again = sv.solve(precision=precision)
        assert np.all(again['status'] == 0)


def test_nan_right_hand_side_in_reference_gmres(ctx):
    p = _ag(2)
    with Solver(p, ctx=ctx) as sv:
        b = sv.rhs(0)[:, 0].copy()
        b[3] = np.nan
        with pytest.raises(_lib.PlxError):
            sv.gmres(0, b, p.tol, 200)
        x, steps, _ = sv.gmres(0, sv.rhs(0)[:, 0], p.tol, 200)
        assert np.all(np.isfinite(x)) and steps > 0


def test_budget_refusal_leaves_nothing_allocated():
    p = configs.particle('Ag', 'sphere', 16.0, n_freq=2, method='iterative')   # dense T of ~60 MB
    c = Context(0, hbm_budget=8 << 20)
    try:
        with pytest.raises(_lib.PlxError) as e:
            Solver(p, ctx=c)
        assert e.value.code == 4
        assert c.bytes_in_use == 0
        small = configs.particle('Na', 'sphere', 6.0, n_freq=2, method='iterative')
        with Solver(small, ctx=c) as sv:
            assert np.all(sv.solve()['status'] == 0)
    finally:
        c.close()


@pytest.mark.parametrize('how', ['bf16x3', 'bf16'])
def test_tensor_core_wait_limit_runs_out_cleanly(how):
    """A wait limit of one poll makes the tensor-core kernel's first pipeline wait
    give up (nothing faults: the loads it issued land, the products finish, the
    kernel returns); plx_contract reports PLX_ERR_CUDA with the timeout message.
    At the default limit the same context contracts correctly again."""
    p = configs.ag_sphere(radius=10.0, n_freq=1, method='iterative')
    c = Context(0)
    try:
        with Solver(p, ctx=c, store_t=True) as sv:
            rng = np.random.default_rng(21)
            X = rng.standard_normal((8, sv.n_var))
            ref = sv.contract(X, 'fp64')
            c.set_wait_limit(1)
            with pytest.raises(_lib.PlxError) as e:
                sv.contract(X, how)
            assert e.value.code == 2 and 'timed out' in str(e.value)
            c.set_wait_limit(0)
            for _ in range(2):
                S = sv.contract(X, how)
                err = np.linalg.norm(S - ref, axis=1) / np.linalg.norm(ref, axis=1)
                assert err.max() < (5e-5 if how == 'bf16x3' else 1e-2), err
    finally:
        c.close()
