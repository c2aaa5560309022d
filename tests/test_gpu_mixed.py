"""Tensor-core (tcgen05) contraction and the mixed-precision refinement solve.

Tolerances:
  * BF16x3 contraction against the FP64 contraction: relative 5e-5 per column
    (operands carry ~16 significant bits, FP32 accumulation);
    single BF16 product: relative 1e-2
  * mixed-precision refined solve: sigma_abs within 1e-6 (relative) of the
    oracle's FP64 LU, the accuracy bar of the mixed path
  * FP64 refined solve: sigma_abs within 1e-10 of the oracle's LU
"""
import numpy as np
import pytest

from oracle import keywords, model, solve as osolve
from plasmonx_b200 import configs
from plasmonx_b200.inputs import Problem
from plasmonx_b200.solver import Context, Solver

pytestmark = pytest.mark.gpu


@pytest.fixture(scope='module')
def ctx():
    c = Context(0)
    yield c
    c.close()


def _ag(radius=10.0, n_freq=4, **kw):
    p0 = configs.ag_sphere(radius=radius, n_freq=n_freq, method='iterative', tolerance=1e-9, **kw)
    text = p0.to_keyword_text()
    return Problem.from_keyword_text(text), model.System.from_keywords(keywords.read_keyword_text(text))


@pytest.mark.parametrize('count', [1, 2, 7, 64, 402])
def test_tensor_core_contraction_accuracy(ctx, count):
    p, _ = _ag(radius=10.0, n_freq=1)
    rng = np.random.default_rng(count)
    X = rng.standard_normal((count, p.n_var))
    with Solver(p, ctx=ctx, store_t=True) as sv:
        ref = sv.contract(X, 'fp64')
        s3 = sv.contract(X, 'bf16x3')
        s1 = sv.contract(X, 'bf16')
    e3 = np.linalg.norm(s3 - ref, axis=1) / np.linalg.norm(ref, axis=1)
    e1 = np.linalg.norm(s1 - ref, axis=1) / np.linalg.norm(ref, axis=1)
    assert e3.max() < 5e-5, e3.max()
    assert e1.max() < 1e-2, e1.max()


def test_contraction_unaligned_size(ctx):
    """n_var not a multiple of the 64-wide k tile nor of the 128-row tile."""
    p, _ = _ag(radius=7.0, n_freq=1)
    assert p.n_var % 64 and p.n_var % 128
    rng = np.random.default_rng(5)
    X = rng.standard_normal((6, p.n_var))
    with Solver(p, ctx=ctx, store_t=True) as sv:
        ref = sv.contract(X, 'fp64')
        s3 = sv.contract(X, 'bf16x3')
    assert np.max(np.linalg.norm(s3 - ref, axis=1) / np.linalg.norm(ref, axis=1)) < 5e-5


@pytest.mark.parametrize('precision,bar', [('mixed_bf16x3', 1e-6), ('mixed_bf16', 1e-6), ('fp64_refined', 1e-10)])
def test_refined_solve_matches_lu(ctx, precision, bar):
    p, s = _ag(radius=10.0, n_freq=5)
    ref = osolve.solve(s, method='inversion')
    with Solver(p, ctx=ctx, store_t=True) as sv:
        b = sv.rhs(0, 1)
        out = sv.solve(mode='iterative', precision=precision, tol=1e-12 * np.linalg.norm(b[:, 0]))
    assert (out['status'] == 0).all(), out['status']
    sig, sref = out['results'][:, 9], ref['results'][:, 9]
    assert np.max(np.abs(sig - sref) / np.abs(sref)) < bar


def _bowtie(edge=24.0, thickness=10.0, n_freq=4):
    p0 = configs.agau_bowtie(edge=edge, thickness=thickness, gap=6.0, n_freq=n_freq, method='iterative on the fly',
                             tolerance=1e-9, polarization='x')
    text = p0.to_keyword_text()
    return Problem.from_keyword_text(text), model.System.from_keywords(keywords.read_keyword_text(text))


def test_generated_split_matches_stored_t(ctx):
    """Without a stored T (on-the-fly geometry) the tensor-core operand is generated
    from the pair formulas; its contraction agrees with the FP64 product of the
    stored T like the stored split does (relative 5e-5)."""
    p, _ = _ag(radius=10.0, n_freq=1)
    rng = np.random.default_rng(3)
    X = rng.standard_normal((9, p.n_var))
    with Solver(p, ctx=ctx, store_t=True) as sv:
        ref = sv.contract(X, 'fp64')
    with Solver(p, ctx=ctx, store_t=False) as sv:
        s3 = sv.contract(X, 'bf16x3')
    assert np.max(np.linalg.norm(s3 - ref, axis=1) / np.linalg.norm(ref, axis=1)) < 5e-5


@pytest.mark.parametrize('case', ['ag_sphere', 'agau_bowtie'])
def test_mixed_on_the_fly_matches_lu(ctx, case):
    """Matrix-free mode with the mixed form: tensor-core inner solves on the generated
    split, FP64 residuals from the on-the-fly product; sigma_abs within 1e-6 of LU
    (one atom type and the two-type Ag-Au bow-tie, whose conductance rows depend on w)."""
    p, s = _ag(radius=10.0, n_freq=4) if case == 'ag_sphere' else _bowtie()
    ref = osolve.solve(s, method='inversion')
    with Solver(p, ctx=ctx, store_t=False) as sv:
        b = sv.rhs(0, 1)
        out = sv.solve(mode='iterative on the fly', precision='mixed_bf16x3', pol_mask=1,
                       tol=1e-12 * np.linalg.norm(b[:, 0]))
    assert (out['status'] == 0).all(), out['status']
    sig, sref = out['results'][:, 9], ref['results'][:, 9]
    assert np.max(np.abs(sig - sref) / np.abs(sref)) < 1e-6


@pytest.mark.parametrize('count', [3, 40])
def test_on_the_fly_fp64_contraction_matches_stored(ctx, count):
    """The matrix-free FP64 product (pair kernel for few columns, tiled product with
    T generated per slab for many) against the stored T: relative 1e-12."""
    p, _ = _ag(radius=10.0, n_freq=1)
    rng = np.random.default_rng(count)
    X = rng.standard_normal((count, p.n_var))
    with Solver(p, ctx=ctx, store_t=True) as sv:
        ref = sv.contract(X, 'fp64')
    with Solver(p, ctx=ctx, store_t=False) as sv:
        otf = sv.contract(X, 'fp64_otf')
    assert np.max(np.linalg.norm(otf - ref, axis=1) / np.linalg.norm(ref, axis=1)) < 1e-12


def test_mixed_alloy_on_memory_matches_lu(ctx):
    """Stored-T alloy: the folded operand carries 1/2 (K + K^T) and the interface rows,
    the w-dependent remainder is the interface correction; sigma_abs within 1e-6 of LU."""
    p, s = _bowtie()
    ref = osolve.solve(s, method='inversion')
    with Solver(p, ctx=ctx, store_t=True) as sv:
        b = sv.rhs(0, 1)
        out = sv.solve(mode='iterative', precision='mixed_bf16x3', pol_mask=1, tol=1e-12 * np.linalg.norm(b[:, 0]))
    assert (out['status'] == 0).all(), out['status']
    sig, sref = out['results'][:, 9], ref['results'][:, 9]
    assert np.max(np.abs(sig - sref) / np.abs(sref)) < 1e-6
