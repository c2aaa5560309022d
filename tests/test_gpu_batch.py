"""Continuous batching (plx_batch_*) and the grouped multi-geometry launch.

  * a request added while another is in flight gets the same results as its
    grid solved alone by plx_solve: mixed BF16x3 within 1e-6 (relative, per
    result column scaled by its largest value), FP64 refined within 1e-10;
  * two geometries stepped together (plx_batch_step_group) give the same
    results as each stepped alone (1e-6), with fewer tensor-core contraction
    launches than the two alone: every inner Arnoldi step of both is one launch;
  * misuse is refused with PLX_ERR_ARG: a repeated tag, plx_set_frequencies on a
    geometry whose batch is open, taking a request still being solved.
"""
import numpy as np
import pytest

from plasmonx_b200 import _lib, configs
from plasmonx_b200 import materials as M
from plasmonx_b200.solver import Batch, Context, Solver

pytestmark = pytest.mark.gpu


@pytest.fixture(scope='module')
def ctx():
    c = Context(0)
    yield c
    c.close()


def _grid(p, lo, hi, nf):
    f0, f1 = p.freqs[0], p.freqs[-1]
    freqs = np.linspace(f0 + lo * (f1 - f0), f0 + hi * (f1 - f0), nf)
    names = {'Ag': 'silver etchegoin', 'Au': 'gold etchegoin'}
    aw = None if p.alpha_w is None else np.array([M.fitted(names[t], freqs, 'polar') for t in p.type_names])
    return freqs, aw


def _alone(sv, freqs, aw, precision, tol):
    sv.set_frequencies(freqs, aw)
    out = sv.solve(precision=precision, pol_mask=1, tol=tol)
    assert (out['status'] == 0).all(), out['status']
    return out['results']


def _close(a, b, bar):
    scale = np.abs(b).max(axis=0) + 1e-300
    return np.max(np.abs(a - b) / scale) < bar


@pytest.mark.parametrize('precision,bar', [('mixed_bf16x3', 1e-6), ('fp64_refined', 1e-10)])
def test_request_joining_in_flight_matches_alone(ctx, precision, bar):
    p = configs.ag_sphere(radius=10.0, n_freq=8, method='iterative')
    tol = 1e-12 * np.sqrt(p.n_var)
    ga, gb = _grid(p, 0.0, 1.0, 6), _grid(p, 0.3, 0.9, 4)
    with Solver(p, ctx=ctx) as sv:
        ref_a = _alone(sv, *ga, precision, tol)
        ref_b = _alone(sv, *gb, precision, tol)
        b = Batch(sv, precision=precision)
        try:
            b.add(0, *ga, pol_mask=1, tol=tol)
            b.step()
            b.add(1, *gb, pol_mask=1, tol=tol)           # joins while request 0 is in flight
            got = {}
            for _ in range(200):
                if not b.active:
                    break
                b.step()
                while (t := b.poll()) is not None:
                    got[t] = b.take(t)
            while (t := b.poll()) is not None:
                got[t] = b.take(t)
            assert set(got) == {0, 1}
            for t, ref in ((0, ref_a), (1, ref_b)):
                assert (got[t]['status'] == 0).all()
                assert _close(got[t]['results'], ref, bar)
        finally:
            b.close()
        # the geometry takes a frequency table again once the batch is closed
        assert _close(_alone(sv, *ga, precision, tol), ref_a, 1e-12)


def test_grouped_step_over_two_geometries(ctx):
    pa = configs.ag_sphere(radius=10.0, n_freq=6, method='iterative')
    pb = configs.particle('Au', 'rod', 7.0, length=20.0, n_freq=5, method='iterative')
    ta, tb = 1e-12 * np.sqrt(pa.n_var), 1e-12 * np.sqrt(pb.n_var)

    def run(batches_and_requests, grouped):
        for b, tag, g, tol in batches_and_requests:
            b.add(tag, *g, pol_mask=1, tol=tol)
        batches = [x[0] for x in batches_and_requests]
        out = {}
        for _ in range(200):
            if not any(b.active for b in batches):
                break
            if grouped:
                Batch.step_group(batches)
            else:
                for b in batches:
                    if b.active:
                        b.step()
            for b in batches:
                while (t := b.poll()) is not None:
                    out[t] = b.take(t)
        return out

    with Solver(pa, ctx=ctx) as sa, Solver(pb, ctx=ctx) as sb:
        ga, gb = (pa.freqs, pa.alpha_w), (pb.freqs, pb.alpha_w)
        res = {}
        for grouped in (False, True):
            ba, bb = Batch(sa), Batch(sb)
            try:
                ctx.profile(True)
                res[grouped] = run([(ba, 0, ga, ta), (bb, 1, gb, tb)], grouped)
                res[grouped]['tc'] = ctx.profile_read(0)['launches']
                ctx.profile(False)
            finally:
                ba.close()
                bb.close()
        for t in (0, 1):
            assert (res[True][t]['status'] == 0).all()
            assert _close(res[True][t]['results'], res[False][t]['results'], 1e-6)
        assert res[True]['tc'] < res[False]['tc']


def test_batch_misuse_is_refused(ctx):
    p = configs.ag_sphere(radius=8.0, n_freq=3, method='iterative')
    with Solver(p, ctx=ctx) as sv:
        b = Batch(sv)
        try:
            b.add(3, p.freqs, p.alpha_w, pol_mask=1, tol=1e-9)
            with pytest.raises(_lib.PlxError) as e:
                b.add(3, p.freqs, p.alpha_w, pol_mask=1, tol=1e-9)
            assert e.value.code == 1
            with pytest.raises(_lib.PlxError) as e:
                sv.set_frequencies(p.freqs, p.alpha_w)
            assert e.value.code == 1
            with pytest.raises(_lib.PlxError) as e:
                b.take(3)
            assert e.value.code == 1
        finally:
            b.close()
