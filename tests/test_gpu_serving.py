"""The serving loop on the GPU: a seeded mix of wFQ, wFQFMu and BEM spectrum
requests arriving as a Poisson stream, solved by concurrent workers with
resident geometries and batching; every request's results are compared with
the same request solved alone.

Tolerances: plain FP64 requests must agree exactly (the FP64 products sum every
column in a batch-independent order); mixed-precision requests within 1e-6
relative (the accuracy of the mixed form), on every one of the 20 result columns
scaled by the column's largest value."""
import copy

import numpy as np
import pytest

from plasmonx_b200 import configs
from plasmonx_b200.bem import bem_surface
from plasmonx_b200.serving import Server, ServeRequest, run_mix

pytestmark = pytest.mark.gpu


def _mix(precision):
    na = configs.particle('Na', 'sphere', 12.0, n_freq=6, method='iterative', tolerance=1e-9, polarization='x')
    ag = configs.particle('Ag', 'rod', 8.0, length=24.0, n_freq=5, method='iterative', tolerance=1e-9,
                          polarization='x')
    bem = bem_surface(320, n_freq=4, method='iterative', tolerance=1e-9, polarization='x')
    for k, p in enumerate((na, ag, bem)):
        p.geometry_key = ('g', k)
    reqs = []
    arrivals = np.cumsum(np.random.default_rng(11).exponential(0.01, size=7))
    for i, (p, lo, hi, nf) in enumerate([(na, 0, 1, 6), (ag, 0, 1, 5), (bem, 0, 1, 4), (na, 0.2, 1, 4),
                                         (ag, 0.3, 1, 3), (bem, 0.5, 1, 3), (na, 0.5, 1, 5)]):
        q = copy.copy(p)
        f0, f1 = p.freqs[0], p.freqs[-1]
        q.freqs = np.linspace(f0 + lo * (f1 - f0), f0 + hi * (f1 - f0), nf)
        if hasattr(q, 'eps'):
            from plasmonx_b200.bem import drude_lorentz
            q.eps = drude_lorentz(q.freqs)
        elif q.alpha_w is not None:
            from plasmonx_b200 import materials as M
            q.alpha_w = np.array([M.fitted('silver etchegoin', q.freqs, 'polar')])
        # the bench's accuracy setting: 1e-12 sqrt(n) (atomistic); BEM right-hand
        # sides scale with E0, so 1e-10 sqrt(n) E0 there
        tol = (1e-10 * q.e0 if hasattr(q, 'eps') else 1e-12) * np.sqrt(q.n_var)
        reqs.append(ServeRequest(i, q, arrival=float(arrivals[i]), precision=precision, pol_mask=1, tol=tol))
    return reqs


def _fresh(r):
    return ServeRequest(r.id, r.problem, precision=r.precision, pol_mask=r.pol_mask, tol=r.tol)


@pytest.mark.parametrize('precision', ['fp64', 'mixed_bf16x3'])
def test_each_result_is_the_same_alone_and_in_the_mix(precision):
    reqs = _mix(precision)
    with Server(workers=2) as srv:
        stats = run_mix(srv, reqs)
    assert stats['errors'] == 0, [r.error for r in reqs if r.error is not None]
    assert stats['p50_ms'] > 0 and stats['p99_ms'] >= stats['p50_ms']
    assert max(r.batch_size for r in reqs) >= 1
    for r in reqs:
        with Server(workers=1) as alone_srv:
            a = alone_srv.submit(_fresh(r))
            assert a.done.wait(600)
        assert a.error is None, a.error
        assert (r.result['status'] == 0).all() and (a.result['status'] == 0).all()
        mine, ref = r.result['results'], a.result['results']
        if precision == 'fp64' and a.mode == r.mode:
            np.testing.assert_array_equal(mine, ref)
        else:
            scale = np.abs(ref).max(axis=0) + 1e-300
            assert np.max(np.abs(mine - ref) / scale) < 1e-6
