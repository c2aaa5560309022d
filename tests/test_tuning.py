"""The per-geometry autotuner (plasmonx_b200.tuning) against a stand-in solver
whose device time is a known function of the settings."""
import numpy as np

from plasmonx_b200.tuning import FORM_CANDIDATES, INNER_CANDIDATES, Tuner


class TimedSolver:
    """solve() reports a device time per frequency from a table; one setting fails."""

    def __init__(self, cost, n_var=5000, failing=()):
        self.cost, self.n_var, self.failing = cost, n_var, set(failing)
        self.freqs = None
        self.calls = []

    def set_frequencies(self, freqs, alpha_w=None):
        self.freqs = np.asarray(freqs)

    def solve(self, mode=None, precision=None, pol_mask=1, tol=None, inner_krylov=0, inner_tol=0.0):
        key = (precision, inner_krylov, inner_tol or 1e-4)
        self.calls.append((key, len(self.freqs)))
        F = len(self.freqs)
        status = np.full(F, 5 if key in self.failing else 0, np.int32)
        return {'device_ms': self.cost(*key) * F, 'status': status}


def test_tuner_picks_the_fastest_setting_and_restores_the_grid():
    def cost(prec, m, itol):
        base = {64: 10.0, 128: 8.0, 256: 9.0}[m]
        return base * (0.7 if (prec, itol) == ('mixed_bf16', 1e-2) else 1.0)
    sv = TimedSolver(cost)
    freqs = np.linspace(3.0, 4.5, 50)
    t = Tuner(n_probe=6)
    got = t.settings(sv, 'g', freqs)
    assert got['inner_krylov'] == 128 and got['precision'] == 'mixed_bf16' and got['inner_tol'] == 1e-2
    np.testing.assert_array_equal(sv.freqs, freqs)            # the request's grid is back
    # the basis sweep, every form at the best basis, the other bases with the best form,
    # each on the probe frequencies
    n_trials = len(INNER_CANDIDATES) + len(FORM_CANDIDATES) + len(INNER_CANDIDATES) - 1
    assert len(sv.calls) == n_trials
    assert all(n == 6 for _, n in sv.calls)
    # cached per geometry key
    assert t.settings(sv, 'g', freqs) is got and len(sv.calls) == n_trials


def test_tuner_resweeps_the_basis_for_the_best_form():
    # BF16x3 is fastest at 128, the one-product form at 64
    def cost(prec, m, itol):
        if prec == 'mixed_bf16':
            return {64: 5.0, 128: 7.0, 256: 9.0}[m] if itol == 3e-2 else 20.0
        return {64: 10.0, 128: 8.0, 256: 9.0}[m]
    sv = TimedSolver(cost)
    got = Tuner(n_probe=6).settings(sv, 'r', np.linspace(3.0, 4.5, 50))
    assert (got['precision'], got['inner_krylov'], got['inner_tol']) == ('mixed_bf16', 64, 3e-2)


def test_tuner_skips_settings_that_do_not_converge():
    def cost(prec, m, itol):
        return 1.0 if prec == 'mixed_bf16' else 5.0 + m / 64.0
    sv = TimedSolver(cost, failing=[('mixed_bf16', 64, 1e-2), ('mixed_bf16', 64, 3e-2)])
    got = Tuner(n_probe=4).settings(sv, 'h', np.linspace(1, 2, 10))
    assert got['precision'] == 'mixed_bf16x3' and got['inner_krylov'] == 64
    rec = [r for r in Tuner().records.values()]
    assert rec == []                                          # records live on the instance


def test_one_product_request_keeps_its_form():
    sv = TimedSolver(lambda prec, m, itol: 1.0)
    Tuner(n_probe=3).settings(sv, 'k', np.linspace(1, 2, 10), precision='mixed_bf16')
    assert {k[0] for k, _ in sv.calls} == {'mixed_bf16'}
