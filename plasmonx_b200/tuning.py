"""Per-geometry autotuning of the mixed-precision spectrum solve.

The tensor-core refinement has two knobs whose best value depends on the
geometry, not on the hardware alone:

  inner_krylov  the inner GMRES basis per cycle (64, 128, 256): a short basis
                orthogonalises cheaply (one Gram-Schmidt pass up to 64 vectors)
                but restarts stagnate on gap-coupled alloys, where a long basis
                (re-orthogonalised) wins;
  freq_block    frequencies solved as one batch: every frequency of the grid
                (the widest tensor-core launches) unless the Krylov state of the
                whole grid does not fit the device budget, then blocks of 64,
                32, 16 or 8.

and, for the best basis, the inner solve's relative tolerance with the
tensor-core form: BF16x3 (three products, ~1e-5 operator error) at 1e-3, 1e-4
or 1e-5, or one BF16 product (half the operand bytes per launch, ~2e-3
operator error) at 1e-2 or 3e-2 -- a looser inner solve costs more FP64
residuals, a tighter one more inner steps, and the one-product operator pays
for its cheaper launches with more outer steps, which wins where the
refinement contracts fast (the silver sphere: 101 against 82 freq-solves/s)
and loses where it does not (the Ag-Au bow-tie: 20 against 42).

``Tuner.settings(solver, key)`` runs a short sweep once per resident geometry
(the basis lengths with the default form; every form at the best of them; the
basis lengths again with the best form)
-- the candidate settings on a few frequencies spread over the grid, each timed
by the library's own CUDA events -- and caches the fastest (device time per
freq-solve) under the geometry's key; later requests on the same geometry reuse
it.  The sweep's records are kept for the report.
"""
import numpy as np

INNER_CANDIDATES = (64, 128, 256)
# (tensor-core form, inner tolerance) tried for the best basis beside the default (BF16x3, 1e-4)
FORM_CANDIDATES = (('mixed_bf16x3', 1e-3), ('mixed_bf16x3', 1e-5), ('mixed_bf16', 1e-2), ('mixed_bf16', 3e-2))
BLOCK_CANDIDATES = (0, 64, 32, 16, 8)


class Tuner:
    def __init__(self, n_probe=6, inner_candidates=INNER_CANDIDATES, form_candidates=FORM_CANDIDATES):
        self.n_probe = int(n_probe)
        self.inner_candidates = tuple(inner_candidates)
        self.form_candidates = tuple(form_candidates)
        self.cache = {}
        self.records = {}

    def settings(self, solver, key, freqs, alpha_w=None, precision='mixed_bf16x3', mode=None, pol_mask=1,
                 tol=None, fits=None):
        """Tuned {'inner_krylov', 'inner_tol', 'precision', 'freq_block'} for the geometry `key`.

        solver  a Solver holding the geometry (its frequency table is restored)
        freqs   the request's grid; alpha_w its (n_types, F) table or None
        fits    optional callable(freq_block) -> bool: whether a block of that many
                frequencies fits the device budget (0 = the whole grid)
        """
        if key in self.cache:
            return self.cache[key]
        F = len(freqs)
        idx = np.unique(np.linspace(0, F - 1, min(self.n_probe, F)).round().astype(int))
        block = 0
        if fits is not None:
            block = next((b for b in BLOCK_CANDIDATES if (b == 0 or b < F) and fits(b)), 8)
        sweep = []
        solver.set_frequencies(np.asarray(freqs)[idx], None if alpha_w is None else np.asarray(alpha_w)[:, idx])
        def trial(m, itol, prec):
            out = solver.solve(mode=mode, precision=prec, pol_mask=pol_mask, tol=tol, inner_krylov=m,
                               inner_tol=itol)
            ok = 'error' not in out and bool(np.all(out['status'] == 0))
            per = out['device_ms'] / max(1, len(idx)) if ok else float('inf')
            sweep.append({'inner_krylov': m, 'inner_tol': itol or 1e-4, 'precision': prec,
                          'ms_per_freq_solve': per, 'ok': ok})

        # from BF16x3 every form is tried; a one-product request keeps its form
        forms = [(f, t) for f, t in self.form_candidates if precision == 'mixed_bf16x3' or f == precision]
        try:
            for m in self.inner_candidates:
                trial(min(m, int(solver.n_var)), 0.0, precision)
            m_best = min(sweep, key=lambda r: (r['ms_per_freq_solve'], r['inner_krylov']))['inner_krylov']
            for prec_, itol in forms:
                trial(m_best, itol, prec_)
            # the basis again for the best form, when that is not the one swept first
            top = min(sweep, key=lambda r: (r['ms_per_freq_solve'], r['inner_krylov']))
            if top['precision'] != precision or top['inner_tol'] != 1e-4:
                for m in self.inner_candidates:
                    m = min(m, int(solver.n_var))
                    if m != top['inner_krylov']:
                        trial(m, top['inner_tol'], top['precision'])
        finally:
            solver.set_frequencies(freqs, alpha_w)
        best = min(sweep, key=lambda r: (r['ms_per_freq_solve'], r['inner_krylov']))
        good = np.isfinite(best['ms_per_freq_solve'])
        chosen = {'inner_krylov': best['inner_krylov'] if good else 64,
                  'inner_tol': best['inner_tol'] if good else 1e-4,
                  'precision': best['precision'] if good else precision, 'freq_block': block}
        self.cache[key] = chosen
        self.records[key] = {'probe_freqs': [int(i) for i in idx], 'sweep': sweep, 'chosen': chosen}
        return chosen
