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

and the inner solve's relative tolerance (1e-3, 1e-4, 1e-5 around the best
basis): a looser inner solve costs more FP64 residuals, a tighter one more
inner steps.

``Tuner.settings(solver, key)`` runs a short sweep once per resident geometry
-- the candidate settings on a few frequencies spread over the grid, each timed
by the library's own CUDA events -- and caches the fastest (device time per
freq-solve) under the geometry's key; later requests on the same geometry reuse
it.  The sweep's records are kept for the report.
"""
import numpy as np

INNER_CANDIDATES = (64, 128, 256)
INNER_TOL_CANDIDATES = (1e-3, 1e-5)       # tried around the default 1e-4 for the best basis
BLOCK_CANDIDATES = (0, 64, 32, 16, 8)


class Tuner:
    def __init__(self, n_probe=6, inner_candidates=INNER_CANDIDATES, inner_tol_candidates=INNER_TOL_CANDIDATES):
        self.n_probe = int(n_probe)
        self.inner_candidates = tuple(inner_candidates)
        self.inner_tol_candidates = tuple(inner_tol_candidates)
        self.cache = {}
        self.records = {}

    def settings(self, solver, key, freqs, alpha_w=None, precision='mixed_bf16x3', mode=None, pol_mask=1,
                 tol=None, fits=None):
        """Tuned {'inner_krylov', 'freq_block'} for the geometry `key`.

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
        def trial(m, itol):
            out = solver.solve(mode=mode, precision=precision, pol_mask=pol_mask, tol=tol, inner_krylov=m,
                               inner_tol=itol)
            ok = 'error' not in out and bool(np.all(out['status'] == 0))
            per = out['device_ms'] / max(1, len(idx)) if ok else float('inf')
            sweep.append({'inner_krylov': m, 'inner_tol': itol or 1e-4, 'ms_per_freq_solve': per, 'ok': ok})

        try:
            for m in self.inner_candidates:
                trial(min(m, int(solver.n_var)), 0.0)
            m_best = min(sweep, key=lambda r: (r['ms_per_freq_solve'], r['inner_krylov']))['inner_krylov']
            for itol in self.inner_tol_candidates:
                trial(m_best, itol)
        finally:
            solver.set_frequencies(freqs, alpha_w)
        best = min(sweep, key=lambda r: (r['ms_per_freq_solve'], r['inner_krylov']))
        good = np.isfinite(best['ms_per_freq_solve'])
        chosen = {'inner_krylov': best['inner_krylov'] if good else 64,
                  'inner_tol': best['inner_tol'] if good else 1e-4, 'freq_block': block}
        self.cache[key] = chosen
        self.records[key] = {'probe_freqs': [int(i) for i in idx], 'sweep': sweep, 'chosen': chosen}
        return chosen
