"""Host-side driver of the B200 solve: the per-frequency loop of the reference
(src/solvers/algorithm_module.f90:150-465) over the C ABI.

    prob = Problem.from_keyword_file('input.kw')   # or BemProblem.from_keyword_file (bem.py)
    with Solver(prob) as s:
        out = s.solve()            # mode taken from the input ('inversion' / 'iterative' /
                                   # 'iterative on the fly'), FP64
        out['results']             # (n_freq, 20): target_%results(i, 1:20)

Errors from the library raise ``PlxError``; a GMRES column that runs out of
Krylov dimension is reported as the reference reports it
("GMRES not converged and restart GMRES NYI.").
"""
import ctypes as C

import numpy as np

from . import _lib
from ._lib import PlxError, ptr


class Context:
    """One CUDA device context of the library (plx_ctx)."""

    def __init__(self, device=0, hbm_budget=0):
        self.lib = _lib.load()
        self.h = self.lib.plx_ctx_create(int(device), int(hbm_budget))
        if not self.h:
            raise MemoryError('plx_ctx_create failed')
        err = self.lib.plx_last_error(self.h).decode()
        if err:
            self.close()
            raise PlxError(2, err)

    def check(self, status):
        if status != _lib.PLX_OK:
            raise PlxError(status, self.lib.plx_last_error(self.h).decode())

    def profile(self, on=True):
        self.check(self.lib.plx_profile_enable(self.h, int(bool(on))))

    PROFILE_CATEGORIES = ('tc_contraction', 'fp64_contraction', 'orthogonalisation', 'operator_rows',
                          'least_squares', 'static_assembly', 'static_factor', 'points', 'neighbours')

    def profile_read(self, category=0):
        ms, fl, by = C.c_double(), C.c_double(), C.c_double()
        n = C.c_int64()
        self.check(self.lib.plx_profile_read(self.h, int(category), C.byref(ms), C.byref(n), C.byref(fl),
                                             C.byref(by)))
        return {'ms': ms.value, 'launches': n.value, 'flops': fl.value, 'bytes': by.value}

    def profile_breakdown(self):
        return {name: self.profile_read(k) for k, name in enumerate(self.PROFILE_CATEGORIES)}

    def set_wait_limit(self, polls=0):
        """Polls after which a pipeline wait in the tensor-core kernels gives up
        (0: the default); a wait that runs out makes the call fail cleanly."""
        self.check(self.lib.plx_set_wait_limit(self.h, int(polls)))

    @property
    def bytes_in_use(self):
        return int(self.lib.plx_ctx_bytes_in_use(self.h))

    @property
    def launches(self):
        """Kernels the library has launched on this context (its own kernels)."""
        return int(self.lib.plx_ctx_launches(self.h))

    def close(self):
        if self.h:
            self.lib.plx_ctx_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Solver:
    """A geometry resident on the device plus its frequency grid."""

    def __init__(self, prob, ctx=None, device=0, store_t=None):
        self.prob = prob
        self.own_ctx = ctx is None
        self.ctx = ctx or Context(device)
        self.lib = self.ctx.lib
        if getattr(prob, 'triangles', None) is not None:
            self._init_bem(prob)
            return
        if store_t is None:
            store_t = prob.method != 'iterative on the fly'
        nt = len(prob.type_names)
        # neighbour counts on the device, from the input Angstrom coordinates
        r0 = np.asfortranarray(prob.r0).ravel(order='F')
        atom_type = np.ascontiguousarray(prob.atom_types, dtype=np.int32)
        nb = np.zeros((prob.n_atoms, nt), dtype=np.int32)                       # (N,nt) row-major == nt x N
        nnb = np.zeros(prob.n_atoms, dtype=np.int32)
        ang = np.ascontiguousarray(prob.coord_ang, dtype=np.float64)
        tz = prob.type_z
        self.ctx.check(self.lib.plx_neighbour_counts(self.ctx.h, prob.n_atoms, nt, ptr(ang), ptr(atom_type, _lib._ip),
                                                     ptr(tz, _lib._ip), ptr(r0), ptr(nb, _lib._ip),
                                                     ptr(nnb, _lib._ip)))
        self.neighbours, self.n_neighbours = nb.T, nnb
        self._keep = dict(
            coord=np.ascontiguousarray(prob.coord, dtype=np.float64),            # (N,3) row-major == 3xN col-major
            atom_type=atom_type, neighbours=nb, n_neighbours=nnb,
            eta=np.ascontiguousarray(prob.eta), r_q=np.ascontiguousarray(prob.r_q),
            r_mu=np.ascontiguousarray(prob.r_mu), tau=np.ascontiguousarray(prob.tau),
            density=np.ascontiguousarray(prob.density), a_ij=np.ascontiguousarray(prob.a_ij),
            fermi_d=np.asfortranarray(prob.fermi_d).ravel(order='F'),
            fermi_s=np.asfortranarray(prob.fermi_s).ravel(order='F'),
            r0=r0)
        k = self._keep
        d = _lib.GeometryDesc(
            _lib.MODEL[prob.model], prob.n_atoms, nt, 1 if prob.rhs_form == 'potential' else 0,
            ptr(k['coord']), ptr(k['atom_type'], _lib._ip), ptr(k['neighbours'], _lib._ip),
            ptr(k['n_neighbours'], _lib._ip), ptr(k['eta']), ptr(k['r_q']), ptr(k['r_mu']), ptr(k['tau']),
            ptr(k['density']), ptr(k['a_ij']), ptr(k['fermi_d']), ptr(k['fermi_s']), ptr(k['r0']), prob.e0)
        h = C.c_void_p()
        self.ctx.check(self.lib.plx_geometry_create(self.ctx.h, C.byref(d), int(bool(store_t)), C.byref(h)))
        self.g = h
        self.n_var = int(self.lib.plx_geometry_n_var(self.g))
        self.set_frequencies(prob.freqs, prob.alpha_w)

    def _init_bem(self, prob):
        self._keep = dict(tri=np.ascontiguousarray(prob.triangles, dtype=np.float64))
        d = _lib.BemDesc(_lib.MODEL[prob.model], prob.n_tess, int(prob.accurate), ptr(self._keep['tri']),
                         prob.normal_factor, prob.sphere_radius, prob.eps_solvent, prob.e0)
        h = C.c_void_p()
        self.ctx.check(self.lib.plx_bem_create(self.ctx.h, C.byref(d), C.byref(h)))
        self.g = h
        self.n_var = int(self.lib.plx_geometry_n_var(self.g))
        self.set_frequencies(prob.freqs, prob.alpha_w)

    def set_frequencies(self, freqs, alpha_w=None):
        self.freqs = np.ascontiguousarray(freqs, dtype=np.float64)
        aw = None
        if alpha_w is not None:
            aw = np.ascontiguousarray(np.asarray(alpha_w, dtype=np.complex128).T).view(np.float64)
        self._aw = aw
        self.ctx.check(self.lib.plx_set_frequencies(self.g, len(self.freqs), ptr(self.freqs), ptr(aw)))

    @property
    def k_nnz(self):
        return int(self.lib.plx_geometry_k_nnz(self.g))

    # ---- reference-shaped entry points -------------------------------------
    def matvec(self, i_freq, x, on_the_fly=False):
        x = np.ascontiguousarray(x, dtype=np.complex128)
        y = np.zeros(self.n_var, dtype=np.complex128)
        self.ctx.check(self.lib.plx_matvec(self.g, i_freq, int(on_the_fly), ptr(x.view(np.float64)),
                                           ptr(y.view(np.float64))))
        return y

    def rhs(self, i_freq, pol_mask=7):
        b = np.zeros((3, self.n_var), dtype=np.complex128)
        self.ctx.check(self.lib.plx_rhs(self.g, i_freq, pol_mask, ptr(b.view(np.float64))))
        return b.T.copy()

    def gmres(self, i_freq, b, tol, restart, on_the_fly=False, max_iter=1):
        x = np.ascontiguousarray(b, dtype=np.complex128).copy()
        steps = C.c_int32(0)
        trace = np.zeros(max(1, min(restart, self.n_var)))
        st = self.lib.plx_gmres_solver(self.g, i_freq, ptr(x.view(np.float64)), int(on_the_fly), float(tol),
                                       int(max_iter), int(restart), C.byref(steps), ptr(trace))
        self.ctx.check(st)
        return x, steps.value, trace[:steps.value]

    def complex_inversion(self, i_freq, variables_w):
        v = np.asfortranarray(np.asarray(variables_w, dtype=np.complex128).reshape(self.n_var, 3))
        buf = np.ascontiguousarray(v.T)
        self.ctx.check(self.lib.plx_complex_inversion(self.g, i_freq, ptr(buf.view(np.float64))))
        return buf.T.copy()

    def field_at_points(self, i_pol, x, points):
        """Induced field (P, 3) and density (P,) of solution x (n_var complex, polarisation
        i_pol) at points (P, 3) in bohr; the external field E0 along i_pol is included."""
        x = np.ascontiguousarray(x, dtype=np.complex128)
        pts = np.ascontiguousarray(points, dtype=np.float64).reshape(-1, 3)
        P = pts.shape[0]
        field = np.zeros((P, 3), dtype=np.complex128)
        dens = np.zeros(P, dtype=np.complex128)
        self.ctx.check(self.lib.plx_field_at_points(self.g, int(i_pol), ptr(x.view(np.float64)), P, ptr(pts),
                                                    ptr(field.view(np.float64)), ptr(dens.view(np.float64))))
        return field, dens

    # ---- the spectrum -------------------------------------------------------
    def contract(self, X, how='fp64'):
        """S = T X for real columns X (count x n_var)."""
        X = np.ascontiguousarray(X, dtype=np.float64).reshape(-1, self.n_var)
        S = np.zeros_like(X)
        self.ctx.check(self.lib.plx_contract(self.g, X.shape[0], ptr(X), ptr(S), _lib.CONTRACT[how]))
        return S

    def solve(self, mode=None, precision='fp64', pol_mask=None, tol=None, max_krylov=None,
              freq_block=0, want_x=False, trace=False, inner_krylov=0, inner_tol=0.0, max_outer=0):
        p = self.prob
        mode = mode or p.method
        pol_mask = p.pol_mask if pol_mask is None else pol_mask
        F = len(self.freqs)
        m = int(max_krylov or p.gmres_dim or 1000)
        desc = _lib.SolveDesc(_lib.MODE[mode], _lib.PRECISION[precision], pol_mask, m,
                              float(p.tol if tol is None else tol), int(freq_block), int(bool(trace)),
                              int(inner_krylov), float(inner_tol), int(max_outer))
        x = np.zeros((F, 3, self.n_var), dtype=np.complex128) if want_x else None
        polar = np.zeros((F, 3, 3), dtype=np.complex128)
        res = np.zeros((F, 20))
        status = np.zeros(F, dtype=np.int32)
        steps = np.zeros((F, 3), dtype=np.int32)
        tr = np.zeros((F, 3, min(m, self.n_var))) if trace else None
        st = self.lib.plx_solve(self.g, C.byref(desc), ptr(None if x is None else x.view(np.float64)),
                                ptr(polar.view(np.float64)), ptr(res), ptr(status, _lib._ip),
                                ptr(steps, _lib._ip), ptr(tr))
        out = {'polar': polar.transpose(0, 2, 1).copy(), 'results': res, 'status': status, 'steps': steps,
               'device_ms': float(self.lib.plx_last_solve_ms(self.g)),
               'launches': int(self.lib.plx_last_solve_launches(self.g))}
        if x is not None:
            out['x'] = x.transpose(0, 2, 1).copy()     # (F, n_var, 3) like variables_w
        if tr is not None:
            out['trace'] = tr
        if st != _lib.PLX_OK:
            out['error'] = PlxError(st, self.lib.plx_last_error(self.ctx.h).decode())
        return out

    def close(self):
        if getattr(self, 'g', None):
            self.lib.plx_geometry_destroy(self.g)
            self.g = None
        if self.own_ctx and self.ctx:
            self.ctx.close()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()


class Batch:
    """Continuous batching on one resident geometry (plx_batch): requests --
    frequency grids with their own tolerance -- join while others are being
    solved, each step() is one outer refinement step of every active column,
    and finished requests are taken out with their results.

        b = Batch(solver, precision='mixed_bf16x3')
        b.add(7, freqs, alpha_w, pol_mask=1, tol=1e-9)
        while b.active:
            b.step()                      # or Batch.step_group([b, b2, ...])
            while (tag := b.poll()) is not None:
                out = b.take(tag)         # 'results' (F, 20), 'polar', 'status', 'steps'

    While a batch is open it owns the solver's frequency table."""

    def __init__(self, solver, mode=None, precision='mixed_bf16x3', inner_krylov=0, inner_tol=0.0, max_outer=0):
        self.solver = solver
        self.ctx = solver.ctx
        self.lib = solver.lib
        mode = mode or solver.prob.method
        if mode == 'inversion':
            mode = 'iterative'
        desc = _lib.SolveDesc(_lib.MODE[mode], _lib.PRECISION[precision], 1, 1, 0.0, 0, 0, int(inner_krylov),
                              float(inner_tol), int(max_outer))
        h = C.c_void_p()
        self.ctx.check(self.lib.plx_batch_open(solver.g, C.byref(desc), C.byref(h)))
        self.h = h
        self.mode, self.precision = mode, precision
        self.n_freq = {}
        self.last_step_ms = 0.0

    def add(self, tag, freqs, alpha_w=None, pol_mask=1, tol=1e-9):
        freqs = np.ascontiguousarray(freqs, dtype=np.float64)
        aw = None
        if alpha_w is not None:
            aw = np.ascontiguousarray(np.asarray(alpha_w, dtype=np.complex128).T).view(np.float64)
        self.ctx.check(self.lib.plx_batch_add(self.h, int(tag), len(freqs), ptr(freqs), ptr(aw), int(pol_mask),
                                              float(tol)))
        self.n_freq[int(tag)] = len(freqs)

    @property
    def active(self):
        return int(self.lib.plx_batch_active(self.h)) if self.h else 0

    def step(self):
        n = C.c_int32(0)
        self.ctx.check(self.lib.plx_batch_step(self.h, C.byref(n)))
        self.last_step_ms = float(self.lib.plx_last_solve_ms(self.solver.g))
        return n.value

    @staticmethod
    def step_group(batches):
        """One outer step of several batches (one per geometry, one context) whose
        inner Arnoldi steps share one grouped tensor-core launch each."""
        arr = (C.c_void_p * len(batches))(*[b.h for b in batches])
        n = C.c_int32(0)
        b0 = batches[0]
        b0.ctx.check(b0.lib.plx_batch_step_group(arr, len(batches), C.byref(n)))
        ms = float(b0.lib.plx_last_solve_ms(b0.solver.g))
        for b in batches:
            b.last_step_ms = ms
        return n.value

    def poll(self):
        """The tag of the earliest request whose columns have all finished, or None."""
        t = C.c_int64(-1)
        self.ctx.check(self.lib.plx_batch_poll(self.h, C.byref(t)))
        return None if t.value < 0 else int(t.value)

    def take(self, tag):
        F = self.n_freq[int(tag)]
        polar = np.zeros((F, 3, 3), dtype=np.complex128)
        res = np.zeros((F, 20))
        status = np.zeros(F, dtype=np.int32)
        steps = np.zeros((F, 3), dtype=np.int32)
        st = self.lib.plx_batch_take(self.h, int(tag), ptr(polar.view(np.float64)), ptr(res), ptr(status, _lib._ip),
                                     ptr(steps, _lib._ip))
        out = {'polar': polar.transpose(0, 2, 1).copy(), 'results': res, 'status': status, 'steps': steps}
        if st not in (_lib.PLX_OK, 5, 6):      # not converged / non-finite: reported per frequency
            self.ctx.check(st)
        del self.n_freq[int(tag)]
        return out

    def close(self):
        if getattr(self, 'h', None):
            self.lib.plx_batch_close(self.h)
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

