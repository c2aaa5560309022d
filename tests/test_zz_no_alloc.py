"""The allocation-free contraction entry point (plx_contract_noalloc).

Callers whose device memory belongs to another allocator, or that must not
allocate inside a timed loop, pass their own device buffers; the entry point
allocates nothing and uses a fixed device scratch array.  This file is
collected last so a failure here comes after every other test has run.
"""
import ctypes as C

import numpy as np
import pytest

from plasmonx_b200 import configs
from plasmonx_b200.solver import Context, Solver

pytestmark = pytest.mark.gpu


def test_noalloc_contraction_matches_allocating_entry_point():
    import torch
    p = configs.ag_sphere(radius=10.0, n_freq=1, method='iterative')
    ctx = Context(0)
    try:
        with Solver(p, ctx=ctx, store_t=True) as sv:
            rng = np.random.default_rng(11)
            for count in (6, 3):                 # two calls in a row, different shapes
                X = rng.standard_normal((count, sv.n_var))
                ref = sv.contract(X, 'fp64')
                dX = torch.from_numpy(X).to('cuda:0')
                dS = torch.full((count, sv.n_var), float('nan'), dtype=torch.float64, device='cuda:0')
                torch.cuda.synchronize()
                st = sv.lib.plx_contract_noalloc(sv.g, count, C.c_void_p(dX.data_ptr()), C.c_void_p(dS.data_ptr()))
                ctx.check(st)
                S = dS.cpu().numpy()
                err = np.linalg.norm(S - ref, axis=1) / np.linalg.norm(ref, axis=1)
                assert err.max() < 1e-12, err
            # sizes beyond the fixed scratch are refused with a clear error
            X = np.zeros((17, sv.n_var))
            dX = torch.zeros((17, sv.n_var), dtype=torch.float64, device='cuda:0')
            st = sv.lib.plx_contract_noalloc(sv.g, 17, C.c_void_p(dX.data_ptr()), C.c_void_p(dX.data_ptr()))
            assert st == 1 and b'1 to 16 columns' in sv.lib.plx_last_error(ctx.h)
    finally:
        ctx.close()


def test_noalloc_refuses_partials_beyond_the_scratch():
    """16 columns of the 7,844-unknown sphere need 20 k-chunks x 16 x 7,844 partial
    sums, more than the 2^21 doubles of the fixed scratch: refused with status 1 and
    the limit in the message; a call that fits still matches the allocating path."""
    import torch
    p = configs.ag_sphere(radius=20.0, n_freq=1, method='iterative')
    ctx = Context(0)
    try:
        with Solver(p, ctx=ctx, store_t=True) as sv:
            assert sv.n_var == 7844
            dX = torch.zeros((16, sv.n_var), dtype=torch.float64, device='cuda:0')
            dS = torch.zeros((16, sv.n_var), dtype=torch.float64, device='cuda:0')
            torch.cuda.synchronize()
            st = sv.lib.plx_contract_noalloc(sv.g, 16, C.c_void_p(dX.data_ptr()), C.c_void_p(dS.data_ptr()))
            assert st == 1 and b'fixed maximum' in sv.lib.plx_last_error(ctx.h)
            rng = np.random.default_rng(12)
            X = rng.standard_normal((6, sv.n_var))
            ref = sv.contract(X, 'fp64')
            dX = torch.from_numpy(X).to('cuda:0')
            dS = torch.full((6, sv.n_var), float('nan'), dtype=torch.float64, device='cuda:0')
            torch.cuda.synchronize()
            ctx.check(sv.lib.plx_contract_noalloc(sv.g, 6, C.c_void_p(dX.data_ptr()), C.c_void_p(dS.data_ptr())))
            S = dS.cpu().numpy()
            assert np.max(np.linalg.norm(S - ref, axis=1) / np.linalg.norm(ref, axis=1)) < 1e-12
    finally:
        ctx.close()
