"""ctypes binding of libplasmonx_b200.so (C ABI in include/plasmonx_b200.h).

The library is built in-tree by ``plasmonx_b200.build``; importing this module
never falls back to anything else: a missing or unloadable library raises.
"""
import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, 'libplasmonx_b200.so')

PLX_OK = 0
STATUS = {0: 'PLX_OK', 1: 'PLX_ERR_ARG', 2: 'PLX_ERR_CUDA', 3: 'PLX_ERR_NOMEM', 4: 'PLX_ERR_BUDGET',
          5: 'PLX_ERR_NOT_CONVERGED', 6: 'PLX_ERR_NAN', 7: 'PLX_ERR_SINGULAR', 8: 'PLX_ERR_UNSUPPORTED'}
MODEL = {'wfq': 0, 'wfqfmu': 1, 'bem_dpcm': 2, 'bem_ief': 3}
MODE = {'inversion': 0, 'iterative': 1, 'iterative on the fly': 2}
PRECISION = {'fp64': 0, 'mixed_bf16x3': 1, 'fp64_refined': 2, 'mixed_bf16': 3}
CONTRACT = {'fp64': 0, 'fp64_otf': 1, 'bf16x3': 2, 'bf16': 3}

EXPORTS = ['plx_ctx_create', 'plx_ctx_destroy', 'plx_last_error', 'plx_ctx_bytes_in_use',
           'plx_geometry_create', 'plx_bem_create', 'plx_geometry_destroy', 'plx_geometry_n_var', 'plx_geometry_k_nnz',
           'plx_set_frequencies', 'plx_matvec', 'plx_rhs', 'plx_gmres_solver', 'plx_complex_inversion',
           'plx_solve', 'plx_last_solve_ms', 'plx_last_solve_launches', 'plx_profile_enable',
           'plx_profile_read', 'plx_contract', 'plx_contract_noalloc', 'plx_field_at_points',
           'plx_static_n_var', 'plx_static_solve', 'plx_principal_axes', 'plx_neighbour_counts',
           'plx_bem_field_at_points', 'plx_ctx_launches', 'plx_set_wait_limit', 'plx_batch_open', 'plx_batch_add',
           'plx_batch_step', 'plx_batch_step_group', 'plx_batch_poll', 'plx_batch_take', 'plx_batch_active',
           'plx_batch_close']
STATIC_FF = {'fq': 0, 'fqfmu': 1}
KERNEL = {'coulomb': 0, 'ohno': 1, 'gaussian': 2}
STATIC_WHAT = {'energy': 0, 'static': 1}

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int32)


class GeometryDesc(C.Structure):
    _fields_ = [('model', C.c_int32), ('n_atoms', C.c_int32), ('n_types', C.c_int32),
                ('rhs_potential', C.c_int32), ('coord', _dp), ('atom_type', _ip), ('neighbours', _ip),
                ('n_neighbours', _ip), ('eta', _dp), ('r_q', _dp), ('r_mu', _dp), ('tau', _dp),
                ('density', _dp), ('a_ij', _dp), ('fermi_d', _dp), ('fermi_s', _dp), ('r0', _dp),
                ('e0', C.c_double)]


class BemDesc(C.Structure):
    _fields_ = [('variant', C.c_int32), ('n_tess', C.c_int32), ('accurate', C.c_int32), ('triangles', _dp),
                ('normal_factor', C.c_double), ('sphere_radius', C.c_double), ('eps_solvent', C.c_double),
                ('e0', C.c_double)]


class StaticDesc(C.Structure):
    _fields_ = [('forcefield', C.c_int32), ('kernel', C.c_int32), ('n_atoms', C.c_int32), ('n_types', C.c_int32),
                ('n_mol', C.c_int32), ('rhs_potential', C.c_int32), ('coord', _dp), ('atom_type', _ip),
                ('atoms_per_molecule', _ip), ('chi', _dp), ('eta', _dp), ('alpha', _dp), ('r_q', _dp),
                ('r_mu', _dp), ('e0', C.c_double), ('factorization', C.c_int32)]


class SolveDesc(C.Structure):
    _fields_ = [('mode', C.c_int32), ('precision', C.c_int32), ('pol_mask', C.c_int32),
                ('max_krylov', C.c_int32), ('tol', C.c_double), ('freq_block', C.c_int32),
                ('record_trace', C.c_int32), ('inner_krylov', C.c_int32), ('inner_tol', C.c_double),
                ('max_outer', C.c_int32)]


class PlxError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__('%s: %s' % (STATUS.get(code, code), msg))
        self.code = code


_lib = None


def load():
    """Load the in-tree library (raises OSError when it is missing)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise OSError('libplasmonx_b200.so is not built; run `python -m plasmonx_b200.build`')
    lib = C.CDLL(LIB_PATH)
    vp = C.c_void_p
    lib.plx_ctx_create.restype = vp
    lib.plx_ctx_create.argtypes = [C.c_int32, C.c_uint64]
    lib.plx_ctx_destroy.argtypes = [vp]
    lib.plx_last_error.restype = C.c_char_p
    lib.plx_last_error.argtypes = [vp]
    lib.plx_ctx_bytes_in_use.restype = C.c_uint64
    lib.plx_ctx_bytes_in_use.argtypes = [vp]
    lib.plx_ctx_launches.restype = C.c_int64
    lib.plx_ctx_launches.argtypes = [vp]
    lib.plx_geometry_create.argtypes = [vp, C.POINTER(GeometryDesc), C.c_int32, C.POINTER(vp)]
    lib.plx_bem_create.argtypes = [vp, C.POINTER(BemDesc), C.POINTER(vp)]
    lib.plx_geometry_destroy.argtypes = [vp]
    lib.plx_geometry_n_var.restype = C.c_int64
    lib.plx_geometry_n_var.argtypes = [vp]
    lib.plx_geometry_k_nnz.restype = C.c_int64
    lib.plx_geometry_k_nnz.argtypes = [vp]
    lib.plx_set_frequencies.argtypes = [vp, C.c_int32, _dp, _dp]
    lib.plx_matvec.argtypes = [vp, C.c_int32, C.c_int32, _dp, _dp]
    lib.plx_rhs.argtypes = [vp, C.c_int32, C.c_int32, _dp]
    lib.plx_gmres_solver.argtypes = [vp, C.c_int32, _dp, C.c_int32, C.c_double, C.c_int32, C.c_int32,
                                     _ip, _dp]
    lib.plx_complex_inversion.argtypes = [vp, C.c_int32, _dp]
    lib.plx_solve.argtypes = [vp, C.POINTER(SolveDesc), _dp, _dp, _dp, _ip, _ip, _dp]
    lib.plx_last_solve_ms.restype = C.c_double
    lib.plx_last_solve_ms.argtypes = [vp]
    lib.plx_last_solve_launches.restype = C.c_int64
    lib.plx_last_solve_launches.argtypes = [vp]
    lib.plx_contract.argtypes = [vp, C.c_int32, _dp, _dp, C.c_int32]
    lib.plx_contract_noalloc.argtypes = [vp, C.c_int32, C.c_void_p, C.c_void_p]
    lib.plx_field_at_points.argtypes = [vp, C.c_int32, _dp, C.c_int32, _dp, _dp, _dp]
    lib.plx_neighbour_counts.argtypes = [vp, C.c_int32, C.c_int32, _dp, _ip, _ip, _dp, _ip, _ip]
    lib.plx_bem_field_at_points.argtypes = [vp, C.c_int32, _dp, _dp, C.c_double, C.c_int32, C.c_int32, _dp, _dp]
    lib.plx_static_n_var.restype = C.c_int64
    lib.plx_static_n_var.argtypes = [C.POINTER(StaticDesc)]
    lib.plx_static_solve.argtypes = [vp, C.POINTER(StaticDesc), C.c_int32, _dp, _dp, _dp]
    lib.plx_principal_axes.argtypes = [C.c_int32, _ip, _dp, _dp, _dp]
    lib.plx_profile_enable.argtypes = [vp, C.c_int32]
    lib.plx_profile_read.argtypes = [vp, C.c_int32, _dp, C.POINTER(C.c_int64), _dp, _dp]
    lib.plx_set_wait_limit.argtypes = [vp, C.c_uint32]
    lib.plx_batch_open.argtypes = [vp, C.POINTER(SolveDesc), C.POINTER(vp)]
    lib.plx_batch_add.argtypes = [vp, C.c_int64, C.c_int32, _dp, _dp, C.c_int32, C.c_double]
    lib.plx_batch_step.argtypes = [vp, _ip]
    lib.plx_batch_step_group.argtypes = [C.POINTER(vp), C.c_int32, _ip]
    lib.plx_batch_poll.argtypes = [vp, C.POINTER(C.c_int64)]
    lib.plx_batch_take.argtypes = [vp, C.c_int64, _dp, _dp, _ip, _ip]
    lib.plx_batch_active.argtypes = [vp]
    lib.plx_batch_active.restype = C.c_int32
    lib.plx_batch_close.argtypes = [vp]
    lib.plx_batch_close.restype = None
    _lib = lib
    return lib


def ptr(a, kind=_dp):
    """Pointer to a contiguous numpy array (or None)."""
    if a is None:
        return None
    return a.ctypes.data_as(kind)
