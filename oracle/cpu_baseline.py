"""ctypes front of oracle/pairs.c, the threaded C restatement of the reference's
on-the-fly matrix-vector product (test infrastructure / timed CPU baseline).

``CpuOperator(system).matvec(i_freq, x)`` returns A(w_i) x computed the way the
reference's on-the-fly GMRES forms it (src/matrix/matrix_module.f90:727-1125 and
new_gmres_diagonal_shift); ``system`` is an ``oracle.model.System``.
"""
import ctypes as C
import os
import subprocess

import numpy as np

from . import model

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, '_ref', 'libplxref.so')

_dp = C.POINTER(C.c_double)


class _Sys(C.Structure):
    _fields_ = [('n_atoms', C.c_int), ('n_types', C.c_int), ('fmu', C.c_int), ('hetero', C.c_int),
                ('coord', _dp), ('type', C.POINTER(C.c_int)), ('rq', _dp), ('rmu', _dp), ('eta', _dp),
                ('aij', _dp), ('fd', _dp), ('fs', _dp), ('r0', _dp), ('dq', _dp), ('dmu', _dp), ('wt', _dp)]


def load():
    if not os.path.exists(LIB):
        subprocess.run(['make', '-s', '-C', HERE], check=True)
    lib = C.CDLL(LIB)
    lib.plxref_matvec.argtypes = [C.POINTER(_Sys), _dp, _dp, C.c_int]
    lib.plxref_matvec.restype = C.c_int
    lib.plxref_max_threads.restype = C.c_int
    return lib


def _p(a):
    return a.ctypes.data_as(_dp)


class CpuOperator:
    def __init__(self, s, n_threads=0):
        self.s = s
        self.lib = load()
        self.n_threads = n_threads or self.lib.plxref_max_threads()
        nt = len(s.type_names)
        self.coord = np.ascontiguousarray(s.coord)
        self.type = np.ascontiguousarray(s.types, dtype=np.int32)
        self.rq, self.rmu, self.eta, self.aij = (np.ascontiguousarray(v, dtype=np.float64)
                                                 for v in (s.rq, s.rmu, s.eta, s.a_ij))
        self.fd = np.asfortranarray(s.fermi_d).ravel(order='F')
        self.fs = np.asfortranarray(s.fermi_s).ravel(order='F')
        r0 = np.zeros((nt, nt))
        for a in range(nt):
            za = s.znum[s.types == a][0]
            for b in range(nt):
                zb = s.znum[s.types == b][0]
                r0[a, b] = model.nearest_distance(int(za), int(zb))
        self.r0 = np.asfortranarray(r0).ravel(order='F')

    def matvec(self, i_freq, x):
        s = self.s
        omega = s.freqs[i_freq]
        nt = len(s.type_names)
        dq = np.zeros(nt, dtype=np.complex128)
        for t in range(nt):
            dq[t] = -(omega * (-omega * s.tau[t] - 1j) / (2.0 * s.density[t] * s.tau[t]))
        dmu = model.z_mu(s, i_freq).astype(np.complex128) if s.model == 'wfqfmu' else np.zeros(1, np.complex128)
        wt = model.drude_w(s, omega).astype(np.complex128)
        keep = [np.ascontiguousarray(v) for v in (dq, dmu, wt)]
        st = _Sys(s.n_atoms, nt, int(s.model == 'wfqfmu'), int(s.heterogeneous), _p(self.coord),
                  self.type.ctypes.data_as(C.POINTER(C.c_int)), _p(self.rq), _p(self.rmu), _p(self.eta),
                  _p(self.aij), _p(self.fd), _p(self.fs), _p(self.r0), _p(keep[0].view(np.float64)),
                  _p(keep[1].view(np.float64)), _p(keep[2].view(np.float64)))
        xin = np.ascontiguousarray(x, dtype=np.complex128)
        y = np.zeros(s.n_var, dtype=np.complex128)
        rc = self.lib.plxref_matvec(C.byref(st), _p(xin.view(np.float64)), _p(y.view(np.float64)),
                                    int(self.n_threads))
        if rc != 0:
            raise MemoryError('plxref_matvec failed')
        return y
