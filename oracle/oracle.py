"""ctypes binding of the CPU oracle (test infrastructure only).

The oracle is a CPU FP64 restatement of the reference single-rank
``FMM3d_MPI::evaluate()`` (aashays/fmm-g).  Only tests/, the smoke check in
``__graft_entry__`` and bench.py's CPU-baseline leg use it, always as the
checker.  Parity against the reference itself is unpinned (no golden vectors
exist and the reference cannot be built); see kifmm_oracle.cpp.
"""
import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "liboracle.so")
_lib = None

_dp = ctypes.POINTER(ctypes.c_double)
_ip = ctypes.POINTER(ctypes.c_int)
_lp = ctypes.POINTER(ctypes.c_long)

STAGE_UP, STAGE_U, STAGE_V, STAGE_W, STAGE_X, STAGE_DOWN = 1, 2, 4, 8, 16, 32
STAGE_ALL = 63


def build():
    subprocess.check_call(["make", "-s", "-C", _HERE])


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        L = ctypes.CDLL(_LIB_PATH)
        L.orc_create.restype = ctypes.c_void_p
        L.orc_create.argtypes = [ctypes.c_int, _dp, ctypes.c_int, ctypes.c_int, ctypes.c_int, _dp,
                                 ctypes.c_int, ctypes.c_int]
        L.orc_destroy.argtypes = [ctypes.c_void_p]
        L.orc_setup.argtypes = [ctypes.c_void_p, ctypes.c_long, _dp, _dp, ctypes.c_long, _dp]
        L.orc_evaluate.argtypes = [ctypes.c_void_p, _dp, _dp, ctypes.c_int]
        L.orc_set_gemv_order.argtypes = [ctypes.c_void_p, ctypes.c_int]
        L.orc_m2l_single.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, _dp, _dp]
        L.orc_dense.argtypes = [ctypes.c_int, _dp, ctypes.c_long, _dp, _dp, _dp, ctypes.c_long, _dp,
                                _dp, ctypes.c_int]
        L.orc_num_nodes.restype = ctypes.c_long
        L.orc_num_nodes.argtypes = [ctypes.c_void_p]
        L.orc_nodes.argtypes = [ctypes.c_void_p, _ip]
        L.orc_lists.restype = ctypes.c_long
        L.orc_lists.argtypes = [ctypes.c_void_p, ctypes.c_int, _lp, _ip]
        L.orc_perms.argtypes = [ctypes.c_void_p, _lp, _lp]
        L.orc_operator.restype = ctypes.c_long
        L.orc_operator.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, _dp, _dp]
        L.orc_sizes.argtypes = [ctypes.c_void_p, _ip]
        L.orc_kernel_matrix.argtypes = [ctypes.c_int, _dp, ctypes.c_int, _dp, _dp, ctypes.c_int, _dp, _dp]
        L.orc_pinv.argtypes = [ctypes.c_int, ctypes.c_int, _dp, ctypes.c_double, _dp]
        L.orc_rfft3.argtypes = [ctypes.c_int, ctypes.c_int, _dp, _dp]
        L.orc_irfft3.argtypes = [ctypes.c_int, ctypes.c_int, _dp, _dp]
        L.orc_sampos.argtypes = [ctypes.c_int, ctypes.c_double, _dp]
        L.orc_regpos.argtypes = [ctypes.c_int, ctypes.c_double, _dp]
        for f in ("orc_src_dof", "orc_trg_dof", "orc_mm_type"):
            getattr(L, f).argtypes = [ctypes.c_int]
        _lib = L
    return _lib


def _d(a):
    return a.ctypes.data_as(_dp)


def _c(a, dtype=np.float64):
    return np.ascontiguousarray(a, dtype=dtype)


def src_dof(kt):
    return lib().orc_src_dof(kt)


def trg_dof(kt):
    return lib().orc_trg_dof(kt)


def mm_type(kt):
    return lib().orc_mm_type(kt)


def kernel_matrix(kt, src, nrm, trg, coefs=(1.0, 0.25)):
    """Column-major dense kernel matrix, returned as a (nt*td, ns*sd) array."""
    src, nrm, trg = _c(src), _c(nrm), _c(trg)
    ns, nt = src.shape[0], trg.shape[0]
    sd, td = src_dof(kt), trg_dof(kt)
    out = np.zeros(nt * td * ns * sd)
    cf = _c(coefs)
    lib().orc_kernel_matrix(kt, _d(cf), ns, _d(src), _d(nrm), nt, _d(trg), _d(out))
    return out.reshape(ns * sd, nt * td).T.copy()


def pinv(A, eps):
    A = np.asfortranarray(A, dtype=np.float64)
    m, n = A.shape
    R = np.zeros((n, m), order="F")
    lib().orc_pinv(m, n, A.ctypes.data_as(_dp), eps, R.ctypes.data_as(_dp))
    return np.array(R)


def rfft3(x, n, howmany):
    """x: real array of n^3*howmany (x index fastest, components interleaved)."""
    x = _c(x).ravel()
    out = np.zeros(n * n * (n // 2 + 1) * howmany * 2)
    lib().orc_rfft3(n, howmany, _d(x), _d(out))
    return out.view(np.complex128)


def irfft3(X, n, howmany):
    X = np.ascontiguousarray(X, dtype=np.complex128).ravel()
    out = np.zeros(n * n * n * howmany)
    lib().orc_irfft3(n, howmany, X.ctypes.data_as(_dp), _d(out))
    return out


def sampos(np_, R):
    n = lib().orc_sampos(np_, R, None)
    out = np.zeros(3 * n)
    lib().orc_sampos(np_, R, _d(out))
    return out.reshape(n, 3)


def regpos(np_, R):
    n = lib().orc_regpos(np_, R, None)
    out = np.zeros(3 * n)
    lib().orc_regpos(np_, R, _d(out))
    return out.reshape(n, 3)


def dense(kt, src, nrm, den, pos, coefs=(1.0, 0.25), nthreads=1):
    """FP64 dense direct sum at pos over all sources (the reference check())."""
    src, nrm, den, pos = _c(src), _c(nrm), _c(den), _c(pos)
    td = trg_dof(kt)
    out = np.zeros(pos.shape[0] * td)
    cf = _c(coefs)
    lib().orc_dense(kt, _d(cf), src.shape[0], _d(src), _d(nrm), _d(den), pos.shape[0], _d(pos), _d(out),
                    nthreads)
    return out


class Oracle:
    """CPU FP64 KIFMM restating FMM3d_MPI setup()/evaluate() on one rank."""

    def __init__(self, kernel_type, np_=6, pts_max=64, max_level=30, coefs=(1.0, 0.25),
                 ctr=(0.5, 0.5, 0.5), root_level=1, nthreads=1):
        self.kt = kernel_type
        self.coefs = _c(coefs)
        c = _c(ctr)
        self.h = lib().orc_create(kernel_type, _d(self.coefs), np_, pts_max, max_level, _d(c), root_level,
                                  nthreads)
        if not self.h:
            raise ValueError("oracle: invalid options")
        self.sd, self.td = src_dof(kernel_type), trg_dof(kernel_type)
        self.ns = self.nt = 0

    def __del__(self):
        if getattr(self, "h", None):
            lib().orc_destroy(self.h)
            self.h = None

    def setup(self, src, nrm, trg):
        self._src, self._nrm, self._trg = _c(src), _c(nrm), _c(trg)
        self.ns, self.nt = self._src.shape[0], self._trg.shape[0]
        lib().orc_setup(self.h, self.ns, _d(self._src), _d(self._nrm), self.nt, _d(self._trg))

    def evaluate(self, den, stages=STAGE_ALL):
        den = _c(den).ravel()
        assert den.size == self.ns * self.sd
        out = np.zeros(self.nt * self.td)
        lib().orc_evaluate(self.h, _d(den), _d(out), stages)
        return out

    GEMV_UP_C2E, GEMV_M2M, GEMV_DN_C2E, GEMV_L2L = 1, 2, 4, 8

    def m2l_single(self, level, tid, den):
        """One V-list interaction at `level` through the oracle's M2L helpers
        (embed and r2c, Hadamard with translation tid, c2r and gather): the DC
        check values of the UE density den."""
        den = _c(den).ravel()
        s = self.sizes()
        out = np.zeros(s["DC"] * trg_dof(mm_type(self.kt)))
        assert lib().orc_m2l_single(self.h, level, tid, _d(den), _d(out)) == 0
        return out

    def set_gemv_order(self, reverse):
        """Sum the columns of the selected operator GEMVs in reverse: a mask of
        GEMV_UP_C2E, GEMV_M2M, GEMV_DN_C2E and GEMV_L2L (True = all of them);
        0 / False keeps the reference BLAS order for all (the default)."""
        lib().orc_set_gemv_order(self.h, 15 if reverse is True else int(reverse))

    def sizes(self):
        out = np.zeros(6, dtype=np.int32)
        lib().orc_sizes(self.h, out.ctypes.data_as(_ip))
        return dict(zip(("UE", "UC", "DE", "DC", "reg", "eff"), out.tolist()))

    def nodes(self):
        nn = lib().orc_num_nodes(self.h)
        out = np.zeros((nn, 11), dtype=np.int32)
        lib().orc_nodes(self.h, out.ctypes.data_as(_ip))
        return out

    def lists(self, which):
        nn = lib().orc_num_nodes(self.h)
        ptr = np.zeros(nn + 1, dtype=np.int64)
        tot = lib().orc_lists(self.h, which, ptr.ctypes.data_as(_lp), None)
        idx = np.zeros(max(tot, 1), dtype=np.int32)
        lib().orc_lists(self.h, which, ptr.ctypes.data_as(_lp), idx.ctypes.data_as(_ip))
        return ptr, idx[:tot]

    def perms(self):
        sp = np.zeros(max(self.ns, 1), dtype=np.int64)
        tp = np.zeros(max(self.nt, 1), dtype=np.int64)
        lib().orc_perms(self.h, sp.ctypes.data_as(_lp), tp.ctypes.data_as(_lp))
        return sp[: self.ns], tp[: self.nt]

    def operator(self, which, idx=0):
        n = lib().orc_operator(self.h, which, idx, None, None)
        out = np.zeros(n)
        lib().orc_operator(self.h, which, idx, _d(out), None)
        return out

    def set_operator(self, which, idx, values):
        v = _c(values).ravel()
        n = lib().orc_operator(self.h, which, idx, None, None)
        assert v.size == n
        lib().orc_operator(self.h, which, idx, None, _d(v))
