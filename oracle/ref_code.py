"""The reference's own kernel and operator code, compiled here (test
infrastructure only).

oracle/ref/Makefile builds fmm3d_mpi/kernel3d_mpi.cpp, fmm3d_mpi/matmgnt3d_mpi.cpp,
common/vecmatop.cpp and common/svdrep.cpp unchanged from the reference tree into
oracle/_ref/libkifmm_ref.so, with stand-in PETSc and FFTW headers and the BLAS
and FFTW arithmetic restated (oracle/ref/ref_shims.cpp).  LAPACK (dgesvd for the
pseudo-inverses, dgetrf/dgetri) comes from scipy's LAPACK, registered here at
load time.  The tests use it to pin the oracle's restatement -- kernel blocks,
surface grids, operator tables and one M2L interaction -- against the
reference's code.  The library is built where the reference tree is present
(build() in __graft_entry__, or the Makefile); available() tells whether it is.
"""
import ctypes
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "_ref", "libkifmm_ref.so")
REF_ROOT = "/root/reference"
_lib = None
_dp = ctypes.POINTER(ctypes.c_double)


def build():
    """Compile the library from the reference tree (where it exists)."""
    import subprocess
    if not os.path.isdir(REF_ROOT):
        return False
    subprocess.check_call(["make", "-s", "-C", os.path.join(_HERE, "ref"), "REF=" + REF_ROOT])
    return os.path.exists(LIB_PATH)


def available():
    return os.path.exists(LIB_PATH) or build()


def _capsule_ptr(capsule):
    get_name = ctypes.pythonapi.PyCapsule_GetName
    get_name.restype = ctypes.c_char_p
    get_name.argtypes = [ctypes.py_object]
    get_ptr = ctypes.pythonapi.PyCapsule_GetPointer
    get_ptr.restype = ctypes.c_void_p
    get_ptr.argtypes = [ctypes.py_object, ctypes.c_char_p]
    return get_ptr(capsule, get_name(capsule))


def lib():
    global _lib
    if _lib is None:
        if not available():
            raise RuntimeError("the reference's code is not built (no reference tree to build it from)")
        import scipy.linalg.cython_lapack as cl
        L = ctypes.CDLL(LIB_PATH)
        L.fmmg_ref_register_lapack.argtypes = [ctypes.c_char_p, ctypes.c_void_p]
        for name in ("dgesvd", "dgetrf", "dgetri"):
            assert L.fmmg_ref_register_lapack(name.encode(), _capsule_ptr(cl.__pyx_capi__[name])) == 0
        L.fmmg_ref_kernel_matrix.argtypes = [ctypes.c_int, _dp, ctypes.c_int, _dp, _dp, ctypes.c_int, _dp, _dp]
        L.fmmg_ref_sampos.argtypes = [ctypes.c_int, ctypes.c_double, _dp]
        L.fmmg_ref_regpos.argtypes = [ctypes.c_int, ctypes.c_double, _dp]
        L.fmmg_ref_operator.restype = ctypes.c_long
        L.fmmg_ref_operator.argtypes = [ctypes.c_int, _dp, ctypes.c_int, ctypes.c_int, ctypes.c_int, _dp]
        L.fmmg_ref_m2l.argtypes = [ctypes.c_int, _dp, ctypes.c_int, ctypes.c_int, ctypes.c_int, _dp, _dp]
        _lib = L
    return _lib


def _c(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def _d(a):
    return a.ctypes.data_as(_dp)


def dofs(kt):
    """(srcDOF, trgDOF) of kernel3d_mpi.cpp:40-104."""
    import oracle as O
    return O.src_dof(kt), O.trg_dof(kt)


def kernel_matrix(kt, src, nrm, trg, coefs=(1.0, 0.25)):
    """Kernel3d_MPI::buildKnlIntCtx, (nt*trgDOF) x (ns*srcDOF) column-major."""
    src, nrm, trg, cf = _c(src), _c(nrm), _c(trg), _c(coefs)
    sd, td = dofs(kt)
    out = np.zeros(trg.shape[0] * td * src.shape[0] * sd)
    assert lib().fmmg_ref_kernel_matrix(kt, _d(cf), src.shape[0], _d(src), _d(nrm), trg.shape[0], _d(trg),
                                        _d(out)) == 0
    return out.reshape(src.shape[0] * sd, trg.shape[0] * td).T


def sampos(np_, R):
    n = lib().fmmg_ref_sampos(np_, R, None)
    out = np.zeros(3 * n)
    lib().fmmg_ref_sampos(np_, R, _d(out))
    return out.reshape(n, 3)


def regpos(np_, R):
    n = lib().fmmg_ref_regpos(np_, R, None)
    out = np.zeros(3 * n)
    lib().fmmg_ref_regpos(np_, R, _d(out))
    return out.reshape(n, 3)


def operator(kt_mm, np_, which, idx=0, coefs=(1.0, 0.25)):
    """The table MatMgnt3d_MPI builds (level 0), flattened as the reference
    stores it; the index conventions of the oracle's operator()."""
    cf = _c(coefs)
    n = lib().fmmg_ref_operator(kt_mm, _d(cf), np_, which, idx, None)
    assert n > 0
    out = np.zeros(n)
    lib().fmmg_ref_operator(kt_mm, _d(cf), np_, which, idx, _d(out))
    return out


def m2l(kt_mm, np_, level, idx, den, coefs=(1.0, 0.25)):
    """One V-list interaction through plnDen2EffDen, UpwEqu2DwnChk_dgemv and
    effVal2PlnVal: the DC check values (from zero) of the UE density den."""
    cf, den = _c(coefs), _c(den).ravel()
    sd, td = dofs(kt_mm)
    n_dc = len(sampos(np_, 1.0))
    val = np.zeros(n_dc * td)
    assert lib().fmmg_ref_m2l(kt_mm, _d(cf), np_, level, idx, _d(den), _d(val)) == 0
    return val
