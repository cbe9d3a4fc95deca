"""ctypes binding of libbsofi_b200_fp32.so, the single-precision variant
(include/bsofi_b200_fp32.h): the reference's names with float arrays.

As with the double library there is no fallback: loading fails loudly when
the shared library has not been built.  The two libraries export the same
names, so each is loaded into its own ctypes namespace (RTLD_LOCAL).
"""
import ctypes
import os

import numpy as np

from ._lib import declared_symbols

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libbsofi_b200_fp32.so")
HEADER = os.path.join(os.path.dirname(HERE), "include", "bsofi_b200_fp32.h")

_ip = ctypes.POINTER(ctypes.c_int)
_fp = ctypes.POINTER(ctypes.c_float)
_dp = ctypes.POINTER(ctypes.c_double)
_vp = ctypes.c_void_p
_i = ctypes.c_int

_HOST = [_i, _i, _fp, _i, _fp, _fp, _i, _ip]
_SIGS = {
    "hybridxinith_": (_i, [_ip] * 4),
    "hybridxbsofilworkh_": (_i, [_ip] * 4),
    "hybridxbsoftrih_": (_i, [_ip, _ip, _ip, _fp, _ip, _fp, _fp, _ip, _ip]),
    "hybridxbsoih_": (_i, [_ip, _ip, _ip, _fp, _ip, _fp, _fp, _ip, _ip]),
    "hybridxfinalizeh_": (_i, [_ip]),
    "fgetwalltime_": (None, [_dp]),
    "felapsed_": (ctypes.c_double, [_dp, _dp]),
    "lapackXbsofiLWork": (_i, [_i] * 3),
    "lapackXbsof": (_i, _HOST),
    "lapackXbstri": (_i, [_i, _i, _fp, _i, _ip]),
    "lapackXbsoi_ormqr": (_i, _HOST),
    "lapackXbsoi_orgqr": (_i, _HOST),
    "hybridXbsofiLWork": (_i, [_i] * 4),
    "hybridXbsoftri": (_i, [_i, _i, _i, _fp, _i, _fp, _fp, _i, _fp, _i, _ip]),
    "hybridXbsoi": (_i, [_i, _i, _i, _fp, _i, _fp, _fp, _i, _fp, _i, _ip]),
    "hybridxbsofilwork_": (_i, [_ip] * 4),
    "hybridxbsoftri_": (_i, [_ip, _ip, _fp, _ip, _fp, _fp, _ip, _fp, _ip, _ip]),
    "hybridxbsoi_": (_i, [_ip, _ip, _fp, _ip, _fp, _fp, _ip, _fp, _ip, _ip]),
    "lapackxbsofilwork_": (_i, [_ip] * 3),
    "lapackxbsof_": (_i, [_ip, _ip, _fp, _ip, _fp, _fp, _ip, _ip]),
    "lapackxbstri_": (_i, [_ip, _ip, _fp, _ip, _ip]),
    "lapackxbsoi_ormqr_": (_i, [_ip, _ip, _fp, _ip, _fp, _fp, _ip, _ip]),
    "lapackxbsoi_orgqr_": (_i, [_ip, _ip, _fp, _ip, _fp, _fp, _ip, _ip]),
    "gpuXbsof": (_i, [_i, _i, _vp, _i, _fp, _fp, _i, _vp, _ip]),
    "gpuXbstri_rseq": (_i, [_i, _i, _vp, _i, _vp, _i, _ip]),
    "gpuXbstri_rbatched": (_i, [_i, _i, _vp, _i, _vp, _i, _ip]),
    "gpuXbsoi_ormqr": (_i, [_i, _i, _vp, _i, _fp, _fp, _i, _vp, _vp, _i, _ip]),
    "gpuXbsoi_orgqr": (_i, [_i, _i, _vp, _i, _fp, _fp, _i, _vp, _vp, _i, _ip]),
    "gpuXbsoi_batched": (_i, [_i, _i, _vp, _i, _fp, _fp, _i, _vp, _vp, _i, _ip]),
    "bsofi_fp32_last_launches": (ctypes.c_longlong, []),
}

_lib = None


def declared():
    """Function names declared in include/bsofi_b200_fp32.h."""
    return declared_symbols(HEADER)


def load():
    """Load the single-precision library (once).  Raises if it is missing."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError("libbsofi_b200_fp32.so is not built (python -m bsofi_b200.build); "
                               "the BSOF/I path has no fallback")
        lib = ctypes.CDLL(LIB_PATH, mode=ctypes.RTLD_LOCAL)
        for name, (res, args) in _SIGS.items():
            f = getattr(lib, name)
            f.restype = res
            f.argtypes = args
        _lib = lib
    return _lib


def _ref(v):
    return ctypes.byref(ctypes.c_int(int(v)))


def _check_host(A, lda):
    if not (isinstance(A, np.ndarray) and A.dtype == np.float32 and A.flags.f_contiguous):
        raise TypeError("A must be a Fortran-ordered float32 numpy array")
    if A.shape[0] != lda:
        raise ValueError("A.shape[0] must equal lda")


class Handle:
    """hybridxinith_ / hybridxfinalizeh_ of the single-precision library
    (src/bsofi_callback.c:101-168 with scalar_t = float)."""

    def __init__(self, n, L, lda=None):
        self.n, self.L = int(n), int(L)
        self.lda = int(lda) if lda is not None else self.n * self.L
        self.words = np.zeros(10, dtype=np.int32)
        rc = load().hybridxinith_(self.words.ctypes.data_as(_ip), _ref(self.n), _ref(self.L),
                                  _ref(self.lda))
        if rc != 0:
            raise RuntimeError("hybridxinith_ failed (%d)" % rc)

    @property
    def ptr(self):
        return self.words.ctypes.data_as(_ip)

    def lwork(self):
        return load().hybridxbsofilworkh_(self.ptr, _ref(self.n), _ref(self.L), _ref(self.lda))

    def _call(self, fname, A, tau, work, lwork):
        _check_host(A, self.lda)
        if work is None:
            work = np.zeros(max(1, self.lwork()), dtype=np.float32)
        lw = len(work) if lwork is None else lwork
        info = ctypes.c_int(0)
        getattr(load(), fname)(self.ptr, _ref(self.n), _ref(self.L), A.ctypes.data_as(_fp),
                               _ref(self.lda), tau.ctypes.data_as(_fp), work.ctypes.data_as(_fp),
                               _ref(lw), ctypes.byref(info))
        return info.value

    def bsoftri(self, A, tau, work=None, lwork=None):
        """hybridxbsoftrih_ in place on A (Fortran-ordered float32); returns info."""
        return self._call("hybridxbsoftrih_", A, tau, work, lwork)

    def bsoi(self, A, tau, work=None, lwork=None):
        return self._call("hybridxbsoih_", A, tau, work, lwork)

    def close(self):
        if self.words is not None:
            load().hybridxfinalizeh_(self.ptr)
            self.words = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def invert(M, n, L):
    """M^{-1} in single precision through the handle API (XbsoftriH +
    XbsoiH).  Returns (X, A_after_bsoftri, tau, info), all float32."""
    A = np.asfortranarray(np.array(M, dtype=np.float32, copy=True))
    tau = np.zeros(n * L, dtype=np.float32)
    with Handle(n, L) as h:
        info = h.bsoftri(A, tau)
        state = A.copy(order="F")
        if info != 0:
            return None, state, tau, info
        info = h.bsoi(A, tau)
    return A, state, tau, info


def last_launches():
    return load().bsofi_fp32_last_launches()
