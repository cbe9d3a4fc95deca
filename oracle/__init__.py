"""CPU checkers for the BSOF/I CUDA path.  TEST INFRASTRUCTURE ONLY.

Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline
and reference legs may import this package.  The product library never routes
through it.

Two checkers, same calling convention (column-major float64, ``lda = n*L``):

* ``ref_*``  -- the reference's own CPU path, compiled unmodified from the
  reference tree into ``oracle/_ref/libbsofi_ref.so`` by ``oracle/Makefile``
  (OpenBLAS 0.3.15).  Called through the reference's Fortran handle API
  ``hybridxinith_ / hybridxbsoftrih_ / hybridxbsoih_`` (src/bsofi_callback.c:
  101-157), which without CUDA is lapackXbsof + lapackXbstri +
  lapackXbsoi_ormqr (src/bsofi_cpu.c:86-248).
* ``port_*`` -- the plain-C restatement in ``oracle/bsofi_oracle.c``.
* ``ref32_*`` -- the reference's single-precision variant (the same sources
  with -D__SINGLE_PREC__, scalar_t = float; config.h:132-136), the checker for
  libbsofi_b200_fp32.so.  Column-major float32.
"""
import ctypes
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_REF_SO = os.path.join(_HERE, "_ref", "libbsofi_ref.so")
_REF32_SO = os.path.join(_HERE, "_ref", "libbsofi_ref_fp32.so")
_PORT_SO = os.path.join(_HERE, "liboracle.so")

_dp = ctypes.POINTER(ctypes.c_double)
_ip = ctypes.POINTER(ctypes.c_int)
_libs = {}


def reference_tree():
    """The reference source tree: $BSOFI_REFERENCE, else the read-only mount
    /root/reference of the build container; None where neither exists (the
    GPU box uses the prebuilt _ref/ libraries)."""
    for d in (os.environ.get("BSOFI_REFERENCE"), "/root/reference"):
        if d and os.path.exists(os.path.join(d, "src", "bsofi_cpu.c")):
            return d
    return None


def build():
    """Compile the checkers (make -C oracle).  The reference library is only
    rebuilt where the reference tree is present."""
    import subprocess
    ref = reference_tree()
    subprocess.run(["make", "-s", "-C", _HERE] + (["REF=" + ref] if ref else []), check=True)


def ref_available():
    return os.path.exists(_REF_SO)


def ref32_available():
    return os.path.exists(_REF32_SO)


def _lib(kind):
    if kind not in _libs:
        path = {"ref": _REF_SO, "ref32": _REF32_SO}.get(kind, _PORT_SO)
        if not os.path.exists(path):
            raise RuntimeError("oracle library missing: %s (run make -C oracle)" % path)
        _libs[kind] = ctypes.CDLL(path)
    return _libs[kind]


def set_ref_threads(k, kind="ref"):
    """Set the OpenBLAS thread count used by the reference library."""
    lib = _lib(kind)
    try:
        f = lib.openblas_set_num_threads
    except AttributeError:
        return False
    f.argtypes = [ctypes.c_int]
    f(int(k))
    return True


def _p(a):
    return a.ctypes.data_as(_dp)


def _i(v):
    return ctypes.byref(ctypes.c_int(int(v)))


def _check(A, n, L):
    N = n * L
    A = np.asfortranarray(np.array(A, dtype=np.float64, copy=True))
    if A.shape != (N, N):
        raise ValueError("A must be %dx%d" % (N, N))
    return A


def _inplace(A, n, L):
    N = n * L
    if A.shape != (N, N) or A.dtype != np.float64 or not A.flags.f_contiguous:
        raise ValueError("A must be a Fortran-ordered float64 %dx%d array" % (N, N))
    return A


# ---------------------------------------------------------------- reference
def ref_bsoftri(A, n, L, inplace=False):
    """hybridxbsoftrih_ on a copy of A (on A itself with inplace=True: A must
    then be a Fortran-ordered float64 N x N array, as the reference's callers
    pass it).  Returns (A_out, tau, info)."""
    lib = _lib("ref")
    A = _inplace(A, n, L) if inplace else _check(A, n, L)
    N = n * L
    h = np.zeros(10, dtype=np.int32)
    hp = h.ctypes.data_as(_ip)
    lib.hybridxinith_(hp, _i(n), _i(L), _i(N))
    lw = lib.hybridxbsofilworkh_(hp, _i(n), _i(L), _i(N))
    work = np.zeros(max(int(lw), 1))
    tau = np.zeros(N)
    info = ctypes.c_int(0)
    lib.hybridxbsoftrih_(hp, _i(n), _i(L), _p(A), _i(N), _p(tau), _p(work),
                         _i(lw), ctypes.byref(info))
    lib.hybridxfinalizeh_(hp)
    return A, tau, info.value


def ref_bsof(A, n, L):
    """lapackXbsof (src/bsofi_cpu.c:86-118) on a copy of A: the factorization
    alone, R in the block upper part and the reflectors below.  Returns
    (A_out, tau, info)."""
    lib = _lib("ref")
    A = _check(A, n, L)
    N = n * L
    lw = int(lib.lapackXbsofiLWork(ctypes.c_int(n), ctypes.c_int(L), ctypes.c_int(N)))
    work = np.zeros(max(lw, 1))
    tau = np.zeros(N)
    info = ctypes.c_int(0)
    lib.lapackXbsof(ctypes.c_int(n), ctypes.c_int(L), _p(A), ctypes.c_int(N), _p(tau), _p(work),
                    ctypes.c_int(lw), ctypes.byref(info))
    return A, tau, info.value


def ref_bsoi(A, tau, n, L, inplace=False):
    """hybridxbsoih_ on a copy of the BSOFTRI state (on A and tau themselves
    with inplace=True).  Returns (A_out, info)."""
    lib = _lib("ref")
    A = _inplace(A, n, L) if inplace else _check(A, n, L)
    N = n * L
    if not inplace:
        tau = np.ascontiguousarray(tau, dtype=np.float64).copy()
    elif not (tau.dtype == np.float64 and tau.flags.c_contiguous):
        raise ValueError("tau must be a contiguous float64 array")
    h = np.zeros(10, dtype=np.int32)
    hp = h.ctypes.data_as(_ip)
    lib.hybridxinith_(hp, _i(n), _i(L), _i(N))
    lw = lib.hybridxbsofilworkh_(hp, _i(n), _i(L), _i(N))
    work = np.zeros(max(int(lw), 1))
    info = ctypes.c_int(0)
    lib.hybridxbsoih_(hp, _i(n), _i(L), _p(A), _i(N), _p(tau), _p(work),
                      _i(lw), ctypes.byref(info))
    lib.hybridxfinalizeh_(hp)
    return A, info.value


def ref_inverse(M, n, L):
    A, tau, info = ref_bsoftri(M, n, L)
    if info != 0:
        raise RuntimeError("reference BSOFTRI info=%d" % info)
    X, info = ref_bsoi(A, tau, n, L)
    return X


def ref_lwork(n, L):
    lib = _lib("ref")
    return int(lib.lapackXbsofiLWork(ctypes.c_int(n), ctypes.c_int(L), ctypes.c_int(n * L)))


# ------------------------------------------------ reference, single precision
_fp = ctypes.POINTER(ctypes.c_float)


def _check32(A, n, L):
    N = n * L
    A = np.asfortranarray(np.array(A, dtype=np.float32, copy=True))
    if A.shape != (N, N):
        raise ValueError("A must be %dx%d" % (N, N))
    return A


def _ref32_call(fname, A, tau, n, L):
    lib = _lib("ref32")
    N = n * L
    h = np.zeros(10, dtype=np.int32)
    hp = h.ctypes.data_as(_ip)
    lib.hybridxinith_(hp, _i(n), _i(L), _i(N))
    lw = lib.hybridxbsofilworkh_(hp, _i(n), _i(L), _i(N))
    work = np.zeros(max(int(lw), 1), dtype=np.float32)
    info = ctypes.c_int(0)
    getattr(lib, fname)(hp, _i(n), _i(L), A.ctypes.data_as(_fp), _i(N), tau.ctypes.data_as(_fp),
                        work.ctypes.data_as(_fp), _i(lw), ctypes.byref(info))
    lib.hybridxfinalizeh_(hp)
    return info.value


def ref32_bsoftri(A, n, L):
    """hybridxbsoftrih_ of the single-precision build on a float32 copy of A.
    Returns (A_out, tau, info)."""
    A = _check32(A, n, L)
    tau = np.zeros(n * L, dtype=np.float32)
    info = _ref32_call("hybridxbsoftrih_", A, tau, n, L)
    return A, tau, info


def ref32_bsoi(A, tau, n, L):
    """hybridxbsoih_ of the single-precision build.  Returns (A_out, info)."""
    A = _check32(A, n, L)
    tau = np.array(tau, dtype=np.float32, copy=True)
    info = _ref32_call("hybridxbsoih_", A, tau, n, L)
    return A, info


# ---------------------------------------------------------------- C port
def port_bsoftri(A, n, L):
    lib = _lib("port")
    A = _check(A, n, L)
    N = n * L
    tau = np.zeros(N)
    lib.oracle_bsof(ctypes.c_int(n), ctypes.c_int(L), _p(A), ctypes.c_int(N), _p(tau))
    info = lib.oracle_bstri(ctypes.c_int(n), ctypes.c_int(L), _p(A), ctypes.c_int(N))
    return A, tau, int(info)


def port_bsoi(A, tau, n, L):
    lib = _lib("port")
    A = _check(A, n, L)
    N = n * L
    tau = np.ascontiguousarray(tau, dtype=np.float64).copy()
    work = np.zeros(4 * n * n)
    lib.oracle_bsoi(ctypes.c_int(n), ctypes.c_int(L), _p(A), ctypes.c_int(N), _p(tau), _p(work))
    return A, 0


def port_inverse(M, n, L):
    A, tau, info = port_bsoftri(M, n, L)
    if info != 0:
        raise RuntimeError("port BSOFTRI info=%d" % info)
    X, _ = port_bsoi(A, tau, n, L)
    return X


def port_geqr2(A):
    """Householder QR (dgeqr2 semantics) of a copy of A; returns (A, tau)."""
    lib = _lib("port")
    A = np.asfortranarray(np.array(A, dtype=np.float64, copy=True))
    m, k = A.shape
    tau = np.zeros(min(m, k))
    lib.oracle_geqr2(ctypes.c_int(m), ctypes.c_int(k), _p(A), ctypes.c_int(m), _p(tau))
    return A, tau


def port_trtri_u(U):
    lib = _lib("port")
    A = np.asfortranarray(np.array(U, dtype=np.float64, copy=True))
    n = A.shape[0]
    info = lib.oracle_trtri_u(ctypes.c_int(n), _p(A), ctypes.c_int(n))
    return A, int(info)
