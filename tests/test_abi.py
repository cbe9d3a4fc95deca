"""The C ABI library: it loads, exports exactly what include/bsofi_b200.h
declares, and rejects illegal arguments LAPACK-style before touching a GPU."""
import ctypes
import subprocess

import numpy as np

from bsofi_b200 import _lib

_ip = ctypes.POINTER(ctypes.c_int)
_dp = ctypes.POINTER(ctypes.c_double)


def _i(v):
    return ctypes.byref(ctypes.c_int(v))


def test_library_loads():
    assert _lib.load() is not None


def test_exports_match_header():
    out = subprocess.run(["nm", "-D", "--defined-only", _lib.LIB_PATH], capture_output=True,
                         text=True, check=True).stdout
    exported = {line.split()[-1] for line in out.splitlines() if line.strip()}
    declared = set(_lib.declared_symbols())
    assert declared <= exported, declared - exported
    # The handle API and C names of the reference are all there.
    for name in ("hybridxinith_", "hybridxbsofilworkh_", "hybridxbsoftrih_", "hybridxbsoih_",
                 "hybridxfinalizeh_", "lapackXbsof", "lapackXbstri", "lapackXbsoi_ormqr",
                 "gpuXbsof", "gpuXbstri_rseq", "gpuXbsoi_batched", "fgetwalltime_"):
        assert name in exported


def test_binding_declares_every_export():
    """Every function of the header has a ctypes signature in the binding."""
    assert set(_lib.declared_symbols()) <= set(_lib._SIGS)


def test_no_oracle_linkage():
    out = subprocess.run(["ldd", _lib.LIB_PATH], capture_output=True, text=True).stdout
    assert "oracle" not in out and "openblas" not in out.lower()


def test_init_rejects_bad_sizes():
    lib = _lib.load()
    h = np.zeros(10, dtype=np.int32)
    hp = h.ctypes.data_as(_ip)
    assert lib.hybridxinith_(hp, _i(0), _i(4), _i(0)) == -1
    assert lib.hybridxinith_(hp, _i(4), _i(1), _i(4)) == -1
    assert lib.hybridxinith_(hp, _i(4), _i(4), _i(8)) == -1  # lda < N
    assert not h.any()


def test_invalid_handle_is_argument_1():
    lib = _lib.load()
    h = np.zeros(10, dtype=np.int32)
    A = np.zeros((8, 8), order="F")
    tau = np.zeros(8)
    w = np.zeros(1)
    info = ctypes.c_int(0)
    rc = lib.hybridxbsoftrih_(h.ctypes.data_as(_ip), _i(4), _i(2), A.ctypes.data_as(_dp), _i(8),
                              tau.ctypes.data_as(_dp), w.ctypes.data_as(_dp), _i(1),
                              ctypes.byref(info))
    assert rc == -1 and info.value == -1
    rc = lib.hybridxbsoih_(h.ctypes.data_as(_ip), _i(4), _i(2), A.ctypes.data_as(_dp), _i(8),
                           tau.ctypes.data_as(_dp), w.ctypes.data_as(_dp), _i(1),
                           ctypes.byref(info))
    assert info.value == -1


def test_c_names_validate_and_query():
    lib = _lib.load()
    A = np.zeros((8, 8), order="F")
    tau = np.zeros(8)
    w = np.zeros(1)
    info = ctypes.c_int(0)
    args = lambda n, L, lda, lw: (n, L, A.ctypes.data_as(_dp), lda, tau.ctypes.data_as(_dp),
                                  w.ctypes.data_as(_dp), lw, ctypes.byref(info))
    lib.lapackXbsof(*args(0, 2, 8, 1))
    assert info.value == -1
    lib.lapackXbsof(*args(4, 1, 8, 1))
    assert info.value == -2
    lib.lapackXbsof(*args(4, 2, 7, 1))
    assert info.value == -4
    lib.lapackXbsof(*args(4, 2, 8, 0))
    assert info.value == -7
    lib.lapackXbsof(*args(4, 2, 8, -1))  # workspace query: no device work
    assert info.value == 0 and w[0] >= 1
    assert lib.lapackXbsofiLWork(4, 2, 8) >= 1
    assert lib.hybridXbsofiLWork(64, 16, 1024, -2) > 1024 * 1024


def test_timers():
    lib = _lib.load()
    t0 = np.zeros(2)
    t1 = np.zeros(2)
    lib.fgetwalltime_(t0.ctypes.data_as(_dp))
    lib.fgetwalltime_(t1.ctypes.data_as(_dp))
    assert lib.felapsed_(t1.ctypes.data_as(_dp), t0.ctypes.data_as(_dp)) >= 0.0


def test_device_api_rejects_bad_arguments():
    """The device entry points validate sizes and pointers before any CUDA
    call (n beyond BSOFI_MAX_BLOCK = 768, L < 2, ldda < n L, NULL)."""
    lib = _lib.load()
    fake = 0x1000  # never dereferenced: the checks come first
    for n, L, ld, p in [(769, 2, 1538, fake), (0, 4, 16, fake), (4, 1, 16, fake), (4, 4, 15, fake),
                        (4, 4, 16, 0)]:
        assert lib.bsofi_device_invert(n, L, p, ld, fake, fake, None) == -1
        assert lib.bsofi_device_bsoftri(n, L, p, ld, fake, fake, None) == -1
        assert lib.bsofi_device_bsoi(n, L, p, ld, fake, fake, None) == -1


def test_device_lwork_query_at_largest_serving_size():
    """n = 576, L = 80 (N = 46080): the device length is past INT_MAX doubles.
    The int-returning query saturates; the lwork = -2 queries that write
    work[0] (a double) give the exact length."""
    lib = _lib.load()
    n, L = 576, 80
    N = n * L
    exact = ((N + 31) // 32 * 32) * N + N + lib.bsofi_device_workspace_bytes(n, L, N) // 8
    assert exact > 2**31 - 1
    assert lib.hybridXbsofiLWork(n, L, N, -2) == 2**31 - 1
    n_, L_, N_, m2 = ctypes.c_int(n), ctypes.c_int(L), ctypes.c_int(N), ctypes.c_int(-2)
    assert lib.hybridxbsofilwork_(ctypes.byref(n_), ctypes.byref(L_), ctypes.byref(N_),
                                  ctypes.byref(m2)) == 2**31 - 1
    w = np.zeros(1)
    info = ctypes.c_int(7)
    A = np.zeros(1)
    tau = np.zeros(1)
    lib.hybridXbsoftri(0, n, L, A.ctypes.data_as(_dp), N, tau.ctypes.data_as(_dp),
                       w.ctypes.data_as(_dp), -2, None, 0, ctypes.byref(info))
    assert info.value == 0 and w[0] == float(exact)


def test_hybrid_fortran_twins_validate_and_query():
    """hybridxbsofilwork_ / hybridxbsoftri_ / hybridxbsoi_ (the reference's
    cb_hybridX* callbacks, src/bsofi_callback.c:62-87) take every argument by
    pointer and answer the lwork queries without a GPU."""
    lib = _lib.load()
    A = np.zeros((8, 8), order="F")
    tau = np.zeros(8)
    w = np.zeros(1)
    info = ctypes.c_int(5)
    n, L, lda, ldw = ctypes.c_int(4), ctypes.c_int(2), ctypes.c_int(8), ctypes.c_int(0)
    for f in (lib.hybridxbsoftri_, lib.hybridxbsoi_):
        lw = ctypes.c_int(-1)
        f(ctypes.byref(n), ctypes.byref(L), A.ctypes.data_as(_dp), ctypes.byref(lda),
          tau.ctypes.data_as(_dp), w.ctypes.data_as(_dp), ctypes.byref(lw), None,
          ctypes.byref(ldw), ctypes.byref(info))
        assert info.value == 0 and w[0] >= 1
        bad = ctypes.c_int(7)  # lda < N
        f(ctypes.byref(n), ctypes.byref(L), A.ctypes.data_as(_dp), ctypes.byref(ctypes.c_int(7)),
          tau.ctypes.data_as(_dp), w.ctypes.data_as(_dp), ctypes.byref(lw), None,
          ctypes.byref(ldw), ctypes.byref(info))
        assert info.value == -4
        f(None, ctypes.byref(L), A.ctypes.data_as(_dp), ctypes.byref(lda),
          tau.ctypes.data_as(_dp), w.ctypes.data_as(_dp), ctypes.byref(lw), None,
          ctypes.byref(ldw), ctypes.byref(info))
        assert info.value == -1
    m1 = ctypes.c_int(-1)
    assert lib.hybridxbsofilwork_(ctypes.byref(n), ctypes.byref(L), ctypes.byref(lda),
                                  ctypes.byref(m1)) == lib.hybridXbsofiLWork(4, 2, 8, -1)
