"""The single-precision library (include/bsofi_b200_fp32.h) on the CPU: it
loads, exports exactly the header's names, rejects illegal arguments before
touching a GPU; and its oracle, the reference built with -D__SINGLE_PREC__,
is pinned against the committed FP32 fixtures."""
import ctypes
import glob
import os
import subprocess

import numpy as np
import pytest

import oracle
from bsofi_b200 import fp32
from bsofi_b200.hubbard import assemble_pcyclic
from conftest import GOLDEN, golden_cases, rel_fro

_ip = ctypes.POINTER(ctypes.c_int)
_fp = ctypes.POINTER(ctypes.c_float)
_dp = ctypes.POINTER(ctypes.c_double)
EPS32 = float(np.finfo(np.float32).eps)


def _i(v):
    return ctypes.byref(ctypes.c_int(v))


def fp32_cases():
    out = []
    for f in sorted(glob.glob(os.path.join(GOLDEN, "fp32", "*.npz"))):
        d = dict(np.load(f))
        d["name"] = os.path.basename(f)[:-4]
        d["n"], d["L"], d["info"] = int(d["n"]), int(d["L"]), int(d["info"])
        out.append(d)
    return out


CASES32 = fp32_cases()


def test_fp32_fixtures_present():
    assert len(CASES32) >= 7
    for c in CASES32:
        assert c["state"].dtype == np.float32 and c["inverse"].dtype == np.float32


def test_library_loads_and_exports_exactly_the_header():
    assert fp32.load() is not None
    out = subprocess.run(["nm", "-D", "--defined-only", fp32.LIB_PATH], capture_output=True,
                         text=True, check=True).stdout
    exported = {line.split()[-1] for line in out.splitlines() if line.strip()}
    assert exported == set(fp32.declared())
    for name in ("hybridxinith_", "hybridxbsoftrih_", "hybridxbsoih_", "hybridxfinalizeh_",
                 "lapackXbsof", "lapackXbstri", "lapackXbsoi_ormqr", "gpuXbsof", "fgetwalltime_"):
        assert name in exported


def test_binding_declares_every_export():
    """Every name of the header has a ctypes signature (no default int
    conversions of pointers)."""
    assert set(fp32._SIGS) == set(fp32.declared())


def test_fortran_twins_validate():
    lib = fp32.load()
    A = np.zeros((8, 8), dtype=np.float32, order="F")
    tau = np.zeros(8, dtype=np.float32)
    w = np.zeros(1, dtype=np.float32)
    info = ctypes.c_int(0)
    lib.lapackxbsof_(_i(0), _i(2), A.ctypes.data_as(_fp), _i(8), tau.ctypes.data_as(_fp),
                     w.ctypes.data_as(_fp), _i(1), ctypes.byref(info))
    assert info.value == -1
    assert lib.lapackxbsofilwork_(_i(4), _i(2), _i(8)) >= 1


def test_no_oracle_linkage():
    out = subprocess.run(["ldd", fp32.LIB_PATH], capture_output=True, text=True).stdout
    assert "oracle" not in out and "openblas" not in out.lower()


def test_init_rejects_bad_sizes_and_handles():
    lib = fp32.load()
    h = np.zeros(10, dtype=np.int32)
    hp = h.ctypes.data_as(_ip)
    assert lib.hybridxinith_(hp, _i(0), _i(4), _i(0)) == -1
    assert lib.hybridxinith_(hp, _i(4), _i(1), _i(4)) == -1
    assert lib.hybridxinith_(hp, _i(4), _i(4), _i(8)) == -1
    assert not h.any()
    A = np.zeros((8, 8), dtype=np.float32, order="F")
    tau = np.zeros(8, dtype=np.float32)
    w = np.zeros(1, dtype=np.float32)
    info = ctypes.c_int(0)
    for f in (lib.hybridxbsoftrih_, lib.hybridxbsoih_):
        rc = f(hp, _i(4), _i(2), A.ctypes.data_as(_fp), _i(8), tau.ctypes.data_as(_fp),
               w.ctypes.data_as(_fp), _i(1), ctypes.byref(info))
        assert rc == -1 and info.value == -1


def test_c_names_validate_and_query():
    lib = fp32.load()
    A = np.zeros((8, 8), dtype=np.float32, order="F")
    tau = np.zeros(8, dtype=np.float32)
    w = np.zeros(1, dtype=np.float32)
    info = ctypes.c_int(0)
    args = lambda n, L, lda, lw: (n, L, A.ctypes.data_as(_fp), lda, tau.ctypes.data_as(_fp),
                                  w.ctypes.data_as(_fp), lw, ctypes.byref(info))
    lib.lapackXbsof(*args(0, 2, 8, 1))
    assert info.value == -1
    lib.lapackXbsof(*args(4, 1, 8, 1))
    assert info.value == -2
    lib.lapackXbsof(*args(4, 2, 7, 1))
    assert info.value == -4
    lib.lapackXbsof(*args(4, 2, 8, 0))
    assert info.value == -7
    lib.lapackXbsof(*args(4, 2, 8, -1))
    assert info.value == 0 and w[0] >= 1
    lib.lapackXbsoi_ormqr(*args(4, 2, 8, -2))
    assert info.value == 0 and w[0] > 64
    assert lib.lapackXbsofiLWork(4, 2, 8) >= 1
    # Device workspace in floats: the FP64 working matrix, its float copy and
    # the pipeline's workspace.
    assert lib.hybridXbsofiLWork(64, 16, 1024, -2) > 3 * 1024 * 1024


def test_timers_are_double():
    lib = fp32.load()
    t0 = np.zeros(2)
    t1 = np.zeros(2)
    lib.fgetwalltime_(t0.ctypes.data_as(_dp))
    lib.fgetwalltime_(t1.ctypes.data_as(_dp))
    assert lib.felapsed_(t1.ctypes.data_as(_dp), t0.ctypes.data_as(_dp)) >= 0.0


@pytest.mark.skipif(not oracle.ref32_available(), reason="FP32 reference library not built")
@pytest.mark.parametrize("case", CASES32, ids=[c["name"] for c in CASES32])
def test_fp32_reference_reproduces_fixtures(case):
    """Pins the FP32 oracle: the single-precision reference library gives the
    committed fixtures (one OpenBLAS thread, as when they were made)."""
    oracle.set_ref_threads(1, kind="ref32")
    n, L = case["n"], case["L"]
    M = assemble_pcyclic(case["diag"], case["sub"]).astype(np.float32)
    A, tau, info = oracle.ref32_bsoftri(M, n, L)
    X, _ = oracle.ref32_bsoi(A, tau, n, L)
    assert info == case["info"] == 0
    np.testing.assert_allclose(tau, case["tau"], rtol=0, atol=4 * EPS32)
    assert rel_fro(A, case["state"]) < 1e-5
    assert rel_fro(X, case["inverse"]) < 1e-5


@pytest.mark.parametrize("case", CASES32, ids=[c["name"] for c in CASES32])
def test_fp32_fixtures_agree_with_fp64_fixtures(case):
    """The FP32 reference's inverse is the FP64 reference's within the FP32
    forward-error bound 8 sqrt(N) kappa_F eps32."""
    by_name = {c["name"]: c for c in golden_cases()}
    c64 = by_name[case["name"]]
    M = assemble_pcyclic(c64["diag"], c64["sub"])
    N = M.shape[0]
    kappa = np.linalg.norm(M) * np.linalg.norm(c64["inverse"]) / N
    assert rel_fro(case["inverse"].astype(np.float64), c64["inverse"]) < \
        8 * np.sqrt(N) * kappa * EPS32
