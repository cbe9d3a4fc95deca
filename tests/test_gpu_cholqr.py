"""The BSOF chain's leaf factorization by CholeskyQR2 and Householder
reconstruction against the column-by-column Householder factorization and
the oracle (the dgeqr2 conventions of src/bsofi_cpu.c:97 via
src/bsofi_lapack.c).

Both settings of bsofi_device_set_bsof_cholqr must give the oracle's state
(tau within 1e-12, reflectors within 1e-10, R^{-1} and M^{-1} within the
kappa-relative FP64 tolerance, determinant sign exact).  Sizes cover 16-wide
leaves (n = 64), a narrower last leaf (n = 100, column by column), 8-wide
leaves (n = 300), and a first panel whose two leading columns agree to 1e-9
(condition number about 1e9, so the leaf falls back to the column-by-column
factorization).
"""
import numpy as np
import pytest

import oracle
from bsofi_b200 import _lib, api
from bsofi_b200.hubbard import hubbard_matrix, random_pcyclic
from conftest import det_sign, inverse_tolerance, rel_fro, residual, split_state

pytestmark = pytest.mark.gpu


def _cases():
    near = random_pcyclic(24, 5, seed=77)
    # Column 1 of block column 0 (rows 0 .. 2n-1, its two p-cyclic blocks)
    # equal to column 0 up to 1e-9.
    near[:48, 1] = near[:48, 0] + 1e-9 * np.random.default_rng(1).standard_normal(48)
    return [("hub64", hubbard_matrix(8, 16, 4.0, seed=3), 64, 16),
            ("rand100", random_pcyclic(100, 5, seed=5), 100, 5),
            ("rand300", random_pcyclic(300, 4, seed=6), 300, 4),
            ("near_dependent", near, 24, 5)]


@pytest.mark.parametrize("name,M,n,L", _cases(), ids=[c[0] for c in _cases()])
@pytest.mark.parametrize("cholqr", [1, 0])
def test_leaf_factorizations_match_oracle(cuda_device, name, M, n, L, cholqr):
    lib = _lib.load()
    Ar, taur, _ = oracle.port_bsoftri(M, n, L)
    Xr, _ = oracle.port_bsoi(Ar, taur, n, L)
    lib.bsofi_device_set_bsof_cholqr(cholqr)
    try:
        X, state, tau, info = api.invert(M, n, L)
    finally:
        lib.bsofi_device_set_bsof_cholqr(1)
    assert info == 0
    tol = inverse_tolerance(M, Xr)
    assert det_sign(state, tau) == det_sign(Ar, taur)
    if name == "near_dependent":
        # The second column's residual after the first reflection is ~1e-9 of
        # its norm: its reflector is determined only to ~1e-7 by any two
        # Householder implementations.
        np.testing.assert_allclose(tau, taur, rtol=0, atol=1e-5)
    else:
        np.testing.assert_allclose(tau, taur, rtol=0, atol=1e-12)
        up, refl = split_state(state, n, L)
        rup, rrefl = split_state(Ar, n, L)
        assert rel_fro(up, rup) < tol
        assert np.abs(refl - rrefl).max() < 1e-10
    assert rel_fro(X, Xr) < tol
    assert residual(M, X) < 1e-13


def test_both_factorizations_agree_at_headline_size(cuda_device):
    """n = 256, p = 32: the two leaf factorizations give the same inverse to
    rounding (both against each other's kappa-relative bound)."""
    lib = _lib.load()
    n, L = 256, 32
    M = hubbard_matrix(16, L, 4.0, seed=8)
    X1, s1, t1, i1 = api.invert(M, n, L)
    lib.bsofi_device_set_bsof_cholqr(0)
    try:
        X0, s0, t0, i0 = api.invert(M, n, L)
    finally:
        lib.bsofi_device_set_bsof_cholqr(1)
    assert i0 == 0 and i1 == 0
    np.testing.assert_allclose(t1, t0, rtol=0, atol=1e-12)
    assert rel_fro(X1, X0) < inverse_tolerance(M, X0)
    assert det_sign(s1, t1) == det_sign(s0, t0)
