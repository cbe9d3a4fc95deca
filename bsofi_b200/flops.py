"""Flop model of BSOF/I, restated from include/bsofi_flops.h:19-30.

The per-routine counts are the LAPACK Working Note 41 formulas for dgeqrf,
dormqr (left and right), dtrtri, dtrmm and dgemm (multiplications plus
additions), composed exactly as bsofi_flops.h composes them.  This is the
count behind every TFLOP/s figure; work the GPU path adds (explicit Q
formation) is not credited.
"""


def _geqrf(m, n):
    m, n = float(m), float(n)
    if m > n:
        mul = n * (n * (0.5 - n / 3.0 + m) + m + 23.0 / 6.0)
        add = n * (n * (0.5 - n / 3.0 + m) + 5.0 / 6.0)
    else:
        mul = m * (m * (-0.5 - m / 3.0 + n) + 2.0 * n + 23.0 / 6.0)
        add = m * (m * (-0.5 - m / 3.0 + n) + n + 5.0 / 6.0)
    return mul + add


def _ormqr(m, n, k, side):
    m, n, k = float(m), float(n), float(k)
    if side == "L":
        mul = 2.0 * n * m * k - n * k * k + 2.0 * n * k
        add = 2.0 * n * m * k - n * k * k + n * k
    else:
        mul = 2.0 * n * m * k - m * k * k + m * k + n * k - 0.5 * k * k + 0.5 * k
        add = 2.0 * n * m * k - m * k * k + m * k
    return mul + add


def _trtri(n):
    n = float(n)
    return n * (n * (n / 6.0 + 0.5) + 1.0 / 3.0) + n * (n * (n / 6.0 - 0.5) + 1.0 / 3.0)


def _trmm(side, m, n):
    m, n = float(m), float(n)
    if side != "L":
        m, n = n, m
    return 0.5 * n * m * (m + 1.0) + 0.5 * n * m * (m - 1.0)


def _gemm(m, n, k):
    return 2.0 * float(m) * float(n) * float(k)


def flops_bsof(n, L):
    return (L - 2) * (2 * _ormqr(2 * n, n, n, "L") + _geqrf(2 * n, n)) + _geqrf(2 * n, 2 * n)


def flops_bstri(n, L):
    # The integer division mirrors the C macro's int arithmetic ((L-3)*(L+2)/2).
    return (_trtri(3 * n) + _trmm("R", n * (L - 3), n)
            + (L - 3) * (_trtri(n) + 2 * _trmm("L", n, n))
            + ((L - 3) * (L + 2) // 2) * _gemm(n, n, n))


def flops_bsoi(n, L):
    return (L - 2) * _ormqr(L * n, 2 * n, n, "R") + _ormqr(L * n, 2 * n, 2 * n, "R")


def bsofi_flops(n, L):
    """FLOPS_BSOFTRI(n, L) + FLOPS_BSOI(n, L): the algorithmic work of one inversion."""
    return flops_bsof(n, L) + flops_bstri(n, L) + flops_bsoi(n, L)
