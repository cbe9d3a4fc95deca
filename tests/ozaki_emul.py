"""numpy restatement of the int8 tensor-core product (the Ozaki splitting
scheme as bsofi_b200/csrc/kernels_ozaki.cu computes it), for tests.

Rows of A and columns of B are scaled by powers of two (frexp of the largest
magnitude) and cut into S signed 7-bit slices by truncation; the diagonal
sums D_d = sum_{s+t=d} A_s B_t (d < S) are exact integers (below 2^31, so
exact in float64 matmul too); the result is sum_{d=S-1..0} D_d 2^-7(d+2),
added in that order starting from 0, scaled by 2^(e_i + f_j).  Every step
but that sum is exact, and the sum is done in the same order as on the GPU,
so the two agree bit for bit.
"""
import numpy as np


def split_rows(A, S):
    """(exponents, [S slices as float64 integers]) of the rows of A."""
    A = np.asarray(A, dtype=np.float64)
    mx = np.abs(A).max(axis=1) if A.shape[1] else np.zeros(A.shape[0])
    _, e = np.frexp(mx)
    e = np.where(mx > 0, e, 0).astype(np.int64)
    r = np.where(mx[:, None] > 0, np.ldexp(A, -e[:, None]), 0.0)
    slices = []
    for _ in range(S):
        t = r * 128.0
        q = np.trunc(t)
        slices.append(q)
        r = t - q
    return e, slices


def ozaki_product(A, B, S):
    """C = A B as the int8 tensor-core kernel computes it."""
    ea, As = split_rows(A, S)
    eb, Bs = split_rows(np.asarray(B).T, S)
    acc = np.zeros((A.shape[0], B.shape[1]))
    for d in range(S - 1, -1, -1):
        D = np.zeros_like(acc)
        for s in range(d + 1):
            D += As[s] @ Bs[d - s].T
        acc = acc + D * np.ldexp(1.0, -7 * (d + 2))
    return np.ldexp(acc, ea[:, None] + eb[None, :])
