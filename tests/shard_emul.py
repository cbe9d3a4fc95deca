"""numpy restatement of the storage-sharded inversion (bsofi_b200/shard.py,
bsofi_shard_* in bsofi_b200/csrc/pipeline.cu), for CPU tests.

From the reference's BSOF state (lapackXbsof, src/bsofi_cpu.c:86-118: R in
the block upper part, reflectors below, tau):
  * factor_terms: X_ii = R_ii^{-1}, W_i = -X_ii R_{i,i+1} (i <= L-3) and
    Z_i = -X_ii R_{i,L-1} X_{L-1,L-1} (i <= L-2);
  * bstri_columns: block columns [c0, c1) of X = R^{-1}, rows 0..c1 n - 1,
    by X_{i,c} = W_i X_{i+1,c} (+ Z_i for c = L-1), i = min(c1-2, L-3)..0
    (the reference's row recurrence, src/bsofi_cpu.c:146-177, read by
    columns);
  * bsoi_rows: rows of M^{-1} = R^{-1} Q_{L-2}^T ... Q_0^T from the same rows
    of X (src/bsofi_cpu.c:211-248), with Q_k the product of panel k's
    Householder reflectors (LAPACK dgeqrf convention, H = I - tau v v^T).
"""
import numpy as np


def _blk(A, n, i, j):
    return A[i * n:(i + 1) * n, j * n:(j + 1) * n]


def factor_terms(A, n, L):
    """(Xd, W, Z) from the BSOF state A (N x N)."""
    Xd = [np.linalg.inv(np.triu(_blk(A, n, i, i))) for i in range(L)]
    Xd = [np.triu(x) for x in Xd]
    W = [-Xd[i] @ _blk(A, n, i, i + 1) for i in range(L - 2)]
    Z = [-Xd[i] @ _blk(A, n, i, L - 1) @ Xd[L - 1] for i in range(L - 1)]
    return Xd, W, Z


def bstri_columns(terms, n, L, c0, c1):
    """Block columns [c0, c1) of X = R^{-1} as a (c1 n) x ((c1 - c0) n) array."""
    Xd, W, Z = terms
    S = np.zeros((c1 * n, (c1 - c0) * n))

    def blk(i, c):
        return S[i * n:(i + 1) * n, (c - c0) * n:(c - c0 + 1) * n]

    for c in range(c0, c1):
        blk(c, c)[:] = Xd[c]
    if c1 == L:
        for i in range(L - 1):
            blk(i, L - 1)[:] = Z[i]
    for i in range(min(c1 - 2, L - 3), -1, -1):
        for c in range(max(i + 1, c0), c1):
            v = W[i] @ blk(i + 1, c)
            if c == L - 1:
                v = v + Z[i]
            blk(i, c)[:] = v
    return S


def panel_q(A, tau, n, L):
    """Q_k (2n x 2n) of every panel k = 0..L-2."""
    out = []
    for k in range(L - 1):
        m = n if k < L - 2 else 2 * n
        Q = np.eye(2 * n)
        for j in range(m):
            v = np.zeros(2 * n)
            v[j] = 1.0
            v[j + 1:] = A[k * n + j + 1:(k + 2) * n, k * n + j]
            Q = Q - tau[k * n + j] * np.outer(Q @ v, v)
        out.append(Q)
    return out


def bsoi_rows(band, Qs, n, L):
    """band: rows [r0, r1) of X in every column ((r1 - r0) x N), overwritten
    with the same rows of M^{-1}."""
    for k in range(L - 2, -1, -1):
        sl = slice(k * n, (k + 2) * n)
        band[:, sl] = band[:, sl] @ Qs[k].T
    return band
