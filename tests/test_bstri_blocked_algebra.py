"""The blocked BSTRI recurrence and its overlapped split, restated in numpy
with the group indexing of bsofi_b200/csrc/pipeline.cu (RowGroups,
groups_seed / groups_rounds / groups_steps, overlap_split) and of the
persistent recurrence kernel's column floor, checked against the inverse of
the block upper-triangular R of BSOF (diagonal, superdiagonal and last block
column) for every group size and block count.  Host logic only: the CUDA path
is checked against the oracle in test_gpu_bstri_blocked.py."""
import numpy as np
import pytest


def _r_matrix(n, L, seed):
    rng = np.random.default_rng(seed)
    N = n * L
    R = np.zeros((N, N))
    for i in range(L):
        blk = np.triu(rng.standard_normal((n, n)))
        blk[np.diag_indices(n)] = 2.0 + rng.random(n)
        R[i * n:(i + 1) * n, i * n:(i + 1) * n] = blk
        if i + 1 < L:
            R[i * n:(i + 1) * n, (i + 1) * n:(i + 2) * n] = rng.standard_normal((n, n)) * 0.5
        if i < L - 2:
            R[i * n:(i + 1) * n, (L - 1) * n:] = rng.standard_normal((n, n)) * 0.5
    return R


class Groups:
    """RowGroups of pipeline.cu."""

    def __init__(self, L, grp):
        self.L, self.grp = L, grp
        self.b0 = L - 3
        self.ngr = (L - 2 + grp - 1) // grp
        self.mlast = (L - 2) - (self.ngr - 1) * grp

    def b(self, g):
        return self.b0 - g * self.grp

    def m(self, g):
        return min(self.b(g) + 1, self.grp)

    def t(self, g):
        return self.b(g) - self.m(g) + 1


def _blocked(R, n, L, grp, split):
    """X = R^{-1} by the blocked recurrence; split: also the overlapped order
    (rows above h first, over columns left of h; then the rest from h on)."""
    B = lambda A, i, j: A[i * n:(i + 1) * n, j * n:(j + 1) * n]
    N = n * L
    X = np.full((N, N), np.nan)
    X[np.tril_indices(N, -1)] = 0.0
    Xd = [np.linalg.inv(B(R, i, i)) for i in range(L)]
    for i in range(L):
        B(X, i, i)[:] = np.triu(Xd[i])
    W = [-Xd[i] @ B(R, i, i + 1) for i in range(L - 2)]
    Z = [-Xd[i] @ B(R, i, L - 1) @ Xd[L - 1] for i in range(L - 1)]
    G = Groups(L, grp)
    P = {}

    def seed(g0, g1):
        for g in range(g0, g1):
            P[(g, grp - 1)] = W[G.b(g)]

    def rounds(g0, g1, what):
        for q in range(1, grp):
            batch = (g1 - g0) - (1 if (g1 == G.ngr and G.mlast <= q) else 0)
            if batch <= 0:
                break
            for z in range(batch):
                g = g0 + z
                r = G.b(g) - q
                assert G.t(g) <= r < G.b(g)
                if "P" in what:
                    P[(g, grp - 1 - q)] = W[r] @ P[(g, grp - q)]
                if "I" in what:
                    for c in range(r + 1, r + q + 1):
                        B(X, r, c)[:] = W[r] @ B(X, r + 1, c)
                if "Z" in what:
                    B(X, r, L - 1)[:] = B(X, r, L - 1) + W[r] @ B(X, r + 1, L - 1)

    def step(g, cfrom, cto):
        b, m, t = G.b(g), G.m(g), G.t(g)
        cs = max(b + 1, cfrom)
        if cto <= cs:
            return
        Pg = np.vstack([P[(g, j)] for j in range(grp - m, grp)])
        rows = slice(t * n, (b + 1) * n)
        cols = slice(cs * n, cto * n)
        prod = Pg @ X[(b + 1) * n:(b + 2) * n, cols]
        if cto == L:
            prod[:, -n:] += X[rows, (L - 1) * n:]
        X[rows, cols] = prod

    for i in range(L - 1):
        B(X, i, L - 1)[:] = Z[i]
    if not split:
        seed(0, G.ngr)
        rounds(0, G.ngr, "PIZ")
        for g in range(G.ngr):
            step(g, 0, L)
        return X
    tailg = max(2, (G.ngr + 3) // 4)
    assert G.ngr > tailg
    h = L - 2 - tailg * grp
    assert h == G.t(tailg - 1)
    # Rows above h, columns left of h (needs only R's rows above h).
    seed(tailg, G.ngr)
    rounds(tailg, G.ngr, "PI")
    for g in range(tailg + 1, G.ngr):
        step(g, 0, h)
    # The rest.
    seed(0, tailg)
    rounds(0, tailg, "PI")
    rounds(0, G.ngr, "Z")
    for g in range(G.ngr):
        step(g, h, L)
    return X


@pytest.mark.parametrize("L", [3, 4, 5, 9, 13, 22, 32])
@pytest.mark.parametrize("grp", [2, 3, 4, 6, 8])
def test_blocked_recurrence_inverts_R(L, grp):
    n = 3
    g = min(grp, L - 2)
    if g < 2:
        pytest.skip("one-row recurrence")
    R = _r_matrix(n, L, seed=L * 10 + grp)
    Xr = np.linalg.inv(R)
    X = _blocked(R, n, L, g, split=False)
    np.testing.assert_allclose(X, Xr, rtol=0, atol=1e-9 * np.abs(Xr).max())
    G = Groups(L, g)
    if G.ngr > max(2, (G.ngr + 3) // 4):
        Xs = _blocked(R, n, L, g, split=True)
        np.testing.assert_allclose(Xs, Xr, rtol=0, atol=1e-9 * np.abs(Xr).max())
