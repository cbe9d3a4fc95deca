"""Seeded block p-cyclic inputs for BSOF/I.

The Hubbard/DQMC generator builds the Green's-function matrix

    M = [[ I,    0,   ...,  0,     +B_p ],
         [-B_1,  I,   ...,  0,      0   ],
         [ 0,   -B_2, ...,  ...,    0   ],
         [ ...                          ],
         [ 0,    ...,      -B_{p-1}, I  ]]

with B_k = expm(dtau*t*K) @ diag(exp(lam*h_k)), K the nearest-neighbour
adjacency of a side x side periodic square lattice (n = side^2 sites),
lam = acosh(exp(U*dtau/2)) and Ising fields h_k in {-1,+1} drawn uniformly from
``numpy.random.default_rng(seed)``.  The chemical potential mu enters as a
factor exp(dtau*mu) on every B_k (mu = 0 in all benchmark configurations).

Matrices are column-major (Fortran order) float64 with leading dimension N.
The reference examples fill the same block positions (identity diagonal,
blocks at (k+1 mod p, k)): examples/ftest_hybrid/ftest_hybrid.f90:12-52.
"""
import numpy as np


def lattice_adjacency(side):
    """Nearest-neighbour adjacency of a periodic side x side square lattice."""
    n = side * side
    K = np.zeros((n, n))
    for x in range(side):
        for y in range(side):
            i = x * side + y
            for dx, dy in ((1, 0), (-1, 0), (0, 1), (0, -1)):
                j = ((x + dx) % side) * side + (y + dy) % side
                if j != i:
                    K[i, j] = 1.0
    return K


def expm_sym(S):
    """exp(S) of a symmetric matrix through its eigendecomposition."""
    w, Q = np.linalg.eigh(S)
    return (Q * np.exp(w)) @ Q.T


def hubbard_blocks(side, p, U, dtau=0.125, t=1.0, mu=0.0, seed=0):
    """Return B of shape (p, n, n): B[k] = B_{k+1} of the DQMC chain."""
    n = side * side
    rng = np.random.default_rng(seed)
    h = rng.choice(np.array([-1.0, 1.0]), size=(p, n))
    lam = np.arccosh(np.exp(U * dtau / 2.0))
    expK = expm_sym(dtau * t * lattice_adjacency(side)) * np.exp(dtau * mu)
    B = np.empty((p, n, n))
    for k in range(p):
        B[k] = expK * np.exp(lam * h[k])[None, :]
    return B


def assemble_pcyclic(diag, sub):
    """Dense column-major p-cyclic matrix.

    diag: (p, n, n) diagonal blocks A_k; sub: (p, n, n) with sub[k] placed at
    block (k+1, k) for k < p-1 and sub[p-1] at block (0, p-1).
    """
    p, n, _ = diag.shape
    N = n * p
    M = np.zeros((N, N), order="F")
    for k in range(p):
        M[k * n:(k + 1) * n, k * n:(k + 1) * n] = diag[k]
        r = (k + 1) % p
        M[r * n:(r + 1) * n, k * n:(k + 1) * n] = sub[k]
    return M


def hubbard_matrix(side, p, U, dtau=0.125, t=1.0, mu=0.0, seed=0):
    """The DQMC matrix M: identity diagonal, -B_k below, +B_p in the corner."""
    B = hubbard_blocks(side, p, U, dtau, t, mu, seed)
    n = side * side
    eye = np.broadcast_to(np.eye(n), (p, n, n))
    sub = -B.copy()
    sub[p - 1] = B[p - 1]
    return assemble_pcyclic(np.array(eye), sub)


def random_pcyclic(n, p, seed=0, diag_scale=1.0):
    """A general p-cyclic matrix with random diagonal and coupling blocks."""
    rng = np.random.default_rng(seed)
    diag = rng.standard_normal((p, n, n)) + diag_scale * np.eye(n)[None]
    sub = rng.standard_normal((p, n, n))
    return assemble_pcyclic(diag, sub)


def pcyclic_blocks(M, n, p):
    """Extract (diag, sub) from a dense p-cyclic matrix (inverse of assemble)."""
    diag = np.empty((p, n, n))
    sub = np.empty((p, n, n))
    for k in range(p):
        diag[k] = M[k * n:(k + 1) * n, k * n:(k + 1) * n]
        r = (k + 1) % p
        sub[k] = M[r * n:(r + 1) * n, k * n:(k + 1) * n]
    return diag, sub
