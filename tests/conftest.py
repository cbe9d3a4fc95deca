import glob
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

GOLDEN = os.path.join(ROOT, "tests", "golden")
EPS = np.finfo(np.float64).eps


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")


def golden_cases():
    out = []
    for f in sorted(glob.glob(os.path.join(GOLDEN, "*.npz"))):
        d = dict(np.load(f))
        d["name"] = os.path.basename(f)[:-4]
        d["n"], d["L"], d["info"] = int(d["n"]), int(d["L"]), int(d["info"])
        out.append(d)
    return out


def golden_matrix(case):
    from bsofi_b200.hubbard import assemble_pcyclic
    return assemble_pcyclic(case["diag"], case["sub"])


def rel_fro(X, Y):
    return float(np.linalg.norm(X - Y) / max(np.linalg.norm(Y), 1e-300))


def inverse_tolerance(M, Xref):
    """Forward-error bound for an FP64 inverse: 8 sqrt(N) kappa_F eps, with
    kappa_F = ||M||_F ||M^{-1}||_F / N (never below 1e-13)."""
    N = M.shape[0]
    kappa = np.linalg.norm(M) * np.linalg.norm(Xref) / N
    return max(1e-13, 8.0 * np.sqrt(N) * kappa * EPS)


def residual(M, X):
    """||M X - I||_F / ||X||_F (the reference's quality metric,
    examples/ftest_hybrid/ftest_hybrid.f90:54-101, without the ||M||_F factor)."""
    N = M.shape[0]
    return float(np.linalg.norm(M @ X - np.eye(N)) / np.linalg.norm(X))


def det_sign(state, tau):
    """Sign of the reference's determinant consumer,
    examples/ftest_hybrid/ftest_hybrid.f90:141-145."""
    s = 1.0
    d = np.diag(state)
    for i in range(len(tau)):
        if tau[i] == 0.0:
            s = -s
        if d[i] < 0.0:
            s = -s
    return s


def split_state(state, n, L):
    """(block upper triangle holding R^{-1} incl. diagonal blocks' upper
    parts, reflector part) of the BSOFTRI state."""
    N = n * L
    up = np.zeros_like(state)
    refl = np.zeros_like(state)
    for k in range(L):
        c0, c1 = k * n, (k + 1) * n
        for c in range(c0, c1):
            # rows 0..c: R^{-1} (block upper triangle, upper part of diagonal block)
            up[: c + 1, c] = state[: c + 1, c]
            if k < L - 2:
                refl[c + 1: (k + 2) * n, c] = state[c + 1: (k + 2) * n, c]
            elif k >= L - 2:
                refl[c + 1: N, c] = state[c + 1: N, c]
        # blocks above the diagonal beyond column: rows < c0 handled above
    return up, refl


@pytest.fixture(scope="session")
def cuda_device():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch.device("cuda:0")
