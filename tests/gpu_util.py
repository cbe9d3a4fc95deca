"""Helpers for GPU tests: column-major device buffers through torch (device
memory plumbing only; the computation is in libbsofi_b200.so)."""
import numpy as np


def to_device_colmajor(torch, A, ld=None, device="cuda:0"):
    """Column-major (ld x ncols) float64 device buffer holding numpy A."""
    m, ncols = A.shape
    ld = ld or m
    t = torch.zeros((ncols, ld), dtype=torch.float64, device=device)
    t[:, :m] = torch.from_numpy(np.ascontiguousarray(A.T)).to(device)
    return t


def from_device_colmajor(t, m):
    return t[:, :m].T.cpu().numpy().copy(order="F")


def block_residual_gpu(torch, diag, sub, X):
    """||M X - I||_F / ||X||_F for the p-cyclic M (diag, sub blocks) and a
    dense device X (torch, row-major N x N view of M^{-1}), in FP64 on the GPU."""
    L, n, _ = diag.shape
    N = n * L
    dev = X.device
    D = torch.from_numpy(diag).to(dev)
    S = torch.from_numpy(sub).to(dev)
    acc = 0.0
    for r in range(L):
        rows = D[r] @ X[r * n:(r + 1) * n, :]
        c = (r - 1) % L  # block (r, r-1) holds sub[r-1]; block (0, L-1) holds sub[L-1]
        rows = rows + S[c] @ X[c * n:(c + 1) * n, :]
        rows[:, r * n:(r + 1) * n] -= torch.eye(n, dtype=torch.float64, device=dev)
        acc += float((rows * rows).sum())
    return (acc ** 0.5) / float(torch.linalg.norm(X))
