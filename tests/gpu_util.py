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


def pcyclic_device(torch, diag, sub, ldd, device):
    """Column-major (ldd x N) device buffer of the p-cyclic matrix with blocks
    diag (p, n, n) and sub (p, n, n; sub[k] at block (k+1 mod p, k)), written
    block by block on the device (no dense host matrix)."""
    L, n, _ = diag.shape
    N = n * L
    t = torch.zeros((N, ldd), dtype=torch.float64, device=device)  # t[col, row]
    D = torch.from_numpy(np.ascontiguousarray(diag)).to(device)
    S = torch.from_numpy(np.ascontiguousarray(sub)).to(device)
    for k in range(L):
        t[k * n:(k + 1) * n, k * n:(k + 1) * n] = D[k].T
        r = (k + 1) % L
        t[k * n:(k + 1) * n, r * n:(r + 1) * n] = S[k].T
    return t


def block_residual_colmajor(torch, diag, sub, T, N):
    """||M X - I||_F / ||X||_F in FP64 on the GPU, X held column-major in the
    device buffer T (T[j, i] = X[i, j], as pcyclic_device lays it out), using
    only M's p-cyclic blocks: block row r of M X is D_r X_r + S_{r-1} X_{r-1}."""
    L, n, _ = diag.shape
    dev = T.device
    Xt = T[:, :N]  # X^T
    acc = 0.0
    eye = torch.eye(n, dtype=torch.float64, device=dev)
    for r in range(L):
        c = (r - 1) % L
        Dr = torch.from_numpy(np.ascontiguousarray(diag[r])).to(dev)
        Sc = torch.from_numpy(np.ascontiguousarray(sub[c])).to(dev)
        # (M X)[rows r, :]^T = X^T[:, rows r] D_r^T + X^T[:, rows c] S_c^T
        Y = Xt[:, r * n:(r + 1) * n] @ Dr.T + Xt[:, c * n:(c + 1) * n] @ Sc.T
        Y[r * n:(r + 1) * n, :] -= eye
        acc += float((Y * Y).sum())
    return (acc ** 0.5) / float(torch.linalg.norm(Xt))


class _DevBuf:
    """__cuda_array_interface__ of raw device memory (no copy)."""

    def __init__(self, ptr, shape):
        self.__cuda_array_interface__ = {"shape": tuple(shape), "typestr": "<f8",
                                         "data": (int(ptr), False), "version": 3,
                                         "strides": None}


def device_view(torch, ptr, ncols, ld, device="cuda:0"):
    """A float64 torch view (ncols, ld) of column-major device memory at ptr,
    laid out as to_device_colmajor lays out its buffers."""
    return torch.as_tensor(_DevBuf(ptr, (ncols, ld)), device=device)
