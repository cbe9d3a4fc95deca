"""The failure path of the bounded waits inside the persistent kernels.

Every spin inside a persistent kernel has an iteration limit; when it runs
out the kernel sets an error word and returns, and the inversion's info word
reads BSOFI_INFO_CUDA - cudaErrorLaunchTimeout.  Here the persistent BSOI
kernel is made to wait on a zeroed word that nothing writes (the diagnostic
switch bsofi_device_set_wait_test), so the waits give up without any fault;
the next inversion on the same buffers, with the switch off, is correct.
"""
import numpy as np
import pytest

from bsofi_b200 import _lib, api
from bsofi_b200.hubbard import hubbard_matrix
from conftest import inverse_tolerance, rel_fro

pytestmark = pytest.mark.gpu

CUDA_ERROR_LAUNCH_TIMEOUT = 702
WAIT_FAILED = -1000 - CUDA_ERROR_LAUNCH_TIMEOUT


def test_bsoi_wait_gives_up_then_next_call_succeeds(cuda_device):
    import torch
    from gpu_util import from_device_colmajor, to_device_colmajor
    lib = _lib.load()
    n, L = 64, 64  # N = 4096: the default plan runs BSOI as one persistent launch
    _, plan = api.plan_get(n, L)
    assert plan[0] in (0, 5)
    N = n * L
    M = hubbard_matrix(8, L, 4.0, seed=51)
    ws = torch.zeros(api.workspace_bytes(n, L, N) // 8 + 1, dtype=torch.float64,
                     device=cuda_device)
    dtau = torch.zeros(N, dtype=torch.float64, device=cuda_device)
    # The info word is the first int of the workspace (bsofi_device_info).
    assert api.device_info_ptr(ws.data_ptr()) == ws.data_ptr()

    def read_info():
        torch.cuda.synchronize()
        w = int(ws.view(torch.int32)[0].item())
        return 0 if w >= 0x7f7f7f7f else w

    lib.bsofi_device_set_wait_test(1)
    try:
        dA = to_device_colmajor(torch, M, ld=N, device=cuda_device)
        assert api.device_invert(n, L, dA.data_ptr(), N, dtau.data_ptr(), ws.data_ptr(), 0) == 0
        assert read_info() == WAIT_FAILED
        # Through the allocation-free entry point, which returns the info word.
        dA = to_device_colmajor(torch, M, ld=N, device=cuda_device)
        assert lib.bsofi_device_invert_noalloc(n, L, dA.data_ptr(), N, dtau.data_ptr(), None,
                                               None) == WAIT_FAILED
    finally:
        lib.bsofi_device_set_wait_test(0)
    # The device and the workspace are still usable: the same call succeeds.
    dA = to_device_colmajor(torch, M, ld=N, device=cuda_device)
    assert api.device_invert(n, L, dA.data_ptr(), N, dtau.data_ptr(), ws.data_ptr(), 0) == 0
    assert read_info() == 0
    X = from_device_colmajor(dA, N)
    Xref = np.linalg.inv(M)
    assert rel_fro(X, Xref) < inverse_tolerance(M, Xref)
    dA = to_device_colmajor(torch, M, ld=N, device=cuda_device)
    assert lib.bsofi_device_invert_noalloc(n, L, dA.data_ptr(), N, dtau.data_ptr(), None,
                                           None) == 0
    assert rel_fro(from_device_colmajor(dA, N), Xref) < inverse_tolerance(M, Xref)
