"""Python view of the BSOF/I C ABI (numpy host buffers and raw device pointers).

Every function calls libbsofi_b200.so; the numerical work runs in the sm_100a
kernels.  Host matrices are column-major float64 (numpy Fortran order).
"""
import ctypes

import numpy as np

from ._lib import load

INFO_CUDA = -1000
_ip = ctypes.POINTER(ctypes.c_int)
_dp = ctypes.POINTER(ctypes.c_double)


def _iref(v):
    return ctypes.byref(ctypes.c_int(int(v)))


def _dptr(a):
    return a.ctypes.data_as(_dp)


class Handle:
    """The reference's integer handler(10) managed by hybridxinith_ /
    hybridxfinalizeh_ (src/bsofi_callback.c:101-168)."""

    def __init__(self, n, L, lda=None):
        self.n, self.L = int(n), int(L)
        self.lda = int(lda) if lda is not None else self.n * self.L
        self.words = np.zeros(10, dtype=np.int32)
        rc = load().hybridxinith_(self.words.ctypes.data_as(_ip), _iref(self.n), _iref(self.L),
                                  _iref(self.lda))
        if rc != 0:
            raise RuntimeError("hybridxinith_ failed (%d)" % rc)

    @property
    def ptr(self):
        return self.words.ctypes.data_as(_ip)

    def lwork(self):
        return load().hybridxbsofilworkh_(self.ptr, _iref(self.n), _iref(self.L), _iref(self.lda))

    def bsoftri(self, A, tau, work=None, lwork=None):
        """hybridxbsoftrih_ in place on A (Fortran-ordered float64); returns info."""
        _check_host(A, self.lda)
        if work is None:
            work = np.zeros(max(1, self.lwork()))
        lw = len(work) if lwork is None else lwork
        info = ctypes.c_int(0)
        load().hybridxbsoftrih_(self.ptr, _iref(self.n), _iref(self.L), _dptr(A), _iref(self.lda),
                                _dptr(tau), _dptr(work), _iref(lw), ctypes.byref(info))
        return info.value

    def bsoi(self, A, tau, work=None, lwork=None):
        _check_host(A, self.lda)
        if work is None:
            work = np.zeros(max(1, self.lwork()))
        lw = len(work) if lwork is None else lwork
        info = ctypes.c_int(0)
        load().hybridxbsoih_(self.ptr, _iref(self.n), _iref(self.L), _dptr(A), _iref(self.lda),
                             _dptr(tau), _dptr(work), _iref(lw), ctypes.byref(info))
        return info.value

    def close(self):
        if self.words is not None:
            load().hybridxfinalizeh_(self.ptr)
            self.words = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def _check_host(A, lda):
    if not (isinstance(A, np.ndarray) and A.dtype == np.float64 and A.flags.f_contiguous):
        raise TypeError("A must be a Fortran-ordered float64 numpy array")
    if A.shape[0] != lda:
        raise ValueError("A.shape[0] must equal lda")


def invert(M, n, L):
    """M^{-1} through the handle API (XbsoftriH + XbsoiH).  Returns
    (X, A_after_bsoftri, tau, info)."""
    A = np.asfortranarray(np.array(M, dtype=np.float64, copy=True))
    tau = np.zeros(n * L)
    with Handle(n, L) as h:
        info = h.bsoftri(A, tau)
        state = A.copy(order="F")
        if info != 0:
            return None, state, tau, info
        info = h.bsoi(A, tau)
    return A, state, tau, info


# ------------------------------------------------------------ device API
def workspace_bytes(n, L, ldda):
    return int(load().bsofi_device_workspace_bytes(n, L, ldda))


def device_invert(n, L, dA, ldda, dtau, dwork, stream=0):
    """bsofi_device_invert on raw device pointers (ints); asynchronous."""
    return load().bsofi_device_invert(n, L, dA, ldda, dtau, dwork, stream)


def device_bsoftri(n, L, dA, ldda, dtau, dwork, stream=0):
    return load().bsofi_device_bsoftri(n, L, dA, ldda, dtau, dwork, stream)


def device_bsoi(n, L, dA, ldda, dtau, dwork, stream=0):
    return load().bsofi_device_bsoi(n, L, dA, ldda, dtau, dwork, stream)


def device_bsoi_rows(n, L, dA, ldda, dtau, dwork, row0, row1, stream=0):
    """BSOI of rows [row0, row1) of M^{-1} (bsofi_device_bsoi_rows)."""
    return load().bsofi_device_bsoi_rows(n, L, dA, ldda, dtau, dwork, row0, row1, stream)


def shard_state_bytes(n, L):
    """Bytes of one rank's state for the storage-sharded inversion."""
    return int(load().bsofi_shard_state_bytes(n, L))


def shard_factor(n, L, dD, dS, dstate, stream=0):
    """bsofi_shard_factor: compact factorization state from packed blocks."""
    return load().bsofi_shard_factor(n, L, dD or None, dS, dstate, stream)


def shard_hubbard_factor(n, L, dExpK, dh, lam, dstate, stream=0):
    """bsofi_shard_hubbard_factor: compact state from expm(K) and the fields."""
    return load().bsofi_shard_hubbard_factor(n, L, dExpK, dh, lam, dstate, stream)


def shard_bstri_columns(n, L, c0, c1, dX, ldx, dstate, stream=0):
    """bsofi_shard_bstri_columns: block columns [c0, c1) of R^{-1} into dX."""
    return load().bsofi_shard_bstri_columns(n, L, c0, c1, dX, ldx, dstate, stream)


def shard_bsoi_rows(n, L, row0, row1, dB, ldb, dstate, stream=0):
    """bsofi_shard_bsoi_rows: rows [row0, row1) of M^{-1} in place in dB."""
    return load().bsofi_shard_bsoi_rows(n, L, row0, row1, dB, ldb, dstate, stream)


def shard_logdet(n, L, dstate, dout, stream=0):
    """bsofi_shard_logdet: dout[0] = sign(det M), dout[1] = log|det M|."""
    return load().bsofi_shard_logdet(n, L, dstate, dout, stream)


def shard_info(state, n, L):
    """The info word of a storage-sharded state (a torch uint8 device
    tensor); synchronises with the device."""
    import torch
    del n, L
    torch.cuda.synchronize()
    ptr = load().bsofi_shard_info(state.data_ptr())
    out = torch.empty(1, dtype=torch.int32)
    base = state.data_ptr()
    off = (ptr - base) // 4
    out.copy_(state.view(torch.int32)[off:off + 1])
    v = int(out.item())
    return 0 if v >= 0x7f7f7f7f else v


def device_assemble(n, L, dD, dS, dA, ldda, stream=0):
    """bsofi_device_assemble: p-cyclic input from packed blocks (dD may be 0 = identity)."""
    return load().bsofi_device_assemble(n, L, dD or None, dS, dA, ldda, stream)


def device_hubbard_assemble(n, L, dExpK, dh, lam, dA, ldda, stream=0):
    """bsofi_device_hubbard_assemble: the DQMC matrix from expm(dtau t K) and the fields."""
    return load().bsofi_device_hubbard_assemble(n, L, dExpK, dh, float(lam), dA, ldda, stream)


def device_logdet(n, L, dA, ldda, dtau, inverted, dout, stream=0):
    """bsofi_device_logdet: dout[0] = sign(det M), dout[1] = log|det M|."""
    return load().bsofi_device_logdet(n, L, dA, ldda, dtau, 1 if inverted else 0, dout, stream)


def device_info_ptr(dwork):
    return load().bsofi_device_info(dwork)


def last_launches():
    return int(load().bsofi_device_last_launches())


def selftest_gemm(M, N, K, alpha, dA, lda, upper_a, dB, ldb, upper_b, beta, dC, ldc, tile=0,
                  stream=0):
    return load().bsofi_selftest_gemm(M, N, K, alpha, dA, lda, int(upper_a), dB, ldb,
                                      int(upper_b), beta, dC, ldc, tile, stream)


def timing(on):
    """Bracket every BSOI step GEMM launch with CUDA events (diagnostics)."""
    load().bsofi_device_timing(1 if on else 0)


def timing_read():
    """(summed BSOI GEMM time in ms, number of timed launches); clears the record."""
    ms = ctypes.c_double(0.0)
    cnt = ctypes.c_longlong(0)
    rc = load().bsofi_device_timing_read(ctypes.byref(ms), ctypes.byref(cnt))
    if rc != 0:
        raise RuntimeError("bsofi_device_timing_read failed (%d)" % rc)
    return ms.value, cnt.value


def batch_workspace_bytes(ns, Ls, lddas, precision=0):
    """Device workspace of a batch: precision 0 FP64, 1 mixed (int8 BSOI)."""
    import numpy as _np
    n = _np.ascontiguousarray(ns, dtype=_np.int32)
    L = _np.ascontiguousarray(Ls, dtype=_np.int32)
    ld = _np.ascontiguousarray(lddas, dtype=_np.int32)
    return int(load().bsofi_batch_workspace_bytes_ex(len(n), n.ctypes.data, L.ctypes.data,
                                                     ld.ctypes.data, precision))


def device_invert_batched(ns, Ls, dAs, lddas, dtaus, dwork, streams=8, stream=0, precision=0):
    """bsofi_device_invert_batched_ex on raw device pointers; asynchronous."""
    import numpy as _np
    n = _np.ascontiguousarray(ns, dtype=_np.int32)
    L = _np.ascontiguousarray(Ls, dtype=_np.int32)
    ld = _np.ascontiguousarray(lddas, dtype=_np.int32)
    pa = _np.ascontiguousarray(dAs, dtype=_np.uint64)
    pt = _np.ascontiguousarray(dtaus, dtype=_np.uint64)
    return load().bsofi_device_invert_batched_ex(len(n), n.ctypes.data, L.ctypes.data,
                                                 pa.ctypes.data, ld.ctypes.data, pt.ctypes.data,
                                                 dwork, streams, precision, stream)


def mixed_workspace_bytes(n, L, ldda, slices=0):
    return int(load().bsofi_device_workspace_bytes_mixed(n, L, ldda, slices))


def device_invert_mixed(n, L, dA, ldda, dtau, dwork, slices=0, stream=0):
    """bsofi_device_invert_mixed: FP64 factorization, BSOI on the int8 tensor
    cores (Ozaki scheme); asynchronous."""
    return load().bsofi_device_invert_mixed(n, L, dA, ldda, dtau, dwork, slices, stream)


def autotune(n, L, reps=3, stream=0):
    """bsofi_autotune: time the launch-plan candidates for (n, L) on the
    device and keep the fastest; returns the plan (4 ints)."""
    plan = np.zeros(4, dtype=np.int32)
    rc = load().bsofi_autotune(n, L, reps, stream, plan.ctypes.data)
    if rc != 0:
        raise RuntimeError("bsofi_autotune failed (%d)" % rc)
    return [int(v) for v in plan]


def plan_get(n, L):
    """(tuned, plan) for (n, L): tuned is False for the default plan."""
    plan = np.zeros(4, dtype=np.int32)
    tuned = load().bsofi_plan_get(n, L, plan.ctypes.data)
    return bool(tuned), [int(v) for v in plan]


def plan_set(n, L, plan):
    p = np.ascontiguousarray(plan, dtype=np.int32)
    return load().bsofi_plan_set(n, L, p.ctypes.data)


def plan_clear():
    load().bsofi_plan_clear()


class BatchGraph:
    """bsofi_batch_graph_*: a batch of inversions captured once into a CUDA
    graph; launch(stream) replays it on the same device buffers."""

    def __init__(self, ns, Ls, dAs, lddas, dtaus, dwork, streams=8):
        import numpy as _np
        self._n = _np.ascontiguousarray(ns, dtype=_np.int32)
        self._L = _np.ascontiguousarray(Ls, dtype=_np.int32)
        self._ld = _np.ascontiguousarray(lddas, dtype=_np.int32)
        self._pa = _np.ascontiguousarray(dAs, dtype=_np.uint64)
        self._pt = _np.ascontiguousarray(dtaus, dtype=_np.uint64)
        self.h = load().bsofi_batch_graph_create(len(self._n), self._n.ctypes.data,
                                                 self._L.ctypes.data, self._pa.ctypes.data,
                                                 self._ld.ctypes.data, self._pt.ctypes.data,
                                                 dwork, streams)
        if not self.h:
            raise RuntimeError("bsofi_batch_graph_create failed")

    def launch(self, stream):
        return load().bsofi_batch_graph_launch(self.h, stream)

    def close(self):
        if self.h:
            load().bsofi_batch_graph_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Server:
    """Continuous-batching inversion server (bsofi_server_*): submit
    device-resident matrices, poll for finished requests."""

    def __init__(self, slots=8, pool_bytes=8 << 30):
        self.ptr = load().bsofi_server_create(int(slots), int(pool_bytes))
        if not self.ptr:
            raise RuntimeError("bsofi_server_create failed")
        import numpy as _np
        self._ids = _np.zeros(256, dtype=_np.int64)
        self._st = _np.zeros(256, dtype=_np.int32)

    def submit(self, n, L, dA, ldda, dtau, precision=0):
        rid = load().bsofi_server_submit(self.ptr, n, L, dA, ldda, dtau, precision)
        if rid < 0:
            raise RuntimeError("bsofi_server_submit failed: %d" % rid)
        return rid

    def submit_blocks(self, n, L, dS, dD=0, precision=0):
        """Server-owned request from packed device blocks (dS: L coupling
        blocks, dD: L diagonal blocks or 0 for identity); the matrix, tau and
        workspace come from the pool at admission."""
        rid = load().bsofi_server_submit_blocks(self.ptr, n, L, dD or None, dS, precision)
        if rid < 0:
            raise RuntimeError("bsofi_server_submit_blocks failed: %d" % rid)
        return rid

    def result(self, rid):
        """(device address of M^{-1}, its leading dimension, address of tau)
        of a finished server-owned request, or None."""
        dA = ctypes.c_void_p(0)
        dtau = ctypes.c_void_p(0)
        ld = ctypes.c_int(0)
        if load().bsofi_server_result(self.ptr, rid, ctypes.byref(dA), ctypes.byref(ld),
                                      ctypes.byref(dtau)) != 0:
            return None
        return dA.value, ld.value, dtau.value

    def release(self, rid):
        return int(load().bsofi_server_release(self.ptr, rid))

    def poll(self):
        """List of (request id, status) that finished since the last poll."""
        k = load().bsofi_server_poll(self.ptr, self._ids.ctypes.data, self._st.ctypes.data,
                                     len(self._ids))
        if k < 0:
            raise RuntimeError("bsofi_server_poll failed")
        return [(int(self._ids[i]), int(self._st[i])) for i in range(k)]

    def pending(self):
        return int(load().bsofi_server_pending(self.ptr))

    def close(self):
        if self.ptr:
            load().bsofi_server_destroy(self.ptr)
            self.ptr = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


def server_request_bytes(n, L, ldda):
    return int(load().bsofi_server_request_bytes(n, L, ldda))


def server_footprint_bytes(n, L, precision=0):
    return int(load().bsofi_server_footprint_bytes(n, L, precision))
