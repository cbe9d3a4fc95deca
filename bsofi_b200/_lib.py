"""ctypes binding of libbsofi_b200.so (the C ABI in include/bsofi_b200.h).

The library is the product: there is no Python or CPU fallback.  Loading fails
loudly when the shared library has not been built.
"""
import ctypes
import os
import re

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libbsofi_b200.so")
HEADER = os.path.join(os.path.dirname(HERE), "include", "bsofi_b200.h")

_c_int_p = ctypes.POINTER(ctypes.c_int)
_c_dbl_p = ctypes.POINTER(ctypes.c_double)
_vp = ctypes.c_void_p

# (restype, argtypes) per exported symbol.
_SIGS = {
    "hybridxinith_": (ctypes.c_int, [_c_int_p, _c_int_p, _c_int_p, _c_int_p]),
    "hybridxbsofilworkh_": (ctypes.c_int, [_c_int_p, _c_int_p, _c_int_p, _c_int_p]),
    "hybridxbsoftrih_": (ctypes.c_int, [_c_int_p, _c_int_p, _c_int_p, _c_dbl_p, _c_int_p,
                                        _c_dbl_p, _c_dbl_p, _c_int_p, _c_int_p]),
    "hybridxbsoih_": (ctypes.c_int, [_c_int_p, _c_int_p, _c_int_p, _c_dbl_p, _c_int_p,
                                     _c_dbl_p, _c_dbl_p, _c_int_p, _c_int_p]),
    "hybridxfinalizeh_": (ctypes.c_int, [_c_int_p]),
    "fgetwalltime_": (None, [_c_dbl_p]),
    "felapsed_": (ctypes.c_double, [_c_dbl_p, _c_dbl_p]),
    "lapackXbsofiLWork": (ctypes.c_int, [ctypes.c_int] * 3),
    "lapackXbsof": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, _c_dbl_p, ctypes.c_int, _c_dbl_p,
                                   _c_dbl_p, ctypes.c_int, _c_int_p]),
    "lapackXbstri": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, _c_dbl_p, ctypes.c_int, _c_int_p]),
    "lapackXbsoi_ormqr": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, _c_dbl_p, ctypes.c_int,
                                         _c_dbl_p, _c_dbl_p, ctypes.c_int, _c_int_p]),
    "lapackXbsoi_orgqr": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, _c_dbl_p, ctypes.c_int,
                                         _c_dbl_p, _c_dbl_p, ctypes.c_int, _c_int_p]),
    "hybridXbsofiLWork": (ctypes.c_int, [ctypes.c_int] * 4),
    "hybridxbsofilwork_": (ctypes.c_int, [_c_int_p] * 4),
    "hybridxbsoftri_": (ctypes.c_int, [_c_int_p, _c_int_p, _c_dbl_p, _c_int_p, _c_dbl_p, _c_dbl_p,
                                       _c_int_p, _c_dbl_p, _c_int_p, _c_int_p]),
    "hybridxbsoi_": (ctypes.c_int, [_c_int_p, _c_int_p, _c_dbl_p, _c_int_p, _c_dbl_p, _c_dbl_p,
                                    _c_int_p, _c_dbl_p, _c_int_p, _c_int_p]),
    "hybridXbsoftri": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, ctypes.c_int, _c_dbl_p,
                                      ctypes.c_int, _c_dbl_p, _c_dbl_p, ctypes.c_int, _c_dbl_p,
                                      ctypes.c_int, _c_int_p]),
    "hybridXbsoi": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, ctypes.c_int, _c_dbl_p,
                                   ctypes.c_int, _c_dbl_p, _c_dbl_p, ctypes.c_int, _c_dbl_p,
                                   ctypes.c_int, _c_int_p]),
    "gpuXbsof": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, _vp, ctypes.c_int, _c_dbl_p,
                                _c_dbl_p, ctypes.c_int, _vp, _c_int_p]),
    "gpuXbstri_rseq": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, _vp, ctypes.c_int, _vp,
                                      ctypes.c_int, _c_int_p]),
    "gpuXbstri_rbatched": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, _vp, ctypes.c_int, _vp,
                                          ctypes.c_int, _c_int_p]),
    "gpuXbsoi_ormqr": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, _vp, ctypes.c_int, _c_dbl_p,
                                      _c_dbl_p, ctypes.c_int, _vp, _vp, ctypes.c_int, _c_int_p]),
    "gpuXbsoi_orgqr": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, _vp, ctypes.c_int, _c_dbl_p,
                                      _c_dbl_p, ctypes.c_int, _vp, _vp, ctypes.c_int, _c_int_p]),
    "lapackxbsofilwork_": (ctypes.c_int, [_c_int_p] * 3),
    "lapackxbsof_": (ctypes.c_int, [_c_int_p, _c_int_p, _c_dbl_p, _c_int_p, _c_dbl_p, _c_dbl_p,
                                    _c_int_p, _c_int_p]),
    "lapackxbstri_": (ctypes.c_int, [_c_int_p, _c_int_p, _c_dbl_p, _c_int_p, _c_int_p]),
    "lapackxbsoi_ormqr_": (ctypes.c_int, [_c_int_p, _c_int_p, _c_dbl_p, _c_int_p, _c_dbl_p,
                                          _c_dbl_p, _c_int_p, _c_int_p]),
    "lapackxbsoi_orgqr_": (ctypes.c_int, [_c_int_p, _c_int_p, _c_dbl_p, _c_int_p, _c_dbl_p,
                                          _c_dbl_p, _c_int_p, _c_int_p]),
    "gpuXbsoi_batched": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, _vp, ctypes.c_int, _c_dbl_p,
                                        _c_dbl_p, ctypes.c_int, _vp, _vp, ctypes.c_int,
                                        _c_int_p]),
    "bsofi_device_workspace_bytes": (ctypes.c_ulonglong, [ctypes.c_int] * 3),
    "bsofi_device_invert": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, _vp, ctypes.c_int, _vp,
                                           _vp, _vp]),
    "bsofi_device_bsoftri": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, _vp, ctypes.c_int, _vp,
                                            _vp, _vp]),
    "bsofi_device_bsoi": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, _vp, ctypes.c_int, _vp,
                                         _vp, _vp]),
    "bsofi_device_bsoi_rows": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, _vp, ctypes.c_int, _vp,
                                              _vp, ctypes.c_int, ctypes.c_int, _vp]),
    "bsofi_device_info": (_vp, [_vp]),
    "bsofi_device_workspace_bytes_mixed": (ctypes.c_ulonglong, [ctypes.c_int] * 4),
    "bsofi_device_invert_mixed": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, _vp, ctypes.c_int,
                                                 _vp, _vp, ctypes.c_int, _vp]),
    "bsofi_selftest_ozaki_scratch_bytes": (ctypes.c_ulonglong, [ctypes.c_int] * 4),
    "bsofi_selftest_ozaki": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, ctypes.c_int, _vp,
                                            ctypes.c_int, _vp, ctypes.c_int, _vp, ctypes.c_int,
                                            ctypes.c_int, _vp, _vp, _vp]),
    "bsofi_device_last_launches": (ctypes.c_longlong, []),
    "bsofi_batch_workspace_bytes": (ctypes.c_ulonglong, [ctypes.c_int, _vp, _vp, _vp]),
    "bsofi_batch_workspace_bytes_ex": (ctypes.c_ulonglong, [ctypes.c_int, _vp, _vp, _vp,
                                                            ctypes.c_int]),
    "bsofi_device_invert_batched_ex": (ctypes.c_int, [ctypes.c_int, _vp, _vp, _vp, _vp, _vp, _vp,
                                                      ctypes.c_int, ctypes.c_int, _vp]),
    "bsofi_device_invert_batched": (ctypes.c_int, [ctypes.c_int, _vp, _vp, _vp, _vp, _vp, _vp,
                                                   ctypes.c_int, _vp]),
    "bsofi_batch_graph_create": (_vp, [ctypes.c_int, _vp, _vp, _vp, _vp, _vp, _vp, ctypes.c_int]),
    "bsofi_batch_graph_launch": (ctypes.c_int, [_vp, _vp]),
    "bsofi_batch_graph_destroy": (None, [_vp]),
    "bsofi_autotune": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, ctypes.c_int, _vp, _vp]),
    "bsofi_plan_get": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, _vp]),
    "bsofi_plan_set": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, _vp]),
    "bsofi_plan_clear": (None, []),
    "bsofi_server_create": (_vp, [ctypes.c_int, ctypes.c_ulonglong]),
    "bsofi_server_request_bytes": (ctypes.c_ulonglong, [ctypes.c_int] * 3),
    "bsofi_server_submit": (ctypes.c_longlong, [_vp, ctypes.c_int, ctypes.c_int, _vp, ctypes.c_int,
                                                _vp, ctypes.c_int]),
    "bsofi_server_footprint_bytes": (ctypes.c_ulonglong, [ctypes.c_int] * 3),
    "bsofi_server_submit_blocks": (ctypes.c_longlong, [_vp, ctypes.c_int, ctypes.c_int, _vp, _vp,
                                                       ctypes.c_int]),
    "bsofi_server_result": (ctypes.c_int, [_vp, ctypes.c_longlong, _vp, _c_int_p, _vp]),
    "bsofi_server_release": (ctypes.c_int, [_vp, ctypes.c_longlong]),
    "bsofi_server_poll": (ctypes.c_int, [_vp, _vp, _vp, ctypes.c_int]),
    "bsofi_server_pending": (ctypes.c_int, [_vp]),
    "bsofi_server_destroy": (None, [_vp]),
    "bsofi_device_assemble": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, _vp, _vp, _vp,
                                             ctypes.c_int, _vp]),
    "bsofi_device_hubbard_assemble": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, _vp, _vp,
                                                     ctypes.c_double, _vp, ctypes.c_int, _vp]),
    "bsofi_device_logdet": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, _vp, ctypes.c_int, _vp,
                                           ctypes.c_int, _vp, _vp]),
    "bsofi_shard_state_bytes": (ctypes.c_ulonglong, [ctypes.c_int] * 2),
    "bsofi_shard_factor": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, _vp, _vp, _vp, _vp]),
    "bsofi_shard_hubbard_factor": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, _vp, _vp,
                                                  ctypes.c_double, _vp, _vp]),
    "bsofi_shard_bstri_columns": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                                 ctypes.c_int, _vp, ctypes.c_longlong, _vp, _vp]),
    "bsofi_shard_bsoi_rows": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                             ctypes.c_int, _vp, ctypes.c_longlong, _vp, _vp]),
    "bsofi_shard_logdet": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, _vp, _vp, _vp]),
    "bsofi_shard_info": (_vp, [_vp]),
    "bsofi_shard_tau": (_vp, [_vp, ctypes.c_int, ctypes.c_int]),
    "bsofi_noalloc_scratch_bytes": (ctypes.c_ulonglong, []),
    "bsofi_noalloc_prepare": (ctypes.c_int, []),
    "bsofi_device_invert_noalloc": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, _vp, ctypes.c_int,
                                                   _vp, _vp, _vp]),
    "bsofi_device_bsof_timeline": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, ctypes.c_int, _vp,
                                                  _vp, ctypes.c_int]),
    "bsofi_device_set_bsof_workers": (None, [ctypes.c_int]),
    "bsofi_device_set_bsof_factor_warps": (None, [ctypes.c_int]),
    "bsofi_device_set_batch_grouped": (None, [ctypes.c_int]),
    "bsofi_device_set_batch_chains": (None, [ctypes.c_int]),
    "bsofi_device_set_batch_pipelined": (None, [ctypes.c_int]),
    "bsofi_device_set_batch_workers": (None, [ctypes.c_int]),
    "bsofi_device_set_gemm_k16": (None, [ctypes.c_int]),
    "bsofi_device_set_bsoi_tma": (None, [ctypes.c_int]),
    "bsofi_device_set_wait_test": (None, [ctypes.c_int]),
    "bsofi_device_set_bstri_overlap": (None, [ctypes.c_int]),
    "bsofi_device_timing": (None, [ctypes.c_int]),
    "bsofi_device_timing_read": (ctypes.c_int, [_c_dbl_p, ctypes.POINTER(ctypes.c_longlong)]),
    "bsofi_selftest_gemm": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                           ctypes.c_double, _vp, ctypes.c_int, ctypes.c_int,
                                           _vp, ctypes.c_int, ctypes.c_int, ctypes.c_double,
                                           _vp, ctypes.c_int, ctypes.c_int, _vp]),
}

_lib = None


def declared_symbols(header=HEADER):
    """Function names declared in include/bsofi_b200.h."""
    text = open(header).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"^\s*(?:unsigned\s+long\s+long|long\s+long|int\s*\*?|(?:const\s+)?double|void|bsofi_\w+)\s*\*?\s*(\w+)\s*\(",
                                 text, flags=re.M)))


def load():
    """Load the library (once).  Raises if it is missing."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError("libbsofi_b200.so is not built (python -m bsofi_b200.build); "
                               "the BSOF/I path has no fallback")
        lib = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in _SIGS.items():
            f = getattr(lib, name)
            f.restype = res
            f.argtypes = args
        _lib = lib
    return _lib
