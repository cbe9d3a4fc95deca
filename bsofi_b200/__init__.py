"""bsofi_b200 -- B200-native BSOF/I (block structured orthogonal factorization
and inversion of block p-cyclic matrices).

The product is the C ABI library ``libbsofi_b200.so`` (include/bsofi_b200.h):
host C over hand-written sm_100a CUDA kernels.  This package builds it
(``bsofi_b200.build``), binds it (``bsofi_b200.api``) and generates inputs
(``bsofi_b200.hubbard``).
"""
from . import hubbard  # noqa: F401
from .flops import bsofi_flops, flops_bsof, flops_bsoi, flops_bstri  # noqa: F401
