"""Generate the golden BSOF/I fixtures from the reference's own CPU path.

Runs in the build container, where oracle/_ref/libbsofi_ref.so (and its
single-precision twin libbsofi_ref_fp32.so) are compiled from the reference
sources (oracle/Makefile).  For every case it stores the p-cyclic input
blocks, the state after the reference's hybridxbsoftrih_ (reflectors +
R^{-1}, tau, info) and the inverse after hybridxbsoih_.  The FP32 cases
(tests/golden/fp32/) hold the same for the single-precision build, whose
input is the FP64 matrix rounded to float32.

    python tests/golden/make_golden.py [--fp32-only]
"""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

import oracle  # noqa: E402
from bsofi_b200.hubbard import hubbard_matrix, pcyclic_blocks, random_pcyclic  # noqa: E402

# (name, n, L, kind, seed, extra)
CASES = [
    ("rand_n1_L2", 1, 2, "rand", 11, {}),
    ("rand_n2_L3", 2, 3, "rand", 12, {}),
    ("rand_n3_L4", 3, 4, "rand", 13, {}),
    ("rand_n5_L4", 5, 4, "rand", 14, {}),
    ("rand_n8_L2", 8, 2, "rand", 15, {}),
    ("rand_n7_L16", 7, 16, "rand", 16, {}),
    ("rand_n17_L5", 17, 5, "rand", 17, {}),
    ("hub_s2_L3", 4, 3, "hub", 21, {"side": 2, "U": 4.0}),
    ("hub_s2_L5", 4, 5, "hub", 22, {"side": 2, "U": 4.0}),
    ("hub_s3_L4", 9, 4, "hub", 23, {"side": 3, "U": 2.0}),
    ("hub_s4_L8", 16, 8, "hub", 24, {"side": 4, "U": 6.0}),
    ("hub_s3_L12", 9, 12, "hub", 25, {"side": 3, "U": 4.0}),
]


# Cases of the single-precision build (names as above).
CASES_FP32 = ["rand_n1_L2", "rand_n5_L4", "rand_n17_L5", "hub_s2_L5", "hub_s3_L4", "hub_s4_L8",
              "hub_s3_L12"]


def case_matrix(n, L, kind, seed, extra):
    if kind == "hub":
        return hubbard_matrix(extra["side"], L, extra["U"], seed=seed)
    return random_pcyclic(n, L, seed=seed)


def make_fp32(path=os.path.join(os.path.dirname(os.path.abspath(__file__)), "fp32")):
    os.makedirs(path, exist_ok=True)
    oracle.set_ref_threads(1, kind="ref32")
    for name, n, L, kind, seed, extra in CASES:
        if name not in CASES_FP32:
            continue
        M = case_matrix(n, L, kind, seed, extra).astype(np.float32)
        diag, sub = (b.astype(np.float32) for b in pcyclic_blocks(M, n, L))
        A, tau, info = oracle.ref32_bsoftri(M, n, L)
        X, info2 = oracle.ref32_bsoi(A, tau, n, L)
        np.savez_compressed(os.path.join(path, name + ".npz"), n=n, L=L, diag=diag, sub=sub,
                            state=A, tau=tau, info=info, inverse=X)
        print("fp32", name, "info", info, info2)


def make(path=os.path.dirname(os.path.abspath(__file__))):
    oracle.set_ref_threads(1)
    for name, n, L, kind, seed, extra in CASES:
        M = case_matrix(n, L, kind, seed, extra)
        diag, sub = pcyclic_blocks(M, n, L)
        A, tau, info = oracle.ref_bsoftri(M, n, L)
        X, info2 = oracle.ref_bsoi(A, tau, n, L)
        np.savez_compressed(os.path.join(path, name + ".npz"), n=n, L=L, diag=diag, sub=sub,
                            state=A, tau=tau, info=info, inverse=X)
        print(name, "info", info, info2)


if __name__ == "__main__":
    if not (oracle.ref_available() and oracle.ref32_available()):
        raise SystemExit("oracle/_ref/libbsofi_ref*.so missing: run make -C oracle")
    if "--fp32-only" not in sys.argv:
        make()
    make_fp32()
