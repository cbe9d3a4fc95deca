"""CPU checks of the numpy restatement of the int8 tensor-core product:
the slices reconstruct each row to 7 S bits, and the product's error against
FP64 falls by about 2^7 per slice."""
import numpy as np

from ozaki_emul import ozaki_product, split_rows


def test_slices_reconstruct_rows():
    rng = np.random.default_rng(0)
    A = rng.standard_normal((40, 33)) * np.exp(rng.uniform(-20, 20, (40, 1)))
    A[3] = 0.0
    for S in (3, 5, 8):
        e, sl = split_rows(A, S)
        assert all(np.abs(s).max() <= 127 for s in sl)
        rec = sum(s * np.ldexp(1.0, -7 * (i + 1)) for i, s in enumerate(sl))
        rec = np.ldexp(rec, e[:, None])
        bound = np.ldexp(1.0, e - 7 * S)[:, None]
        assert (np.abs(rec - A) < bound + 0.0).all()
        assert (rec[3] == 0).all()


def test_product_accuracy_per_slice():
    rng = np.random.default_rng(1)
    A = rng.standard_normal((64, 96))
    B = rng.standard_normal((96, 48))
    C = A @ B
    errs = []
    for S in (3, 4, 5, 6, 7, 8):
        errs.append(np.linalg.norm(ozaki_product(A, B, S) - C) / np.linalg.norm(C))
    assert errs[-1] < 1e-15
    for a, b in zip(errs, errs[1:]):
        assert b < a / 30 or b < 1e-15
