"""A numpy model of the mixed form's tensor-core product, Y = F X with F
stored in FP32: X split into TF32 parts X_hi + X_lo, F's FP32 value used as
A_hi (a TF32 operand's low 13 bits do not enter the product) plus the
rounded remainder A_lo, the products A_hi X_hi + A_hi X_lo + A_lo X_hi summed
in FP32 per 32-column slab of F and the slabs summed in FP64.

What it pins: the scheme's error is at FP32 level (a few 1e-7 relative:
the dropped A_lo X_lo term, about 2^-22, FP32 accumulation inside a slab and
FP32 storage of F), while a single TF32 product is ~5e-4 — the level at
which the GPU operator tests fail when the remainder terms are missing —
which is why the kernel issues three."""
import numpy as np


def tf32_rna(a):
    """FP32 -> TF32 (10 explicit mantissa bits), round to nearest, ties away
    from zero: add half an ulp of TF32 to the magnitude bits, clear the low 13."""
    b = np.ascontiguousarray(a, dtype=np.float32).view(np.uint32)
    return ((b + np.uint32(0x1000)) & np.uint32(0xFFFFE000)).view(np.float32)


def tf32_trunc(a):
    b = np.ascontiguousarray(a, dtype=np.float32).view(np.uint32)
    return (b & np.uint32(0xFFFFE000)).view(np.float32)


def model_product(F, X, terms=3):
    A = F.astype(np.float32)
    A_hi = tf32_trunc(A)                                    # what the MMA reads of the FP32 slab
    A_lo = tf32_rna(A - A_hi)
    X_hi = tf32_rna(X.astype(np.float32))
    X_lo = tf32_rna((X - X_hi.astype(np.float64)).astype(np.float32))
    Y = np.zeros((F.shape[0], X.shape[1]))
    for k0 in range(0, F.shape[1], 32):                     # one FP32 accumulator per slab
        s = slice(k0, k0 + 32)
        acc = A_hi[:, s] @ X_hi[s]
        if terms == 3:
            acc = acc + A_hi[:, s] @ X_lo[s] + A_lo[:, s] @ X_hi[s]
        Y += acc.astype(np.float64)
    return Y


def _local_schur_like(n, seed):
    """A dense SPD inverse with the spread of magnitudes of an explicit F_i."""
    rng = np.random.default_rng(seed)
    Q, _ = np.linalg.qr(rng.normal(size=(n, n)))
    K = (Q * np.logspace(0, 4, n)) @ Q.T
    return np.linalg.inv(K + K.T) * 1e3


def rel(a, b):
    return np.linalg.norm(a - b) / np.linalg.norm(b)


def test_tf32_rounding_helpers():
    x = np.array([1.0 + 2.0 ** -11, 1.0 + 3 * 2.0 ** -11, -(1.0 + 2.0 ** -11), 1.0 + 2.0 ** -12], np.float32)
    # ties go away from zero; below half an ulp rounds down
    assert np.array_equal(tf32_rna(x), np.array([1.0 + 2.0 ** -10, 1.0 + 2 * 2.0 ** -10, -(1.0 + 2.0 ** -10), 1.0],
                                                np.float32))
    assert np.array_equal(tf32_trunc(x)[:2], np.array([1.0, 1.0 + 2.0 ** -10], np.float32))


def test_three_products_reach_fp32_level_accuracy():
    F = _local_schur_like(256, 1)
    X = np.random.default_rng(2).normal(size=(256, 32))
    exact = F @ X
    storage = rel(F.astype(np.float32).astype(np.float64) @ X, exact)
    three = rel(model_product(F, X, 3), exact)
    one = rel(model_product(F, X, 1), exact)
    assert storage < three < 5e-7                           # FP32-level accuracy
    assert 1e-4 < one and one > 100 * three                 # a single TF32 product is far worse
