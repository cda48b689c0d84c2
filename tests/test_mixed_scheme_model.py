"""Numpy models of the mixed form's tensor-core product Y = F X, the
products A_hi X_hi + A_hi X_lo + A_lo X_hi summed in FP32 per 32-column slab
of F and the slabs summed in FP64, for two operand formats of 4 bytes per
entry:

* scaled FP16 pairs (the kernel's form): F and every column of X scaled by a
  power of two below 2^14, each split into FP16 hi + lo;
* 3xTF32 (the form it replaced): F stored in FP32, whose value serves as A_hi
  (a TF32 operand's low 13 bits do not enter the product) plus the rounded
  remainder A_lo, X split into TF32 parts X_hi + X_lo.

What it pins: both schemes' error is at FP32 level (a few 1e-7 relative:
the dropped A_lo X_lo term, about 2^-22, FP32 accumulation inside a slab and
the 4-byte storage of F), while a single TF32 product is ~5e-4 — the level
at which the GPU operator tests fail when the remainder terms are missing —
which is why the kernel issues three products."""
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


def pow2_exponent(m, mult=1.0):
    """The exponent E that scales values of magnitude <= m * mult to at most
    2^14 (a quarter of the FP16 range): m * mult = f 2^e, f in [0.5, 1),
    E = 14 - e; 0 for an all-zero operand."""
    m = float(m) * mult
    if not m > 0.0:
        return 0
    _, e = np.frexp(m)
    return 14 - int(e)


def f16_pair(v):
    """v (FP64, already scaled) as FP16 hi + FP16 lo, both rounded to nearest."""
    hi = v.astype(np.float16)
    lo = (v - hi.astype(np.float64)).astype(np.float16)
    return hi, lo


def model_product_f16(F, X, nent=1.0):
    """The FP16-pair form of the product: F scaled by one power of two per
    matrix, every column of X by one power of two from its maximum times the
    bound nent, each split into FP16 hi + lo planes (4 bytes per entry, like
    FP32), products A_hi X_hi + A_hi X_lo + A_lo X_hi (exact in FP32) summed in
    FP32 per 32-column slab, slabs summed and unscaled in FP64."""
    ea = pow2_exponent(np.abs(F).max())
    ex = np.array([pow2_exponent(np.abs(X[:, j]).max(), nent) for j in range(X.shape[1])])
    A_hi, A_lo = f16_pair(np.ldexp(F, ea))
    X_hi, X_lo = f16_pair(np.ldexp(X, ex[None, :]))
    A_hi, A_lo, X_hi, X_lo = (a.astype(np.float32) for a in (A_hi, A_lo, X_hi, X_lo))
    Y = np.zeros((F.shape[0], X.shape[1]))
    for k0 in range(0, F.shape[1], 32):
        s = slice(k0, k0 + 32)
        acc = A_hi[:, s] @ X_hi[s] + A_hi[:, s] @ X_lo[s] + A_lo[:, s] @ X_hi[s]
        Y += acc.astype(np.float64)
    return np.ldexp(Y, -(ea + ex)[None, :])


def test_pow2_exponent_keeps_fp16_in_range():
    for m in (1e-300, 3e-9, 0.7, 1.0, 2.0 ** 14, 6e12):
        e = pow2_exponent(m, 8.0)
        assert 2.0 ** 13 <= np.ldexp(m * 8.0, e) < 2.0 ** 14
    assert pow2_exponent(0.0) == 0


def test_fp16_pairs_reach_the_accuracy_of_three_tf32_products():
    """Same operands as the 3xTF32 model: the FP16-pair form with power-of-two
    scales is at FP32 level too, also when the columns of X span many orders of
    magnitude and the scale is taken from a bound 8x above their maximum."""
    F = _local_schur_like(256, 1)
    X = np.random.default_rng(2).normal(size=(256, 32))
    X[:, 1] *= np.logspace(-10, 0, 256)
    X[:, 2] *= 1e-200
    exact = F @ X
    three = rel(model_product(F, X, 3), exact)
    pair = rel(model_product_f16(F, X, nent=8.0), exact)
    assert pair < 5e-7 and pair < 2 * three
    got = model_product_f16(F, X, nent=8.0)
    for j in (1, 2):                        # max norms: the 1e-200 column's 2-norm underflows
        assert np.abs(got[:, j] - exact[:, j]).max() < 5e-7 * np.abs(exact[:, j]).max()
