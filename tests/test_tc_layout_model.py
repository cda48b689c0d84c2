"""A CPU model of the tensor-core product's shared-memory layouts: the
FP16-pair slab planes as k_make_slabs writes them, the X planes as
k_gather_multi writes them, the pieces the producer of k_tc_gemm copies for
a K step above the diagonal, and the operand reads of tcgen05.mma through
the canonical SWIZZLE_64B layouts its descriptors name (K-major: 8-row
groups of 64-byte rows, SBO = 512 B between groups, a K step of 16 is
32 bytes along a row; MN-major: 64-byte rows of 32 consecutive M elements,
LBO = 2 KB between the four 32-row pieces, SBO = 512 B between groups of 8 K
indices, a K step of 16 is 1 KB).  Both K-step kinds must read A(m, k) of
the symmetric matrix, and the X operand X(k, j), with every byte inside its
plane.  The arithmetic mirrors tc_gemm.cu and pcpg_multi.cu; what the model
cannot pin is the hardware's reading of the descriptors, which the GPU
operator tests check."""
import numpy as np

PLANE = 8192          # bytes of one plane of a 128 x 32 slab (128 rows x 64 B)
PIECE = 2048          # bytes of 32 stored rows of one plane


def swz64(b):
    """SWIZZLE_64B: the 16-byte granule (bits 4-5) XOR address bits 7-8."""
    return b ^ (((b >> 7) & 3) << 4)


def write_plane(block):
    """rows x 32 values -> plane bytes (as an element array indexed by byte / 2)."""
    rows = block.shape[0]
    plane = np.zeros(rows * 32, dtype=np.int64)
    for r in range(rows):
        for c in range(32):
            plane[swz64(r * 64 + c * 2) // 2] = block[r, c]
    return plane


def read_kmajor(smem, rows, kstep):
    """Operand (row, k) for k < 16 of K step kstep through a K-major SW64 descriptor."""
    out = np.zeros((rows, 16), dtype=np.int64)
    for m in range(rows):
        for k in range(16):
            pre = 32 * kstep + (m % 8) * 64 + (m // 8) * 512 + k * 2
            assert pre < len(smem) * 2
            out[m, k] = smem[swz64(pre) // 2]
    return out


def read_mnmajor(smem, kstep, lbo=PIECE, sbo=512):
    """Operand (m, k), m < 128, k < 16 of K step kstep through an MN-major SW64 descriptor."""
    out = np.zeros((128, 16), dtype=np.int64)
    for m in range(128):
        for k in range(16):
            pre = 1024 * kstep + (m % 32) * 2 + (m // 32) * lbo + (k % 8) * 64 + (k // 8) * sbo
            assert pre < PLANE
            out[m, k] = smem[swz64(pre) // 2]
    return out


def test_direct_and_transposed_k_steps_read_the_symmetric_matrix():
    rng = np.random.default_rng(0)
    n = 384                                            # three 128-row blocks
    A = rng.integers(-1000, 1000, size=(n, n))
    A = A + A.T
    # stored slabs: block mb keeps K slabs kk < 4 (mb + 1) (one plane modelled)
    stored = {(mb, kk): write_plane(A[128 * mb:128 * mb + 128, 32 * kk:32 * kk + 32])
              for mb in range(3) for kk in range(4 * (mb + 1))}
    ks = n // 32
    for m in range(3):
        for kk in range(ks):
            if kk < 4 * (m + 1):                       # stored slab, one bulk copy
                smem = stored[(m, kk)]
                for q in range(2):
                    got = read_kmajor(smem, 128, q)
                    assert np.array_equal(got, A[128 * m:128 * m + 128, 32 * kk + 16 * q:32 * kk + 16 * q + 16])
            else:                                      # four 2 KB pieces of the slabs below
                mp, q = kk >> 2, kk & 3
                smem = np.zeros(PLANE // 2, dtype=np.int64)
                for p in range(4):
                    src = stored[(mp, 4 * m + p)]
                    smem[p * PIECE // 2:(p + 1) * PIECE // 2] = src[q * PIECE // 2:(q + 1) * PIECE // 2]
                for kst in range(2):
                    got = read_mnmajor(smem, kst)
                    c0 = 32 * kk + 16 * kst
                    assert np.array_equal(got, A[128 * m:128 * m + 128, c0:c0 + 16])


def test_x_planes_read_as_the_b_operand():
    rng = np.random.default_rng(1)
    for K in (16, 32):
        X = rng.integers(-100, 100, size=(32, K))      # 32 slots x K load cases
        hi = write_plane(X.T)                          # rows = load cases, 64 B each
        lo = write_plane(-X.T)
        smem = np.concatenate([hi, lo])                # X_hi rows, then X_lo rows: the N = 2K operand
        assert len(smem) * 2 == K * 128
        for q in range(2):
            got = read_kmajor(smem, 2 * K, q)          # B(n, k): n < 2K load-case rows
            assert np.array_equal(got[:K], X[16 * q:16 * q + 16].T)
            assert np.array_equal(got[K:], -X[16 * q:16 * q + 16].T)
