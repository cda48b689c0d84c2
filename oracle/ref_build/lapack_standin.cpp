// Stand-ins for the LAPACKE routines and the METIS entry point that the
// reference links against (MKL and METIS are not in this image).  Written
// from the LAPACK interface descriptions; dense, column-major, FP64.
//   dpotrf/dpotri : Cholesky and inverse from it        (Cluster.cpp:1254,1260)
//   dspev         : symmetric eigen-decomposition, packed (Matrix.cpp:1489,2352)
//   dgesvd        : singular values only                (Matrix.cpp:1526)
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <vector>
#include <algorithm>
#include "shim/mkl.h"
#include "shim/metis.h"

extern "C" int LAPACKE_dpotrf(int layout, char uplo, int n, double *a, int lda) {
    if (layout != LAPACK_COL_MAJOR || (uplo != 'L' && uplo != 'l')) return -1;
    for (int j = 0; j < n; ++j) {
        double d = a[j + j * lda];
        for (int k = 0; k < j; ++k) d -= a[j + k * lda] * a[j + k * lda];
        if (!(d > 0.0)) return j + 1;
        d = std::sqrt(d);
        a[j + j * lda] = d;
        for (int i = j + 1; i < n; ++i) {
            double s = a[i + j * lda];
            for (int k = 0; k < j; ++k) s -= a[i + k * lda] * a[j + k * lda];
            a[i + j * lda] = s / d;
        }
    }
    return 0;
}

extern "C" int LAPACKE_dpotri(int layout, char uplo, int n, double *a, int lda) {
    if (layout != LAPACK_COL_MAJOR || (uplo != 'L' && uplo != 'l')) return -1;
    // W = L^{-1} (lower), then A^{-1} = W^T W, lower triangle written back.
    std::vector<double> W(size_t(n) * n, 0.0);
    for (int j = 0; j < n; ++j) {
        W[j + j * n] = 1.0 / a[j + j * lda];
        for (int i = j + 1; i < n; ++i) {
            double s = 0.0;
            for (int k = j; k < i; ++k) s += a[i + k * lda] * W[k + j * n];
            W[i + j * n] = -s / a[i + i * lda];
        }
    }
    for (int j = 0; j < n; ++j)
        for (int i = j; i < n; ++i) {
            double s = 0.0;
            for (int k = i; k < n; ++k) s += W[k + i * n] * W[k + j * n];
            a[i + j * lda] = s;
        }
    return 0;
}

// Cyclic Jacobi eigen-decomposition of a dense symmetric n x n matrix A
// (column-major, overwritten); eigenvalues in w (unsorted), vectors in V.
static void jacobi_eig(int n, std::vector<double> &A, std::vector<double> &w, std::vector<double> &V) {
    V.assign(size_t(n) * n, 0.0);
    for (int i = 0; i < n; ++i) V[i + i * n] = 1.0;
    for (int sweep = 0; sweep < 100; ++sweep) {
        double off = 0.0, tot = 0.0;
        for (int j = 0; j < n; ++j)
            for (int i = 0; i < n; ++i) {
                double v = A[i + j * n] * A[i + j * n];
                tot += v;
                if (i != j) off += v;
            }
        if (off <= 1e-30 * tot || off == 0.0) break;
        for (int p = 0; p < n - 1; ++p)
            for (int q = p + 1; q < n; ++q) {
                double apq = A[p + q * n];
                if (apq == 0.0) continue;
                double app = A[p + p * n], aqq = A[q + q * n];
                double theta = (aqq - app) / (2.0 * apq);
                double t = (theta >= 0 ? 1.0 : -1.0) / (std::fabs(theta) + std::sqrt(theta * theta + 1.0));
                double c = 1.0 / std::sqrt(t * t + 1.0), s = t * c;
                for (int k = 0; k < n; ++k) {       // A <- A J (columns p,q)
                    double akp = A[k + p * n], akq = A[k + q * n];
                    A[k + p * n] = c * akp - s * akq;
                    A[k + q * n] = s * akp + c * akq;
                }
                for (int k = 0; k < n; ++k) {       // A <- J^T A (rows p,q)
                    double apk = A[p + k * n], aqk = A[q + k * n];
                    A[p + k * n] = c * apk - s * aqk;
                    A[q + k * n] = s * apk + c * aqk;
                }
                for (int k = 0; k < n; ++k) {
                    double vkp = V[k + p * n], vkq = V[k + q * n];
                    V[k + p * n] = c * vkp - s * vkq;
                    V[k + q * n] = s * vkp + c * vkq;
                }
            }
    }
    w.resize(n);
    for (int i = 0; i < n; ++i) w[i] = A[i + i * n];
}

extern "C" int LAPACKE_dspev(int layout, char jobz, char uplo, int n, double *ap, double *w,
                             double *z, int ldz) {
    if (layout != LAPACK_COL_MAJOR || (uplo != 'U' && uplo != 'u')) return -1;
    std::vector<double> A(size_t(n) * n), ev, V;
    for (int j = 0; j < n; ++j)
        for (int i = 0; i <= j; ++i) {
            double v = ap[i + size_t(j) * (j + 1) / 2];
            A[i + j * n] = v;
            A[j + i * n] = v;
        }
    jacobi_eig(n, A, ev, V);
    std::vector<int> idx(n);
    for (int i = 0; i < n; ++i) idx[i] = i;
    std::sort(idx.begin(), idx.end(), [&](int a, int b) { return ev[a] < ev[b]; });
    for (int i = 0; i < n; ++i) {
        w[i] = ev[idx[i]];
        if (jobz == 'V' || jobz == 'v')
            for (int k = 0; k < n; ++k) z[k + size_t(i) * ldz] = V[k + idx[i] * n];
    }
    return 0;
}

// One-sided Jacobi: singular values of the m x n matrix (only S is consumed
// by the reference); U and VT are left zeroed.
extern "C" int LAPACKE_dgesvd(int layout, char, char, int m, int n, double *a, int lda,
                              double *s, double *u, int ldu, double *vt, int ldvt, double *) {
    // Treat the data as column-major C (rows x cols); singular values are the
    // same for a matrix and its transpose, so the layout only fixes strides.
    int rows = (layout == LAPACK_ROW_MAJOR) ? n : m;
    int cols = (layout == LAPACK_ROW_MAJOR) ? m : n;
    std::vector<double> C(size_t(rows) * cols);
    for (int j = 0; j < cols; ++j)
        for (int i = 0; i < rows; ++i) C[i + size_t(j) * rows] = a[i + size_t(j) * lda];
    for (int sweep = 0; sweep < 100; ++sweep) {
        double maxrot = 0.0;
        for (int p = 0; p < cols - 1; ++p)
            for (int q = p + 1; q < cols; ++q) {
                double alpha = 0, beta = 0, gamma = 0;
                for (int k = 0; k < rows; ++k) {
                    double x = C[k + size_t(p) * rows], y = C[k + size_t(q) * rows];
                    alpha += x * x; beta += y * y; gamma += x * y;
                }
                if (gamma == 0.0) continue;
                double r = std::fabs(gamma) / std::sqrt(alpha * beta);
                if (r > maxrot) maxrot = r;
                double zeta = (beta - alpha) / (2.0 * gamma);
                double t = (zeta >= 0 ? 1.0 : -1.0) / (std::fabs(zeta) + std::sqrt(1.0 + zeta * zeta));
                double c = 1.0 / std::sqrt(1.0 + t * t), sn = c * t;
                for (int k = 0; k < rows; ++k) {
                    double x = C[k + size_t(p) * rows], y = C[k + size_t(q) * rows];
                    C[k + size_t(p) * rows] = c * x - sn * y;
                    C[k + size_t(q) * rows] = sn * x + c * y;
                }
            }
        if (maxrot < 1e-15) break;
    }
    std::vector<double> sv(cols);
    for (int j = 0; j < cols; ++j) {
        double t = 0;
        for (int k = 0; k < rows; ++k) t += C[k + size_t(j) * rows] * C[k + size_t(j) * rows];
        sv[j] = std::sqrt(t);
    }
    std::sort(sv.begin(), sv.end(), [](double x, double y) { return x > y; });
    int ns = std::min(m, n);
    for (int i = 0; i < ns; ++i) s[i] = sv[i];
    (void)u; (void)ldu; (void)vt; (void)ldvt;
    return 0;
}

extern "C" int METIS_PartMeshDual(idx_t *, idx_t *, idx_t *, idx_t *, idx_t *, idx_t *, idx_t *,
                                  idx_t *, real_t *, idx_t *, idx_t *, idx_t *, idx_t *) {
    std::fprintf(stderr, "METIS is not available in this build (run with metis=false)\n");
    std::abort();
}
