// Direct-solver stand-in for MKL PARDISO as the reference drives it
// (Matrix.cpp:1115-1327): mtype -2, 0-based upper-triangular CSR input,
// phases 11 (analysis), 22 (numeric factorisation), 33 (solve with
// iparm[7] steps of iterative refinement against the matrix passed at the
// solve) and -1 (release; kept as a no-op so the harness can still apply
// operators after Cluster::initialization returned).
//
// Factorisation: envelope (skyline) Cholesky in the given ordering; if a
// non-positive pivot appears (indefinite saddle-point matrices such as Ac)
// it falls back to dense LU with partial pivoting.  PARDISO equilibrates
// (iparm[10] = 1) before it perturbs pivots (iparm[9] = 8); without that
// scaling a relative 1e-8 threshold would perturb the legitimate small
// Schur pivots of a badly scaled saddle-point matrix, so only numerically
// zero pivots (below 1e-15 * max|a|) are perturbed here.
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>
#include <algorithm>
#include "shim/mkl_pardiso.h"

namespace {
struct Factor {
    int n = 0;
    bool skyline = false;
    std::vector<int> first;              // skyline: first column of row i
    std::vector<size_t> rowptr;          // skyline: start of row i in L
    std::vector<double> L;               // skyline rows, L[rowptr[i] + (j - first[i])]
    std::vector<double> LU;              // dense fallback, column-major
    std::vector<int> piv;
};

void dense_from_csr(int n, const double *a, const int *ia, const int *ja, std::vector<double> &A) {
    A.assign(size_t(n) * n, 0.0);
    for (int i = 0; i < n; ++i)
        for (int k = ia[i]; k < ia[i + 1]; ++k) {
            int j = ja[k];
            A[i + size_t(j) * n] += a[k];
            if (j != i) A[j + size_t(i) * n] += a[k];
        }
}

bool skyline_factor(Factor &F, int n, const double *a, const int *ia, const int *ja) {
    F.first.assign(n, 0);
    for (int i = 0; i < n; ++i) F.first[i] = i;
    for (int r = 0; r < n; ++r)
        for (int k = ia[r]; k < ia[r + 1]; ++k) {
            int c = ja[k];
            int lo = std::min(r, c), hi = std::max(r, c);
            F.first[hi] = std::min(F.first[hi], lo);
        }
    F.rowptr.assign(n + 1, 0);
    for (int i = 0; i < n; ++i) F.rowptr[i + 1] = F.rowptr[i] + size_t(i - F.first[i] + 1);
    F.L.assign(F.rowptr[n], 0.0);
    for (int r = 0; r < n; ++r)
        for (int k = ia[r]; k < ia[r + 1]; ++k) {
            int c = ja[k];
            int hi = std::max(r, c), lo = std::min(r, c);
            F.L[F.rowptr[hi] + (lo - F.first[hi])] += a[k];
        }
    for (int i = 0; i < n; ++i) {
        double *Li = &F.L[F.rowptr[i]];
        int fi = F.first[i];
        for (int j = fi; j < i; ++j) {
            const double *Lj = &F.L[F.rowptr[j]];
            int fj = F.first[j];
            int k0 = std::max(fi, fj);
            double s = Li[j - fi];
            for (int k = k0; k < j; ++k) s -= Li[k - fi] * Lj[k - fj];
            Li[j - fi] = s / Lj[j - fj];
        }
        double d = Li[i - fi];
        for (int k = fi; k < i; ++k) d -= Li[k - fi] * Li[k - fi];
        if (!(d > 0.0)) return false;
        Li[i - fi] = std::sqrt(d);
    }
    F.skyline = true;
    return true;
}

void dense_lu(Factor &F, int n, const double *a, const int *ia, const int *ja) {
    dense_from_csr(n, a, ia, ja, F.LU);
    double amax = 0.0;
    for (double v : F.LU) amax = std::max(amax, std::fabs(v));
    double tiny = 1e-15 * (amax > 0 ? amax : 1.0);
    F.piv.assign(n, 0);
    double *A = F.LU.data();
    for (int k = 0; k < n; ++k) {
        int p = k;
        double pm = std::fabs(A[k + size_t(k) * n]);
        for (int i = k + 1; i < n; ++i) {
            double v = std::fabs(A[i + size_t(k) * n]);
            if (v > pm) { pm = v; p = i; }
        }
        F.piv[k] = p;
        if (p != k)
            for (int j = 0; j < n; ++j) std::swap(A[k + size_t(j) * n], A[p + size_t(j) * n]);
        double d = A[k + size_t(k) * n];
        if (std::fabs(d) < tiny) {
            d = (d < 0 ? -tiny : tiny);
            A[k + size_t(k) * n] = d;
        }
        for (int i = k + 1; i < n; ++i) A[i + size_t(k) * n] /= d;
        for (int j = k + 1; j < n; ++j) {
            double akj = A[k + size_t(j) * n];
            if (akj == 0.0) continue;
            double *cj = A + size_t(j) * n;
            const double *ck = A + size_t(k) * n;
            for (int i = k + 1; i < n; ++i) cj[i] -= akj * ck[i];
        }
    }
    F.skyline = false;
}

void apply_inverse(const Factor &F, double *x) {
    int n = F.n;
    if (F.skyline) {
        for (int i = 0; i < n; ++i) {
            const double *Li = &F.L[F.rowptr[i]];
            int fi = F.first[i];
            double s = x[i];
            for (int k = fi; k < i; ++k) s -= Li[k - fi] * x[k];
            x[i] = s / Li[i - fi];
        }
        for (int i = n - 1; i >= 0; --i) {
            const double *Li = &F.L[F.rowptr[i]];
            int fi = F.first[i];
            x[i] /= Li[i - fi];
            double xi = x[i];
            for (int k = fi; k < i; ++k) x[k] -= Li[k - fi] * xi;
        }
    } else {
        const double *A = F.LU.data();
        for (int k = 0; k < n; ++k) std::swap(x[k], x[F.piv[k]]);
        for (int k = 0; k < n; ++k) {
            double xk = x[k];
            for (int i = k + 1; i < n; ++i) x[i] -= A[i + size_t(k) * n] * xk;
        }
        for (int k = n - 1; k >= 0; --k) {
            x[k] /= A[k + size_t(k) * n];
            double xk = x[k];
            for (int i = 0; i < k; ++i) x[i] -= A[i + size_t(k) * n] * xk;
        }
    }
}

void sym_csr_mult(int n, const double *a, const int *ia, const int *ja, const double *x, double *y) {
    for (int i = 0; i < n; ++i) y[i] = 0.0;
    for (int i = 0; i < n; ++i)
        for (int k = ia[i]; k < ia[i + 1]; ++k) {
            int j = ja[k];
            y[i] += a[k] * x[j];
            if (j != i) y[j] += a[k] * x[i];
        }
}
}  // namespace

extern "C" void pardiso(void *pt_, const MKL_INT *, const MKL_INT *, const MKL_INT *mtype,
                        const MKL_INT *phase, const MKL_INT *n_, const void *a_, const MKL_INT *ia,
                        const MKL_INT *ja, MKL_INT *, const MKL_INT *nrhs_, MKL_INT *iparm,
                        const MKL_INT *, void *b_, void *x_, MKL_INT *error) {
    void **pt = static_cast<void **>(pt_);
    const double *a = static_cast<const double *>(a_);
    int n = *n_;
    *error = 0;
    if (*mtype != -2 && *mtype != 2) { *error = -3; return; }
    Factor *F = static_cast<Factor *>(pt[0]);
    switch (*phase) {
    case 11:
        if (!F) { F = new Factor(); pt[0] = F; }
        F->n = n;
        return;
    case 22:
    case 12:
        if (!F) { F = new Factor(); pt[0] = F; }
        F->n = n;
        if (!skyline_factor(*F, n, a, ia, ja)) {
            F->L.clear(); F->first.clear(); F->rowptr.clear();
            dense_lu(*F, n, a, ia, ja);
        }
        if (iparm) iparm[13] = 0;
        return;
    case 33: {
        if (!F) { *error = -1; return; }
        const double *b = static_cast<const double *>(b_);
        double *x = static_cast<double *>(x_);
        int nrhs = *nrhs_;
        int steps = iparm ? iparm[7] : 0;
        std::vector<double> r(n), ax(n);
        for (int k = 0; k < nrhs; ++k) {
            const double *bk = b + size_t(k) * n;
            double *xk = x + size_t(k) * n;
            std::memcpy(xk, bk, sizeof(double) * n);
            apply_inverse(*F, xk);
            for (int s = 0; s < steps; ++s) {
                sym_csr_mult(n, a, ia, ja, xk, ax.data());
                double rn = 0.0;
                for (int i = 0; i < n; ++i) { r[i] = bk[i] - ax[i]; rn += r[i] * r[i]; }
                if (rn == 0.0) break;
                apply_inverse(*F, r.data());
                for (int i = 0; i < n; ++i) xk[i] += r[i];
            }
        }
        if (iparm) iparm[6] = steps;
        return;
    }
    case -1:
        return;
    default:
        *error = -1;
        return;
    }
}
