// Kernel basis and fix DOFs of every subdomain on the GPU, one CTA per
// subdomain: the analytic rigid-body modes of the subdomain's nodes
// (Data::create_analytic_ker_K, Data.cpp:61-109) orthonormalised by
// classical Gram-Schmidt (Matrix::GramSchmidtOrtho, Matrix.cpp:2450-2472),
// then the full-pivot elimination of Matrix::getNullPivots
// (Matrix.cpp:835-884) on the rows of R at the Bf column set, which picks
// the 6 fix DOFs of the regularisation.
//
// The results are bit for bit those of the host code (host/problem.cpp
// kernel_of, null_pivots) that the layout inspection entry points use
// without a device: every dot product and norm is a left-to-right sum by one
// thread, every other operation is elementwise with the same rounding
// (__dmul_rn, __dadd_rn, __ddiv_rn: no contraction into FMAs), and the pivot
// search takes the last maximum in column-major order, as std::max_element
// with <= does.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <string>
#include <vector>

#include "../host/problem.hpp"

namespace htf {

namespace {

constexpr int KF_THREADS = 128;

// left-to-right sum of a[k] b[k]: the adds stay in order, the loads of b
// (global memory) are issued eight at a time ahead of them
__device__ double seq_dot(const double *a, const double *b, int n) {
    double s = 0.0;
    int k = 0;
    for (; k + 8 <= n; k += 8) {
        double r[8];
#pragma unroll
        for (int u = 0; u < 8; ++u) r[u] = b[k + u];
#pragma unroll
        for (int u = 0; u < 8; ++u) s = __dadd_rn(s, __dmul_rn(a[k + u], r[u]));
    }
    for (; k < n; ++k) s = __dadd_rn(s, __dmul_rn(a[k], b[k]));
    return s;
}

// R (n x 6, column-major at R + r_off) and the work copy N (nb x 6 at
// N + nb_off) of subdomain d; fix[6 d ..] = the 6 fix DOFs (local, sorted)
__global__ void __launch_bounds__(KF_THREADS) k_kernel_fix(const double *__restrict__ coords,
                                                           const int *__restrict__ node_ptr,
                                                           const int *__restrict__ nodes,
                                                           const int *__restrict__ b_ptr,
                                                           const int *__restrict__ bidx,
                                                           const long long *__restrict__ r_off, double *__restrict__ R,
                                                           const long long *__restrict__ n_off,
                                                           double *__restrict__ N, double *__restrict__ Wg,
                                                           int *__restrict__ piv_buf, int *__restrict__ fix) {
    const int d = blockIdx.x, t = threadIdx.x;
    const int nn = node_ptr[d + 1] - node_ptr[d], n = 3 * nn;
    const int nb = b_ptr[d + 1] - b_ptr[d];
    extern __shared__ double wsm[];
    // the column being orthogonalised (n doubles): shared memory, or global
    // scratch for subdomains too large for it
    double *w = Wg ? Wg + r_off[d] / 6 : wsm;
    double *Rd = R + r_off[d];
    double *Nd = N + n_off[d];
    int *piv = piv_buf + n_off[d] / 6;
    const int *bd = bidx + b_ptr[d];
    __shared__ double coef[6], last_row[6], nrm;
    __shared__ double red_v[KF_THREADS];
    __shared__ long long red_i[KF_THREADS];
    // analytic modes, column order x, y, z, (-y, x, 0), (-z, 0, x), (0, -z, y)
    for (int i = t; i < nn; i += KF_THREADS) {
        const int node = nodes[node_ptr[d] + i];
        const double x = coords[3 * (size_t)node], y = coords[3 * (size_t)node + 1], z = coords[3 * (size_t)node + 2];
        for (int j = 0; j < 6; ++j)
            for (int c = 0; c < 3; ++c) Rd[3 * i + c + (size_t)j * n] = 0.0;
        Rd[3 * i + 0 + (size_t)n * 0] = 1.0;
        Rd[3 * i + 1 + (size_t)n * 1] = 1.0;
        Rd[3 * i + 2 + (size_t)n * 2] = 1.0;
        Rd[3 * i + 0 + (size_t)n * 3] = -y;
        Rd[3 * i + 1 + (size_t)n * 3] = x;
        Rd[3 * i + 0 + (size_t)n * 4] = -z;
        Rd[3 * i + 2 + (size_t)n * 4] = x;
        Rd[3 * i + 1 + (size_t)n * 5] = -z;
        Rd[3 * i + 2 + (size_t)n * 5] = y;
    }
    __syncthreads();
    // classical Gram-Schmidt, column by column
    for (int j = 0; j < 6; ++j) {
        for (int k = t; k < n; k += KF_THREADS) w[k] = Rd[k + (size_t)j * n];
        __syncthreads();
        if (t < j) coef[t] = seq_dot(w, Rd + (size_t)t * n, n);
        __syncthreads();
        for (int k = t; k < n; k += KF_THREADS) {
            double v = w[k];
            for (int i = 0; i < j; ++i) v = __dsub_rn(v, __dmul_rn(Rd[k + (size_t)i * n], coef[i]));
            w[k] = v;
        }
        __syncthreads();
        if (t == 0) nrm = sqrt(seq_dot(w, w, n));
        __syncthreads();
        for (int k = t; k < n; k += KF_THREADS) Rd[k + (size_t)j * n] = __ddiv_rn(w[k], nrm);
        __syncthreads();
    }
    // null pivots of R at the Bf columns (nb x 6, column-major)
    for (int j = 0; j < 6; ++j)
        for (int i = t; i < nb; i += KF_THREADS) Nd[i + (size_t)j * nb] = Rd[bd[i] + (size_t)j * n];
    for (int i = t; i < nb; i += KF_THREADS) piv[i] = i;
    __syncthreads();
    const int m = 6;
    for (int j = 0; j < m; ++j) {
        // last maximum of |N| over the first m - j columns in column-major order
        const long long len = (long long)nb * (m - j);
        double bv = -1.0;
        long long bi = 0;
        for (long long q = t; q < len; q += KF_THREADS) {
            const double v = fabs(Nd[q]);
            if (v >= bv) { bv = v; bi = q; }
        }
        red_v[t] = bv;
        red_i[t] = bi;
        __syncthreads();
        for (int o = KF_THREADS / 2; o > 0; o >>= 1) {
            if (t < o) {
                const double v2 = red_v[t + o];
                const long long i2 = red_i[t + o];
                if (v2 > red_v[t] || (v2 == red_v[t] && i2 > red_i[t])) { red_v[t] = v2; red_i[t] = i2; }
            }
            __syncthreads();
        }
        const long long I = red_i[0];
        const int col = int(I / nb), row = int(I - (long long)col * nb);
        const int last = nb - 1 - j;
        __syncthreads();
        if (t < m - j) {                          // swap rows last and row in the first m - j columns
            const double a = Nd[last + (size_t)t * nb];
            Nd[last + (size_t)t * nb] = Nd[row + (size_t)t * nb];
            Nd[row + (size_t)t * nb] = a;
        }
        if (t == 0) {
            const int a = piv[row];
            piv[row] = piv[last];
            piv[last] = a;
        }
        __syncthreads();
        if (m - 1 - j != col)
            for (int i = t; i < nb; i += KF_THREADS) {
                const double a = Nd[i + (size_t)(m - 1 - j) * nb];
                Nd[i + (size_t)(m - 1 - j) * nb] = Nd[i + (size_t)col * nb];
                Nd[i + (size_t)col * nb] = a;
            }
        __syncthreads();
        if (t < m) last_row[t] = Nd[last + (size_t)t * nb];
        __syncthreads();
        const double p = last_row[m - 1 - j];
        for (int J = 0; J < m - j - 1; ++J)
            for (int i = t; i < nb - j; i += KF_THREADS) {
                const double a = Nd[i + (size_t)(m - 1 - j) * nb];
                Nd[i + (size_t)J * nb] = __dsub_rn(Nd[i + (size_t)J * nb], __ddiv_rn(__dmul_rn(a, last_row[J]), p));
            }
        __syncthreads();
    }
    if (t == 0) {
        int out[6];
        for (int i = 0; i < 6; ++i) out[i] = bd[piv[nb - 1 - i]];
        for (int a = 1; a < 6; ++a)               // sort the 6 local DOFs
            for (int b = a; b > 0 && out[b - 1] > out[b]; --b) {
                const int x = out[b];
                out[b] = out[b - 1];
                out[b - 1] = x;
            }
        for (int i = 0; i < 6; ++i) fix[6 * d + i] = out[i];
    }
}

template <typename T> int upload(T *&dst, const std::vector<T> &src, std::string &err, size_t n_alloc = 0) {
    const size_t bytes = std::max<size_t>(std::max(src.size(), n_alloc), 1) * sizeof(T);
    cudaError_t e = cudaMalloc(&dst, bytes);
    if (e == cudaSuccess && !src.empty()) e = cudaMemcpy(dst, src.data(), src.size() * sizeof(T), cudaMemcpyHostToDevice);
    if (e != cudaSuccess) {
        err = std::string("kernel detection upload: ") + cudaGetErrorString(e);
        return e == cudaErrorMemoryAllocation ? HTF_ENOMEM : HTF_ECUDA;
    }
    return HTF_OK;
}

}  // namespace

int kernels_fix_on_device(const Mesh &m, std::vector<Subdomain> &subs, int device, std::string &err,
                          double *timing_ms) {
    const int ns = int(subs.size());
    if (ns == 0) return HTF_OK;
    int count = 0;
    const auto t0 = std::chrono::steady_clock::now();   // runtime initialisation and context creation
    cudaGetLastError();                 // an error left by an earlier, failed call is not this one's
    if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0) {
        cudaGetLastError();
        err = "no CUDA device";
        return HTF_ENODEV;
    }
    if (cudaSetDevice(device) != cudaSuccess || cudaFree(nullptr) != cudaSuccess) {
        err = "kernel detection: cudaSetDevice failed";
        return HTF_ECUDA;
    }
    const auto t1 = std::chrono::steady_clock::now();
    std::vector<int> node_ptr(ns + 1, 0), nodes, b_ptr(ns + 1, 0), bidx;
    std::vector<long long> r_off(ns + 1, 0), n_off(ns + 1, 0);
    int max_n = 0;
    for (int d = 0; d < ns; ++d) {
        const Subdomain &s = subs[d];
        max_n = std::max(max_n, s.n);
        for (int i = 0; i < s.n / 3; ++i) nodes.push_back(s.l2g[3 * i] / 3);
        node_ptr[d + 1] = int(nodes.size());
        bidx.insert(bidx.end(), s.b.begin(), s.b.end());
        b_ptr[d + 1] = int(bidx.size());
        r_off[d + 1] = r_off[d] + 6LL * s.n;
        n_off[d + 1] = n_off[d] + 6LL * s.nb;
    }
    double *dc = nullptr, *dR = nullptr, *dN = nullptr, *dW = nullptr;
    int *dnp = nullptr, *dn = nullptr, *dbp = nullptr, *db = nullptr, *dpiv = nullptr, *dfix = nullptr;
    long long *dro = nullptr, *dno = nullptr;
    int rc = upload(dc, m.coords, err);
    if (!rc) rc = upload(dnp, node_ptr, err);
    if (!rc) rc = upload(dn, nodes, err);
    if (!rc) rc = upload(dbp, b_ptr, err);
    if (!rc) rc = upload(db, bidx, err);
    if (!rc) rc = upload(dro, r_off, err);
    if (!rc) rc = upload(dno, n_off, err);
    if (!rc) rc = upload(dR, std::vector<double>(), err, size_t(r_off[ns]));
    if (!rc) rc = upload(dN, std::vector<double>(), err, size_t(n_off[ns]) + 1);
    if (!rc) rc = upload(dpiv, std::vector<int>(), err, size_t(n_off[ns] / 6) + 1);
    if (!rc) rc = upload(dfix, std::vector<int>(), err, size_t(6 * ns));
    std::vector<double> R(r_off[ns]);
    std::vector<int> fix(6 * ns);
    int smem = max_n * int(sizeof(double)), optin = 0;
    cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, device);
    if (!rc && smem > optin - 4096) {          // too large for shared memory: global scratch
        smem = 0;
        rc = upload(dW, std::vector<double>(), err, size_t(r_off[ns] / 6) + 1);
    } else if (!rc && smem > 0) {
        // static + dynamic shared memory above 48 KB needs the opt-in; set it
        // for every size (the static arrays count against the same 48 KB)
        const cudaError_t e = cudaFuncSetAttribute(k_kernel_fix, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
        if (e != cudaSuccess) {
            err = std::string("kernel detection: shared memory opt-in of ") + std::to_string(smem) +
                  " B: " + cudaGetErrorString(e);
            rc = HTF_ECUDA;
        }
    }
    if (!rc) {
        const char *step = "launch";
        k_kernel_fix<<<ns, KF_THREADS, smem>>>(dc, dnp, dn, dbp, db, dro, dR, dno, dN, dW, dpiv, dfix);
        cudaError_t e = cudaGetLastError();
        if (e == cudaSuccess) {
            step = "copy of R";
            e = cudaMemcpy(R.data(), dR, R.size() * sizeof(double), cudaMemcpyDeviceToHost);
        }
        if (e == cudaSuccess) {
            step = "copy of the fix DOFs";
            e = cudaMemcpy(fix.data(), dfix, fix.size() * sizeof(int), cudaMemcpyDeviceToHost);
        }
        if (e != cudaSuccess) {
            err = std::string("kernel detection: ") + step + " (" + std::to_string(ns) + " CTAs, " +
                  std::to_string(smem) + " B dynamic shared memory): " + cudaGetErrorString(e);
            rc = HTF_ECUDA;
        }
    }
    for (void *p : {(void *)dc, (void *)dR, (void *)dN, (void *)dW, (void *)dnp, (void *)dn, (void *)dbp, (void *)db,
                    (void *)dpiv, (void *)dfix, (void *)dro, (void *)dno})
        if (p) cudaFree(p);
    if (rc) return rc;
    if (timing_ms) {
        timing_ms[0] = std::chrono::duration<double, std::milli>(t1 - t0).count();
        timing_ms[1] = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t1).count();
    }
    for (int d = 0; d < ns; ++d) {
        Subdomain &s = subs[d];
        s.R.assign(R.begin() + r_off[d], R.begin() + r_off[d + 1]);
        s.fix.assign(fix.begin() + 6 * d, fix.begin() + 6 * d + 6);
    }
    return HTF_OK;
}

}  // namespace htf
