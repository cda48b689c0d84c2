// Cluster coarse problem on the GPU (FP64), all clusters at once.
//
// Cluster::create_Ac_clust (Cluster.cpp:582-678) builds the extended
// saddle-point matrix Ac = [Fc Gc 0; Gc^T 0 H; 0 H^T 0] of every cluster and
// factors it with PARDISO (Cluster.cpp:283-324); each F apply then solves with
// it.  Here the solve is a GEMV with the explicit restriction
// M = [Ac^{-1}]_{(lambda_c, alpha), (lambda_c, alpha)}, formed by block
// elimination with SPD pieces only:
//   L L^T = Fc                       batched Cholesky (the subdomain kernels)
//   [Z | Fi] = Fc^{-1} [Gc | I]      batched multi-RHS triangular solves
//   Sr = Gc^T Z + H H^T              batched GEMM
//   Ls Ls^T = Sr, Si = Sr^{-1}       Cholesky + triangular solves
//   ZS = Z Si                        GEMM
//   M11 = Fi - ZS Z^T, M12 = ZS, M21 = ZS^T, M22 = H H^T - Si
// with H the orthonormal basis of ker(Gc) (the cluster's rigid modes).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "engine.hpp"

namespace htf {

__global__ void k_potrf_diag(const StepDesc *, const SubDev *, double *, int *);
__global__ void k_trsm_panel(const StepDesc *, int, const SubDev *, double *, const int *);
__global__ void k_syrk_update(const StepDesc *, int, const SubDev *, double *, const int *);
__global__ void k_trsm_fwd_multi(const SubDev *, const double *, double *, long long, int, const int *);
__global__ void k_trsm_bwd_multi(const SubDev *, const double *, double *, long long, int, const int *);
__global__ void k_build_Fc(const SubDev *, const double *, const int *, const int *, const double *,
                           const long long *, double *);

// C = alpha op(A) op(B) + beta C (column-major; beta == 0 does not read C)
struct GemmDesc {
    int m, n, k;
    int ta, tb;
    int lda, ldb, ldc;
    const double *A, *B;
    double *C;
    double alpha, beta;
};

// dst = alpha op(src) (rows x cols); src == nullptr: dst = alpha I
struct CopyDesc {
    int rows, cols, trans, lds, ldd;
    const double *src;
    double *dst;
    double alpha;
};

// 64x64 tile per CTA, k in chunks of 16 staged in shared memory (the next
// chunk register-prefetched while the current one multiplies); the
// products on the FP64 tensor path (mma.sync m8n8k4 .f64): warp w owns rows
// 32 (w / 4) .. +31 and columns 16 (w % 4) .. +15 of the tile as 4 x 2 tiles
// of 8 x 8 (row stride 68 doubles: conflict-free fragment loads).
// grid: (tiles of the largest problem, problems)
__device__ __forceinline__ void dmma_gemm(double &d0, double &d1, double a, double b) {
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};"
                 : "+d"(d0), "+d"(d1)
                 : "d"(a), "d"(b));
}

__global__ void __launch_bounds__(256) k_gemm_batched(const GemmDesc *__restrict__ desc) {
    constexpr int LD = 68;
    __shared__ double As[16][LD];
    __shared__ double Bs[16][LD];
    const GemmDesc g = desc[blockIdx.y];
    const int tm = (g.m + 63) / 64, tn = (g.n + 63) / 64;
    if ((int)blockIdx.x >= tm * tn) return;
    const int i0 = 64 * (blockIdx.x % tm), j0 = 64 * (blockIdx.x / tm);
    const int t = threadIdx.x, warp = t >> 5, lane = t & 31;
    const int gq = lane >> 2, t4 = lane & 3;
    const int wr = 32 * (warp >> 2), wc = 16 * (warp & 3);
    double acc[4][2][2];
#pragma unroll
    for (int a = 0; a < 4; ++a)
#pragma unroll
        for (int b = 0; b < 2; ++b) acc[a][b][0] = acc[a][b][1] = 0.0;
    // the next k chunk is loaded into registers while the current one multiplies
    double ra[4], rb[4];
    auto load = [&](int p0) {
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const int e = t + 256 * q;                       // 0..1023
            // A: op(A)[i][p], i in tile (64), p in chunk (16)
            int i, p;
            if (!g.ta) { i = e % 64; p = e / 64; } else { p = e % 16; i = e / 16; }
            const int gi = i0 + i, gp = p0 + p;
            ra[q] = (gi < g.m && gp < g.k) ? (g.ta ? g.A[gp + (size_t)gi * g.lda] : g.A[gi + (size_t)gp * g.lda])
                                           : 0.0;
            int j, pb;
            if (!g.tb) { pb = e % 16; j = e / 16; } else { j = e % 64; pb = e / 64; }
            const int gj = j0 + j, gpb = p0 + pb;
            rb[q] = (gj < g.n && gpb < g.k) ? (g.tb ? g.B[gj + (size_t)gpb * g.ldb] : g.B[gpb + (size_t)gj * g.ldb])
                                            : 0.0;
        }
    };
    if (g.k > 0) load(0);
    for (int p0 = 0; p0 < g.k; p0 += 16) {
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const int e = t + 256 * q;
            int i, p;
            if (!g.ta) { i = e % 64; p = e / 64; } else { p = e % 16; i = e / 16; }
            As[p][i] = ra[q];
            int j, pb;
            if (!g.tb) { pb = e % 16; j = e / 16; } else { j = e % 64; pb = e / 64; }
            Bs[pb][j] = rb[q];
        }
        __syncthreads();
        if (p0 + 16 < g.k) load(p0 + 16);
#pragma unroll
        for (int kg = 0; kg < 4; ++kg) {
            const int kr = 4 * kg + t4;
            double av[4], bv[2];
#pragma unroll
            for (int a = 0; a < 4; ++a) av[a] = As[kr][wr + 8 * a + gq];
#pragma unroll
            for (int b = 0; b < 2; ++b) bv[b] = Bs[kr][wc + 8 * b + gq];
#pragma unroll
            for (int a = 0; a < 4; ++a)
#pragma unroll
                for (int b = 0; b < 2; ++b) dmma_gemm(acc[a][b][0], acc[a][b][1], av[a], bv[b]);
        }
        __syncthreads();
    }
#pragma unroll
    for (int b = 0; b < 2; ++b)
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            const int j = j0 + wc + 8 * b + 2 * t4 + h;
            if (j >= g.n) continue;
#pragma unroll
            for (int a = 0; a < 4; ++a) {
                const int i = i0 + wr + 8 * a + gq;
                if (i >= g.m) continue;
                double *c = g.C + i + (size_t)j * g.ldc;
                *c = g.alpha * acc[a][b][h] + (g.beta != 0.0 ? g.beta * *c : 0.0);
            }
        }
}

// Cluster Fc = sum_d Bc_d F_d Bc_d^T (Cluster.cpp:190-198) assembled in place
// from the subdomains' c x c blocks: one CTA per cluster adds its subdomains'
// blocks one after another (in cluster order, the host's order; the targets
// inside one block are distinct), so every entry gets its contributions in
// the same order as a sequential host loop.  F is zero on entry.
__global__ void __launch_bounds__(1024) k_assemble_Fc(const SubDev *__restrict__ subs,
                                                      const int *__restrict__ cl_ptr, const int *__restrict__ cl_subs,
                                                      const int *__restrict__ bcr, const long long *__restrict__ fco,
                                                      const double *__restrict__ Fc, const long long *__restrict__ oF,
                                                      const int *__restrict__ ncs, double *__restrict__ F) {
    const int ci = blockIdx.x, nc = ncs[ci];
    double *Fcl = F + oF[ci];
    for (int k = cl_ptr[ci]; k < cl_ptr[ci + 1]; ++k) {
        const int d = cl_subs[k];
        const SubDev &sd = subs[d];
        const int c = sd.c;
        const int *rows = bcr + sd.bcr_off;
        const double *B = Fc + fco[d];
        for (int e = threadIdx.x; e < c * c; e += blockDim.x) {
            const int i = e % c, j = e / c;
            double *t = Fcl + rows[i] + (size_t)rows[j] * nc;
            *t = __dadd_rn(*t, B[i + (size_t)j * c]);
        }
        __syncthreads();
    }
}

// Cluster Gc = -Bc R (Cluster.cpp:190-198): thread (subdomain d, mode j) owns
// column 6 k + j of its cluster's Gc (k = d's position in the cluster) and
// subtracts its Bc entries' products in the host's entry order, rounded as
// the host rounds them (product, then difference).  G is zero on entry.
__global__ void k_assemble_Gc(int ns, const SubDev *__restrict__ subs, const int *__restrict__ cl_index,
                              const int *__restrict__ e_ptr, const int *__restrict__ e_row,
                              const int *__restrict__ e_pl, const double *__restrict__ e_val,
                              const double *__restrict__ R, const long long *__restrict__ oG,
                              const int *__restrict__ ncs, double *__restrict__ G) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= 6 * ns) return;
    const int d = t / 6, j = t % 6;
    const SubDev &sd = subs[d];
    const int nc = ncs[sd.cluster];
    double *col = G + oG[sd.cluster] + (size_t)(6 * cl_index[d] + j) * nc;
    const double *Rj = R + sd.R_off + (size_t)j * sd.N;
    for (int e = e_ptr[d]; e < e_ptr[d + 1]; ++e)
        col[e_row[e]] = __dsub_rn(col[e_row[e]], __dmul_rn(e_val[e], Rj[e_pl[e]]));
}

// grid: (blocks of the largest copy, copies)
__global__ void k_copy_batched(const CopyDesc *__restrict__ desc) {
    const CopyDesc c = desc[blockIdx.y];
    const long long n = (long long)c.rows * c.cols;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n; e += (long long)gridDim.x * blockDim.x) {
        const int i = int(e % c.rows), j = int(e / c.rows);
        double v;
        if (!c.src) v = (i == j) ? c.alpha : 0.0;
        else v = c.alpha * (c.trans ? c.src[j + (size_t)i * c.lds] : c.src[i + (size_t)j * c.lds]);
        c.dst[i + (size_t)j * c.ldd] = v;
    }
}

namespace {

struct DevTmp {                        // device scratch freed when the coarse set-up ends
    std::vector<void *> p;
    ~DevTmp() {
        for (void *q : p) cudaFree(q);
    }
    template <typename T> T *get(size_t n, cudaError_t &e) {
        void *q = nullptr;
        if (e == cudaSuccess) e = cudaMalloc(&q, std::max<size_t>(n, 1) * sizeof(T));
        if (e == cudaSuccess) p.push_back(q);
        return static_cast<T *>(q);
    }
};

// step tables of the batched right-looking Cholesky of the given matrices
void chol_steps(const std::vector<SubDev> &m, std::vector<std::vector<StepDesc>> &steps) {
    steps.clear();
    for (int d = 0; d < int(m.size()); ++d)
        for (int k = 0, s = 0; k < m[d].N; k += CHOL_STEP, ++s) {
            if (int(steps.size()) <= s) steps.resize(s + 1);
            steps[s].push_back({d, k, std::min(CHOL_STEP, m[d].N - k), 0, 0});
        }
}

int cdivc(long long a, long long b) { return int((a + b - 1) / b); }

}  // namespace

// Launches the batched Cholesky of the matrices described by hm / dm (N, K_off).
static cudaError_t chol_batched(const std::vector<SubDev> &hm, const SubDev *dm, double *buf, int *status,
                                DevTmp &tmp, cudaStream_t s) {
    std::vector<std::vector<StepDesc>> steps;
    chol_steps(hm, steps);
    std::vector<StepDesc> flat;
    std::vector<size_t> off;
    std::vector<int> ntri, nrb;
    for (auto &v : steps) {
        int tri = 0, rb = 0;
        for (auto &x : v) {
            const int rows = hm[x.d].N - x.k - x.nb, nbr = (rows + 63) / 64;
            x.tri0 = tri; tri += nbr * (nbr + 1) / 2;
            x.rb0 = rb; rb += (rows + 127) / 128;
        }
        ntri.push_back(tri);
        nrb.push_back(rb);
        off.push_back(flat.size());
        flat.insert(flat.end(), v.begin(), v.end());
    }
    if (flat.empty()) return cudaSuccess;
    cudaError_t e = cudaFuncSetAttribute(k_syrk_update, cudaFuncAttributeMaxDynamicSharedMemorySize, SYRK_SMEM);
    if (e != cudaSuccess) return e;
    std::vector<int> hints;
    std::vector<size_t> htri, hrb;
    for (size_t st = 0; st < steps.size(); ++st) {
        htri.push_back(hints.size());
        step_hints(steps[st], ntri[st], true, hints);
        hrb.push_back(hints.size());
        step_hints(steps[st], nrb[st], false, hints);
    }
    StepDesc *d = tmp.get<StepDesc>(flat.size(), e);
    int *dh = tmp.get<int>(hints.size(), e);
    if (e != cudaSuccess) return e;
    e = cudaMemcpyAsync(d, flat.data(), flat.size() * sizeof(StepDesc), cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(dh, hints.data(), hints.size() * sizeof(int), cudaMemcpyHostToDevice, s);
    if (e != cudaSuccess) return e;
    for (size_t st = 0; st < steps.size(); ++st) {
        const int cnt = int(steps[st].size());
        k_potrf_diag<<<cnt, CHOL_STEP, 0, s>>>(d + off[st], dm, buf, status);
        if (nrb[st] > 0) k_trsm_panel<<<nrb[st], 128, 0, s>>>(d + off[st], cnt, dm, buf, dh + hrb[st]);
        if (ntri[st] > 0) k_syrk_update<<<ntri[st], 256, SYRK_SMEM, s>>>(d + off[st], cnt, dm, buf, dh + htri[st]);
    }
    return cudaGetLastError();
}

static cudaError_t gemm_batched(const std::vector<GemmDesc> &g, DevTmp &tmp, cudaStream_t s) {
    std::vector<GemmDesc> v;
    int tiles = 0;
    for (auto &x : g)
        if (x.m > 0 && x.n > 0) {
            v.push_back(x);
            tiles = std::max(tiles, cdivc(x.m, 64) * cdivc(x.n, 64));
        }
    if (v.empty()) return cudaSuccess;
    cudaError_t e = cudaSuccess;
    GemmDesc *d = tmp.get<GemmDesc>(v.size(), e);
    if (e == cudaSuccess) e = cudaMemcpyAsync(d, v.data(), v.size() * sizeof(GemmDesc), cudaMemcpyHostToDevice, s);
    if (e != cudaSuccess) return e;
    k_gemm_batched<<<dim3(tiles, int(v.size())), 256, 0, s>>>(d);
    return cudaGetLastError();
}

static cudaError_t copy_batched(const std::vector<CopyDesc> &c, DevTmp &tmp, cudaStream_t s) {
    std::vector<CopyDesc> v;
    long long mx = 0;
    for (auto &x : c)
        if (x.rows > 0 && x.cols > 0) {
            v.push_back(x);
            mx = std::max(mx, (long long)x.rows * x.cols);
        }
    if (v.empty()) return cudaSuccess;
    cudaError_t e = cudaSuccess;
    CopyDesc *d = tmp.get<CopyDesc>(v.size(), e);
    if (e == cudaSuccess) e = cudaMemcpyAsync(d, v.data(), v.size() * sizeof(CopyDesc), cudaMemcpyHostToDevice, s);
    if (e != cudaSuccess) return e;
    k_copy_batched<<<dim3(std::min(cdivc(mx, 256), 4096), int(v.size())), 256, 0, s>>>(d);
    return cudaGetLastError();
}

// triangular solves L L^T X = X for the matrices hm / dm; X of matrix c at
// x + hm[c].nfull_off with leading dimension hm[c].N and ncols[c] columns
static cudaError_t solve_batched(const std::vector<SubDev> &hm, const SubDev *dm, const double *buf, double *x,
                                 const std::vector<int> &ncols, DevTmp &tmp, cudaStream_t s) {
    int chunks = 0;
    for (int c : ncols) chunks = std::max(chunks, cdivc(c, 32));
    if (chunks == 0 || hm.empty()) return cudaSuccess;
    cudaError_t e = cudaSuccess;
    int *d = tmp.get<int>(ncols.size(), e);
    if (e == cudaSuccess) e = cudaMemcpyAsync(d, ncols.data(), ncols.size() * sizeof(int), cudaMemcpyHostToDevice, s);
    if (e != cudaSuccess) return e;
    const dim3 grid(int(hm.size()), chunks);
    k_trsm_fwd_multi<<<grid, 256, 0, s>>>(dm, buf, x, 0, 0, d);
    k_trsm_bwd_multi<<<grid, 256, 0, s>>>(dm, buf, x, 0, 0, d);
    return cudaGetLastError();
}

#define CKC(call)                                                          \
    do {                                                                   \
        int _rc = check((call), #call, err, "coarse.cu", __LINE__);        \
        if (_rc) return _rc;                                               \
    } while (0)

int Engine::coarse(Problem &p, std::string &err) {
    int rc = HTF_OK;
    // Fc_d = Bc_d F_d Bc_d^T of every subdomain, on the device
    std::vector<long long> fco(nsub_);
    long long fct = 0;
    for (int d = 0; d < nsub_; ++d) { fco[d] = fct; fct += (long long)hs_[d].c * hs_[d].c; }
    DevTmp tmp;
    cudaError_t ce = cudaSuccess;
    long long *d_fco = tmp.get<long long>(nsub_, ce);
    double *d_Fc = tmp.get<double>(fct, ce);
    CKC(ce);
    CKC(cudaMemcpyAsync(d_fco, fco.data(), nsub_ * sizeof(long long), cudaMemcpyHostToDevice, s_));
    k_build_Fc<<<nsub_, 256, 0, s_>>>(d_subs_, d_V_, d_bce_ptr_, d_bce_pos_, d_bce_val_, d_fco, d_Fc);
    CKC(cudaGetLastError());
    // cluster Fc and Gc = -Bc R (Cluster.cpp:190-198) on the device (below);
    // host: H = ker(Gc) (orthonormal rigid modes of the cluster)
    std::vector<long long> oF(ncl_), oW(ncl_), oG(ncl_), oH(ncl_), oS(ncl_), oZS(ncl_);
    long long nF = 0, nW = 0, nG = 0, nH = 0, nS = 0, nZS = 0;
    for (int c = 0; c < ncl_; ++c) {
        const long long nc = p.clu[c].nlam_c, na = 6 * (long long)p.clu[c].subs.size();
        oF[c] = nF; nF += nc * nc;
        oW[c] = nW; nW += nc * (na + nc);
        oG[c] = nG; nG += nc * na;
        oH[c] = nH; nH += na * 6;
        oS[c] = nS; nS += na * na;
        oZS[c] = nZS; nZS += nc * na;
    }
    if (nW > 0x7fffffffLL || nS > 0x7fffffffLL) { err = "cluster coarse problems too large"; return HTF_EINVAL; }
    std::vector<double> hH(nH, 0.0);
    Hd_.assign(nsub_, std::vector<double>(36, 0.0));
#pragma omp parallel for schedule(dynamic)
    for (int ci = 0; ci < ncl_; ++ci) {
        const Cluster &cl = p.clu[ci];
        const int ns = int(cl.subs.size()), na = 6 * ns;
        double *H = hH.data() + oH[ci];
        for (int k = 0; k < ns; ++k) {
            const int d = cl.subs[k];
            const Subdomain &s = p.sub[d];
            // ker(Gc): alpha_d = R_d^T r for the (unnormalised) rigid modes r of the cluster
            const int n = s.n;
            for (int q = 0; q < 6; ++q)
                for (int j = 0; j < 6; ++j) {
                    double v = 0.0;
                    for (int l = 0; l < n / 3; ++l) {
                        const int node = s.l2g[3 * l] / 3;
                        const double x = p.mesh.coords[3 * size_t(node)], y = p.mesh.coords[3 * size_t(node) + 1],
                                     z = p.mesh.coords[3 * size_t(node) + 2];
                        double g[3] = {0, 0, 0};
                        switch (q) {
                            case 0: g[0] = 1; break;
                            case 1: g[1] = 1; break;
                            case 2: g[2] = 1; break;
                            case 3: g[0] = -y; g[1] = x; break;
                            case 4: g[0] = -z; g[2] = x; break;
                            default: g[1] = -z; g[2] = y; break;
                        }
                        for (int cc = 0; cc < 3; ++cc) v += s.R[3 * l + cc + size_t(j) * n] * g[cc];
                    }
                    H[6 * k + j + size_t(q) * na] = v;
                }
        }
        for (int pass = 0; pass < 2; ++pass)               // two passes of Gram-Schmidt
            for (int q = 0; q < 6; ++q) {
                double *hq = H + size_t(q) * na;
                for (int o = 0; o < q; ++o) {
                    const double *ho = H + size_t(o) * na;
                    double dd = 0.0;
                    for (int i = 0; i < na; ++i) dd += hq[i] * ho[i];
                    for (int i = 0; i < na; ++i) hq[i] -= dd * ho[i];
                }
                double nn = 0.0;
                for (int i = 0; i < na; ++i) nn += hq[i] * hq[i];
                nn = std::sqrt(nn);
                for (int i = 0; i < na; ++i) hq[i] /= nn;
            }
        for (int k = 0; k < ns; ++k)
            for (int j = 0; j < 6; ++j)
                for (int q = 0; q < 6; ++q) Hd_[cl.subs[k]][j * 6 + q] = H[6 * k + j + size_t(q) * na];
    }
    // device: factor Fc and Sr, solve, multiply, assemble M
    double *dF = tmp.get<double>(nF, ce), *dW = tmp.get<double>(nW, ce), *dG = tmp.get<double>(nG, ce);
    double *dH = tmp.get<double>(nH, ce), *dS = tmp.get<double>(nS, ce), *dSi = tmp.get<double>(nS, ce);
    double *dZS = tmp.get<double>(nZS, ce);
    SubDev *dmF = tmp.get<SubDev>(ncl_, ce), *dmS = tmp.get<SubDev>(ncl_, ce);
    int *dst = tmp.get<int>(2 * ncl_, ce);
    CKC(ce);
    CKC(cudaMemcpyAsync(dH, hH.data(), nH * sizeof(double), cudaMemcpyHostToDevice, s_));
    {
        // cluster Fc and Gc assembled on the device, in the host loop's order
        std::vector<int> cl_ptr(ncl_ + 1, 0), cl_subs, cl_index(nsub_), ncs(ncl_), e_ptr(nsub_ + 1, 0), e_row, e_pl;
        std::vector<double> e_val;
        for (int c = 0; c < ncl_; ++c) {
            ncs[c] = p.clu[c].nlam_c;
            for (size_t k = 0; k < p.clu[c].subs.size(); ++k) {
                cl_subs.push_back(p.clu[c].subs[k]);
                cl_index[p.clu[c].subs[k]] = int(k);
            }
            cl_ptr[c + 1] = int(cl_subs.size());
        }
        for (int d = 0; d < nsub_; ++d) {
            const Subdomain &s = p.sub[d];
            for (size_t e = 0; e < s.bc_row.size(); ++e) {
                e_row.push_back(s.bc_row[e]);
                e_pl.push_back(s.perm[s.bc_col[e]]);
                e_val.push_back(s.bc_val[e]);
            }
            e_ptr[d + 1] = int(e_row.size());
        }
        int *d_clp = tmp.get<int>(cl_ptr.size(), ce), *d_cls = tmp.get<int>(cl_subs.size(), ce);
        int *d_cli = tmp.get<int>(cl_index.size(), ce), *d_ncs = tmp.get<int>(ncs.size(), ce);
        int *d_ep = tmp.get<int>(e_ptr.size(), ce), *d_er = tmp.get<int>(e_row.size(), ce);
        int *d_epl = tmp.get<int>(e_pl.size(), ce);
        double *d_ev = tmp.get<double>(e_val.size(), ce);
        long long *d_oF = tmp.get<long long>(ncl_, ce), *d_oG = tmp.get<long long>(ncl_, ce);
        CKC(ce);
        auto up = [&](void *dst, const void *src, size_t bytes) {
            return bytes ? cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, s_) : cudaSuccess;
        };
        CKC(up(d_clp, cl_ptr.data(), cl_ptr.size() * sizeof(int)));
        CKC(up(d_cls, cl_subs.data(), cl_subs.size() * sizeof(int)));
        CKC(up(d_cli, cl_index.data(), cl_index.size() * sizeof(int)));
        CKC(up(d_ncs, ncs.data(), ncs.size() * sizeof(int)));
        CKC(up(d_ep, e_ptr.data(), e_ptr.size() * sizeof(int)));
        CKC(up(d_er, e_row.data(), e_row.size() * sizeof(int)));
        CKC(up(d_epl, e_pl.data(), e_pl.size() * sizeof(int)));
        CKC(up(d_ev, e_val.data(), e_val.size() * sizeof(double)));
        CKC(up(d_oF, oF.data(), ncl_ * sizeof(long long)));
        CKC(up(d_oG, oG.data(), ncl_ * sizeof(long long)));
        CKC(cudaMemsetAsync(dF, 0, std::max<long long>(nF, 1) * sizeof(double), s_));
        CKC(cudaMemsetAsync(dG, 0, std::max<long long>(nG, 1) * sizeof(double), s_));
        k_assemble_Fc<<<ncl_, 1024, 0, s_>>>(d_subs_, d_clp, d_cls, d_bcr_, d_fco, d_Fc, d_oF, d_ncs, dF);
        k_assemble_Gc<<<cdivc(6LL * nsub_, 256), 256, 0, s_>>>(nsub_, d_subs_, d_cli, d_ep, d_er, d_epl, d_ev, d_R_,
                                                              d_oG, d_ncs, dG);
        CKC(cudaGetLastError());
        // the scratch above is released with tmp at the end of the coarse set-up, after the stream's work
    }
    CKC(cudaMemsetAsync(dst, 0, 2 * ncl_ * sizeof(int), s_));
    std::vector<SubDev> mF(ncl_), mS(ncl_);
    std::vector<int> colsW(ncl_), colsS(ncl_);
    std::vector<CopyDesc> cp;
    for (int c = 0; c < ncl_; ++c) {
        const int nc = p.clu[c].nlam_c, na = 6 * int(p.clu[c].subs.size());
        mF[c] = SubDev{};
        mF[c].N = nc; mF[c].K_off = oF[c]; mF[c].K_bset = -1; mF[c].nfull_off = int(oW[c]);
        mS[c] = SubDev{};
        mS[c].N = na; mS[c].K_off = oS[c]; mS[c].K_bset = -1; mS[c].nfull_off = int(oS[c]);
        colsW[c] = nc > 0 ? na + nc : 0;
        colsS[c] = na;
        cp.push_back(CopyDesc{nc, na, 0, nc, nc, dG + oG[c], dW + oW[c], 1.0});                 // W = [Gc | I]
        cp.push_back(CopyDesc{nc, nc, 0, 0, nc, nullptr, dW + oW[c] + (size_t)nc * na, 1.0});
        cp.push_back(CopyDesc{na, na, 0, 0, na, nullptr, dSi + oS[c], 1.0});                    // Si = I
    }
    CKC(cudaMemcpyAsync(dmF, mF.data(), ncl_ * sizeof(SubDev), cudaMemcpyHostToDevice, s_));
    CKC(cudaMemcpyAsync(dmS, mS.data(), ncl_ * sizeof(SubDev), cudaMemcpyHostToDevice, s_));
    CKC(copy_batched(cp, tmp, s_));
    CKC(chol_batched(mF, dmF, dF, dst, tmp, s_));
    CKC(solve_batched(mF, dmF, dF, dW, colsW, tmp, s_));               // [Z | Fi]
    std::vector<GemmDesc> gm;
    for (int c = 0; c < ncl_; ++c) {                                     // Sr = Gc^T Z + H H^T
        const int nc = p.clu[c].nlam_c, na = 6 * int(p.clu[c].subs.size());
        if (nc > 0) gm.push_back(GemmDesc{na, na, nc, 1, 0, nc, nc, na, dG + oG[c], dW + oW[c], dS + oS[c], 1.0, 0.0});
        gm.push_back(GemmDesc{na, na, 6, 0, 1, na, na, na, dH + oH[c], dH + oH[c], dS + oS[c], 1.0, nc > 0 ? 1.0 : 0.0});
    }
    // (the k = 6 update of a cluster runs after its k = nc product: separate launches)
    {
        std::vector<GemmDesc> a, b;
        for (auto &g : gm) (g.k == 6 ? b : a).push_back(g);
        CKC(gemm_batched(a, tmp, s_));
        CKC(gemm_batched(b, tmp, s_));
    }
    CKC(chol_batched(mS, dmS, dS, dst + ncl_, tmp, s_));
    CKC(solve_batched(mS, dmS, dS, dSi, colsS, tmp, s_));              // Si = Sr^{-1}
    gm.clear();
    for (int c = 0; c < ncl_; ++c) {                                     // ZS = Z Si
        const int nc = p.clu[c].nlam_c, na = 6 * int(p.clu[c].subs.size());
        gm.push_back(GemmDesc{nc, na, na, 0, 0, nc, na, nc, dW + oW[c], dSi + oS[c], dZS + oZS[c], 1.0, 0.0});
    }
    CKC(gemm_batched(gm, tmp, s_));
    cp.clear();
    gm.clear();
    for (int c = 0; c < ncl_; ++c) {
        const int nc = p.clu[c].nlam_c, na = 6 * int(p.clu[c].subs.size()), ng = nc + na;
        double *M = d_M_ + hc_[c].M_off;
        cp.push_back(CopyDesc{nc, nc, 0, nc, ng, dW + oW[c] + (size_t)nc * na, M, 1.0});            // M11 = Fi
        cp.push_back(CopyDesc{nc, na, 0, nc, ng, dZS + oZS[c], M + (size_t)nc * ng, 1.0});           // M12 = ZS
        cp.push_back(CopyDesc{na, nc, 1, nc, ng, dZS + oZS[c], M + nc, 1.0});                        // M21 = ZS^T
        cp.push_back(CopyDesc{na, na, 0, na, ng, dSi + oS[c], M + nc + (size_t)nc * ng, -1.0});      // M22 = -Si
        gm.push_back(GemmDesc{nc, nc, na, 0, 1, nc, nc, ng, dZS + oZS[c], dW + oW[c], M, -1.0, 1.0});  // M11 -= ZS Z^T
        gm.push_back(GemmDesc{na, na, 6, 0, 1, na, na, ng, dH + oH[c], dH + oH[c], M + nc + (size_t)nc * ng, 1.0,
                              1.0});                                                                  // M22 += H H^T
    }
    CKC(copy_batched(cp, tmp, s_));
    CKC(gemm_batched(gm, tmp, s_));
    std::vector<int> status(2 * ncl_);
    CKC(cudaMemcpyAsync(status.data(), dst, 2 * ncl_ * sizeof(int), cudaMemcpyDeviceToHost, s_));
    std::vector<double> Hflat(36 * (size_t)nsub_);
    for (int d = 0; d < nsub_; ++d) std::memcpy(&Hflat[36 * (size_t)d], Hd_[d].data(), 36 * sizeof(double));
    CKC(cudaMemcpyAsync(d_H_, Hflat.data(), Hflat.size() * sizeof(double), cudaMemcpyHostToDevice, s_));
    CKC(cudaStreamSynchronize(s_));
    for (int c = 0; c < 2 * ncl_; ++c)
        if (status[c]) {
            err = "cluster coarse matrix of cluster " + std::to_string(c % ncl_) + " is not positive definite";
            return HTF_ENOTSPD;
        }
    return rc;
}

}  // namespace htf
