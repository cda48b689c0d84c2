// Engine: GPU setup and PCPG of the HTFETI path.
//   setup   Cluster::initialization (Cluster.cpp:21-360)
//   pcpg    Cluster::pcpg + printVTK reconstruction (Cluster.cpp:1363-1458, 1648-1678)
#include <algorithm>
#include <chrono>
#include <climits>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <numeric>

#include "engine.hpp"

namespace htf {

// kernels (setup_kernels.cu / pcpg_kernels.cu)
cudaError_t set_gauss_points(cudaStream_t s);
__global__ void k_assemble(const int *, int, const double *, const int *, const int *, const double *,
                           const double *, const SubDev *, double *, double *, double, double, double);
__global__ void k_regularize(SubDev *, int, double *);
__global__ void k_potrf_diag(const StepDesc *, const SubDev *, double *, int *);
__global__ void k_trsm_panel(const StepDesc *, int, const SubDev *, double *, const int *);
__global__ void k_syrk_update(const StepDesc *, int, const SubDev *, double *, const int *);
__global__ void k_snapshot(const int *, const SubDev *, const double *, double *, long long);
__global__ void k_make_slabs(const GemmBlock *, const SubDev *, const double *, float *, long long,
                             const unsigned *);
__global__ void k_slab_amax(const GemmBlock *, const SubDev *, const double *, long long, unsigned *);
__global__ void k_trtri_step(int, const int *, const SubDev *, const double *, double *);
__global__ void k_lauum_tiles(const int *, const SubDev *, const double *, double *);
__global__ void k_build_V(const SubDev *, const double *, const int *, const int *, const double *,
                          const double *, double *);
__global__ void k_build_Fc(const SubDev *, const double *, const int *, const int *, const double *,
                           const long long *, double *);
__global__ void k_trsv_fwd(const SubDev *, const double *, double *, long long);
__global__ void k_trsv_bwd(const SubDev *, const double *, double *, long long);
__global__ void k_gather_b(int, const int *, const int *, const double *, const double *, double *,
                           const PcpgState *);
template <typename T>
__global__ void k_symv_units(const SymvUnit *, const SubDev *, const T *, const double *, const double *, double *,
                             double *, const PcpgState *);
__global__ void k_reduce_correct(const SubDev *, const SymvUnit *, const int *, const int *, const double *, const ClusterDev *,
                                 const double *, const int *, const double *, double *, const PcpgState *);
__global__ void k_lbt_x(const int2 *, const SubDev *, const double *, const double *, double *, const PcpgState *);
__global__ void k_lb_t(const int2 *, const SubDev *, const double *, const double *, const double *, double *,
                       const PcpgState *);
__global__ void k_pack_M(const int2 *, const ClusterDev *, const double *, double *);
__global__ void k_msym_rows(const int2 *, const ClusterDev *, const double *, const double *, double *, double *,
                            const PcpgState *);
__global__ void k_msym_reduce(const int2 *, const ClusterDev *, const double *, const double *, double *,
                              const PcpgState *);
__global__ void k_gf_coef(int, const int *, const double *, const double *, double *, double *, const PcpgState *);
__global__ void k_gf_apply(int, int, const double *, const int *, const double *, const double *, double *,
                           const double *, double *, const PcpgState *);
__global__ void k_gf_apply_fused(int, int, const int *, const double *, const double *, const int *,
                                 const double *, const double *, double *, double *, double *, const double *,
                                 double *, const PcpgState *);
__global__ void k_gc(int, const int *, const int *, const double *, double *, const PcpgState *);
__global__ void k_coarse(const ClusterDev *, const double *, const double *, double *, const PcpgState *);
__global__ void k_correct(const SubDev *, const ClusterDev *, const double *, const int *, const double *,
                          double *, const PcpgState *);
__global__ void k_rows(int, const int *, const double *, const double *, const double *, double *,
                       const double *, double *, const PcpgState *);
__global__ void k_gft_partial(const int *, const int *, const int *, const int *, const double *,
                              const double *, double *, const PcpgState *);
__global__ void k_gf_mult(int, const int *, const double *, const double *, double *);
__global__ void k_update_lam_g(int, const double *, int, const double *, const double *, double *, double *,
                               PcpgState *);
__global__ void k_update_w(int, const double *, int, const double *, double *, PcpgState *);
__global__ void k_finish_iter(const double *, int, PcpgState *, double *);
__global__ void k_init_state(const double *, int, PcpgState *, double, int);
__global__ void k_axpby(int, double, const double *, double, double *);

// ---- glue kernels on full (permuted local) vectors ----------------------
// t_d = [Bc_b z_b ; -R^T y]  (y full, z full)
__global__ void k_bc_rt(const SubDev *__restrict__ subs, const int *__restrict__ bce_ptr,
                        const int *__restrict__ bce_pos, const double *__restrict__ bce_val,
                        const double *__restrict__ Rbuf, const double *__restrict__ z,
                        const double *__restrict__ y, double *__restrict__ t) {
    const SubDev &sd = subs[blockIdx.x];
    const int lane = threadIdx.x % 32, warp = threadIdx.x / 32, nw = blockDim.x / 32;
    const double *zb = z + sd.nfull_off + sd.nr;
    for (int q = threadIdx.x; q < sd.c; q += blockDim.x) {
        double v = 0.0;
        for (int e = bce_ptr[sd.bce_off + q]; e < bce_ptr[sd.bce_off + q + 1]; ++e) v += bce_val[e] * zb[bce_pos[e]];
        t[sd.t_off + q] = v;
    }
    for (int j = warp; j < 6; j += nw) {
        const double *R = Rbuf + sd.R_off + (size_t)j * sd.N;
        const double *yy = y + sd.nfull_off;
        double s = 0.0;
        for (int i = lane; i < sd.N; i += 32) s += R[i] * yy[i];
        for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
        if (lane == 0) t[sd.t_off + sd.c + j] = -s;
    }
}

// copy the b block of a full vector into b space
__global__ void k_full_to_b(const SubDev *__restrict__ subs, const double *__restrict__ z, double *__restrict__ xb) {
    const SubDev &sd = subs[blockIdx.x];
    for (int i = threadIdx.x; i < sd.nbp; i += blockDim.x) xb[sd.xb_off + i] = (i < sd.nb) ? z[sd.nfull_off + sd.nr + i] : 0.0;
}

// y_full -= x_b on the b block
__global__ void k_full_minus_b(const SubDev *__restrict__ subs, const double *__restrict__ xb, double *__restrict__ y) {
    const SubDev &sd = subs[blockIdx.x];
    for (int i = threadIdx.x; i < sd.nb; i += blockDim.x) y[sd.nfull_off + sd.nr + i] -= xb[sd.xb_off + i];
}

// y_full -= Bc^T lambda_c
__global__ void k_sub_bct(const SubDev *__restrict__ subs, const ClusterDev *__restrict__ cl,
                          const int *__restrict__ bcr, const int *__restrict__ bce_ptr,
                          const int *__restrict__ bce_pos, const double *__restrict__ bce_val,
                          const double *__restrict__ s, double *__restrict__ y) {
    const SubDev &sd = subs[blockIdx.x];
    if (threadIdx.x != 0) return;      // few entries; sequential keeps the order fixed
    const ClusterDev &c = cl[sd.cluster];
    for (int q = 0; q < sd.c; ++q) {
        const double lc = s[c.gc_off + bcr[sd.bcr_off + q]];
        for (int e = bce_ptr[sd.bce_off + q]; e < bce_ptr[sd.bce_off + q + 1]; ++e)
            y[sd.nfull_off + sd.nr + bce_pos[e]] -= bce_val[e] * lc;
    }
}

// u_full += R_d (alpha_c,d - H_d alpha_f,cluster)
__global__ void k_add_R(const SubDev *__restrict__ subs, const ClusterDev *__restrict__ cl,
                        const double *__restrict__ Rbuf, const double *__restrict__ Hbuf,
                        const double *__restrict__ s, const double *__restrict__ alpha_f, double *__restrict__ u) {
    __shared__ double coef[6];
    const SubDev &sd = subs[blockIdx.x];
    const ClusterDev &c = cl[sd.cluster];
    if (threadIdx.x < 6) {
        const int j = threadIdx.x;
        double v = s[c.gc_off + sd.alpha_pos + j];
        const double *H = Hbuf + 36 * (size_t)blockIdx.x;      // H_d row-major 6x6: H[j*6+k]
        for (int k = 0; k < 6; ++k) v -= H[j * 6 + k] * alpha_f[6 * sd.cluster + k];
        coef[j] = v;
    }
    __syncthreads();
    for (int i = threadIdx.x; i < sd.N; i += blockDim.x) {
        double a = u[sd.nfull_off + i];
        for (int j = 0; j < 6; ++j) a += Rbuf[sd.R_off + (size_t)j * sd.N + i] * coef[j];
        u[sd.nfull_off + i] = a;
    }
}

// e_c = sum_{d in c} H_d^T (R_d^T f_d) = -sum_d H_d^T t_alpha,d ; one thread per (c, k)
__global__ void k_e_vec(int ncl, const int *__restrict__ cl_sub_ptr, const int *__restrict__ cl_sub,
                        const SubDev *__restrict__ subs, const double *__restrict__ Hbuf,
                        const double *__restrict__ t, double *__restrict__ e) {
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= 6 * ncl) return;
    const int c = q / 6, k = q % 6;
    double v = 0.0;
    for (int p = cl_sub_ptr[c]; p < cl_sub_ptr[c + 1]; ++p) {
        const int d = cl_sub[p];
        const SubDev &sd = subs[d];
        for (int j = 0; j < 6; ++j) v -= Hbuf[36 * (size_t)d + j * 6 + k] * t[sd.t_off + sd.c + j];
    }
    e[q] = v;
}

// a = A x (m x m, col-major), one CTA
__global__ void k_small_gemv(int m, const double *__restrict__ A, const double *__restrict__ x, double *__restrict__ a) {
    for (int q = threadIdx.x; q < m; q += blockDim.x) {
        double s = 0.0;
        for (int p = 0; p < m; ++p) s += A[q + (size_t)p * m] * x[p];
        a[q] = s;
    }
}

// f[r][i] = fbody[i] + fn[r][own[i]]
__global__ void k_build_f(int nfull, int ndof, int nrhs, const double *__restrict__ fbody, const int *__restrict__ own,
                          const double *__restrict__ fn, double *__restrict__ f) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nfull) return;
    const int g = own[i];
    for (int r = 0; r < nrhs; ++r) f[(size_t)r * nfull + i] = fbody[i] + ((fn && g >= 0) ? fn[(size_t)r * ndof + g] : 0.0);
}

// u[g] = uloc[win[g]]
__global__ void k_gather_u(int ndof, const int *__restrict__ win, const double *__restrict__ uloc, double *__restrict__ u) {
    const int g = blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= ndof) return;
    const int s = win[g];
    u[g] = (s >= 0) ? uloc[s] : 0.0;
}

// ---------------------------------------------------------------------------
// free one of the engine's buffers before the end of its life
void Engine::release(void *p) {
    for (size_t i = 0; i < bufs_.size(); ++i)
        if (bufs_[i].p == p) {
            cudaFree(p);
            bufs_.erase(bufs_.begin() + i);
            return;
        }
}

// s = M gc for every cluster (M = [Ac^{-1}] restricted), from the packed symmetric tiles
void Engine::coarse_apply(const double *gc, double *s, const PcpgState *st) {
    k_msym_rows<<<nmt_, 128, 0, s_>>>(d_mt_, d_cl_, d_MT_, gc, d_mD_, d_mP_, st);
    k_msym_reduce<<<nmt_, TILE, 0, s_>>>(d_mt_, d_cl_, d_mD_, d_mP_, s, st);
}

Engine::~Engine() {
    if (own_s_) cudaStreamSynchronize(own_s_);
    if (s_ && s_ != own_s_) cudaStreamSynchronize(s_);
    if (graph_) cudaGraphExecDestroy(graph_);
    if (bgraph_) cudaGraphExecDestroy(bgraph_);
    if (run_e0_) cudaEventDestroy(run_e0_);
    if (run_e1_) cudaEventDestroy(run_e1_);
    for (auto &b : bufs_) cudaFree(b.p);
    if (own_s_) cudaStreamDestroy(own_s_);
}

size_t Engine::device_bytes() const {
    size_t t = 0;
    for (auto &b : bufs_) t += b.bytes;
    return t;
}

int Engine::check(cudaError_t e, const char *what, std::string &err, const char *file, int line) {
    if (e == cudaSuccess) return HTF_OK;
    err = std::string(what) + ": " + cudaGetErrorString(e);
    if (file) err += " (" + std::string(file) + ":" + std::to_string(line) + ")";
    return (e == cudaErrorMemoryAllocation) ? HTF_ENOMEM : HTF_ECUDA;
}

#define CK(call)                                                   \
    do {                                                           \
        int _rc = check((call), #call, err, "engine.cu", __LINE__); \
        if (_rc) return _rc;                                       \
    } while (0)

static inline int cdiv(long long a, long long b) { return int((a + b - 1) / b); }

// ---------------------------------------------------------------------------
int Engine::upload_layout(Problem &p, std::string &err) {
    int rc = HTF_OK;
    nsub_ = int(p.sub.size());
    ncl_ = int(p.clu.size());
    nlam_ = p.n_lam;
    hs_.assign(nsub_, SubDev());
    long long K_off = 0, T_off = 0, X_off = 0, V_off = 0, R_off = 0;
    const long long XWAVE = 1LL << 29;           // 4 GiB
    xwave_.assign(1, 0);
    xwave_max_ = 0;
    // factor waves of at most FCAP doubles of panels (a subdomain larger than that is a wave of its own)
    const long long FCAP = opt_.factor_wave_gb > 0.0 ? std::max(1LL, (long long)(opt_.factor_wave_gb * 1e9 / 8.0))
                                                     : LLONG_MAX;
    fwave_.assign(1, 0);
    long long kwave_max = 0;
    int xb = 0, nf = 0, t_off = 0, bcr = 0, bce = 0;
    for (int d = 0; d < nsub_; ++d) {
        const Subdomain &s = p.sub[d];
        SubDev &h = hs_[d];
        h.n = s.n; h.nr = s.nr; h.nb = s.nb;
        h.nt = (s.nb + TILE - 1) / TILE;
        h.nbp = h.nt * TILE;
        h.N = h.nr + h.nbp;
        const long long kp = kpanel_doubles(h.nr, h.nbp);
        const bool new_fwave = K_off > 0 && K_off + kp > FCAP;
        if (new_fwave) {
            fwave_.push_back(d);
            K_off = 0;
        }
        h.K_off = K_off; K_off += kp;
        kwave_max = std::max(kwave_max, K_off);
        h.K_bset = kpanel_interior(h.nr, h.N);
        h.T_off = T_off; T_off += (long long)h.nt * (h.nt + 1) / 2;
        // L_bb^{-1} scratch of the F_i set-up, in waves of subdomains of at most XWAVE doubles that
        // never cross a factor wave
        const long long xs = (long long)h.nbp * h.nbp;
        if (X_off > 0 && (new_fwave || X_off + xs > XWAVE)) {
            xwave_.push_back(d);
            X_off = 0;
        }
        h.X_off = X_off; X_off += xs;
        xwave_max_ = std::max(xwave_max_, X_off);
        h.xb_off = xb; xb += h.nbp;
        h.nfull_off = nf; nf += h.N;
        h.c = s.c();
        if (h.c + 6 > 256) {
            err = "subdomain " + std::to_string(d) + " has " + std::to_string(h.c) +
                  " Bc rows; at most 250 are supported";
            return HTF_EINVAL;
        }
        h.cluster = s.cluster;
        h.alpha_pos = p.clu[s.cluster].nlam_c + 6 * s.cl_index;
        h.V_off = V_off; V_off += (long long)h.nbp * (h.c + 6);
        h.t_off = t_off; t_off += h.c + 6;
        h.bcr_off = bcr; bcr += h.c;
        h.bce_off = bce; bce += h.c + 1;
        h.R_off = R_off; R_off += (long long)h.N * 6;
        for (int q = 0; q < 6; ++q) { h.fix[q] = s.perm[s.fix[q]]; h.fix_diag[q] = 0.0; }
    }
    xwave_.push_back(nsub_);
    fwave_.push_back(nsub_);
    waves_ = fwave_.size() > 2;
    if (waves_ && (!opt_.mixed || opt_.preconditioner == "Dirichlet_implicit" || opt_.print_matrices >= 2)) {
        err = "factor_wave_gb needs precision=mixed, an explicit preconditioner and print_matrices < 2";
        return HTF_EINVAL;
    }
    s_lean_ = !opt_.S_fp64;
    if (s_lean_ && (!opt_.mixed || opt_.preconditioner == "Dirichlet_implicit")) {
        err = "S_fp64=0 needs precision=mixed and an explicit preconditioner";
        return HTF_EINVAL;
    }
    // S tiles of the largest factor wave (S_fp64=0) or of all subdomains
    long long s_tiles = T_off;
    if (s_lean_) {
        s_tiles = 0;
        for (size_t w = 0; w + 1 < fwave_.size(); ++w) {
            const int a = fwave_[w], b = fwave_[w + 1];
            const SubDev &hl = hs_[b - 1];
            s_tiles = std::max(s_tiles, hl.T_off + (long long)hl.nt * (hl.nt + 1) / 2 - hs_[a].T_off);
        }
    }
    nslots_ = xb;
    nfull_ = nf;
    ntiles_ = T_off;
    // SYMV work units (default schedule; autotune_symv may replace it after set-up)
    for (auto &h : hs_) max_nbp_ = std::max(max_nbp_, h.nbp);
    if ((rc = alloc_units(err))) return rc;
    // clusters
    hc_.assign(ncl_, ClusterDev());
    long long M_off = 0;
    int gc_off = 0;
    long long MT_off = 0;
    int mt_rows = 0;
    std::vector<int2> mtl;
    for (int c = 0; c < ncl_; ++c) {
        hc_[c].nlam_c = p.clu[c].nlam_c;
        hc_[c].ngc = p.clu[c].ngc();
        hc_[c].M_off = M_off; M_off += (long long)hc_[c].ngc * hc_[c].ngc;
        hc_[c].gc_off = gc_off; gc_off += hc_[c].ngc;
        hc_[c].mt = (hc_[c].ngc + TILE - 1) / TILE;
        hc_[c].MT_off = MT_off; MT_off += (long long)hc_[c].mt * (hc_[c].mt + 1) / 2;
        hc_[c].mt_row_off = mt_rows; mt_rows += hc_[c].mt;
        for (int I = 0; I < hc_[c].mt; ++I) mtl.push_back(make_int2(c, I));
    }
    ngc_total_ = gc_off;
    // device allocations
    d_subs_ = alloc<SubDev>(nsub_, err, rc);
    d_cl_ = alloc<ClusterDev>(ncl_, err, rc);
    d_all_subs_ = alloc<int>(nsub_, err, rc);
    d_K_ = alloc<double>(kwave_max, err, rc);
    kpanel_total_ = kwave_max;
    d_F_ = alloc<double>(ntiles_ * TILE_ELEMS, err, rc);
    implicit_ = opt_.preconditioner == "Dirichlet_implicit";
    if (!implicit_) d_S_ = alloc<double>(s_tiles * TILE_ELEMS, err, rc);   // implicit: S applied through L_bb
    d_V_ = alloc<double>(V_off, err, rc);
    d_R_ = alloc<double>(R_off, err, rc);
    d_M_ = alloc<double>(M_off, err, rc);
    // the plain form's coarse solves read M as packed symmetric tiles (the dense M is freed after
    // set-up unless the batched mixed form needs it)
    nmt_ = int(mtl.size());
    d_mt_ = alloc<int2>(mtl.size(), err, rc);
    d_MT_ = alloc<double>(MT_off * TILE_ELEMS, err, rc);
    d_mP_ = alloc<double>(MT_off * TILE, err, rc);
    d_mD_ = alloc<double>((size_t)mt_rows * TILE, err, rc);
    if (!rc) CK(cudaMemcpyAsync(d_mt_, mtl.data(), mtl.size() * sizeof(int2), cudaMemcpyHostToDevice, s_));
    d_H_ = alloc<double>(36 * (size_t)nsub_, err, rc);
    d_status_ = alloc<int>(nsub_, err, rc);
    if (rc) return rc;
    // R in permuted order, Bc rows / entries
    {
        std::vector<double> R(R_off, 0.0);
        std::vector<int> bcrows(std::max(bcr, 1)), bptr(std::max(bce, 1));
        std::vector<int> bpos;
        std::vector<double> bval;
#pragma omp parallel for schedule(dynamic, 16)
        for (int d = 0; d < nsub_; ++d) {              // disjoint ranges of R per subdomain
            const Subdomain &s = p.sub[d];
            const SubDev &h = hs_[d];
            for (int j = 0; j < 6; ++j)
                for (int l = 0; l < s.n; ++l) R[h.R_off + (size_t)j * h.N + s.perm[l]] = s.R[l + (size_t)j * s.n];
        }
        for (int d = 0; d < nsub_; ++d) {
            const Subdomain &s = p.sub[d];
            const SubDev &h = hs_[d];
            for (int q = 0; q < h.c; ++q) bcrows[h.bcr_off + q] = s.bc_rows[q];
            // entries grouped by compressed row
            std::vector<std::vector<std::pair<int, double>>> rows(h.c);
            for (size_t e = 0; e < s.bc_row.size(); ++e) {
                int q = int(std::lower_bound(s.bc_rows.begin(), s.bc_rows.end(), s.bc_row[e]) - s.bc_rows.begin());
                rows[q].push_back({s.perm[s.bc_col[e]] - s.nr, s.bc_val[e]});
            }
            bptr[h.bce_off] = int(bpos.size());
            for (int q = 0; q < h.c; ++q) {
                for (auto &pr : rows[q]) { bpos.push_back(pr.first); bval.push_back(pr.second); }
                bptr[h.bce_off + q + 1] = int(bpos.size());
            }
        }
        d_bcr_ = alloc<int>(bcrows.size(), err, rc);
        d_bce_ptr_ = alloc<int>(bptr.size(), err, rc);
        d_bce_pos_ = alloc<int>(std::max<size_t>(bpos.size(), 1), err, rc);
        d_bce_val_ = alloc<double>(std::max<size_t>(bval.size(), 1), err, rc);
        if (rc) return rc;
        CK(cudaMemcpyAsync(d_R_, R.data(), R.size() * sizeof(double), cudaMemcpyHostToDevice, s_));
        CK(cudaMemcpyAsync(d_bcr_, bcrows.data(), bcrows.size() * sizeof(int), cudaMemcpyHostToDevice, s_));
        CK(cudaMemcpyAsync(d_bce_ptr_, bptr.data(), bptr.size() * sizeof(int), cudaMemcpyHostToDevice, s_));
        if (!bpos.empty()) {
            CK(cudaMemcpyAsync(d_bce_pos_, bpos.data(), bpos.size() * sizeof(int), cudaMemcpyHostToDevice, s_));
            CK(cudaMemcpyAsync(d_bce_val_, bval.data(), bval.size() * sizeof(double), cudaMemcpyHostToDevice, s_));
        }
        CK(cudaStreamSynchronize(s_));
    }
    // Bf gather (b slots) and row tables
    {
        std::vector<int> sptr(nslots_ + 1, 0), sent;
        for (int d = 0; d < nsub_; ++d) {
            const Subdomain &s = p.sub[d];
            const SubDev &h = hs_[d];
            for (int i = 0; i < h.nbp; ++i) {
                int slot = h.xb_off + i;
                if (i < h.nb)
                    for (int e = s.bf_ptr[i]; e < s.bf_ptr[i + 1]; ++e)
                        sent.push_back(2 * s.bf_lam[e] + (s.bf_sign[e] < 0 ? 1 : 0));
                sptr[slot + 1] = int(sent.size());
            }
        }
        std::vector<int> rslot(2 * (size_t)nlam_, -1);
        std::vector<double> rsign(2 * (size_t)nlam_, 0.0);
        for (int r = 0; r < nlam_; ++r)
            for (int k = 0; k < 2; ++k) {
                int d = p.rows[r].sub[k];
                if (d < 0) continue;
                const Subdomain &s = p.sub[d];
                int l = int(std::lower_bound(s.l2g.begin(), s.l2g.end(), p.rows[r].dof[k]) - s.l2g.begin());
                rslot[2 * r + k] = hs_[d].xb_off + (s.perm[l] - s.nr);
                rsign[2 * r + k] = p.rows[r].sign[k];
            }
        d_slot_ptr_ = alloc<int>(sptr.size(), err, rc);
        d_slot_ent_ = alloc<int>(std::max<size_t>(sent.size(), 1), err, rc);
        d_rslot_ = alloc<int>(rslot.size(), err, rc);
        d_rsign_ = alloc<double>(rsign.size(), err, rc);
        d_weight_ = alloc<double>(nlam_, err, rc);
        if (rc) return rc;
        CK(cudaMemcpyAsync(d_slot_ptr_, sptr.data(), sptr.size() * sizeof(int), cudaMemcpyHostToDevice, s_));
        CK(cudaMemcpyAsync(d_slot_ent_, sent.data(), sent.size() * sizeof(int), cudaMemcpyHostToDevice, s_));
        CK(cudaMemcpyAsync(d_rslot_, rslot.data(), rslot.size() * sizeof(int), cudaMemcpyHostToDevice, s_));
        CK(cudaMemcpyAsync(d_rsign_, rsign.data(), rsign.size() * sizeof(double), cudaMemcpyHostToDevice, s_));
        CK(cudaMemcpyAsync(d_weight_, p.weight.data(), nlam_ * sizeof(double), cudaMemcpyHostToDevice, s_));
        CK(cudaStreamSynchronize(s_));
    }
    // coarse gather map: gc[q] <- t slots
    {
        std::vector<std::vector<int>> lists(ngc_total_);
        for (int d = 0; d < nsub_; ++d) {
            const SubDev &h = hs_[d];
            const ClusterDev &c = hc_[h.cluster];
            for (int q = 0; q < h.c; ++q) lists[c.gc_off + p.sub[d].bc_rows[q]].push_back(h.t_off + q);
            for (int j = 0; j < 6; ++j) lists[c.gc_off + h.alpha_pos + j].push_back(h.t_off + h.c + j);
        }
        std::vector<int> gptr(ngc_total_ + 1, 0), gidx;
        for (int q = 0; q < ngc_total_; ++q) {
            for (int v : lists[q]) gidx.push_back(v);
            gptr[q + 1] = int(gidx.size());
        }
        d_gptr_ = alloc<int>(gptr.size(), err, rc);
        d_gidx_ = alloc<int>(std::max<size_t>(gidx.size(), 1), err, rc);
        if (rc) return rc;
        CK(cudaMemcpyAsync(d_gptr_, gptr.data(), gptr.size() * sizeof(int), cudaMemcpyHostToDevice, s_));
        CK(cudaMemcpyAsync(d_gidx_, gidx.data(), gidx.size() * sizeof(int), cudaMemcpyHostToDevice, s_));
    }
    // vectors
    const int nrhs = p.nrhs;
    d_f_ = alloc<double>((size_t)nfull_ * nrhs, err, rc);
    d_full_ = alloc<double>(nfull_, err, rc);
    d_full2_ = alloc<double>(nfull_, err, rc);
    d_lam_ = alloc<double>(nlam_, err, rc);
    d_g_ = alloc<double>(nlam_, err, rc);
    d_w_ = alloc<double>(nlam_, err, rc);
    d_Fw_ = alloc<double>(nlam_, err, rc);
    d_Pg_ = alloc<double>(nlam_, err, rc);
    d_z_ = alloc<double>(nlam_, err, rc);
    d_Pz_ = alloc<double>(nlam_, err, rc);
    d_d_ = alloc<double>(nlam_, err, rc);
    d_tmp_ = alloc<double>(nlam_, err, rc);
    d_xb_ = alloc<double>(nslots_, err, rc);
    d_yb_ = alloc<double>(nslots_, err, rc);
    if (implicit_) {              // (subdomain, 32-block) list of the two L_bb passes and their b-space vector
        std::vector<int2> lb;
        for (int d = 0; d < nsub_; ++d)
            for (int q = 0; q < hs_[d].nt; ++q) lb.push_back(make_int2(d, q));
        nlblk_ = int(lb.size());
        d_lblk_ = alloc<int2>(lb.size(), err, rc);
        d_tb_ = alloc<double>(nslots_, err, rc);
        if (!rc) CK(cudaMemcpyAsync(d_lblk_, lb.data(), lb.size() * sizeof(int2), cudaMemcpyHostToDevice, s_));
    }
    d_t_ = alloc<double>(t_off, err, rc);
    d_gc_ = alloc<double>(ngc_total_, err, rc);
    d_s_ = alloc<double>(ngc_total_, err, rc);
    d_a_ = alloc<double>(6 * (size_t)ncl_, err, rc);
    d_alpha_ = alloc<double>(6 * (size_t)ncl_, err, rc);
    npart_ = cdiv(nlam_, 256);
    d_partial_ = alloc<double>(npart_, err, rc);
    d_st_ = alloc<PcpgState>(1, err, rc);
    d_hist_ = alloc<double>(size_t(std::max(opt_.max_iter, 0)) + 1, err, rc);
    if (rc) return rc;
    {
        std::vector<int> csp(ncl_ + 1, 0), cs;
        for (int c = 0; c < ncl_; ++c) {
            for (int d : p.clu[c].subs) cs.push_back(d);
            csp[c + 1] = int(cs.size());
        }
        d_csp_ = alloc<int>(csp.size(), err, rc);
        d_cs_ = alloc<int>(cs.size(), err, rc);
        if (rc) return rc;
        CK(cudaMemcpyAsync(d_csp_, csp.data(), csp.size() * sizeof(int), cudaMemcpyHostToDevice, s_));
        CK(cudaMemcpyAsync(d_cs_, cs.data(), cs.size() * sizeof(int), cudaMemcpyHostToDevice, s_));
    }
    std::vector<int> ids(nsub_);
    std::iota(ids.begin(), ids.end(), 0);
    CK(cudaMemcpyAsync(d_all_subs_, ids.data(), nsub_ * sizeof(int), cudaMemcpyHostToDevice, s_));
    CK(cudaMemcpyAsync(d_cl_, hc_.data(), ncl_ * sizeof(ClusterDev), cudaMemcpyHostToDevice, s_));
    CK(cudaMemsetAsync(d_status_, 0, nsub_ * sizeof(int), s_));
    return HTF_OK;
}

// ---------------------------------------------------------------------------
int Engine::factorize(Problem &p, std::string &err) {
    int rc = HTF_OK;
    const Mesh &m = p.mesh;
    const int ne = m.n_elems();
    // element data: coordinates, permuted DOF positions, colours
    std::vector<double> ec(24 * (size_t)ne);
    std::vector<int> ep(24 * (size_t)ne);
#pragma omp parallel for schedule(dynamic, 4)
    for (int d = 0; d < nsub_; ++d) {
        const Subdomain &s = p.sub[d];
        for (int e : s.elems) {
            const int *q = &m.elems[8 * (size_t)e];
            for (int a = 0; a < 8; ++a) {
                for (int c = 0; c < 3; ++c) ec[24 * (size_t)e + 3 * a + c] = m.coords[3 * (size_t)q[a] + c];
                for (int c = 0; c < 3; ++c) {
                    int g = 3 * q[a] + c;
                    int l = int(std::lower_bound(s.l2g.begin(), s.l2g.end(), g) - s.l2g.begin());
                    ep[24 * (size_t)e + 8 * c + a] = s.perm[l];
                }
            }
        }
    }
    // greedy colouring: elements sharing a node get different colours
    std::vector<uint32_t> mask(m.n_nodes, 0u);
    std::vector<int> col(ne);
    int ncol = 0;
    for (int e = 0; e < ne; ++e) {
        uint32_t used = 0;
        for (int a = 0; a < 8; ++a) used |= mask[m.elems[8 * (size_t)e + a]];
        int c = 0;
        while (c < 32 && (used >> c & 1u)) ++c;
        if (c >= 32) { err = "element colouring needs more than 32 colours"; return HTF_EINVAL; }
        col[e] = c;
        ncol = std::max(ncol, c + 1);
        for (int a = 0; a < 8; ++a) mask[m.elems[8 * (size_t)e + a]] |= 1u << c;
    }
    // elements grouped by factor wave, then colour (with one wave: colour order)
    const int nfw = int(fwave_.size()) - 1;
    std::vector<int> wave_of(nsub_);
    for (int w = 0; w < nfw; ++w)
        for (int d = fwave_[w]; d < fwave_[w + 1]; ++d) wave_of[d] = w;
    std::vector<int> order(ne);
    ecptr_.assign((size_t)nfw * ncol + 1, 0);
    for (int e = 0; e < ne; ++e) ecptr_[(size_t)wave_of[m.elem_sub[e]] * ncol + col[e] + 1]++;
    for (size_t i = 0; i + 1 < ecptr_.size(); ++i) ecptr_[i + 1] += ecptr_[i];
    {
        std::vector<int> pos(ecptr_.begin(), ecptr_.end() - 1);
        for (int e = 0; e < ne; ++e) order[pos[(size_t)wave_of[m.elem_sub[e]] * ncol + col[e]]++] = e;
    }
    ncol_ = ncol;
    d_ec_ = alloc<double>(ec.size(), err, rc);
    d_ep_ = alloc<int>(ep.size(), err, rc);
    d_es_ = alloc<int>(ne, err, rc);
    d_order_ = alloc<int>(ne, err, rc);
    d_E_ = alloc<double>(nsub_, err, rc);
    d_nu_ = alloc<double>(nsub_, err, rc);
    if (rc) return rc;
    CK(cudaMemcpyAsync(d_ec_, ec.data(), ec.size() * sizeof(double), cudaMemcpyHostToDevice, s_));
    CK(cudaMemcpyAsync(d_ep_, ep.data(), ep.size() * sizeof(int), cudaMemcpyHostToDevice, s_));
    CK(cudaMemcpyAsync(d_es_, m.elem_sub.data(), ne * sizeof(int), cudaMemcpyHostToDevice, s_));
    CK(cudaMemcpyAsync(d_order_, order.data(), ne * sizeof(int), cudaMemcpyHostToDevice, s_));
    CK(cudaMemcpyAsync(d_E_, m.sub_E.data(), nsub_ * sizeof(double), cudaMemcpyHostToDevice, s_));
    CK(cudaMemcpyAsync(d_nu_, m.sub_nu.data(), nsub_ * sizeof(double), cudaMemcpyHostToDevice, s_));
    CK(cudaMemcpyAsync(d_subs_, hs_.data(), nsub_ * sizeof(SubDev), cudaMemcpyHostToDevice, s_));
    CK(set_gauss_points(s_));
    for (int c = 0; c < 3; ++c) bf_[c] = m.body_force[c];
    CK(cudaMemsetAsync(d_f_, 0, (size_t)nfull_ * p.nrhs * sizeof(double), s_));
    // explicit Dirichlet: snapshot S_reg - D_fix as tiles; implicit: nothing (L_bb stays in the factor)
    const bool dirichlet = opt_.preconditioner == "Dirichlet_explicit";
    const bool lumped = opt_.preconditioner == "lumped";
    max_tiles_ = 0;
    for (auto &h : hs_) max_tiles_ = std::max(max_tiles_, h.nt * (h.nt + 1) / 2);
    if ((dirichlet || lumped) && !d_S_) {
        err = "preconditioner blocks were not allocated";
        return HTF_EINVAL;
    }
    // step tables of every wave
    fw_.assign(nfw, FactorWave());
    for (int w = 0; w < nfw; ++w) {
        FactorWave &W = fw_[w];
        W.a = fwave_[w];
        W.b = fwave_[w + 1];
        W.eoff = (size_t)w * ncol;
        if (!sub_blk0_.empty()) {
            W.blk0 = sub_blk0_[W.a];
            W.blk1 = sub_blk0_[W.b];
        }
        std::vector<std::vector<StepDesc>> steps;
        std::vector<std::vector<int>> snap_after;      // subdomains whose interior ends after step s
        std::vector<int> snap_first;                   // nr == 0
        for (int d = W.a; d < W.b; ++d) {
            const SubDev &h = hs_[d];
            W.kdoubles += kpanel_doubles(h.nr, h.nbp);
            std::vector<std::pair<int, int>> blocks;      // steps never cross from the interior into the b set
            for (int k = 0; k < h.nr; k += CHOL_STEP) blocks.push_back({k, std::min(CHOL_STEP, h.nr - k)});
            int interior_steps = int(blocks.size());
            for (int k = h.nr; k < h.N; k += CHOL_STEP) blocks.push_back({k, std::min(CHOL_STEP, h.N - k)});
            if (steps.size() < blocks.size()) { steps.resize(blocks.size()); snap_after.resize(blocks.size()); }
            for (size_t s = 0; s < blocks.size(); ++s) steps[s].push_back({d, blocks[s].first, blocks[s].second, 0, 0});
            if (interior_steps == 0) snap_first.push_back(d);
            else snap_after[interior_steps - 1].push_back(d);
        }
        std::vector<StepDesc> flat;
        for (auto &v : steps) {
            int tri = 0, rb = 0;
            for (auto &x : v) {
                const int rows = hs_[x.d].N - x.k - x.nb, nbr = (rows + 63) / 64;
                x.tri0 = tri; tri += nbr * (nbr + 1) / 2;
                x.rb0 = rb; rb += (rows + 127) / 128;
            }
            W.cnt.push_back(int(v.size()));
            W.ntri.push_back(tri);
            W.nrb.push_back(rb);
            W.soff.push_back(flat.size());
            flat.insert(flat.end(), v.begin(), v.end());
        }
        std::vector<int> snap_flat;
        for (auto &v : snap_after) {
            W.snap_off.push_back(snap_flat.size());
            W.nsnap.push_back(int(v.size()));
            snap_flat.insert(snap_flat.end(), v.begin(), v.end());
        }
        W.snap_first_off = snap_flat.size();
        W.nsnap_first = int(snap_first.size());
        snap_flat.insert(snap_flat.end(), snap_first.begin(), snap_first.end());
        // entry hints of every step's SYRK and panel-solve grids
        std::vector<int> hints;
        for (size_t s = 0; s < steps.size(); ++s) {
            W.htri.push_back(hints.size());
            step_hints(steps[s], W.ntri[s], true, hints);
            W.hrb.push_back(hints.size());
            step_hints(steps[s], W.nrb[s], false, hints);
        }
        W.steps = alloc<StepDesc>(std::max<size_t>(flat.size(), 1), err, rc);
        W.snap = alloc<int>(std::max<size_t>(snap_flat.size(), 1), err, rc);
        W.hints = alloc<int>(std::max<size_t>(hints.size(), 1), err, rc);
        if (rc) return rc;
        CK(cudaMemcpyAsync(W.steps, flat.data(), flat.size() * sizeof(StepDesc), cudaMemcpyHostToDevice, s_));
        if (!hints.empty())
            CK(cudaMemcpyAsync(W.hints, hints.data(), hints.size() * sizeof(int), cudaMemcpyHostToDevice, s_));
        if (!snap_flat.empty())
            CK(cudaMemcpyAsync(W.snap, snap_flat.data(), snap_flat.size() * sizeof(int), cudaMemcpyHostToDevice, s_));
        // the host copies of flat, hints and snap_flat must outlive the asynchronous copies
        CK(cudaStreamSynchronize(s_));
    }
    CK(cudaFuncSetAttribute(k_syrk_update, cudaFuncAttributeMaxDynamicSharedMemorySize, SYRK_SMEM));
    {
        double *X = nullptr;
        CK(cudaMalloc(&X, std::max<long long>(xwave_max_, 1) * sizeof(double)));
        for (int w = 0; w < nfw; ++w) factor_wave(w, true, X);
        const cudaError_t le = cudaGetLastError();
        const cudaError_t se = cudaStreamSynchronize(s_);
        cudaFree(X);
        CK(le);
        CK(se);
    }
    int max_cols = 0;
    for (auto &h : hs_) max_cols = std::max(max_cols, h.c + 6);
    k_build_V<<<dim3(nsub_, max_cols), 256, 0, s_>>>(d_subs_, d_F_, d_bce_ptr_, d_bce_pos_, d_bce_val_, d_R_, d_V_);
    CK(cudaGetLastError());
    std::vector<int> status(nsub_);
    CK(cudaMemcpyAsync(status.data(), d_status_, nsub_ * sizeof(int), cudaMemcpyDeviceToHost, s_));
    CK(cudaStreamSynchronize(s_));
    for (int d = 0; d < nsub_; ++d)
        if (status[d]) {
            status_sub = d;
            err = "K_reg of subdomain " + std::to_string(d) + " is not positive definite (column " +
                  std::to_string(status[d] - 1) + ")";
            return HTF_ENOTSPD;
        }
    if (!waves_) {                  // resident factors: the element data is not needed again
        for (void *q : {(void *)d_ec_, (void *)d_ep_, (void *)d_es_, (void *)d_order_, (void *)d_E_, (void *)d_nu_})
            release(q);
        d_ec_ = d_E_ = d_nu_ = nullptr;
        d_ep_ = d_es_ = d_order_ = nullptr;
    }
    return HTF_OK;
}

void Engine::factor_wave(int w, bool build, double *X) {
    const FactorWave &W = fw_[w];
    const bool dirichlet = opt_.preconditioner == "Dirichlet_explicit";
    const bool lumped = opt_.preconditioner == "lumped";
    const int nw = W.b - W.a;
    // S tiles: all resident (from tile 0), or this wave's only, made into tensor-core slabs below
    const long long st0 = s_lean_ ? hs_[W.a].T_off : 0;
    cudaMemsetAsync(d_K_, 0, W.kdoubles * sizeof(double), s_);
    for (int c = 0; c < ncol_; ++c) {
        const int e0 = ecptr_[W.eoff + c], cnt = ecptr_[W.eoff + c + 1] - e0;
        if (cnt == 0) continue;
        k_assemble<<<cnt, 64, 0, s_>>>(d_order_ + e0, cnt, d_ec_, d_es_, d_ep_, d_E_, d_nu_, d_subs_, d_K_,
                                       build ? d_f_ : nullptr, bf_[0], bf_[1], bf_[2]);
    }
    k_regularize<<<nw, 128, 0, s_>>>(d_subs_ + W.a, nw, d_K_);
    if (build && opt_.print_matrices >= 2) {      // K_reg panels before the factorisation, for htf_dump (one wave)
        dumpK_.assign(size_t(kpanel_total_), 0.0);
        cudaMemcpyAsync(dumpK_.data(), d_K_, dumpK_.size() * sizeof(double), cudaMemcpyDeviceToHost, s_);
        cudaStreamSynchronize(s_);
    }
    if (build && lumped)            // lumped: K_bb before any elimination
        k_snapshot<<<dim3(nw, max_tiles_), 256, 0, s_>>>(d_all_subs_ + W.a, d_subs_, d_K_, d_S_, st0);
    if (build && dirichlet && W.nsnap_first > 0)
        k_snapshot<<<dim3(W.nsnap_first, max_tiles_), 256, 0, s_>>>(W.snap + W.snap_first_off, d_subs_, d_K_, d_S_,
                                                                    st0);
    for (size_t s = 0; s < W.soff.size(); ++s) {
        const int cnt = W.cnt[s];
        const StepDesc *ds = W.steps + W.soff[s];
        k_potrf_diag<<<cnt, CHOL_STEP, 0, s_>>>(ds, d_subs_, d_K_, d_status_);
        if (W.nrb[s] > 0) k_trsm_panel<<<W.nrb[s], 128, 0, s_>>>(ds, cnt, d_subs_, d_K_, W.hints + W.hrb[s]);
        if (W.ntri[s] > 0)
            k_syrk_update<<<W.ntri[s], 256, SYRK_SMEM, s_>>>(ds, cnt, d_subs_, d_K_, W.hints + W.htri[s]);
        if (build && dirichlet && W.nsnap[s] > 0)
            k_snapshot<<<dim3(W.nsnap[s], max_tiles_), 256, 0, s_>>>(W.snap + W.snap_off[s], d_subs_, d_K_, d_S_,
                                                                     st0);
    }
    if (!build) return;
    if (s_lean_ && (dirichlet || lumped) && W.blk1 > W.blk0) {
        const GemmBlock *wb = static_cast<const GemmBlock *>(d_blocks_) + W.blk0;
        k_slab_amax<<<dim3(W.blk1 - W.blk0, maxks_), 256, 0, s_>>>(wb, d_subs_, d_S_, st0, d_amaxS_);
        k_make_slabs<<<dim3(W.blk1 - W.blk0, maxks_), 256, 0, s_>>>(wb, d_subs_, d_S_, d_AS_, st0, d_amaxS_);
    }
    // X = L_bb^{-1}, F = X^T X, in the L_bb^{-1} waves of this factor wave, sharing one scratch buffer
    for (size_t x = 0; x + 1 < xwave_.size(); ++x) {
        const int a = xwave_[x], b = xwave_[x + 1];
        if (a < W.a || b > W.b) continue;
        int wnt = 0, wtiles = 0;
        for (int d = a; d < b; ++d) {
            wnt = std::max(wnt, hs_[d].nt);
            wtiles = std::max(wtiles, hs_[d].nt * (hs_[d].nt + 1) / 2);
        }
        for (int i = 0; i < wnt; ++i)
            k_trtri_step<<<dim3(b - a, i + 1), 256, 0, s_>>>(i, d_all_subs_ + a, d_subs_, d_K_, X);
        k_lauum_tiles<<<dim3(b - a, wtiles), 256, 0, s_>>>(d_all_subs_ + a, d_subs_, X, d_F_);
    }
}

// Gf = Bf Rf, Rf_d = R_d H_d (Cluster.cpp:1332-1352); (Gf^T Gf)^{-1} (1227-1273)
int Engine::outer_coarse(Problem &p, std::string &err) {
    int rc = HTF_OK;
    const int m = 6 * ncl_;
    std::vector<int> gcl(2 * (size_t)nlam_, -1);
    std::vector<double> gval(12 * (size_t)nlam_, 0.0);
#pragma omp parallel for schedule(static, 4096)
    for (int r = 0; r < nlam_; ++r) {
        for (int k = 0; k < 2; ++k) {
            int d = p.rows[r].sub[k];
            if (d < 0) continue;
            const Subdomain &s = p.sub[d];
            int l = int(std::lower_bound(s.l2g.begin(), s.l2g.end(), p.rows[r].dof[k]) - s.l2g.begin());
            double rf[6];
            for (int q = 0; q < 6; ++q) {
                double v = 0.0;
                for (int j = 0; j < 6; ++j) v += s.R[l + size_t(j) * s.n] * Hd_[d][j * 6 + q];
                rf[q] = p.rows[r].sign[k] * v;
            }
            int slot = (k == 1 && gcl[2 * r] == s.cluster) ? 0 : k;
            gcl[2 * r + slot] = s.cluster;
            for (int q = 0; q < 6; ++q) gval[6 * (2 * (size_t)r + slot) + q] += rf[q];
        }
    }
    std::vector<double> GtG(size_t(m) * m, 0.0);
    // per-cluster entry lists for the reduction
    std::vector<std::vector<int>> crow(ncl_);
    std::vector<std::vector<double>> cval(ncl_);
    for (int r = 0; r < nlam_; ++r)
        for (int k = 0; k < 2; ++k) {
            int c = gcl[2 * r + k];
            if (c < 0) continue;
            crow[c].push_back(r);
            for (int q = 0; q < 6; ++q) cval[c].push_back(gval[6 * (2 * (size_t)r + k) + q]);
        }
    // Gf^T Gf: partial sums over a fixed number of row chunks (independent of
    // the thread count), added in chunk order; small problems keep one chunk
    const int nch = (nlam_ >= (1 << 16) && m <= 512) ? 32 : 1;
    std::vector<std::vector<double>> gpartial(nch);
#pragma omp parallel for schedule(dynamic, 1)
    for (int ch = 0; ch < nch; ++ch) {
        std::vector<double> &P = gpartial[ch];
        P.assign(size_t(m) * m, 0.0);
        const int r0 = int((long long)nlam_ * ch / nch), r1 = int((long long)nlam_ * (ch + 1) / nch);
        for (int r = r0; r < r1; ++r)
            for (int k1 = 0; k1 < 2; ++k1)
                for (int k2 = 0; k2 < 2; ++k2) {
                    int c1 = gcl[2 * r + k1], c2 = gcl[2 * r + k2];
                    if (c1 < 0 || c2 < 0) continue;
                    for (int a = 0; a < 6; ++a)
                        for (int b = 0; b < 6; ++b)
                            P[(6 * c1 + a) + size_t(6 * c2 + b) * m] +=
                                gval[6 * (2 * (size_t)r + k1) + a] * gval[6 * (2 * (size_t)r + k2) + b];
                }
    }
    if (nch == 1) GtG.swap(gpartial[0]);
    else
        for (int ch = 0; ch < nch; ++ch)
            for (size_t i = 0; i < GtG.size(); ++i) GtG[i] += gpartial[ch][i];
    if (opt_.print_matrices >= 2) {               // for htf_dump
        gtg_ = GtG;
        gcl_ = gcl;
        gval_ = gval;
    }
    std::vector<double> L(GtG);
    if (!chol_lower(m, L.data(), m)) { err = "Gf^T Gf is not positive definite"; return HTF_ENOTSPD; }
    invGtG_.assign(size_t(m) * m, 0.0);
    for (int i = 0; i < m; ++i) invGtG_[i + size_t(i) * m] = 1.0;
    chol_solve(m, L.data(), m, invGtG_.data(), m, m);
    // chunks
    const int CH = 1024;
    std::vector<int> ch_cl, ch_beg, ch_end, clp(ncl_ + 1, 0), rows_all;
    std::vector<double> vals_all;
    for (int c = 0; c < ncl_; ++c) {
        int base = int(rows_all.size());
        rows_all.insert(rows_all.end(), crow[c].begin(), crow[c].end());
        vals_all.insert(vals_all.end(), cval[c].begin(), cval[c].end());
        int n = int(crow[c].size());
        for (int b = 0; b < std::max(n, 1); b += CH) {
            ch_cl.push_back(c);
            ch_beg.push_back(base + b);
            ch_end.push_back(base + std::min(n, b + CH));
        }
        clp[c + 1] = int(ch_cl.size());
    }
    nchunks_ = int(ch_cl.size());
    d_gcl_ = alloc<int>(gcl.size(), err, rc);
    d_gval_ = alloc<double>(gval.size(), err, rc);
    d_chunk_cl_ = alloc<int>(nchunks_, err, rc);
    d_chunk_beg_ = alloc<int>(nchunks_, err, rc);
    d_chunk_end_ = alloc<int>(nchunks_, err, rc);
    d_cl_chunk_ptr_ = alloc<int>(ncl_ + 1, err, rc);
    d_crow_ = alloc<int>(std::max<size_t>(rows_all.size(), 1), err, rc);
    d_cval_ = alloc<double>(std::max<size_t>(vals_all.size(), 1), err, rc);
    d_invGtG_ = alloc<double>(invGtG_.size(), err, rc);
    d_gpart_ = alloc<double>(6 * (size_t)nchunks_, err, rc);
    if (rc) return rc;
    CK(cudaMemcpyAsync(d_gcl_, gcl.data(), gcl.size() * sizeof(int), cudaMemcpyHostToDevice, s_));
    CK(cudaMemcpyAsync(d_gval_, gval.data(), gval.size() * sizeof(double), cudaMemcpyHostToDevice, s_));
    CK(cudaMemcpyAsync(d_chunk_cl_, ch_cl.data(), nchunks_ * sizeof(int), cudaMemcpyHostToDevice, s_));
    CK(cudaMemcpyAsync(d_chunk_beg_, ch_beg.data(), nchunks_ * sizeof(int), cudaMemcpyHostToDevice, s_));
    CK(cudaMemcpyAsync(d_chunk_end_, ch_end.data(), nchunks_ * sizeof(int), cudaMemcpyHostToDevice, s_));
    CK(cudaMemcpyAsync(d_cl_chunk_ptr_, clp.data(), (ncl_ + 1) * sizeof(int), cudaMemcpyHostToDevice, s_));
    if (!rows_all.empty()) {
        CK(cudaMemcpyAsync(d_crow_, rows_all.data(), rows_all.size() * sizeof(int), cudaMemcpyHostToDevice, s_));
        CK(cudaMemcpyAsync(d_cval_, vals_all.data(), vals_all.size() * sizeof(double), cudaMemcpyHostToDevice, s_));
    }
    CK(cudaMemcpyAsync(d_invGtG_, invGtG_.data(), invGtG_.size() * sizeof(double), cudaMemcpyHostToDevice, s_));
    CK(cudaStreamSynchronize(s_));
    return HTF_OK;
}

// ---------------------------------------------------------------------------
int Engine::setup(Problem &p, std::string &err) {
    int dev_count = 0;
    if (cudaGetDeviceCount(&dev_count) != cudaSuccess || dev_count == 0) {
        err = "no CUDA device";
        return HTF_ENODEV;
    }
    cudaGetLastError();           // an error left by an earlier, unrelated call is not this setup's
    auto clk = std::chrono::steady_clock::now();
    auto lap = [&](int i) {
        const auto now = std::chrono::steady_clock::now();
        phase_ms[i] = std::chrono::duration<double, std::milli>(now - clk).count();
        clk = now;
    };
    CK(cudaSetDevice(opt_.device));
    CK(cudaStreamCreateWithFlags(&own_s_, cudaStreamNonBlocking));
    s_ = own_s_;
    cudaEvent_t e0, e1;
    CK(cudaEventCreate(&e0));
    CK(cudaEventCreate(&e1));
    CK(cudaEventRecord(e0, s_));
    CK(cudaStreamSynchronize(s_));
    lap(1);
    int rc = upload_layout(p, err);
    if (!rc) rc = check(cudaStreamSynchronize(s_), "sync", err);
    if (!rc) {                    // the projector keeps 12 doubles per cluster in shared memory
        const int smem = 12 * ncl_ * int(sizeof(double));
        int optin = 0;
        rc = check(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, opt_.device),
                   "cudaDeviceGetAttribute", err);
        // the kernel's 2 KB of static shared memory count against the same limits
        if (!rc && smem + 2048 > optin) {
            err = "projector: " + std::to_string(ncl_) + " clusters need " + std::to_string(smem + 2048) +
                  " bytes of shared memory, the device allows " + std::to_string(optin) + " per block";
            rc = HTF_EINVAL;
        }
        if (!rc)
            rc = check(cudaFuncSetAttribute(k_gf_apply_fused, cudaFuncAttributeMaxDynamicSharedMemorySize, smem),
                       "cudaFuncSetAttribute(k_gf_apply_fused)", err);
        if (!rc)
            rc = check(cudaFuncSetAttribute(k_gf_coef, cudaFuncAttributeMaxDynamicSharedMemorySize, smem / 2),
                       "cudaFuncSetAttribute(k_gf_coef)", err);
        if (!rc)
            rc = check(cudaFuncSetAttribute(k_gf_apply, cudaFuncAttributeMaxDynamicSharedMemorySize, smem / 2),
                       "cudaFuncSetAttribute(k_gf_apply)", err);
    }
    lap(2);
    if (!rc && s_lean_) rc = plan_slabs(opt_.batch, err);   // S_i goes into its slabs wave by wave
    if (!rc) rc = factorize(p, err);
    lap(3);
    if (!rc) {                    // body-force load, load ownership and the displacement gather map
        ndof_ = 3 * p.mesh.n_nodes;
        std::vector<int> own(nfull_, -1), win(ndof_, -1), owner(ndof_, -1);
        for (int d = 0; d < nsub_; ++d)
            for (int g : p.sub[d].l2g)
                if (owner[g] < 0) owner[g] = d;
        for (int d = 0; d < nsub_; ++d) {
            const Subdomain &s = p.sub[d];
            for (int l = 0; l < s.n; ++l) {
                const int slot = hs_[d].nfull_off + s.perm[l], g = s.l2g[l];
                if (owner[g] == d) own[slot] = g;
                win[g] = slot;              // highest subdomain index wins (Cluster.cpp:1672-1676)
            }
        }
        d_fbody_ = alloc<double>(nfull_, err, rc);
        d_own_ = alloc<int>(nfull_, err, rc);
        d_win_ = alloc<int>(ndof_, err, rc);
        if (!rc) rc = check(cudaMemcpyAsync(d_fbody_, d_f_, nfull_ * sizeof(double), cudaMemcpyDeviceToDevice, s_), "copy", err);
        if (!rc) rc = check(cudaMemcpyAsync(d_own_, own.data(), nfull_ * sizeof(int), cudaMemcpyHostToDevice, s_), "copy", err);
        if (!rc) rc = check(cudaMemcpyAsync(d_win_, win.data(), ndof_ * sizeof(int), cudaMemcpyHostToDevice, s_), "copy", err);
        if (!rc) rc = check(cudaStreamSynchronize(s_), "sync", err);
    }
    lap(4);
    if (!rc) rc = coarse(p, err);
    if (!rc) {
        k_pack_M<<<nmt_, 256, 0, s_>>>(d_mt_, d_cl_, d_M_, d_MT_);
        rc = check(cudaGetLastError(), "k_pack_M", err);
        if (!rc) rc = check(cudaStreamSynchronize(s_), "sync", err);
        if (!rc && !opt_.mixed) {
            release(d_M_);
            d_M_ = nullptr;
        }
    }
    lap(5);
    if (!rc) rc = outer_coarse(p, err);
    lap(6);
    if (!rc) rc = autotune_symv(err);             // SYMV work-unit schedule of this problem class
    if (!rc && opt_.mixed) {
        // FP16-pair slabs for the tensor-core products of the batched form; the
        // FP64 tiles stay resident for the FP64 residuals
        mixed_ = true;
        rc = setup_batch(opt_.batch, err);
        if (!rc && s_lean_) {         // the FP64 S tiles of the last wave are not needed again
            rc = check(cudaStreamSynchronize(s_), "sync", err);
            release(d_S_);
            d_S_ = nullptr;
        }
    }
    if (!rc) rc = check(cudaEventRecord(e1, s_), "cudaEventRecord", err);
    if (!rc) rc = check(cudaEventSynchronize(e1), "cudaEventSynchronize", err);
    lap(7);
    float ms = 0.f;
    if (!rc) cudaEventElapsedTime(&ms, e0, e1);
    setup_ms = ms;
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    // algorithmic bytes of one FP64 F apply (triangular tiles, V, lambda gather/scatter)
    double bytes = 0.0;
    const double sz = 8.0;
    for (int d = 0; d < nsub_; ++d) {
        const Subdomain &s = p.sub[d];
        const double nb = s.nb;
        int m_i = s.bf_ptr[s.nb];
        bytes += sz * nb * (nb + 1) / 2 + 8.0 * nb * (s.c() + 6) + m_i * (8.0 + 4.0) + m_i * 8.0;
    }
    fapply_bytes_ = bytes;
    return rc;
}

// ---------------------------------------------------------------------------
void Engine::op_F(const double *w, double *Fw, const double *dotv, double *partial, PcpgState *st) {
    k_gather_b<<<cdiv(nslots_, 256), 256, 0, s_>>>(nslots_, d_slot_ptr_, d_slot_ent_, w, nullptr, d_xb_, st);
    k_symv_units<double><<<nunits_ + nsub_, SYMV_WARPS * 32, symv_smem_, s_>>>(d_units_, d_subs_, d_F_, d_V_, d_xb_, d_ypart_, d_t_, st);
    k_gc<<<cdiv(ngc_total_, 256), 256, 0, s_>>>(ngc_total_, d_gptr_, d_gidx_, d_t_, d_gc_, st);
    coarse_apply(d_gc_, d_s_, st);
    k_reduce_correct<<<dim3(nsub_, cdiv(max_nbp_, 256)), 256, 0, s_>>>(d_subs_, d_units_, d_rbptr_, d_rbunit_, d_ypart_, d_cl_, d_V_, d_bcr_,
                                                                       d_s_, d_yb_, st);
    k_rows<<<npart_, 256, 0, s_>>>(nlam_, d_rslot_, d_rsign_, d_yb_, nullptr, Fw, dotv, partial, st);
}

void Engine::op_M(const double *x, double *z, PcpgState *st) {
    k_gather_b<<<cdiv(nslots_, 256), 256, 0, s_>>>(nslots_, d_slot_ptr_, d_slot_ent_, x, d_weight_, d_xb_, st);
    if (implicit_) {
        k_lbt_x<<<nlblk_, 128, 0, s_>>>(d_lblk_, d_subs_, d_K_, d_xb_, d_tb_, st);
        k_lb_t<<<nlblk_, 128, 0, s_>>>(d_lblk_, d_subs_, d_K_, d_tb_, d_xb_, d_yb_, st);
        k_rows<<<npart_, 256, 0, s_>>>(nlam_, d_rslot_, d_rsign_, d_yb_, d_weight_, z, nullptr, nullptr, st);
        return;
    }
    k_symv_units<double><<<nunits_, SYMV_WARPS * 32, symv_smem_, s_>>>(d_units_, d_subs_, d_S_, d_V_, d_xb_, d_ypart_, d_t_, st);
    k_reduce_correct<<<dim3(nsub_, cdiv(max_nbp_, 256)), 256, 0, s_>>>(d_subs_, d_units_, d_rbptr_, d_rbunit_, d_ypart_, d_cl_, d_V_, d_bcr_,
                                                                       nullptr, d_yb_, st);
    k_rows<<<npart_, 256, 0, s_>>>(nlam_, d_rslot_, d_rsign_, d_yb_, d_weight_, z, nullptr, nullptr, st);
}

void Engine::op_P(const double *x, double *Px, double *alpha_out, const double *dotv, double *partial,
                  PcpgState *st) {
    k_gft_partial<<<nchunks_, 256, 0, s_>>>(d_chunk_cl_, d_chunk_beg_, d_chunk_end_, d_crow_, d_cval_, x, d_gpart_, st);
    // the coarse coefficient once, then the rows (k_gf_apply_fused, which
    // recomputes it in every CTA, stays for the allocation-free entry point)
    k_gf_coef<<<1, 256, 6 * ncl_ * sizeof(double), s_>>>(ncl_, d_cl_chunk_ptr_, d_gpart_, d_invGtG_, d_a_, alpha_out,
                                                          st);
    k_gf_apply<<<npart_, 256, 6 * ncl_ * sizeof(double), s_>>>(nlam_, ncl_, d_a_, d_gcl_, d_gval_, x, Px, dotv,
                                                                partial, st);
}

void Engine::iteration(PcpgState *st) {
    op_F(d_w_, d_Fw_, d_w_, d_partial_, st);
    k_update_lam_g<<<std::min(npart_, 1184), 256, 0, s_>>>(nlam_, d_partial_, npart_, d_w_, d_Fw_, d_lam_, d_g_, st);
    op_P(d_g_, d_Pg_, d_alpha_, nullptr, nullptr, st);
    op_M(d_Pg_, d_z_, st);
    op_P(d_z_, d_Pz_, nullptr, d_g_, d_partial_, st);
    k_update_w<<<std::min(npart_, 1184), 256, 0, s_>>>(nlam_, d_partial_, npart_, d_Pz_, d_w_, st);
    k_finish_iter<<<1, 256, 0, s_>>>(d_partial_, npart_, st, d_hist_);
}

int Engine::apply(int op, const double *x, double *y, int nrhs, std::string &err) {
    cudaGetLastError();
    if (mixed_ && bK_ > 0) return apply_batch(op, x, y, nrhs, err);
    for (int k = 0; k < nrhs; ++k) {
        CK(cudaMemcpyAsync(d_tmp_, x + (size_t)k * nlam_, nlam_ * sizeof(double), cudaMemcpyHostToDevice, s_));
        if (op == 0) op_F(d_tmp_, d_Fw_, nullptr, nullptr, nullptr);
        else if (op == 1) op_P(d_tmp_, d_Fw_, nullptr, nullptr, nullptr, nullptr);
        else op_M(d_tmp_, d_Fw_, nullptr);
        CK(cudaGetLastError());
        CK(cudaMemcpyAsync(y + (size_t)k * nlam_, d_Fw_, nlam_ * sizeof(double), cudaMemcpyDeviceToHost, s_));
    }
    CK(cudaStreamSynchronize(s_));
    return HTF_OK;
}

// x = K_HT^+ f, d = Bf x, lambda0 = Gf (GfTGf)^{-1} Rf^T f  (Cluster.cpp:1385-1394, 967-1040);
// with x_solved the triangular solves K_reg^{-1} f were done already (for
// several load cases at once) and x_solved holds them
void Engine::init_rhs(const double *f, const double *x_solved) {
    const double *x = x_solved;
    if (!x) {
        cudaMemcpyAsync(d_full_, f, nfull_ * sizeof(double), cudaMemcpyDeviceToDevice, s_);
        k_trsv_fwd<<<dim3(nsub_, 1), 256, 0, s_>>>(d_subs_, d_K_, d_full_, 0);
        k_trsv_bwd<<<dim3(nsub_, 1), 256, 0, s_>>>(d_subs_, d_K_, d_full_, 0);
        x = d_full_;
    }
    k_bc_rt<<<nsub_, 256, 0, s_>>>(d_subs_, d_bce_ptr_, d_bce_pos_, d_bce_val_, d_R_, x, f, d_t_);
    k_gc<<<cdiv(ngc_total_, 256), 256, 0, s_>>>(ngc_total_, d_gptr_, d_gidx_, d_t_, d_gc_, nullptr);
    coarse_apply(d_gc_, d_s_, nullptr);
    k_full_to_b<<<nsub_, 256, 0, s_>>>(d_subs_, x, d_yb_);
    k_correct<<<nsub_, 256, 0, s_>>>(d_subs_, d_cl_, d_V_, d_bcr_, d_s_, d_yb_, nullptr);
    k_rows<<<npart_, 256, 0, s_>>>(nlam_, d_rslot_, d_rsign_, d_yb_, nullptr, d_d_, nullptr, nullptr, nullptr);
    k_e_vec<<<cdiv(6 * ncl_, 128), 128, 0, s_>>>(ncl_, d_csp_, d_cs_, d_subs_, d_H_, d_t_, d_gc_);
    k_small_gemv<<<1, 256, 0, s_>>>(6 * ncl_, d_invGtG_, d_gc_, d_a_);
    k_gf_mult<<<npart_, 256, 0, s_>>>(nlam_, d_gcl_, d_gval_, d_a_, d_lam_);
}

// g = F lambda - d ; Pg (alpha) ; z = M Pg ; Pz ; g.Pz partials -> st  (Cluster.cpp:1398-1412)
double Engine::pcpg_start(PcpgState *st) {
    op_F(d_lam_, d_g_, nullptr, nullptr, nullptr);
    k_axpby<<<npart_, 256, 0, s_>>>(nlam_, -1.0, d_d_, 1.0, d_g_);
    op_P(d_g_, d_Pg_, d_alpha_, nullptr, nullptr, nullptr);
    op_M(d_Pg_, d_z_, nullptr);
    op_P(d_z_, d_Pz_, nullptr, d_g_, d_partial_, nullptr);
    k_init_state<<<1, 256, 0, s_>>>(d_partial_, npart_, st, opt_.eps_iter, opt_.max_iter);
    return 0.0;
}

// u = K_HT^+(f - Bf^T lambda) - Rf alpha  (Cluster.cpp:1648-1678)
void Engine::reconstruct(const double *f, double *u_dev) {
    cudaMemcpyAsync(d_full_, f, nfull_ * sizeof(double), cudaMemcpyDeviceToDevice, s_);
    k_gather_b<<<cdiv(nslots_, 256), 256, 0, s_>>>(nslots_, d_slot_ptr_, d_slot_ent_, d_lam_, nullptr, d_xb_, nullptr);
    k_full_minus_b<<<nsub_, 256, 0, s_>>>(d_subs_, d_xb_, d_full_);
    cudaMemcpyAsync(d_full2_, d_full_, nfull_ * sizeof(double), cudaMemcpyDeviceToDevice, s_);
    k_trsv_fwd<<<dim3(nsub_, 1), 256, 0, s_>>>(d_subs_, d_K_, d_full2_, 0);
    k_trsv_bwd<<<dim3(nsub_, 1), 256, 0, s_>>>(d_subs_, d_K_, d_full2_, 0);
    k_bc_rt<<<nsub_, 256, 0, s_>>>(d_subs_, d_bce_ptr_, d_bce_pos_, d_bce_val_, d_R_, d_full2_, d_full_, d_t_);
    k_gc<<<cdiv(ngc_total_, 256), 256, 0, s_>>>(ngc_total_, d_gptr_, d_gidx_, d_t_, d_gc_, nullptr);
    coarse_apply(d_gc_, d_s_, nullptr);
    k_sub_bct<<<nsub_, 32, 0, s_>>>(d_subs_, d_cl_, d_bcr_, d_bce_ptr_, d_bce_pos_, d_bce_val_, d_s_, d_full_);
    k_trsv_fwd<<<dim3(nsub_, 1), 256, 0, s_>>>(d_subs_, d_K_, d_full_, 0);
    k_trsv_bwd<<<dim3(nsub_, 1), 256, 0, s_>>>(d_subs_, d_K_, d_full_, 0);
    k_add_R<<<nsub_, 256, 0, s_>>>(d_subs_, d_cl_, d_R_, d_H_, d_s_, d_alpha_, d_full_);
    if (u_dev) k_gather_u<<<cdiv(ndof_, 256), 256, 0, s_>>>(ndof_, d_win_, d_full_, u_dev);
}

// one load case: Cluster::pcpg (Cluster.cpp:1363-1458) + printVTK (1648-1678)
int Engine::solve_one(Problem &p, int rhs, double *u_dev, int &iters, double &norm0, double &rel,
                      double &solve_ms, std::string &err) {
    (void)p;
    const double *f = d_f_ + (size_t)rhs * nfull_;
    cudaEvent_t e0, e1;
    CK(cudaEventCreate(&e0));
    CK(cudaEventCreate(&e1));
    init_rhs(f);
    CK(cudaEventRecord(e0, s_));
    pcpg_start(d_st_);
    CK(cudaMemcpyAsync(d_w_, d_Pz_, nlam_ * sizeof(double), cudaMemcpyDeviceToDevice, s_));
    CK(cudaGetLastError());
    if (!graph_) {
        cudaGraph_t g;
        CK(cudaStreamBeginCapture(s_, cudaStreamCaptureModeThreadLocal));
        iteration(d_st_);
        CK(cudaStreamEndCapture(s_, &g));
        size_t nn = 0;
        CK(cudaGraphGetNodes(g, nullptr, &nn));
        kernels_per_iter_ = int(nn);
        CK(cudaGraphInstantiate(&graph_, g, 0));
        cudaGraphDestroy(g);
    }
    PcpgState hst;
    const int every = std::max(1, opt_.check_every);
    launches_ += 27 + 12;     // kernels of the start (x, d, lambda0, g0, Pz) and of the reconstruction
    for (;;) {
        for (int k = 0; k < every; ++k) CK(cudaGraphLaunch(graph_, s_));
        launches_ += (long long)every * kernels_per_iter_;
        CK(cudaMemcpyAsync(&hst, d_st_, sizeof(PcpgState), cudaMemcpyDeviceToHost, s_));
        CK(cudaStreamSynchronize(s_));
        if (hst.done) break;
    }
    CK(cudaEventRecord(e1, s_));
    CK(cudaEventSynchronize(e1));
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    solve_ms = ms;
    iters = hst.it;
    norm0 = hst.norm0;
    rel = hst.rel;
    if (rhs < 64) {                           // relative residual per iteration, for htf_residual_history
        std::vector<double> h(size_t(std::min(hst.it, opt_.max_iter)) + 1, 1.0);
        if (h.size() > 1)
            CK(cudaMemcpy(h.data() + 1, d_hist_ + 1, (h.size() - 1) * sizeof(double), cudaMemcpyDeviceToHost));
        if (int(hist_.size()) <= rhs) hist_.resize(rhs + 1);
        hist_[rhs] = std::move(h);
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    reconstruct(f, u_dev);
    CK(cudaGetLastError());
    if (hst.done == 2) { err = "PCPG breakdown (w'Fw <= 0 or non-finite)"; return HTF_EBREAKDOWN; }
    return HTF_OK;
}

int Engine::history(int rhs, double *out, int cap, std::string &err) const {
    if (rhs < 0 || rhs >= int(hist_.size()) || hist_[rhs].empty()) {
        err = "no residual history for load case " + std::to_string(rhs) +
              " (the plain FP64 form records the first 64 load cases of the last solve)";
        return HTF_EINVAL;
    }
    const int n = int(hist_[rhs].size());
    if (out) std::copy(hist_[rhs].begin(), hist_[rhs].begin() + std::min(n, std::max(cap, 0)), out);
    return n;
}

int Engine::ensure_rhs(int nrhs, std::string &err) {
    if (nrhs <= rhs_cap_) return HTF_OK;
    int rc = HTF_OK;
    d_fn_ = alloc<double>((size_t)ndof_ * nrhs, err, rc);
    d_u_ = alloc<double>((size_t)ndof_ * nrhs, err, rc);
    d_f_ = alloc<double>((size_t)nfull_ * nrhs, err, rc);
    if (rc) return rc;
    rhs_cap_ = nrhs;
    return HTF_OK;
}

int Engine::solve(Problem &p, int nrhs, const double *f_nodal, double *u, htf_stats *stats, std::string &err) {
    cudaGetLastError();           // an error left by an earlier, unrelated call is not this solve's
    if (mixed_ && bK_ > 0) return solve_batch(p, nrhs, f_nodal, u, stats, err);
    int rc = ensure_rhs(nrhs, err);
    if (rc) return rc;
    launches_ = 1;            // k_build_f
    if (f_nodal)
        CK(cudaMemcpyAsync(d_fn_, f_nodal, (size_t)ndof_ * nrhs * sizeof(double), cudaMemcpyHostToDevice, s_));
    k_build_f<<<cdiv(nfull_, 256), 256, 0, s_>>>(nfull_, ndof_, nrhs, d_fbody_, d_own_, f_nodal ? d_fn_ : nullptr, d_f_);
    CK(cudaGetLastError());
    double total_ms = 0.0;
    for (int r = 0; r < nrhs; ++r) {
        int it = 0;
        double n0 = 0, rel = 0, ms = 0;
        rc = solve_one(p, r, d_u_ + (size_t)r * ndof_, it, n0, rel, ms, err);
        total_ms += ms;
        if (stats && r < 64) { stats->iterations[r] = it; stats->norm_gPz0[r] = n0; stats->final_rel[r] = rel; }
        if (rc) return rc;
        if (it >= opt_.max_iter && !(rel < opt_.eps_iter)) {
            if (stats) stats->solve_ms = total_ms;
            err = "PCPG did not converge within max_iter";
            return HTF_ENOCONV;
        }
    }
    if (u) CK(cudaMemcpyAsync(u, d_u_, (size_t)ndof_ * nrhs * sizeof(double), cudaMemcpyDeviceToHost, s_));
    CK(cudaStreamSynchronize(s_));
    if (stats) {
        stats->solve_ms = total_ms;
        stats->setup_ms = setup_ms;
        stats->fapply_bytes = fapply_bytes_;
        stats->n_lambda = nlam_;
        stats->n_sub = nsub_;
        stats->n_clusters = ncl_;
        stats->n_rhs = nrhs;
        stats->status_sub = status_sub;
        stats->kernel_launches = launches_;
    }
    return HTF_OK;
}

// projector with the reduction scratch in the static array of noalloc.cu
int Engine::project_noalloc(const double *x, double *Px, cudaStream_t stream, std::string &err) {
    double *scr = nullptr;
    size_t cap = 0;
    int rc = noalloc_scratch(&scr, &cap, err);
    if (rc) return rc;
    const size_t need = 6 * (size_t)nchunks_;
    if (need > cap) {
        err = "htf_projection_noalloc: problem needs " + std::to_string(need) +
              " doubles of scratch, the static array holds " + std::to_string(cap);
        return HTF_EINVAL;
    }
    k_gft_partial<<<nchunks_, 256, 0, stream>>>(d_chunk_cl_, d_chunk_beg_, d_chunk_end_, d_crow_, d_cval_, x, scr,
                                                nullptr);
    k_gf_apply_fused<<<npart_, 256, 12 * ncl_ * sizeof(double), stream>>>(
        nlam_, ncl_, d_cl_chunk_ptr_, scr, d_invGtG_, d_gcl_, d_gval_, x, nullptr, nullptr, Px,
        nullptr, nullptr, nullptr);
    return check(cudaGetLastError(), "htf_projection_noalloc launch", err);
}

int Engine::profile(int reps, htf_profile_info *info, std::string &err) {
    if (!info || reps < 1) { err = "bad arguments"; return HTF_EINVAL; }
    std::memset(info, 0, sizeof(*info));
    for (int i = 0; i < 8; ++i) info->setup_phase_ms[i] = phase_ms[i];
    for (int b = 0; b < SYMV_BUCKETS && b < int(schedule_.size()); ++b) info->symv_unit_tiles[b] = schedule_[b];
    info->symv_tuned = tuned_ ? 1 : 0;
    info->device_bytes = double(device_bytes());
    info->kernel_detection_ms = kernel_detection_ms;
    info->frontend_ms = frontend_ms;
    cudaEvent_t e0, e1;
    CK(cudaEventCreate(&e0));
    CK(cudaEventCreate(&e1));
    float ms = 0.f;
    auto timeit = [&](auto &&fn) -> double {
        fn();
        cudaEventRecord(e0, s_);
        for (int r = 0; r < reps; ++r) fn();
        cudaEventRecord(e1, s_);
        cudaEventSynchronize(e1);
        cudaEventElapsedTime(&ms, e0, e1);
        return double(ms) / reps;
    };
    k_gather_b<<<cdiv(nslots_, 256), 256, 0, s_>>>(nslots_, d_slot_ptr_, d_slot_ent_, d_lam_, nullptr, d_xb_, nullptr);
    const double sz = 8.0;
    double tri = 0.0, vec = 0.0;
    for (auto &h : hs_) { tri += sz * double(h.nb) * (h.nb + 1) / 2; vec += 16.0 * h.nb; }
    info->symv_F_ms = timeit([&] {
        k_symv_units<double><<<nunits_, SYMV_WARPS * 32, symv_smem_, s_>>>(d_units_, d_subs_, d_F_, d_V_, d_xb_, d_ypart_, d_t_, nullptr);
    });
    info->symv_F_bytes = tri + vec;
    if (implicit_) {              // the two passes over L_bb (its triangle read twice)
        info->symv_S_ms = timeit([&] {
            k_lbt_x<<<nlblk_, 128, 0, s_>>>(d_lblk_, d_subs_, d_K_, d_xb_, d_tb_, nullptr);
            k_lb_t<<<nlblk_, 128, 0, s_>>>(d_lblk_, d_subs_, d_K_, d_tb_, d_xb_, d_yb_, nullptr);
        });
        info->symv_S_bytes = 2.0 * tri + 2.0 * vec;
    } else if (d_S_) {
        info->symv_S_ms = timeit([&] {
            k_symv_units<double><<<nunits_, SYMV_WARPS * 32, symv_smem_, s_>>>(d_units_, d_subs_, d_S_, d_V_, d_xb_, d_ypart_, d_t_,
                                                                   nullptr);
        });
        info->symv_S_bytes = tri + vec;
    }
    info->fapply_ms = timeit([&] { op_F(d_lam_, d_Fw_, nullptr, nullptr, nullptr); });
    info->fapply_bytes = fapply_bytes_;
    if (graph_) {
        // a state with done=1 would skip the work: time with a live state copy
        PcpgState st{};
        st.gPz = 1.0; st.norm0 = 1.0; st.eps = 0.0; st.max_iter = 1 << 30; st.wFw = 1.0;
        PcpgState saved;
        CK(cudaMemcpyAsync(&saved, d_st_, sizeof(PcpgState), cudaMemcpyDeviceToHost, s_));
        CK(cudaStreamSynchronize(s_));
        std::vector<double> lam(nlam_), g(nlam_), w(nlam_);
        CK(cudaMemcpy(lam.data(), d_lam_, nlam_ * sizeof(double), cudaMemcpyDeviceToHost));
        CK(cudaMemcpy(g.data(), d_g_, nlam_ * sizeof(double), cudaMemcpyDeviceToHost));
        CK(cudaMemcpy(w.data(), d_w_, nlam_ * sizeof(double), cudaMemcpyDeviceToHost));
        CK(cudaMemcpyAsync(d_st_, &st, sizeof(PcpgState), cudaMemcpyHostToDevice, s_));
        info->iteration_ms = timeit([&] { cudaGraphLaunch(graph_, s_); });
        CK(cudaMemcpyAsync(d_st_, &saved, sizeof(PcpgState), cudaMemcpyHostToDevice, s_));
        CK(cudaMemcpyAsync(d_lam_, lam.data(), nlam_ * sizeof(double), cudaMemcpyHostToDevice, s_));
        CK(cudaMemcpyAsync(d_g_, g.data(), nlam_ * sizeof(double), cudaMemcpyHostToDevice, s_));
        CK(cudaMemcpyAsync(d_w_, w.data(), nlam_ * sizeof(double), cudaMemcpyHostToDevice, s_));
        CK(cudaStreamSynchronize(s_));
        info->kernels_per_iteration = kernels_per_iter_;
    }
    if (mixed_ && bK_ > 0) {
        const int K = bK_;
        info->batch_width = K;
        CK(cudaMemsetAsync(b_tmp_, 0, (size_t)nlam_ * K * sizeof(double), s_));
        CK(cudaMemsetAsync(b_s_, 0, (size_t)ngc_total_ * K * sizeof(double), s_));
        profile_batch_gather(b_tmp_);
        info->tc_F_ms = timeit([&] { tc_apply(0); });
        // algorithmic bytes of one launch (the product's per-subdomain terms for k
        // load cases): the FP32 triangle n_b (n_b + 1) / 2, X_hi + X_lo in (FP32)
        // and Y out (FP64) per load case; padding rows and the diagonal blocks'
        // upper halves the kernel also reads are not counted (the coarse
        // correction runs in its own kernel after it)
        double bytes = 0.0;
        for (auto &h : hs_) bytes += 4.0 * h.nb * (h.nb + 1.0) / 2.0 + (4.0 + 4.0 + 8.0) * h.nb * K;
        info->tc_F_bytes = bytes;
        if (bgraph_) {
            std::vector<PcpgState> st(K), saved(K);
            for (auto &x : st) {
                x = PcpgState{};
                x.gPz = 1.0; x.norm0 = 1.0; x.eps = 0.0; x.max_iter = 1 << 30; x.wFw = 1.0;
            }
            CK(cudaMemcpyAsync(saved.data(), b_st_, K * sizeof(PcpgState), cudaMemcpyDeviceToHost, s_));
            CK(cudaMemcpyAsync(b_st_, st.data(), K * sizeof(PcpgState), cudaMemcpyHostToDevice, s_));
            info->batch_iteration_ms = timeit([&] { cudaGraphLaunch(bgraph_, s_); });
            CK(cudaMemcpyAsync(b_st_, saved.data(), K * sizeof(PcpgState), cudaMemcpyHostToDevice, s_));
            CK(cudaStreamSynchronize(s_));
            info->kernels_per_batch_iteration = bkernels_per_iter_;
        }
    }
    CK(cudaGetLastError());
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    return HTF_OK;
}

}  // namespace htf
