// Batched mixed-precision PCPG (K load cases at once).
//
// F_i and S_i are applied on the tensor cores as scaled FP16 hi + lo pairs
// (tc_gemm.cu: three FP16 products per K step, FP32 accumulation in TMEM,
// 22 significant bits per operand); gather, coarse problem, projector and
// recurrences stay FP64.  Each load case follows
// Cluster::pcpg (Cluster.cpp:1363-1458) with reliable updates: its residual
// is replaced by the FP64 one g = F lambda - d (FP64 F_i, one load case at a
// time) whenever its recursive g'Pz has dropped 100x or it looks converged,
// and convergence is declared only on the FP64 residual with the reference's
// rule sqrt(g'Pz) < eps * sqrt(g0'Pz0) (Cluster.cpp:1424-1426).
//
// A solve is batch_loads -> per chunk of K load cases batch_begin, then
// {check_every iterations; batch_check} until done, batch_finish.  One
// iteration is iter_a | F product | iter_b | S product | iter_c, so a
// server can run the phases of several problems around one tensor-core
// launch over all their blocks.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <vector>

#include "engine.hpp"

namespace htf {

template <int K>
__global__ void k_tc_gemm(const GemmBlock *, const TcSet *, int, int *);
__global__ void k_make_slabs(const GemmBlock *, const SubDev *, const double *, float *, long long,
                             const unsigned *);
__global__ void k_slab_amax(const GemmBlock *, const SubDev *, const double *, long long, unsigned *);
__global__ void k_colmax(int, int, const double *, unsigned *);
__global__ void k_gather_multi(int, int, const int *, const int *, const double *, const double *, double *, float *,
                               const unsigned *, float);
template <int K, int QN>
__global__ void k_vt_multi(int, const SubDev *, const double *, const double *, double *);
__global__ void k_gc_multi(int, int, int, const int *, const int *, const double *, double *);
template <int K>
__global__ void k_coarse_multi(const ClusterDev *, const double *, const double *, double *);
template <int K>
__global__ void k_correct_multi(const SubDev *, const ClusterDev *, const double *, const int *, const double *,
                                double *);
__global__ void k_rows_multi(int, int, const int *, const double *, const double *, const double *, double *,
                             const double *, double *);
__global__ void k_gft_partial_multi(int, const int *, const int *, const int *, const double *, const double *,
                                    double *);
__global__ void k_gt_sum_multi(int, const int *, const double *, double *);
__global__ void k_gf_coef_multi(int, int, const double *, const double *, double *, double *);
__global__ void k_gf_apply_multi(int, int, const double *, const int *, const double *, const double *, double *,
                                 const double *, double *);
__global__ void k_colsum(const double *, int, int, double *);
__global__ void k_update_lam_g_multi(int, int, const double *, const double *, const double *, const double *, double *,
                                     double *, PcpgState *);
__global__ void k_dot_multi(int, int, const double *, const double *, double *);
__global__ void k_update_w_multi(int, int, const double *, const double *, double *, const PcpgState *);
__global__ void k_finish_multi(int, const double *, const double *, PcpgState *);
__global__ void k_col_get(int, int, int, const double *, double *);
__global__ void k_col_set(int, int, int, const double *, double *);
__global__ void k_build_f(int, int, int, const double *, const int *, const double *, double *);
template <int K>
__global__ void k_symv_rows_multi(const int2 *, const SubDev *, const double *, const double *, double *,
                                  const ClusterDev *, const double *, const int *, const double *);
__global__ void k_cols_copy(long long, int, const int *, const double *, double *);
__global__ void k_alpha_cols(int, int, const int *, const double *, double *);
__global__ void k_axpby(int, double, const double *, double, double *);
__global__ void k_trsm_fwd_multi(const SubDev *, const double *, double *, long long, int, const int *);
__global__ void k_trsm_bwd_multi(const SubDev *, const double *, double *, long long, int, const int *);
__global__ void k_gather_b(int, const int *, const int *, const double *, const double *, double *,
                           const PcpgState *);
__global__ void k_full_minus_b(const SubDev *, const double *, double *);
__global__ void k_bc_rt(const SubDev *, const int *, const int *, const double *, const double *, const double *,
                        const double *, double *);
__global__ void k_gc(int, const int *, const int *, const double *, double *, const PcpgState *);
__global__ void k_coarse(const ClusterDev *, const double *, const double *, double *, const PcpgState *);
__global__ void k_sub_bct(const SubDev *, const ClusterDev *, const int *, const int *, const int *, const double *,
                          const double *, double *);
__global__ void k_add_R(const SubDev *, const ClusterDev *, const double *, const double *, const double *,
                        const double *, double *);
__global__ void k_gather_u(int, const int *, const double *, double *);

static inline int cdivb(long long a, long long b) { return int((a + b - 1) / b); }

#define CKB(call)                                                  \
    do {                                                           \
        int _rc = check((call), #call, err, "engine_batch.cu", __LINE__); \
        if (_rc) return _rc;                                       \
    } while (0)

// tensor-core blocks and slab buffers (once; before the factorisation
// when S_i is made into slabs wave by wave)
int Engine::plan_slabs(int K, std::string &err) {
    if (d_blocks_) return HTF_OK;
    if (K != 16 && K != 32) { err = "batch width must be 16 or 32"; return HTF_EINVAL; }
    int rc = HTF_OK;
    // tensor-core blocks and slabs: the lower triangle at 128-row block
    // granularity (block m stores its slabs kk < min(4 (m + 1), ks), so the
    // block's first slab is 2 m (m + 1) slabs after the subdomain's first)
    std::vector<GemmBlock> blocks;
    long long aoff = 0;
    sub_blk0_.assign(nsub_ + 1, 0);
    for (int d = 0; d < nsub_; ++d) {
        sub_blk0_[d] = int(blocks.size());
        const SubDev &h = hs_[d];
        const int mb = (h.nbp + 127) / 128, ks = h.nbp / 32;
        long long stored = 0;
        for (int m = 0; m < mb; ++m) {
            const int kd = std::min(4 * (m + 1), ks);
            if (stored != 2LL * m * (m + 1)) { err = "tensor-core slab layout"; return HTF_EINVAL; }
            GemmBlock g{d, m, aoff + stored * 4096, ks, std::min(128, h.nb - 128 * m),
                        (long long)h.xb_off * K, (long long)h.xb_off + 128 * m, 0, kd};
            blocks.push_back(g);
            stored += kd;
        }
        aoff += stored * 4096;
    }
    sub_blk0_[nsub_] = int(blocks.size());
    nblocks_ = int(blocks.size());
    d_blocks_ = alloc<GemmBlock>(blocks.size(), err, rc);
    d_AF_ = alloc<float>(aoff, err, rc);               // FP16-pair slabs (4 bytes per entry)
    d_AS_ = alloc<float>(aoff, err, rc);
    d_amaxF_ = alloc<unsigned>(nsub_, err, rc);        // largest |F_i|, |S_i| per subdomain: the slabs' scales
    d_amaxS_ = alloc<unsigned>(nsub_, err, rc);
    aoff_ = aoff;
    hblocks_ = blocks;
    maxks_ = 0;
    for (auto &h : hs_) maxks_ = std::max(maxks_, h.nbp / 32);
    if (rc) return rc;
    CKB(cudaMemcpyAsync(d_blocks_, blocks.data(), blocks.size() * sizeof(GemmBlock), cudaMemcpyHostToDevice, s_));
    CKB(cudaMemsetAsync(d_amaxF_, 0, nsub_ * sizeof(unsigned), s_));
    CKB(cudaMemsetAsync(d_amaxS_, 0, nsub_ * sizeof(unsigned), s_));
    CKB(cudaStreamSynchronize(s_));
    return HTF_OK;
}

int Engine::setup_batch(int K, std::string &err) {
    if (K != 16 && K != 32) { err = "batch width must be 16 or 32"; return HTF_EINVAL; }
    if (implicit_) {
        err = "precision=mixed needs the explicit preconditioner blocks (Dirichlet_explicit or lumped)";
        return HTF_EINVAL;
    }
    int rc = HTF_OK;
    for (auto &h : hs_)
        if ((h.c + 6) * K > 2048) {
            err = "too many Bc rows for the batched form";
            return HTF_EINVAL;
        }
    if ((rc = plan_slabs(K, err))) return rc;
    d_Xs_ = alloc<float>((size_t)nslots_ * K, err, rc);
    d_xmax_ = alloc<unsigned>(K, err, rc);
    d_slot_sub_ = alloc<int>(nslots_, err, rc);
    d_tcerr_ = alloc<int>(1, err, rc);
    d_tcset_ = alloc<TcSet>(1, err, rc);
    if (rc) return rc;
    std::vector<int> ss(nslots_);
    for (int d = 0; d < nsub_; ++d)
        for (int i = 0; i < hs_[d].nbp; ++i) ss[hs_[d].xb_off + i] = d;
    CKB(cudaMemcpyAsync(d_slot_sub_, ss.data(), nslots_ * sizeof(int), cudaMemcpyHostToDevice, s_));
    CKB(cudaMemsetAsync(d_Xs_, 0, (size_t)nslots_ * K * sizeof(float), s_));
    CKB(cudaMemsetAsync(d_tcerr_, 0, sizeof(int), s_));
    {
        // |x_b| <= (entries of a slot) x (largest weight) x max|w|: the bound behind X's scale
        std::vector<int> sp(nslots_ + 1);
        std::vector<double> wt(nlam_);
        CKB(cudaMemcpy(sp.data(), d_slot_ptr_, sp.size() * sizeof(int), cudaMemcpyDeviceToHost));
        CKB(cudaMemcpy(wt.data(), d_weight_, wt.size() * sizeof(double), cudaMemcpyDeviceToHost));
        int nent = 1;
        for (int i = 0; i < nslots_; ++i) nent = std::max(nent, sp[i + 1] - sp[i]);
        double wmax = 1.0;
        for (double x : wt) wmax = std::max(wmax, std::fabs(x));
        xbound_ = float(nent * wmax);
    }
    const GemmBlock *db = static_cast<const GemmBlock *>(d_blocks_);
    k_slab_amax<<<dim3(nblocks_, maxks_), 256, 0, s_>>>(db, d_subs_, d_F_, 0, d_amaxF_);
    k_make_slabs<<<dim3(nblocks_, maxks_), 256, 0, s_>>>(db, d_subs_, d_F_, d_AF_, 0, d_amaxF_);
    if (!s_lean_) {
        k_slab_amax<<<dim3(nblocks_, maxks_), 256, 0, s_>>>(db, d_subs_, d_S_, 0, d_amaxS_);
        k_make_slabs<<<dim3(nblocks_, maxks_), 256, 0, s_>>>(db, d_subs_, d_S_, d_AS_, 0, d_amaxS_);
    }
    CKB(cudaGetLastError());
    // TC_STAGES stages of A (16 KB) and X (k x 128 B) + alignment slack
    tc_smem_ = tc_smem_bytes(K);
    if (K == 16)
        CKB(cudaFuncSetAttribute(k_tc_gemm<16>, cudaFuncAttributeMaxDynamicSharedMemorySize, tc_smem_));
    else
        CKB(cudaFuncSetAttribute(k_tc_gemm<32>, cudaFuncAttributeMaxDynamicSharedMemorySize, tc_smem_));
    // batch vectors
    const size_t nl = (size_t)nlam_ * K;
    int ntot = 0;
    vt_nch_ = 1;
    int maxcol = 0;
    for (auto &h : hs_) {
        ntot = std::max(ntot, h.t_off + h.c + 6);
        vt_nch_ = std::max(vt_nch_, (h.nb + 127) / 128);
        maxcol = std::max(maxcol, h.c + 6);
    }
    vt_qn_ = maxcol <= 32 ? 32 : maxcol <= 64 ? 64 : 128;     // columns of V^T x_b computed per chunk
    // row kernels stride over row groups with a fixed grid: few partials per column
    bnpart_ = std::min(cdivb(nlam_, 256 / K), 1184);
    b_lam_ = alloc<double>(nl, err, rc); b_g_ = alloc<double>(nl, err, rc); b_w_ = alloc<double>(nl, err, rc);
    b_Fw_ = alloc<double>(nl, err, rc); b_Pg_ = alloc<double>(nl, err, rc); b_z_ = alloc<double>(nl, err, rc);
    b_Pz_ = alloc<double>(nl, err, rc); b_d_ = alloc<double>(nl, err, rc); b_tmp_ = alloc<double>(nl, err, rc);
    b_xb_ = alloc<double>((size_t)nslots_ * K, err, rc); b_yb_ = alloc<double>((size_t)nslots_ * K, err, rc);
    b_t_ = alloc<double>((size_t)ntot * vt_nch_ * K, err, rc);     // V^T x_b partials per 128-row chunk
    b_gc_ = alloc<double>((size_t)ngc_total_ * K, err, rc); b_s_ = alloc<double>((size_t)ngc_total_ * K, err, rc);
    b_part_ = alloc<double>((size_t)bnpart_ * K, err, rc);
    b_gpart_ = alloc<double>((size_t)nchunks_ * 6 * K, err, rc);
    b_wFw_ = alloc<double>(K, err, rc); b_gPz_ = alloc<double>(K, err, rc);
    b_gw_ = alloc<double>(K, err, rc);
    b_gt_ = alloc<double>((size_t)6 * ncl_ * K, err, rc); b_acoef_ = alloc<double>((size_t)6 * ncl_ * K, err, rc);
    b_alpha_ = alloc<double>((size_t)6 * ncl_ * K, err, rc);
    b_st_ = alloc<PcpgState>(K, err, rc);
    b_alpha2_ = alloc<double>((size_t)6 * ncl_ * K, err, rc);
    d_mask_ = alloc<int>(2 * K, err, rc);
    {
        std::vector<int2> rb;                       // (subdomain, 32-row block) of the FP64 multi-RHS SYMV
        for (int d = 0; d < nsub_; ++d)
            for (int I = 0; I < hs_[d].nt; ++I) rb.push_back(make_int2(d, I));
        nrowblk_ = int(rb.size());
        d_rowblk_ = alloc<int2>(rb.size(), err, rc);
        if (!rc) CKB(cudaMemcpyAsync(d_rowblk_, rb.data(), rb.size() * sizeof(int2), cudaMemcpyHostToDevice, s_));
    }
    b_fullA_ = alloc<double>((size_t)nfull_ * K, err, rc);
    b_fullB_ = alloc<double>((size_t)nfull_ * K, err, rc);
    b_srec_ = alloc<double>((size_t)ngc_total_ * K, err, rc);
    if (rc) return rc;
    bK_ = K;
    const TcSet ts = tc_set();
    CKB(cudaMemcpyAsync(d_tcset_, &ts, sizeof(TcSet), cudaMemcpyHostToDevice, s_));
    CKB(cudaStreamSynchronize(s_));
    return HTF_OK;
}

// the coarse correction of the F product runs after it (k_correct_multi in
// f_post), so the product's epilogue gets no coarse solution
TcSet Engine::tc_set() const {
    return TcSet{d_AF_, d_AS_, d_Xs_, b_yb_, d_amaxF_, d_amaxS_, d_xmax_, xbound_};
}

// x_b = Bf^T w (weighted when weight != nullptr; into xb when xb != nullptr)
// and the X slabs of the tensor-core product, scaled from w's column maxima
void Engine::gather_x(const double *w, const double *weight, double *xb) {
    const int K = bK_;
    cudaMemsetAsync(d_xmax_, 0, K * sizeof(unsigned), s_);
    k_colmax<<<std::max(1, std::min(cdivb((long long)nlam_ * K, 256), 1184)), 256, 0, s_>>>(nlam_, K, w, d_xmax_);
    k_gather_multi<<<nslots_ / 32, 256, 0, s_>>>(nslots_, K, d_slot_ptr_, d_slot_ent_, w, weight, xb, d_Xs_, d_xmax_,
                                                 xbound_);
}

// X slabs of a batch vector (for timing the tensor-core product alone)
void Engine::profile_batch_gather(const double *w) { gather_x(w, nullptr, b_xb_); }

// one tensor-core launch over the given blocks / operand sets (which: 0 = F,
// 1 = S; the coarse correction of F follows in k_correct_multi)
int tc_launch(int K, const GemmBlock *blocks, int nblocks, const TcSet *sets, int which, int smem, int *err,
              cudaStream_t s) {
    if (nblocks <= 0) return 0;
    if (K == 16) k_tc_gemm<16><<<nblocks, TC_THREADS, smem, s>>>(blocks, sets, which, err);
    else k_tc_gemm<32><<<nblocks, TC_THREADS, smem, s>>>(blocks, sets, which, err);
    return 0;
}

int tc_smem_bytes(int K) { return 1024 + TC_STAGES * (128 * 32 + K * 32) * 4; }

void Engine::tc_apply(int which) {
    tc_launch(bK_, static_cast<const GemmBlock *>(d_blocks_), nblocks_, d_tcset_, which, tc_smem_, d_tcerr_, s_);
}

// F w = Bf [F_d x_b - V_d M_c V_d^T x_b]: the coarse solve before the
// tensor-core product, whose epilogue applies the correction
void Engine::f_pre(const double *w) {
    gather_x(w, nullptr, b_xb_);
    coarse_batch();
}

// s = M_c [Bc_b F x_b ; -R_b^T x_b] per cluster from the batch vector b_xb_:
// V^T x_b per 128-row chunk, the coarse right-hand side, M G
void Engine::coarse_batch() {
    const int K = bK_;
    int maxg = 0;
    for (auto &c : hc_) maxg = std::max(maxg, c.ngc);
    const dim3 gv(nsub_, vt_nch_);
    if (K == 32) {
        if (vt_qn_ == 32) k_vt_multi<32, 32><<<gv, 256, 0, s_>>>(vt_nch_, d_subs_, d_V_, b_xb_, b_t_);
        else k_vt_multi<32, 64><<<gv, 256, 0, s_>>>(vt_nch_, d_subs_, d_V_, b_xb_, b_t_);
    } else {
        if (vt_qn_ == 32) k_vt_multi<16, 32><<<gv, 256, 0, s_>>>(vt_nch_, d_subs_, d_V_, b_xb_, b_t_);
        else if (vt_qn_ == 64) k_vt_multi<16, 64><<<gv, 256, 0, s_>>>(vt_nch_, d_subs_, d_V_, b_xb_, b_t_);
        else k_vt_multi<16, 128><<<gv, 256, 0, s_>>>(vt_nch_, d_subs_, d_V_, b_xb_, b_t_);
    }
    k_gc_multi<<<cdivb((long long)ngc_total_ * K, 256), 256, 0, s_>>>(ngc_total_, K, vt_nch_, d_gptr_, d_gidx_, b_t_,
                                                                      b_gc_);
    if (K == 32) k_coarse_multi<32><<<dim3(ncl_, cdivb(maxg, 32)), 128, 0, s_>>>(d_cl_, d_M_, b_gc_, b_s_);
    else k_coarse_multi<16><<<dim3(ncl_, cdivb(maxg, 32)), 128, 0, s_>>>(d_cl_, d_M_, b_gc_, b_s_);
}

void Engine::f_post(double *Fw, const double *dotv, double *partial) {
    const dim3 gc(nsub_, cdivb(max_nbp_, 128));
    if (bK_ == 32) k_correct_multi<32><<<gc, 256, 0, s_>>>(d_subs_, d_cl_, d_V_, d_bcr_, b_s_, b_yb_);
    else k_correct_multi<16><<<gc, 256, 0, s_>>>(d_subs_, d_cl_, d_V_, d_bcr_, b_s_, b_yb_);
    k_rows_multi<<<bnpart_, 256, 0, s_>>>(nlam_, bK_, d_rslot_, d_rsign_, b_yb_, nullptr, Fw, dotv, partial);
}

// the preconditioner uses the same FP16-pair products as F
void Engine::m_pre(const double *x) { gather_x(x, d_weight_, nullptr); }

void Engine::m_post(double *z) {
    k_rows_multi<<<bnpart_, 256, 0, s_>>>(nlam_, bK_, d_rslot_, d_rsign_, b_yb_, d_weight_, z, nullptr, nullptr);
}

void Engine::op_F_batch(const double *w, double *Fw, const double *dotv, double *partial) {
    f_pre(w);
    tc_apply(0);
    f_post(Fw, dotv, partial);
}

void Engine::op_M_batch(const double *x, double *z) {
    m_pre(x);
    tc_apply(1);
    m_post(z);
}

void Engine::op_P_batch(const double *x, double *Px, double *alpha_out, const double *dotv, double *partial) {
    const int K = bK_;
    k_gft_partial_multi<<<nchunks_, 256, 0, s_>>>(K, d_chunk_beg_, d_chunk_end_, d_crow_, d_cval_, x, b_gpart_);
    k_gt_sum_multi<<<ncl_, 6 * K, 0, s_>>>(K, d_cl_chunk_ptr_, b_gpart_, b_gt_);
    k_gf_coef_multi<<<1, 1024, 0, s_>>>(K, ncl_, d_invGtG_, b_gt_, b_acoef_, alpha_out);
    k_gf_apply_multi<<<bnpart_, 256, 0, s_>>>(nlam_, K, b_acoef_, d_gcl_, d_gval_, x, Px, dotv, partial);
}

// one batched iteration = iter_a | F product | iter_b | S product | iter_c
void Engine::iter_a() { f_pre(b_w_); }

void Engine::iter_b() {
    const int K = bK_;
    const int nk = cdivb((long long)nlam_ * K, 256);
    f_post(b_Fw_, b_w_, b_part_);
    k_colsum<<<K, 256, 0, s_>>>(b_part_, bnpart_, K, b_wFw_);
    k_dot_multi<<<bnpart_, 256, 0, s_>>>(nlam_, K, b_g_, b_w_, b_part_);
    k_colsum<<<K, 256, 0, s_>>>(b_part_, bnpart_, K, b_gw_);
    k_update_lam_g_multi<<<nk, 256, 0, s_>>>(nlam_, K, b_wFw_, b_gw_, b_w_, b_Fw_, b_lam_, b_g_, b_st_);
    op_P_batch(b_g_, b_Pg_, nullptr, nullptr, nullptr);
    m_pre(b_Pg_);
}

void Engine::iter_c() {
    const int K = bK_;
    const int nk = cdivb((long long)nlam_ * K, 256);
    m_post(b_z_);
    op_P_batch(b_z_, b_Pz_, nullptr, b_g_, b_part_);
    k_colsum<<<K, 256, 0, s_>>>(b_part_, bnpart_, K, b_gPz_);
    k_update_w_multi<<<nk, 256, 0, s_>>>(nlam_, K, b_gPz_, b_Pz_, b_w_, b_st_);
    k_finish_multi<<<1, 32, 0, s_>>>(K, b_wFw_, b_gPz_, b_st_);
}

void Engine::iteration_batch() {
    iter_a();
    tc_apply(0);
    iter_b();
    tc_apply(1);
    iter_c();
}

int Engine::apply_batch(int op, const double *x, double *y, int nrhs, std::string &err) {
    const int K = bK_;
    if (nrhs > K) { err = "more load cases than the batch width"; return HTF_EINVAL; }
    std::vector<double> hx((size_t)nlam_ * K, 0.0), hy((size_t)nlam_ * K);
    for (int j = 0; j < nrhs; ++j)
        for (int r = 0; r < nlam_; ++r) hx[(size_t)r * K + j] = x[(size_t)j * nlam_ + r];
    CKB(cudaMemcpyAsync(b_tmp_, hx.data(), hx.size() * sizeof(double), cudaMemcpyHostToDevice, s_));
    if (op == 0) op_F_batch(b_tmp_, b_Fw_, nullptr, nullptr);
    else if (op == 2) op_M_batch(b_tmp_, b_Fw_);
    else op_P_batch(b_tmp_, b_Fw_, nullptr, nullptr, nullptr);
    CKB(cudaGetLastError());
    CKB(cudaMemcpyAsync(hy.data(), b_Fw_, hy.size() * sizeof(double), cudaMemcpyDeviceToHost, s_));
    CKB(cudaStreamSynchronize(s_));
    int tcerr = 0;
    CKB(cudaMemcpy(&tcerr, d_tcerr_, sizeof(int), cudaMemcpyDeviceToHost));
    if (tcerr) { err = "tensor-core product timed out on a barrier"; return tcerr; }
    for (int j = 0; j < nrhs; ++j)
        for (int r = 0; r < nlam_; ++r) y[(size_t)j * nlam_ + r] = hy[(size_t)r * K + j];
    return HTF_OK;
}

// ---------------------------------------------------------------------------
// load cases of a solve: f for nrhs columns on the device
int Engine::batch_loads(int nrhs, const double *f_nodal, std::string &err) {
    int rc = ensure_rhs(nrhs, err);
    if (rc) return rc;
    if (f_nodal)
        CKB(cudaMemcpyAsync(d_fn_, f_nodal, (size_t)ndof_ * nrhs * sizeof(double), cudaMemcpyHostToDevice, s_));
    k_build_f<<<cdivb(nfull_, 256), 256, 0, s_>>>(nfull_, ndof_, nrhs, d_fbody_, d_own_, f_nodal ? d_fn_ : nullptr,
                                                  d_f_);
    CKB(cudaGetLastError());
    return HTF_OK;
}

// FP64 residuals of the load cases j with sel[j] (Cluster.cpp:1398-1412 from
// the current lambda), all in one pass over the FP64 tiles: g = F lambda - d,
// P g (alpha), z = M P g, P z and g'Pz.  They replace the batch residual
// columns of the selected load cases, and the search directions of those with
// reset[j].  Every column is computed independently of the others, so a load
// case gets the same bits alone and in a batch.
int Engine::fp64_residual_batch(const std::vector<int> &sel, const std::vector<int> &reset, std::string &err) {
    BatchRun &r = run_;
    const auto t_start = std::chrono::steady_clock::now();
    const int K = bK_;
    const long long nk = (long long)nlam_ * K;
    auto symv = [&](const double *tiles, const double *scoarse) {
        if (K == 32)
            k_symv_rows_multi<32><<<nrowblk_, 256, 0, s_>>>(static_cast<const int2 *>(d_rowblk_), d_subs_, tiles, b_xb_,
                                                           b_yb_, d_cl_, d_V_, d_bcr_, scoarse);
        else
            k_symv_rows_multi<16><<<nrowblk_, 256, 0, s_>>>(static_cast<const int2 *>(d_rowblk_), d_subs_, tiles, b_xb_,
                                                           b_yb_, d_cl_, d_V_, d_bcr_, scoarse);
    };
    // g = F lambda - d
    k_gather_multi<<<nslots_ / 32, 256, 0, s_>>>(nslots_, K, d_slot_ptr_, d_slot_ent_, b_lam_, nullptr, b_xb_, nullptr,
                                                 nullptr, 0.f);
    coarse_batch();
    symv(d_F_, b_s_);
    k_rows_multi<<<bnpart_, 256, 0, s_>>>(nlam_, K, d_rslot_, d_rsign_, b_yb_, nullptr, b_tmp_, nullptr, nullptr);
    k_axpby<<<cdivb(nk, 256), 256, 0, s_>>>(int(nk), -1.0, b_d_, 1.0, b_tmp_);
    op_P_batch(b_tmp_, b_Pg_, b_alpha2_, nullptr, nullptr);
    // z = M P g, P z, g'Pz
    if (d_S_) {
        k_gather_multi<<<nslots_ / 32, 256, 0, s_>>>(nslots_, K, d_slot_ptr_, d_slot_ent_, b_Pg_, d_weight_, b_xb_,
                                                     nullptr, nullptr, 0.f);
        symv(d_S_, nullptr);
        k_rows_multi<<<bnpart_, 256, 0, s_>>>(nlam_, K, d_rslot_, d_rsign_, b_yb_, d_weight_, b_z_, nullptr, nullptr);
    } else {
        op_M_batch(b_Pg_, b_z_);      // S_i only as tensor-core slabs: the tensor-core product
    }
    op_P_batch(b_z_, b_Pz_, nullptr, b_tmp_, b_part_);
    k_colsum<<<K, 256, 0, s_>>>(b_part_, bnpart_, K, b_gPz_);
    // the selected columns back into the recurrence
    std::vector<int> masks(2 * K, 0);
    for (int j = 0; j < K; ++j) {
        masks[j] = sel[j];
        masks[K + j] = sel[j] && reset[j];
    }
    CKB(cudaMemcpyAsync(d_mask_, masks.data(), 2 * K * sizeof(int), cudaMemcpyHostToDevice, s_));
    k_cols_copy<<<cdivb(nk, 256), 256, 0, s_>>>(nlam_, K, d_mask_, b_tmp_, b_g_);
    k_cols_copy<<<cdivb(nk, 256), 256, 0, s_>>>(nlam_, K, d_mask_ + K, b_Pz_, b_w_);
    k_alpha_cols<<<1, 256, 0, s_>>>(6 * ncl_, K, d_mask_, b_alpha2_, b_alpha_);
    CKB(cudaGetLastError());
    launches_ += 19 + 8;
    std::vector<double> gPz(K);
    CKB(cudaMemcpyAsync(gPz.data(), b_gPz_, K * sizeof(double), cudaMemcpyDeviceToHost, s_));
    CKB(cudaStreamSynchronize(s_));
    if (opt_.verbose) {
        int m = 0;
        for (int j = 0; j < K; ++j) m += sel[j];
        std::fprintf(stderr, "[htf mixed] FP64 residuals of %d load cases: %.3f ms\n", m,
                     std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t_start).count());
    }
    for (int j = 0; j < K; ++j) {
        if (!sel[j]) continue;
        PcpgState &st = r.st[j];
        st.gPz = gPz[j];
        st.gPz_prev = gPz[j];
        r.last[j] = gPz[j];
        if (st.norm0 == 0.0) st.norm0 = std::sqrt(gPz[j]);
        const double cur = std::sqrt(gPz[j]);
        r.rel[j] = st.norm0 > 0 ? cur / st.norm0 : 0.0;
        if (opt_.verbose)
            std::fprintf(stderr, "[htf mixed] rhs %d it %d FP64 sqrt(gPz)/norm0 = %.3e\n", r.r0 + j, st.it, r.rel[j]);
        if (!(gPz[j] > 0.0) || !std::isfinite(gPz[j]) || cur < opt_.eps_iter * opt_.mixed_eps_factor * st.norm0) {
            r.conv[j] = 1;
            st.done = 1;
        } else {
            st.done = 0;
        }
    }
    return HTF_OK;
}

int Engine::batch_begin(int r0, int kc, std::string &err) {
    const int K = bK_;
    if (kc < 1 || kc > K) { err = "bad load-case chunk"; return HTF_EINVAL; }
    if (!run_e0_) {
        CKB(cudaEventCreate(&run_e0_));
        CKB(cudaEventCreate(&run_e1_));
    }
    BatchRun &r = run_;
    r.r0 = r0;
    r.kc = kc;
    r.st.assign(K, PcpgState{});
    r.last.assign(K, 0.0);
    r.rel.assign(K, 0.0);
    r.best.assign(K, 0.0);
    r.best_it.assign(K, 0);
    r.stall.assign(K, 0);
    r.conv.assign(K, 0);
    CKB(cudaMemsetAsync(b_lam_, 0, (size_t)nlam_ * K * sizeof(double), s_));
    CKB(cudaMemsetAsync(b_d_, 0, (size_t)nlam_ * K * sizeof(double), s_));
    CKB(cudaMemsetAsync(d_tcerr_, 0, sizeof(int), s_));
    // K_reg^{-1} f for the whole chunk: the factor is read once
    CKB(cudaMemcpyAsync(b_fullB_, d_f_ + (size_t)r0 * nfull_, (size_t)kc * nfull_ * sizeof(double),
                        cudaMemcpyDeviceToDevice, s_));
    trsm_multi(b_fullB_, kc);
    launches_ += 2;
    for (int j = 0; j < kc; ++j) {
        init_rhs(d_f_ + (size_t)(r0 + j) * nfull_, b_fullB_ + (size_t)j * nfull_);
        k_col_set<<<npart_, 256, 0, s_>>>(nlam_, K, j, d_d_, b_d_);
        k_col_set<<<npart_, 256, 0, s_>>>(nlam_, K, j, d_lam_, b_lam_);
        launches_ += 25;
    }
    CKB(cudaEventRecord(run_e0_, s_));
    for (int j = 0; j < K; ++j) r.st[j].done = 1;
    int rc;
    std::vector<int> sel(K, 0), reset(K, 0);
    for (int j = 0; j < kc; ++j) {
        r.st[j].eps = opt_.eps_iter * opt_.mixed_eps_factor;
        r.st[j].max_iter = opt_.max_iter;
        r.st[j].wFw = 1.0;
        sel[j] = reset[j] = 1;
    }
    if ((rc = fp64_residual_batch(sel, reset, err))) return rc;
    for (int j = kc; j < K; ++j) r.conv[j] = 1;
    CKB(cudaMemcpyAsync(b_st_, r.st.data(), K * sizeof(PcpgState), cudaMemcpyHostToDevice, s_));
    return HTF_OK;
}

// after some iterations: FP64 residuals where due; all_done when every load
// case has converged (or hit max_iter)
int Engine::batch_check(bool &all_done, std::string &err) {
    BatchRun &r = run_;
    const int K = bK_;
    const double ru2 = 1e-2;
    CKB(cudaMemcpyAsync(r.st.data(), b_st_, K * sizeof(PcpgState), cudaMemcpyDeviceToHost, s_));
    CKB(cudaStreamSynchronize(s_));
    int tcerr = 0;
    CKB(cudaMemcpy(&tcerr, d_tcerr_, sizeof(int), cudaMemcpyDeviceToHost));
    if (tcerr) { err = "tensor-core product timed out on a barrier"; return tcerr; }
    bool changed = false;
    int rc;
    std::vector<int> sel(K, 0), reset(K, 0);
    for (int j = 0; j < K; ++j) {
        if (r.conv[j]) continue;
        const bool broke = r.st[j].done == 2;
        if (r.st[j].it >= opt_.max_iter) { r.conv[j] = 2; continue; }
        if (r.st[j].done != 0 || r.st[j].gPz < ru2 * r.last[j]) {
            r.st[j].eps = opt_.eps_iter * opt_.mixed_eps_factor;
            sel[j] = 1;
            reset[j] = broke;
            changed = true;
        }
    }
    if (changed && (rc = fp64_residual_batch(sel, reset, err))) return rc;
    for (int j = 0; j < K; ++j) {
        if (!sel[j] || r.conv[j]) continue;
        if (r.best[j] == 0.0 || r.rel[j] < 0.5 * r.best[j]) {
            r.best[j] = r.rel[j];
            r.best_it[j] = r.st[j].it;
            r.stall[j] = 0;
        } else if (++r.stall[j] >= MIXED_STALL_LIMIT && r.st[j].it - r.best_it[j] >= MIXED_STALL_ITERATIONS) {
            r.conv[j] = 3;
            r.st[j].done = 1;          // the iterations leave it alone from here on
        }
    }
    if (changed) CKB(cudaMemcpyAsync(b_st_, r.st.data(), K * sizeof(PcpgState), cudaMemcpyHostToDevice, s_));
    all_done = true;
    for (int j = 0; j < K; ++j) all_done &= r.conv[j] != 0;
    return HTF_OK;
}

// displacements of the chunk's load cases into d_u_; per-load-case stats
int Engine::batch_finish(htf_stats *stats, double &ms, std::string &err) {
    BatchRun &r = run_;
    const int K = bK_;
    CKB(cudaEventRecord(run_e1_, s_));
    CKB(cudaEventSynchronize(run_e1_));
    float fms = 0.f;
    cudaEventElapsedTime(&fms, run_e0_, run_e1_);
    ms = fms;
    // u_j = K_HT^+(f_j - Bf^T lambda_j) - Rf alpha_j (Cluster.cpp:1648-1678) for the whole
    // chunk, with the two K_reg^{-1} solves of every load case done at once
    const int kc = r.kc;
    int maxg = 0;
    for (auto &c : hc_) maxg = std::max(maxg, c.ngc);
    CKB(cudaMemcpyAsync(b_fullA_, d_f_ + (size_t)r.r0 * nfull_, (size_t)kc * nfull_ * sizeof(double),
                        cudaMemcpyDeviceToDevice, s_));
    for (int j = 0; j < kc; ++j) {
        double *fa = b_fullA_ + (size_t)j * nfull_;
        k_col_get<<<npart_, 256, 0, s_>>>(nlam_, K, j, b_lam_, d_lam_);
        k_gather_b<<<cdivb(nslots_, 256), 256, 0, s_>>>(nslots_, d_slot_ptr_, d_slot_ent_, d_lam_, nullptr, d_xb_,
                                                        nullptr);
        k_full_minus_b<<<nsub_, 256, 0, s_>>>(d_subs_, d_xb_, fa);
    }
    CKB(cudaMemcpyAsync(b_fullB_, b_fullA_, (size_t)kc * nfull_ * sizeof(double), cudaMemcpyDeviceToDevice, s_));
    trsm_multi(b_fullB_, kc);
    for (int j = 0; j < kc; ++j) {
        double *fa = b_fullA_ + (size_t)j * nfull_;
        k_bc_rt<<<nsub_, 256, 0, s_>>>(d_subs_, d_bce_ptr_, d_bce_pos_, d_bce_val_, d_R_, b_fullB_ + (size_t)j * nfull_,
                                       fa, d_t_);
        k_gc<<<cdivb(ngc_total_, 256), 256, 0, s_>>>(ngc_total_, d_gptr_, d_gidx_, d_t_, d_gc_, nullptr);
        k_coarse<<<dim3(ncl_, cdivb(maxg, 8)), 256, 0, s_>>>(d_cl_, d_M_, d_gc_, b_srec_ + (size_t)j * ngc_total_,
                                                            nullptr);
        k_sub_bct<<<nsub_, 32, 0, s_>>>(d_subs_, d_cl_, d_bcr_, d_bce_ptr_, d_bce_pos_, d_bce_val_,
                                        b_srec_ + (size_t)j * ngc_total_, fa);
    }
    trsm_multi(b_fullA_, kc);
    for (int j = 0; j < kc; ++j) {
        double *fa = b_fullA_ + (size_t)j * nfull_;
        k_add_R<<<nsub_, 256, 0, s_>>>(d_subs_, d_cl_, d_R_, d_H_, b_srec_ + (size_t)j * ngc_total_,
                                       b_alpha_ + (size_t)j * 6 * ncl_, fa);
        k_gather_u<<<cdivb(ndof_, 256), 256, 0, s_>>>(ndof_, d_win_, fa, d_u_ + (size_t)(r.r0 + j) * ndof_);
    }
    launches_ += 4 + 9 * kc;
    for (int j = 0; j < kc; ++j) {
        if (stats && r.r0 + j < 64) {
            stats->iterations[r.r0 + j] = r.st[j].it;
            stats->norm_gPz0[r.r0 + j] = r.st[j].norm0 * r.st[j].norm0;
            stats->final_rel[r.r0 + j] = r.rel[j];
        }
    }
    CKB(cudaGetLastError());
    for (int j = 0; j < r.kc; ++j)
        if (r.conv[j] == 2) { err = "PCPG did not converge within max_iter"; return HTF_ENOCONV; }
    for (int j = 0; j < r.kc; ++j)
        if (r.conv[j] == 3) {
            char msg[256];
            std::snprintf(msg, sizeof msg,
                          "PCPG stagnated: load case %d stayed at a relative FP64 residual of %.3e (target %.1e) "
                          "from iteration %d to %d (%d residual replacements); the mixed form cannot reach "
                          "eps_iter on this problem",
                          r.r0 + j, r.best[j], opt_.eps_iter * opt_.mixed_eps_factor, r.best_it[j], r.st[j].it,
                          r.stall[j]);
            err = msg;
            return HTF_ENOCONV;
        }
    return HTF_OK;
}

void Engine::trsm_multi(double *v, int nrhs) {
    if (!waves_) {
        k_trsm_fwd_multi<<<nsub_, 256, 0, s_>>>(d_subs_, d_K_, v, nfull_, nrhs, nullptr);
        k_trsm_bwd_multi<<<nsub_, 256, 0, s_>>>(d_subs_, d_K_, v, nfull_, nrhs, nullptr);
        return;
    }
    // the factor panels were dropped: assemble and factorise each wave again, then solve its subdomains
    for (size_t w = 0; w < fw_.size(); ++w) {
        factor_wave(int(w), false, nullptr);
        const int a = fw_[w].a, nw = fw_[w].b - fw_[w].a;
        k_trsm_fwd_multi<<<nw, 256, 0, s_>>>(d_subs_ + a, d_K_, v, nfull_, nrhs, nullptr);
        k_trsm_bwd_multi<<<nw, 256, 0, s_>>>(d_subs_ + a, d_K_, v, nfull_, nrhs, nullptr);
    }
}

int Engine::batch_graph(std::string &err) {
    if (bgraph_) return HTF_OK;
    cudaGraph_t g;
    CKB(cudaStreamBeginCapture(s_, cudaStreamCaptureModeThreadLocal));
    iteration_batch();
    CKB(cudaStreamEndCapture(s_, &g));
    size_t nn = 0;
    CKB(cudaGraphGetNodes(g, nullptr, &nn));
    bkernels_per_iter_ = int(nn);
    CKB(cudaGraphInstantiate(&bgraph_, g, 0));
    cudaGraphDestroy(g);
    return HTF_OK;
}

int Engine::solve_batch(Problem &p, int nrhs, const double *f_nodal, double *u, htf_stats *stats, std::string &err) {
    (void)p;
    const int K = bK_;
    launches_ = 1;
    int rc = batch_loads(nrhs, f_nodal, err);
    if (!rc) rc = batch_graph(err);
    if (rc) return rc;
    double total_ms = 0.0;
    for (int r0 = 0; r0 < nrhs; r0 += K) {
        if ((rc = batch_begin(r0, std::min(K, nrhs - r0), err))) return rc;
        for (bool done = false; !done;) {
            for (int k = 0; k < opt_.check_every; ++k) CKB(cudaGraphLaunch(bgraph_, s_));
            launches_ += (long long)opt_.check_every * bkernels_per_iter_;
            if ((rc = batch_check(done, err))) return rc;
        }
        double ms = 0.0;
        if ((rc = batch_finish(stats, ms, err))) return rc;
        total_ms += ms;
    }
    if (u) CKB(cudaMemcpyAsync(u, d_u_, (size_t)ndof_ * nrhs * sizeof(double), cudaMemcpyDeviceToHost, s_));
    CKB(cudaStreamSynchronize(s_));
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

}  // namespace htf
