// Host-side engine of the HTFETI path: owns the device buffers of one
// problem, runs the GPU setup and the PCPG iterations.
#pragma once
#include <cuda_runtime.h>

#include <string>
#include <vector>

#include "../host/problem.hpp"
#include "device.cuh"

namespace htf {

// static scratch of the allocation-free entry point (noalloc.cu)
int noalloc_scratch(double **ptr, size_t *cap, std::string &err);

// tensor-core product over blocks of one or more problems (engine_batch.cu)
int tc_launch(int K, const GemmBlock *blocks, int nblocks, const TcSet *sets, int which, int smem, int *err,
              cudaStream_t s);
int tc_smem_bytes(int K);

// host-side state of one chunk of load cases in the batched form
struct BatchRun {
    int r0 = 0, kc = 0;
    std::vector<PcpgState> st;
    std::vector<double> last;      // g'Pz at the last FP64 residual
    std::vector<double> rel;       // last FP64 sqrt(g'Pz)/norm0
    std::vector<double> best;      // smallest FP64 rel seen at a residual replacement
    std::vector<int> best_it;      // iteration at which best was set
    std::vector<int> stall;        // residual replacements since best was set
    std::vector<int> conv;         // 0 running, 1 converged, 2 max_iter, 3 stagnated
};

// A load case of the batched mixed form is stopped as stagnated (HTF_ENOCONV)
// when MIXED_STALL_LIMIT FP64 residual replacements, over at least
// MIXED_STALL_ITERATIONS iterations, have passed without its FP64 residual
// falling below half of its smallest value so far.  A replacement follows a
// 100x drop of the recursive g'Pz or a recursion that says converged; while
// the form converges the FP64 residual follows the recursive one down, so a
// run of replacements without progress means the FP32 operator cannot carry
// the FP64 residual any lower (its rounding times the problem's conditioning
// is above eps), and the iterations left to max_iter would only add FP64
// replacements.
constexpr int MIXED_STALL_LIMIT = 10;
constexpr int MIXED_STALL_ITERATIONS = 500;

struct DevBuf {
    void *p = nullptr;
    size_t bytes = 0;
};

class Engine {
public:
    explicit Engine(const Options &o) : opt_(o) {}
    ~Engine();
    int setup(Problem &p, std::string &err);
    int solve(Problem &p, int nrhs, const double *f_nodal, double *u, htf_stats *stats, std::string &err);
    int profile(int reps, htf_profile_info *info, std::string &err);
    int project_noalloc(const double *x, double *Px, cudaStream_t stream, std::string &err);
    // MatrixMarket files of the problem's matrices (dump.cpp)
    int dump(const Problem &p, const std::string &folder, int level, std::string &err);
    // relative residuals per iteration of load case rhs of the last plain solve; returns their count
    int history(int rhs, double *out, int cap, std::string &err) const;
    // batched mixed-precision form (engine_batch.cu)
    int setup_batch(int K, std::string &err);
    int plan_slabs(int K, std::string &err);       // tensor-core blocks and slab buffers
    int solve_batch(Problem &p, int nrhs, const double *f_nodal, double *u, htf_stats *stats, std::string &err);
    int apply_batch(int op, const double *x, double *y, int nrhs, std::string &err);
    bool batch_ready() const { return bK_ > 0; }
    // steps of a batched solve, for callers that interleave several problems
    int batch_loads(int nrhs, const double *f_nodal, std::string &err);
    int batch_begin(int r0, int kc, std::string &err);
    int batch_check(bool &all_done, std::string &err);
    int batch_finish(htf_stats *stats, double &ms, std::string &err);
    int batch_graph(std::string &err);
    void iter_a();                                  // before the F product
    void iter_b();                                  // between the F and S products
    void iter_c();                                  // after the S product
    TcSet tc_set() const;
    const std::vector<GemmBlock> &tc_blocks() const { return hblocks_; }
    int batch_width() const { return bK_; }
    int *tc_err() const { return d_tcerr_; }
    int n_dof() const { return ndof_; }
    const double *u_dev() const { return d_u_; }
    size_t device_bytes() const;
    // stream of every later launch (the engine's own one by default)
    void set_stream(cudaStream_t s) { s_ = s ? s : own_s_; }
    cudaStream_t stream() const { return s_; }
    int device() const { return opt_.device; }
    int apply(int op, const double *x, double *y, int nrhs, std::string &err);   // 0=F, 1=P, 2=M
    double setup_ms = 0.0;
    const std::vector<int> &symv_schedule() const { return schedule_; }
    bool symv_tuned() const { return tuned_; }
    double phase_ms[8] = {0, 0, 0, 0, 0, 0, 0, 0};   // see htf_profile_info::setup_phase_ms
    double kernel_detection_ms = 0.0;                 // part of phase 0 run on the device
    double frontend_ms = 0.0;                         // part of phase 0 run on the device
    int status_sub = -1;

private:
    template <typename T> T *alloc(size_t n, std::string &err, int &rc);
    void init_rhs(const double *f, const double *x_solved = nullptr);   // d = Bf K_HT^+ f, lambda0
    void trsm_multi(double *v, int nrhs);                 // v_j = K_reg^{-1} v_j, nrhs <= 32 columns of nfull
    void reconstruct(const double *f, double *u_dev);     // u from lambda, alpha
    double pcpg_start(PcpgState *st);                     // g0, Pg, z, Pz; returns nothing useful
    void tc_apply(int which);
    void f_pre(const double *w);
    void coarse_batch();
    void f_post(double *Fw, const double *dotv, double *partial);
    void m_pre(const double *x);
    void gather_x(const double *w, const double *weight, double *xb);   // x_b and the X slabs
    void m_post(double *z);
    int fp64_residual_batch(const std::vector<int> &sel, const std::vector<int> &reset, std::string &err);
    void profile_batch_gather(const double *w);
    void op_F_batch(const double *w, double *Fw, const double *dotv, double *partial);
    void op_M_batch(const double *x, double *z);
    void op_P_batch(const double *x, double *Px, double *alpha_out, const double *dotv, double *partial);
    void iteration_batch();
    int check(cudaError_t e, const char *what, std::string &err, const char *file = nullptr, int line = 0);
    int upload_layout(Problem &p, std::string &err);
    // SYMV work-unit schedules (autotune.cu)
    void build_units(const std::vector<int> &tiles, std::vector<SymvUnit> &units, long long &yoff, int &smem,
                     std::vector<int> &rbptr, std::vector<int> &rbunit);
    int apply_schedule(const std::vector<int> &tiles, bool subs_on_device, std::string &err);
    int alloc_units(std::string &err);
    std::string schedule_key() const;
    int autotune_symv(std::string &err);
    int factorize(Problem &p, std::string &err);
    int coarse(Problem &p, std::string &err);
    int outer_coarse(Problem &p, std::string &err);
    // device operators on device vectors (length n_lam)
    void op_F(const double *w, double *Fw, const double *dotv, double *partial, PcpgState *st);
    void op_M(const double *x, double *z, PcpgState *st);
    void op_P(const double *x, double *Px, double *alpha_out, const double *dotv, double *partial,
              PcpgState *st);
    void iteration(PcpgState *st);
    void coarse_apply(const double *gc, double *s, const PcpgState *st);
    void release(void *p);
    int solve_one(Problem &p, int rhs, double *u_dev, int &iters, double &norm0, double &rel,
                  double &solve_ms, std::string &err);
    int ensure_rhs(int nrhs, std::string &err);

    Options opt_;
    cudaStream_t s_ = nullptr, own_s_ = nullptr;
    std::vector<DevBuf> bufs_;
    int nsub_ = 0, ncl_ = 0, nlam_ = 0, nslots_ = 0, nfull_ = 0, ngc_total_ = 0, nt_total_ = 0;
    long long ntiles_ = 0;
    std::vector<SubDev> hs_;
    std::vector<ClusterDev> hc_;
    SubDev *d_subs_ = nullptr;
    ClusterDev *d_cl_ = nullptr;
    int *d_all_subs_ = nullptr;          // 0..nsub-1
    double *d_K_ = nullptr, *d_F_ = nullptr, *d_S_ = nullptr;
    std::vector<int> xwave_;             // subdomain boundaries of the L_bb^{-1} scratch waves
    long long xwave_max_ = 0;            // doubles of the largest wave
    // factor waves: consecutive subdomains whose panels share d_K_ (one wave
    // over all subdomains unless opt_.factor_wave_gb > 0); each is a union of
    // L_bb^{-1} waves, and K_off of a subdomain counts from its wave's start
    struct FactorWave {
        int a = 0, b = 0;                        // subdomains [a, b)
        long long kdoubles = 0;                  // its panels
        size_t eoff = 0;                         // its first (wave, colour) entry of ecptr_
        int blk0 = 0, blk1 = 0;                  // its tensor-core blocks (tensor-core slab layout)
        StepDesc *steps = nullptr;               // Cholesky step tables of its subdomains
        int *snap = nullptr, *hints = nullptr;
        std::vector<size_t> soff, htri, hrb, snap_off;
        std::vector<int> cnt, ntri, nrb, nsnap;
        size_t snap_first_off = 0;
        int nsnap_first = 0;
    };
    std::vector<int> fwave_;             // subdomain boundaries of the factor waves
    std::vector<FactorWave> fw_;
    std::vector<int> ecptr_;             // element ranges of d_order_ per (wave, colour)
    int ncol_ = 0, max_tiles_ = 0;
    bool waves_ = false;                 // factors dropped between uses (more than one wave)
    bool s_lean_ = false;                // S_i only as tensor-core slabs: d_S_ holds one wave's FP64 tiles during set-up
    int maxks_ = 0;                      // largest nbp / 32
    std::vector<int> sub_blk0_;          // first tensor-core block of each subdomain (nsub + 1)
    double *d_ec_ = nullptr, *d_E_ = nullptr, *d_nu_ = nullptr;   // element data for re-assembly
    int *d_ep_ = nullptr, *d_es_ = nullptr, *d_order_ = nullptr;
    double bf_[3] = {0.0, 0.0, 0.0};
    // assemble, regularise and factorise wave w; with build also the preconditioner
    // snapshots, the body-force load and F_i (X: L_bb^{-1} scratch)
    void factor_wave(int w, bool build, double *X);
    double *d_V_ = nullptr, *d_R_ = nullptr, *d_M_ = nullptr, *d_H_ = nullptr;
    double *d_MT_ = nullptr, *d_mP_ = nullptr, *d_mD_ = nullptr;   // packed symmetric M, its partial sums
    int2 *d_mt_ = nullptr;                     // (cluster, tile row) pairs of M
    int nmt_ = 0;
    int *d_bcr_ = nullptr, *d_bce_ptr_ = nullptr, *d_bce_pos_ = nullptr;
    double *d_bce_val_ = nullptr;
    int *d_slot_ptr_ = nullptr, *d_slot_ent_ = nullptr;
    int *d_rslot_ = nullptr;
    double *d_rsign_ = nullptr, *d_weight_ = nullptr;
    int *d_gptr_ = nullptr, *d_gidx_ = nullptr;
    int *d_gcl_ = nullptr;
    double *d_gval_ = nullptr;
    int *d_chunk_cl_ = nullptr, *d_chunk_beg_ = nullptr, *d_chunk_end_ = nullptr, *d_crow_ = nullptr,
        *d_cl_chunk_ptr_ = nullptr;
    double *d_cval_ = nullptr, *d_invGtG_ = nullptr;
    int nchunks_ = 0;
    int *d_status_ = nullptr;
    int *d_csp_ = nullptr, *d_cs_ = nullptr;   // cluster -> subdomain lists
    double *d_fbody_ = nullptr;                // assembled body-force load (full vectors)
    int *d_own_ = nullptr;                     // full slot -> global DOF it owns, or -1
    int *d_win_ = nullptr;                     // global DOF -> full slot of the highest subdomain
    double *d_fn_ = nullptr, *d_u_ = nullptr;  // nodal loads / displacements (global DOFs x nrhs)
    int rhs_cap_ = 0, ndof_ = 0;
    int kernels_per_iter_ = 0;
    long long launches_ = 0;                   // kernels launched by the current solve call
    SymvUnit *d_units_ = nullptr;              // SYMV work units (+ one V^T x unit per subdomain)
    int *d_rbptr_ = nullptr, *d_rbunit_ = nullptr;   // per 32-row block of every subdomain: the units covering it
    long long rbptr_cap_ = 0, rbunit_cap_ = 0;
    double *d_ypart_ = nullptr;                // partial y sums of the units (scratch)
    int nunits_ = 0, max_nbp_ = 0;
    long long units_cap_ = 0, ypart_cap_ = 0;    // unit buffers, sized for every candidate schedule
    int symv_smem_cap_ = 0;
    std::vector<int> schedule_;                  // unit tiles per size bucket in use
    bool tuned_ = false;
    // batched mixed-precision form
    int bK_ = 0, nblocks_ = 0, bnpart_ = 0, bnpartP_ = 0;
    float *d_AF_ = nullptr, *d_AS_ = nullptr, *d_Xs_ = nullptr;
    unsigned *d_amaxF_ = nullptr, *d_amaxS_ = nullptr;   // scales of the FP16-pair slabs (largest |A| per subdomain)
    unsigned *d_xmax_ = nullptr;                         // scale of the X slabs (largest |w_j| per column)
    float xbound_ = 1.f;                                 // |x_b| <= xbound_ max|w_j|
    void *d_blocks_ = nullptr;
    TcSet *d_tcset_ = nullptr;
    std::vector<GemmBlock> hblocks_;
    BatchRun run_;
    cudaEvent_t run_e0_ = nullptr, run_e1_ = nullptr;
    int *d_slot_sub_ = nullptr, *d_tcerr_ = nullptr;
    double *b_lam_ = nullptr, *b_g_ = nullptr, *b_w_ = nullptr, *b_Fw_ = nullptr, *b_Pg_ = nullptr, *b_z_ = nullptr,
           *b_Pz_ = nullptr, *b_d_ = nullptr, *b_xb_ = nullptr, *b_yb_ = nullptr, *b_t_ = nullptr, *b_gc_ = nullptr,
           *b_s_ = nullptr, *b_part_ = nullptr, *b_gpart_ = nullptr, *b_wFw_ = nullptr, *b_gPz_ = nullptr, *b_gw_ = nullptr, *b_gt_ = nullptr, *b_acoef_ = nullptr,
           *b_alpha_ = nullptr, *b_tmp_ = nullptr;
    double *b_fullA_ = nullptr, *b_fullB_ = nullptr;   // full vectors of the batch (nfull x K)
    double *b_srec_ = nullptr;                         // coarse solutions of the reconstruction (ngc x K)
    double *b_alpha2_ = nullptr;                       // alpha of the FP64 residuals, K-interleaved
    int *d_mask_ = nullptr;                            // selected / reset columns of an FP64 residual batch
    void *d_rowblk_ = nullptr;                         // (subdomain, 32-row block) list of the FP64 multi-RHS SYMV
    int nrowblk_ = 0;
    PcpgState *b_st_ = nullptr;
    cudaGraphExec_t bgraph_ = nullptr;
    int bkernels_per_iter_ = 0;
    int tc_smem_ = 0, vt_nch_ = 1, vt_qn_ = 64;
    long long aoff_ = 0;                       // 4-byte words per slab array
    // vectors
    double *d_f_ = nullptr, *d_full_ = nullptr, *d_full2_ = nullptr;
    double *d_lam_ = nullptr, *d_g_ = nullptr, *d_w_ = nullptr, *d_Fw_ = nullptr, *d_Pg_ = nullptr,
           *d_z_ = nullptr, *d_Pz_ = nullptr, *d_d_ = nullptr, *d_tmp_ = nullptr;
    double *d_xb_ = nullptr, *d_yb_ = nullptr, *d_t_ = nullptr, *d_gc_ = nullptr, *d_s_ = nullptr;
    double *d_a_ = nullptr, *d_alpha_ = nullptr, *d_partial_ = nullptr, *d_gpart_ = nullptr;
    PcpgState *d_st_ = nullptr;
    double *d_hist_ = nullptr;                 // relative residual per iteration of the running solve
    std::vector<std::vector<double>> hist_;    // per load case (first 64) of the last plain solve
    int npart_ = 0;
    int symv_smem_ = 0;
    bool mixed_ = false;
    bool implicit_ = false;                    // Dirichlet_implicit: S_d applied through L_bb, no S tiles
    int2 *d_lblk_ = nullptr;                   // (subdomain, 32-block) pairs of the L_bb passes
    int nlblk_ = 0;
    double *d_tb_ = nullptr;                   // b-space L_bb^T x of the implicit preconditioner
    cudaGraphExec_t graph_ = nullptr;
    double fapply_ms_ = 0.0, fapply_bytes_ = 0.0;
    std::vector<std::vector<double>> Hd_;   // per subdomain 6x6 rows of ker(Gc)
    long long kpanel_total_ = 0;            // doubles of all factor panels
    std::vector<double> dumpK_;             // K_reg panels before the factorisation (print_matrices >= 2)
    std::vector<double> gtg_, gval_;        // Gf^T Gf and the Gf rows (print_matrices >= 2)
    std::vector<int> gcl_;
    std::vector<double> invGtG_;
};

template <typename T> T *Engine::alloc(size_t n, std::string &err, int &rc) {
    if (rc) return nullptr;
    void *p = nullptr;
    const size_t bytes = (n > 0 ? n : 1) * sizeof(T);
    const cudaError_t e = cudaMalloc(&p, bytes);
    if (e != cudaSuccess) {
        rc = check(e, "cudaMalloc", err);
        err += " (" + std::to_string(bytes) + " bytes)";
        return nullptr;
    }
    bufs_.push_back({p, bytes});
    return static_cast<T *>(p);
}

}  // namespace htf
