// Host-side problem description of the HTFETI path: mesh, per-subdomain
// DOF maps, the dual layout (Bf, Bc, weights), kernels and fix DOFs, and the
// small dense coarse objects.  Integer/index work and the O(n) FP64 pieces
// live here; everything O(n^2) and above runs on the GPU.
#pragma once
#include <cstdint>
#include <string>
#include <vector>

#include "htfeti.h"

namespace htf {

// splitmix64 counter hash -> uniform [0,1)
uint64_t mix64(uint64_t z);
double u01(uint64_t seed, uint64_t stream, uint64_t i);

struct Mesh {
    int n_nodes = 0;
    std::vector<double> coords;     // 3*n_nodes
    std::vector<int> elems;         // 8*n_elems
    std::vector<int> elem_sub;      // n_elems
    std::vector<int> sub_cluster;   // n_sub
    std::vector<double> sub_E, sub_nu;
    std::vector<int> dirichlet;     // reference order
    std::vector<int> corner;        // sorted
    double body_force[3] = {0, 0, 0};
    int n_elems() const { return int(elem_sub.size()); }
    int n_sub() const { return int(sub_cluster.size()); }
};

// Mesh::createMesh generalised (Mesh.cpp:69-289).
int generate_mesh(const htf_mesh_spec &s, Mesh &m, std::string &err);
// sum over subdomains of 8 (n_d^2/2 + 16 n_d) (n_d = 3 x nodes of subdomain
// d): the column-panel factors alone, a lower bound of the device footprint
// of a spec's problem
int mesh_sizes(const htf_mesh_spec &s, int *nn, int *ne, int *ns, int *nc, int *nd, int *ncr,
               std::string &err);
int mesh_traction(const htf_mesh_spec &s, uint64_t seed, int n_rhs, double scale, double *f,
                  std::string &err);
// box.vtk of the displacement field (vtk.cpp)
int write_vtk(const char *path, int n_nodes, const double *coords, int n_elems, const int *elems,
              const int *elem_sub, const int *elem_mat, const double *u);

struct Options {
    std::string typeBc = "cor";                       // cor | ker | all
    std::string preconditioner = "Dirichlet_explicit";
    double eps_iter = 1e-8;
    int max_iter = 500;
    bool mixed = false;                               // precision=mixed
    double mixed_eps_factor = 0.1;                    // the batched mixed form stops at eps_iter x this factor:
                                                      // the reference's criterion at eps_iter alone leaves the
                                                      // displacements ~1e-7 from converged on ill-conditioned
                                                      // meshes, the mixed form's bound against the FP64 oracle
    int device = 0;
    int check_every = 8;                              // iterations between host convergence checks
    int batch = 32;                                   // load cases per batched mixed-precision solve (16 | 32)
    int verbose = 0;                                  // progress lines on stderr
    int print_matrices = 0;                           // the reference's dump level (Cluster.cpp:31): >= 2 keeps
                                                      // K_i for htf_dump (MatrixMarket files)
    int autotune = 1;                                 // time SYMV work-unit sizes at setup (once per process and
                                                      // problem class) for problems of >= 1 GiB of FP64 tiles;
                                                      // 2 = every problem; 0 = fixed default schedule
    std::string tune_file;                            // JSON file of tuned schedules, read and extended
    double factor_wave_gb = 0.0;                      // > 0: the factor panels of at most this many GB of
                                                      // subdomains are held at a time; set-up and every later
                                                      // K_reg solve assemble and factorise them again, wave
                                                      // by wave (batched mixed form, explicit preconditioners)
    bool S_fp64 = true;                               // false: S_i is kept only as the 4-byte slabs of the tensor-
                                                      // core product, which the FP64 residual replacements apply
                                                      // too (batched mixed form, explicit preconditioners)
    bool admit_oversize = false;                      // server: a request that does not fit the budget alone is
                                                      // admitted with factor waves (and S_fp64 = 0 if needed)
                                                      // instead of being refused with HTF_ENOMEM
};
int parse_options(const char *s, Options &o, std::string &err);

// One Bf row: up to two (subdomain, global DOF, sign) entries.
struct BfRow {
    int sub[2];
    int dof[2];
    double sign[2];
};

struct Subdomain {
    int id = 0, cluster = 0, cl_index = 0;   // index inside its cluster
    std::vector<int> elems;                  // element ids in increasing order
    std::vector<int> l2g;                    // sorted global DOFs (Data.cpp:111-144)
    std::vector<int> b;                      // sorted local DOFs touched by Bf (j_col_cmpr)
    std::vector<int> perm;                   // local DOF -> position in [interior | b] order
    int n = 0, nb = 0, nr = 0;
    std::vector<double> R;                   // n x 6, column-major, orthonormal columns
    std::vector<int> fix;                    // 6 sorted local DOFs (all in b)
    // Bc entries of this subdomain: cluster row, local DOF, value
    std::vector<int> bc_row, bc_col;
    std::vector<double> bc_val;
    std::vector<int> bc_rows;                // sorted distinct cluster rows (l2g_i_coo of Bc)
    int c() const { return int(bc_rows.size()); }
    // Bf entries grouped per b position: CSR
    std::vector<int> bf_ptr;                 // nb+1
    std::vector<int> bf_lam;                 // lambda row
    std::vector<double> bf_sign;
    std::vector<double> f;                   // assembled load per local DOF, n x nrhs (filled on device)
};

struct Cluster {
    std::vector<int> subs;   // global subdomain ids in this cluster
    int nlam_c = 0;          // Bc rows
    int ngc() const { return nlam_c + 6 * int(subs.size()); }
};

struct Problem {
    Mesh mesh;
    Options opt;
    std::vector<Subdomain> sub;
    std::vector<Cluster> clu;
    std::vector<BfRow> rows;
    std::vector<double> weight;
    int n_lam = 0;
    int nrhs = 1;
    std::vector<double> f_nodal;            // 3*n_nodes*nrhs (optional)
    double context_ms = 0.0;                // host wall of the device context creation (set-up only)
    double kernel_ms = 0.0;                 // host wall of the device kernel detection (set-up only)
    double frontend_ms = 0.0;               // host wall of the device front-end (set-up only)
};

// Data::buildMappingStruct + Cluster::create_cluster_constraints +
// kernels/fix DOFs.  Returns HTF_OK or an error code with err set.
// on_device: kernels and fix DOFs on the GPU (kernel_fix.cu), bit-identical
// to the host code used otherwise
int build_problem(Problem &p, std::string &err, bool on_device = false);
// l2g, Bf rows and weights, b sets and Bf CSR of all subdomains on the GPU
// (frontend.cu), bit-identical to the host front-end; node_ptr / node_subs:
// the sorted subdomains of every node.  HTF_ESTATE: a Dirichlet list with a
// repeated DOF, HTF_ENODEV: no device; the host front-end builds both
int frontend_on_device(Problem &p, std::vector<int> &node_ptr, std::vector<int> &node_subs, std::string &err);
// kernel bases and fix DOFs of all subdomains on the GPU (kernel_fix.cu)
// timing_ms (optional): [0] device context creation, [1] the rest (uploads,
// kernel, copies back), host wall milliseconds
int kernels_fix_on_device(const Mesh &m, std::vector<Subdomain> &subs, int device, std::string &err,
                          double *timing_ms = nullptr);

// Analytic rigid body modes of the nodes of l2g (column order of
// Data::create_analytic_ker_K, Data.cpp:61-109), Gram-Schmidt'ed
// (Matrix.cpp:2450-2472).
void kernel_of(const Mesh &m, const std::vector<int> &l2g, std::vector<double> &R);
// Matrix::getNullPivots (Matrix.cpp:835-884) on an n x m column-major matrix.
std::vector<int> null_pivots(const std::vector<double> &R, int n, int m);

// ---- small dense FP64 helpers (column-major) ----
bool chol_lower(int n, double *A, int lda);   // in place; false if not numerically SPD
void chol_solve(int n, const double *L, int lda, double *B, int ldb, int nrhs);
void sym_eig(int n, std::vector<double> &A, std::vector<double> &w, std::vector<double> &V);

}  // namespace htf
