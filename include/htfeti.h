/*
 * htfeti.h - C ABI of the B200 HTFETI (hybrid total FETI) solve path.
 *
 * The reference (ostravaTokyo/hfls) exposes its solver only as C++ classes
 * (Driver, Cluster, Solver, Matrix, Mesh; no FFI).  Every entry point below
 * replaces one of those class members and says which.  Conventions:
 *   - return 0 on success, a negative HTF_E* code on failure (never exit());
 *     htf_last_error() gives a message for the last failing call on a context;
 *   - caller-owned host buffers, library-owned device memory;
 *   - one context per host thread; contexts are independent.
 * Arrays are 0-based.  DOF g = 3*node + component.  Dense matrices are
 * column-major.
 */
#ifndef HTFETI_H
#define HTFETI_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- error codes ------------------------------------------------------- */
#define HTF_OK 0
#define HTF_EINVAL -1       /* bad argument or option                          */
#define HTF_ENOMEM -2       /* device or host allocation failed                */
#define HTF_ECUDA -3        /* CUDA runtime error (message has the detail)     */
#define HTF_ENOTSPD -4      /* a regularised K_i or coarse matrix is not SPD   */
#define HTF_EBREAKDOWN -5   /* PCPG: w'Fw <= 0, NaN or Inf                      */
#define HTF_ENOCONV -6      /* PCPG: max_iter reached                          */
#define HTF_ESTATE -7       /* call out of order (e.g. pcpg before setup)      */
#define HTF_ETIMEDOUT -8    /* a bounded device wait gave up                   */
#define HTF_ENODEV -9       /* no CUDA device                                  */
#define HTF_EIO -10         /* a file could not be written                     */

/* ---- mesh generation ----------------------------------------------------
 * Replaces Mesh::createMesh (Mesh.cpp:69-289), generalised to clusters,
 * non-uniform subdomain slabs, node jitter, per-subdomain materials and the
 * boundary conditions of the benchmark configurations.                     */
#define HTF_BC_ROLLERS 0    /* u_x=0 on x=0, u_y=0 on y=0, u_z=0 on z=0 (Mesh.cpp:221-239) */
#define HTF_BC_CLAMP_X0 1   /* u=0 on the face x=0                                         */

#define HTF_MAT_CONST 0     /* E everywhere                                                 */
#define HTF_MAT_CHECKER 1   /* E*ratio on even subdomains (Data.cpp:47-48, Mesh.cpp:281)    */
#define HTF_MAT_LOGUNIFORM 2 /* E_i ~ logU[E_lo, E_hi] per subdomain, seeded                */

typedef struct htf_mesh_spec {
    int clusters[3];         /* clusters per axis                                   */
    int subs[3];             /* subdomains per cluster per axis                     */
    int elems[3];            /* elements per subdomain per axis (uniform slabs)     */
    const int *widths[3];    /* optional: element count of every subdomain slab
                                along axis a (clusters[a]*subs[a] entries); NULL =
                                uniform elems[a]                                    */
    double jitter;           /* interior nodes moved by U(-jitter*h, jitter*h)      */
    uint64_t seed;           /* seed of jitter, materials and tractions             */
    int bc;                  /* HTF_BC_*                                            */
    int material;            /* HTF_MAT_*                                           */
    double E, E_hi, nu;      /* CONST: E; CHECKER: E, ratio=E_hi; LOGUNIFORM: [E,E_hi] */
    double body_force[3];    /* rho*a per unit volume                               */
} htf_mesh_spec;

/* Sizes of the generated mesh (two-call pattern with htf_mesh_fill). */
int htf_mesh_sizes(const htf_mesh_spec *spec, int *n_nodes, int *n_elems, int *n_sub,
                   int *n_clusters, int *n_dirichlet, int *n_corner);

/* Fill caller buffers: coords[3*n_nodes], elems[8*n_elems] (node order of
 * Mesh.cpp:250-257), elem_sub[n_elems], sub_cluster[n_sub], sub_E[n_sub],
 * sub_nu[n_sub], dirichlet[n_dirichlet], corner[n_corner] (corner DOFs of
 * Mesh.cpp:175-208).  Any pointer may be NULL to skip that array.          */
int htf_mesh_fill(const htf_mesh_spec *spec, double *coords, int *elems, int *elem_sub,
                  int *sub_cluster, double *sub_E, double *sub_nu, int *dirichlet, int *corner);

/* Seeded N(0,1) nodal forces on the face x=1 for n_rhs load cases, added to
 * f[3*n_nodes*n_rhs] (column-major: load case k at f + k*3*n_nodes).  The
 * reference has no traction; it is a configuration load.                   */
int htf_mesh_traction(const htf_mesh_spec *spec, uint64_t seed, int n_rhs, double scale, double *f);

/* ---- solution output ----------------------------------------------------
 * Replaces Mesh::SaveVTK (Mesh.cpp:292-351), which Cluster::printVTK
 * (Cluster.cpp:1648-1678) calls with the displacement field at the end of
 * the solve: writes `path` as the reference's box.vtk (legacy ASCII VTK,
 * unstructured grid of hex8 cells, same layout and number formats), with
 * u[3*n_nodes] as the point field "displacements", elem_sub as the cell field
 * "decomposition" and elem_mat as "materialId".  elem_mat may be NULL: the
 * reference's rule is used, remainder(elem_sub, 2) (Mesh.cpp:280-281; 0, 1
 * or -1).  Host only, no context.  HTF_EINVAL for a NULL array or a node id
 * out of range, HTF_EIO if the file cannot be written.                     */
int htf_write_vtk(const char *path, int n_nodes, const double *coords, int n_elems, const int *elems,
                  const int *elem_sub, const int *elem_mat, const double *u);

/* ---- solver context ------------------------------------------------------
 * Replaces Driver::Driver(map) / Cluster::initialization's options map
 * (Driver.cpp:14-18, htfeti.cpp:12-57).  `options` is a ';'-separated list
 * of key=value with the reference's keys (eps_iter, max_iter,
 * preconditioner = Dirichlet_explicit | Dirichlet_implicit | lumped,
 * typeBc = cor | ker | all, Ac_extended_by_kerGc) and this library's keys:
 * precision = fp64 | mixed, device = <cuda ordinal>, batch = 16 | 32 (load
 * cases per batched mixed solve), check_every = <iterations between host
 * convergence checks>, autotune = 1 | 2 | 0 (time the FP64 SYMV work-unit
 * sizes per subdomain-size bucket at set-up, once per process and problem
 * class: 1 for problems of at least 1 GiB of FP64 tiles, 2 for every
 * problem, 0 never), tune_file = <path of a JSON file of tuned schedules,
 * read and extended>, factor_wave_gb = <GB> (0: every factor panel stays
 * resident; > 0: the panels of at most that many GB of subdomains are held
 * at a time and are assembled and factorised again, wave by wave, for each
 * later K_reg solve — the batched mixed form with an explicit
 * preconditioner only), S_fp64 = 1 | 0 (0: S_i is kept only as the 4-byte
 * slabs of the tensor-core product, which the FP64 residual replacements
 * apply too — batched mixed form, explicit preconditioner), verbose = 0 | 1,
 * admit_oversize = 0 | 1 (server only; 1: a request whose footprint does not
 * fit the budget alone is admitted with factor_wave_gb and, if still needed,
 * S_fp64 = 0 picked for it, instead of failing with HTF_ENOMEM).
 * The batched mixed form stops a load case whose FP64 residual has not halved
 * over ten residual replacements and at least 500 iterations with
 * HTF_ENOCONV ("stagnated"): its FP32 products cannot reach eps_iter.     */
typedef struct htf_ctx htf_ctx;

int htf_create(const char *options, htf_ctx **ctx);
int htf_destroy(htf_ctx *ctx);
const char *htf_last_error(const htf_ctx *ctx);
/* Subdomain whose regularised K_i was found not positive definite by the
 * last htf_setup that returned HTF_ENOTSPD (-1 otherwise; also reported as
 * htf_stats.status_sub by later solves).  The reference exits from inside
 * PARDISO's factorisation instead (Matrix.cpp:1174-1178).                  */
int htf_status_sub(const htf_ctx *ctx);

/* Mesh of one problem.  Replaces the Mesh& argument of
 * Cluster::initialization (Cluster.cpp:21, 42) and the public Mesh fields
 * it reads (points, elements, DirichletDOFs, cornerDOFs, Mesh.hpp:72-84).
 * All arrays are copied.                                                   */
int htf_set_mesh(htf_ctx *ctx, int n_nodes, const double *coords, int n_elems, const int *elems,
                 const int *elem_sub, int n_sub, const int *sub_cluster, const double *sub_E,
                 const double *sub_nu, int n_dirichlet, const int *dirichlet, int n_corner,
                 const int *corner, const double body_force[3]);

/* Extra nodal forces for n_rhs load cases (f_nodal[3*n_nodes*n_rhs],
 * column-major), added to the body-force load of every case.  Without this
 * call there is one load case: the body force.                            */
int htf_set_loads(htf_ctx *ctx, int n_rhs, const double *f_nodal);

/* Setup.  Replaces Cluster::initialization up to the PCPG call
 * (Cluster.cpp:21-360): assembly (Data.cpp:25-273), kernels and fix-DOF
 * regularisation (Matrix.cpp:835-884, 1029-1057), constraints
 * (Cluster.cpp:682-959), Dirichlet preconditioner (Matrix.cpp:1708-1871),
 * local and cluster coarse objects (Cluster.cpp:150-352).  On the GPU: hex8
 * assembly, batched dense Cholesky, explicit F_i = (K_reg^{-1})_bb and S_i. */
int htf_setup(htf_ctx *ctx);

typedef struct htf_stats {
    int iterations[64];      /* PCPG iterations per load case (first 64)      */
    double norm_gPz0[64];
    double final_rel[64];    /* sqrt(g'Pz)/sqrt(g0'Pz0) at exit               */
    double setup_ms;         /* device time of htf_setup                      */
    double solve_ms;         /* device time of the PCPG loops (g0 -> exit)    */
    double fapply_ms;        /* mean device time of one F apply               */
    double fapply_bytes;     /* algorithmic bytes of one F apply              */
    int n_lambda, n_sub, n_clusters, n_rhs;
    int status_sub;          /* subdomain index of an HTF_ENOTSPD failure     */
    long long kernel_launches; /* kernels this call launched on the device    */
} htf_stats;

/* PCPG for every load case and the displacement field.  Replaces
 * Cluster::pcpg (Cluster.cpp:1363-1458) and the solution assembly of
 * Cluster::printVTK (Cluster.cpp:1648-1678): u[3*n_nodes*n_rhs] receives
 * the displacements (for DOFs shared by several subdomains the highest
 * subdomain index wins, as in the reference).  u may be NULL.             */
int htf_pcpg(htf_ctx *ctx, double *u, htf_stats *stats);

/* Solve n_rhs new load cases with the factors resident on the device.
 * f_nodal[3*n_nodes*n_rhs] (column-major, may be NULL) is added to the body
 * force; u[3*n_nodes*n_rhs] receives the displacements as in htf_pcpg.
 * Host buffers in and out; this is the call a serving loop makes per
 * request.  Replaces a repeated Cluster::pcpg with a new rhs
 * (Cluster.cpp:1385-1458) without redoing the setup.                     */
int htf_solve(htf_ctx *ctx, int n_rhs, const double *f_nodal, double *u, htf_stats *stats);

/* Device timing of the dominant kernels on the library's own stream
 * (CUDA events, averaged over `reps` launches after one warm-up), with the
 * algorithmic bytes each launch moves.  No counterpart in the reference
 * (it only prints clock() totals, Cluster.cpp:378-379, 1451-1452).        */
typedef struct htf_profile_info {
    double symv_F_ms, symv_F_bytes;     /* y_b = F_i x_b over all subdomains        */
    double symv_S_ms, symv_S_bytes;     /* preconditioner block, same layout        */
    double fapply_ms, fapply_bytes;     /* whole F apply (gather .. scatter)        */
    double iteration_ms;                /* one captured PCPG iteration              */
    int kernels_per_iteration;          /* kernel launches in one iteration graph   */
    /* batched mixed-precision form (precision=mixed after a solve; else 0)  */
    int batch_width;                    /* load cases per batch                     */
    double tc_F_ms, tc_F_bytes;         /* Y_b = F_i X_b for the whole batch on the
                                           tensor cores: 4-byte slabs + X + Y bytes   */
    double batch_iteration_ms;          /* one captured batched PCPG iteration      */
    int kernels_per_batch_iteration;
    /* host wall time of the phases of htf_setup (ms): 0 problem build (maps,
     * Bf/Bc, kernels, fix DOFs), 1 device context and stream, 2 layout upload
     * and allocation, 3 assembly + factorisation + F_i/S_i, 4 load and
     * displacement maps, 5 cluster coarse problems, 6 outer coarse problem,
     * 7 SYMV schedule tuning and tensor-core slabs of the batched form              */
    double setup_phase_ms[8];
    /* SYMV schedule in use: work-unit tiles for subdomains with at most
     * 8, 16, 32, 64 and more tile rows; tuned = 1 when it came from the
     * autotuner (option autotune) or its cache                             */
    int symv_unit_tiles[5];
    int symv_tuned;
    double device_bytes;                /* device memory the context holds          */
    double kernel_detection_ms;         /* host wall of the kernel bases and fix
                                           DOFs computed on the device (part of
                                           setup phase 0)                           */
    double frontend_ms;                 /* host wall of the l2g / Bf rows / b sets
                                           built on the device (part of phase 0)    */
} htf_profile_info;
int htf_profile(htf_ctx *ctx, int reps, htf_profile_info *info);

/* The dual operators on host vectors of length n_lambda (nrhs columns,
 * column-major).  Replace Cluster::mult_Ff (Cluster.cpp:1114-1188),
 * Cluster::Projection (Cluster.cpp:1314-1329) and Cluster::Preconditioning
 * (Cluster.cpp:1043-1112).                                                */
int htf_mult_Ff(htf_ctx *ctx, const double *w, double *Fw, int nrhs);
int htf_projection(htf_ctx *ctx, const double *x, double *Px, int nrhs);
int htf_preconditioning(htf_ctx *ctx, const double *x, double *Mx, int nrhs);

/* Projector P x = x - Gf (Gf^T Gf)^{-1} Gf^T x on caller-owned DEVICE
 * vectors of n_lambda doubles (on the context's device), enqueued on
 * `stream` (a cudaStream_t, NULL = legacy default stream) and returning
 * without waiting.  It allocates nothing: its reduction scratch is a static
 * device array of HTF_NOALLOC_SCRATCH_DOUBLES doubles (8 MiB, held by every
 * GPU that loads the library until exit), for callers that cannot allocate
 * while they project — a serving loop held to a fixed device-memory budget,
 * or a latency-bound loop that must not trigger the synchronisation an
 * allocation can cause.  No counterpart in the reference.  The first call on
 * a device looks the array up and should come before any stream capture;
 * all calls share the array, so calls that overlap on the GPU race.
 * Returns HTF_EINVAL when the problem needs more scratch than the array
 * holds (6 doubles per chunk of up to 1024 dual rows of one cluster: about
 * 170 million (row, cluster) entries of Gf), or when a vector is not device
 * memory of the context's device.                                         */
#define HTF_NOALLOC_SCRATCH_DOUBLES 1048576
int htf_projection_noalloc(htf_ctx *ctx, const double *x_dev, double *Px_dev, void *stream);

/* Relative residual sqrt(g'Pz)/sqrt(g0'Pz0) at every PCPG iteration of load
 * case rhs (< 64) of the last plain FP64 htf_pcpg / htf_solve: hist[0] = 1,
 * hist[i] after iteration i, as the reference prints them (Cluster.cpp:
 * 1422-1424).  Copies at most cap values; returns their total count (or a
 * negative code).                                                         */
int htf_residual_history(htf_ctx *ctx, int rhs, double *hist, int cap);

/* MatrixMarket files of the set-up problem, written as the reference's
 * Matrix::printToFile writes them (Matrix.cpp:556-632; names
 * <folder>/dump_<name>_<index>.txt, 1-based coordinates, "%.16e" values) at
 * the reference's print_matrices levels (Cluster.cpp:118-358): level >= 2
 * K_i (upper triangle, symmetric), rhs_i (the element load), Bc_i, Bf_i;
 * >= 3 also R_i, Rf_i, Gf_clust, GfTGf, iGfTGf; >= 4 also S_i (explicit
 * Dirichlet preconditioner).  K_i needs the option print_matrices >= 2 at
 * htf_create (the set-up keeps a host copy before factorising; HTF_ESTATE
 * otherwise).  HTF_EIO if a file cannot be written.                       */
int htf_dump(htf_ctx *ctx, const char *folder, int level);

/* Dual layout for checking: n_lambda, and for every Bf row its entries as
 * (subdomain, global DOF, sign) with up to two entries per row
 * (Cluster.cpp:846-924); weights (Cluster.cpp:893-895, 918).  Arrays of
 * length 2*n_lambda (second entry sub = -1 when the row has one).         */
int htf_dual_sizes(htf_ctx *ctx, int *n_lambda, int *n_sub, int *n_clusters);
int htf_dual_layout(htf_ctx *ctx, int *row_sub, int *row_dof, double *row_sign, double *weight);

/* Fix DOFs (6 per subdomain, global DOF ids) chosen for the regularisation
 * (Matrix.cpp:835-884 restricted to the Bf column set).                   */
int htf_fix_dofs(htf_ctx *ctx, int *fix_global);

/* ---- Continuous-batching solve server (no counterpart in the reference,
 * which solves one problem per process, htfeti.cpp:8-21).  Requests — a
 * mesh spec and 1..batch load cases — are admitted in arrival order while
 * the estimated device footprint of their factors, F_i / S_i and vectors fits
 * the HBM budget and fewer than max_live are set up or running; their setup
 * overlaps the iterations of running requests; all running requests advance
 * together in the batched mixed-precision form (options as for htf_create,
 * precision forced to mixed), their F and S products in one tensor-core
 * launch.  A request's result does not depend on the others in the mix.
 * htf_server_destroy lets every submitted request finish first.            */
typedef struct htf_server htf_server;

#define HTF_REQ_QUEUED 0
#define HTF_REQ_SETUP 1
#define HTF_REQ_RUNNING 2
#define HTF_REQ_DONE 3
#define HTF_REQ_FAILED 4

typedef struct htf_request_info {
    int status;                         /* HTF_REQ_*                                */
    int rc;                             /* HTF_OK or the failed request's code      */
    int n_rhs, iterations_max;
    double t_submit_ms, t_admit_ms;     /* wall times since the server was created  */
    double t_start_ms, t_done_ms;       /* joined the iterations / finished         */
    double setup_ms, solve_ms;          /* device time of setup and of the solve    */
    double bytes;                       /* device bytes held by the request         */
    double bytes_estimate;              /* the footprint estimate it was admitted on */
} htf_request_info;

/* hbm_budget_bytes <= 0: 85 % of the device's free memory; max_live <= 0: 8 */
int htf_server_create(const char *options, double hbm_budget_bytes, int max_live, htf_server **srv);
int htf_server_destroy(htf_server *srv);
/* f_nodal: 3*n_nodes*n_rhs nodal loads (copied; NULL = body force only);
 * u: caller-owned 3*n_nodes*n_rhs displacements, written at completion    */
int htf_server_submit(htf_server *srv, const htf_mesh_spec *spec, int n_rhs, const double *f_nodal, double *u,
                      long long *ticket);
/* timeout_ms < 0 waits for completion; HTF_ETIMEDOUT if still running;
 * returns the request's own code once it has finished                     */
int htf_server_wait(htf_server *srv, long long ticket, double timeout_ms, htf_request_info *info);
int htf_server_info(htf_server *srv, long long ticket, htf_request_info *info);
/* message of a failed request (ticket > 0) or of the last failed submit   */
const char *htf_server_error(htf_server *srv, long long ticket);

#ifdef __cplusplus
}
#endif
#endif /* HTFETI_H */
