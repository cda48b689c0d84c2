// Driver for the reference's own classes (Mesh, Cluster, Data, Matrix) built
// unmodified from the reference sources.  It replaces htfeti.cpp's main:
// options come as key=value arguments (same keys as htfeti.cpp:12-57), and
// after Cluster::initialization (setup + PCPG + VTK of u) it writes the data
// used to pin the oracle:
//   mesh.txt    points, elements, partition/material ids, Dirichlet and corner DOFs
//   layout.txt  per subdomain l2g, Bf CSR + compressed-row ids, weights
//   probe.txt   w, P F P w and P M P w for a seeded w (Projection, mult_Ff,
//               Preconditioning of the reference, Cluster.cpp:1043-1188,1314-1329)
//   elem.txt    Data::stf_mtrx_solid45 on an axis-aligned and a distorted hex
//   timing.txt  wall seconds of the reference's own timed intervals (below)
// The displacement field is the reference's own box.vtk in path2data.
//
// Timing: clock() is wrapped too (--wrap=clock).  The reference calls it four
// times in a run: at the start of Cluster::initialization (Cluster.cpp:24),
// at the start and end of Cluster::pcpg's timed region (Cluster.cpp:1364,
// 1451; the final printVTK is outside it) and at the end of the setup +
// solve (Cluster.cpp:374).  The wrapper returns the real clock() and records
// a steady-clock wall time per call, so timing.txt holds the reference's own
// "Solver time" and "Total time" intervals in wall seconds at microsecond
// resolution (the reference prints them with one decimal).  `dumps=false`
// skips the layout, probe and element dumps.
//
// Two process-level measures keep the run deterministic without touching the
// sources: time() is wrapped (link flag --wrap=time) so the srand(time(NULL))
// seeds of the kernel detection (Matrix.cpp:2164,2172,2188) are constant, and
// the global allocator pads every block with 0xFF bytes so the read past the
// end of nullPivots in Matrix::num_factor (Matrix.cpp:1040) sees -1 and never
// triggers the out-of-bounds write at Matrix.cpp:1043.
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <ctime>
#include <new>
#include <string>
#include <map>
#include <vector>
#include <cmath>
#include <sys/stat.h>
#include "Cluster.hpp"

extern "C" time_t __wrap_time(time_t *t) {
    if (t) *t = 12345;
    return 12345;
}

extern "C" clock_t __real_clock(void);
static std::vector<double> g_clock_wall;
extern "C" clock_t __wrap_clock(void) {
    g_clock_wall.push_back(std::chrono::duration<double>(
        std::chrono::steady_clock::now().time_since_epoch()).count());
    return __real_clock();
}

static const size_t kPad = 64;
void *operator new(size_t n) {
    void *p = std::malloc(n + kPad);
    if (!p) throw std::bad_alloc();
    std::memset(static_cast<char *>(p) + n, 0xFF, kPad);
    return p;
}
void operator delete(void *p) noexcept { std::free(p); }
void operator delete(void *p, size_t) noexcept { std::free(p); }
void *operator new[](size_t n) { return operator new(n); }
void operator delete[](void *p) noexcept { std::free(p); }
void operator delete[](void *p, size_t) noexcept { std::free(p); }

// splitmix64-based uniform in [0,1): the same counter hash the framework's
// mesh generator uses for node jitter.
static uint64_t mix64(uint64_t z) {
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    return z ^ (z >> 31);
}
static double u01(uint64_t seed, uint64_t stream, uint64_t i) {
    uint64_t z = mix64(seed * 0x9E3779B97F4A7C15ULL + stream * 0xD1B54A32D192ED03ULL + i + 0x632BE59BD9B4E019ULL);
    return double(z >> 11) * (1.0 / 9007199254740992.0);
}

static void dump_vec(FILE *f, const char *name, const std::vector<double> &v) {
    std::fprintf(f, "%s %zu\n", name, v.size());
    for (double x : v) std::fprintf(f, "%.17g\n", x);
}
static void dump_ivec(FILE *f, const char *name, const std::vector<int> &v) {
    std::fprintf(f, "%s %zu\n", name, v.size());
    for (int x : v) std::fprintf(f, "%d\n", x);
}

int main(int argc, char **argv) {
    std::map<std::string, std::string> o;
    o["eps_iter"] = "1e-8";
    o["max_iter"] = "500";
    o["vtkWithinIter"] = "false";
    o["metis"] = "false";
    o["preconditioner"] = "Dirichlet_explicit";
    o["Ac_clust_explicit"] = "true";
    o["path2data"] = "data/";
    o["young_modulus"] = "1000";
    o["ratio_mat"] = "1";
    o["poissons_ratio"] = "0.3";
    o["linear_solver"] = "pardiso";
    o["print_matrices"] = "0";
    o["typeBc"] = "ker";
    o["Ac_extended_by_kerGc"] = "true";
    o["GcTGc_assembl_block_by_block"] = "true";
    o["Bc_fullRank"] = "true";
    o["create_analytic_ker_K"] = "true";
    o["Nx"] = "2"; o["Ny"] = "2"; o["Nz"] = "2";
    o["nx"] = "5"; o["ny"] = "5"; o["nz"] = "5";
    o["nparts"] = "1";
    // harness-only keys
    std::string out = "out";
    long jitter_seed = -1;
    bool clamp = false;
    long probe_seed = 7;
    bool dumps = true;
    for (int i = 1; i < argc; ++i) {
        std::string a = argv[i];
        size_t eq = a.find('=');
        if (eq == std::string::npos) { std::fprintf(stderr, "bad arg %s\n", argv[i]); return 2; }
        std::string k = a.substr(0, eq), v = a.substr(eq + 1);
        if (k == "out") out = v;
        else if (k == "jitter_seed") jitter_seed = std::atol(v.c_str());
        else if (k == "clamp") clamp = (v == "true");
        else if (k == "probe_seed") probe_seed = std::atol(v.c_str());
        else if (k == "dumps") dumps = (v != "false");
        else o[k] = v;
    }
    mkdir(out.c_str(), 0755);
    o["path2data"] = out;

    Mesh mesh;
    mesh.createMesh(o);
    mesh.ddm_metis(o);
    int NEx = mesh.nElSubXYZ[0] * mesh.nSubXYZ[0];
    int NEy = mesh.nElSubXYZ[1] * mesh.nSubXYZ[1];
    int NEz = mesh.nElSubXYZ[2] * mesh.nSubXYZ[2];
    if (jitter_seed >= 0) {                 // interior nodes, +-0.1 h per coordinate
        int n = 0;
        for (int k = 0; k <= NEz; ++k)
            for (int j = 0; j <= NEy; ++j)
                for (int i = 0; i <= NEx; ++i, ++n) {
                    if (i == 0 || j == 0 || k == 0 || i == NEx || j == NEy || k == NEz) continue;
                    Point &p = mesh.points[n];
                    double dx = 0.1 * (1.0 / NEx) * (2.0 * u01(jitter_seed, 0, 3 * uint64_t(n) + 0) - 1.0);
                    double dy = 0.1 * (1.0 / NEy) * (2.0 * u01(jitter_seed, 0, 3 * uint64_t(n) + 1) - 1.0);
                    double dz = 0.1 * (1.0 / NEz) * (2.0 * u01(jitter_seed, 0, 3 * uint64_t(n) + 2) - 1.0);
                    p.set(p.get_x() + dx, p.get_y() + dy, p.get_z() + dz);
                }
    }
    if (clamp) {                            // u = 0 on the face x = 0 (all components)
        mesh.DirichletDOFs.clear();
        for (int i = 0; i < (int)mesh.points.size(); ++i)
            if (std::fabs(mesh.points[i].get_x()) < 1e-8)
                for (int c = 0; c < 3; ++c) mesh.DirichletDOFs.push_back(3 * i + c);
    }

    FILE *fm = std::fopen((out + "/mesh.txt").c_str(), "w");
    std::vector<double> pts;
    for (auto &p : mesh.points) { pts.push_back(p.get_x()); pts.push_back(p.get_y()); pts.push_back(p.get_z()); }
    dump_vec(fm, "points", pts);
    std::vector<int> el, part, mat;
    for (auto &e : mesh.elements) {
        for (int j = 0; j < 8; ++j) el.push_back(e.getInd(j));
        part.push_back(e.getPartitionId());
        mat.push_back(e.getMaterialId());
    }
    dump_ivec(fm, "elements", el);
    dump_ivec(fm, "partition", part);
    dump_ivec(fm, "material", mat);
    dump_ivec(fm, "dirichlet", mesh.DirichletDOFs);
    dump_ivec(fm, "corner", mesh.cornerDOFs);
    std::fclose(fm);

    Cluster cluster;
    g_clock_wall.clear();
    cluster.initialization(o, mesh);          // setup + PCPG + box.vtk
    FILE *ft = std::fopen((out + "/timing.txt").c_str(), "w");
    if (g_clock_wall.size() == 4) {           // Cluster.cpp:24, 1364, 1451, 374
        const std::vector<double> &c = g_clock_wall;
        std::fprintf(ft, "setup_s %.6f\npcpg_s %.6f\ntotal_s %.6f\n", c[1] - c[0], c[2] - c[1], c[3] - c[0]);
    } else {
        std::fprintf(ft, "clock_calls %zu\n", g_clock_wall.size());
    }
    std::fclose(ft);
    if (!dumps) return 0;

    FILE *fl = std::fopen((out + "/layout.txt").c_str(), "w");
    int ns = cluster.get_nSubClst();
    std::fprintf(fl, "nsub %d\nnlam %d\nnlam_c %d\n", ns, cluster.get_nLam_f(), cluster.get_nLam_c());
    for (int d = 0; d < ns; ++d) {
        dump_ivec(fl, "l2g", cluster.data.l2g[d]);
        dump_ivec(fl, "bf_rows", cluster.Bf[d].l2g_i_coo);
        dump_ivec(fl, "bf_iptr", cluster.Bf[d].i_ptr);
        dump_ivec(fl, "bf_jcol", cluster.Bf[d].j_col);
        dump_vec(fl, "bf_val", cluster.Bf[d].val);
    }
    dump_vec(fl, "weight", cluster.weigth);
    std::fclose(fl);

    // projected operators on a seeded probe vector
    int nl = cluster.get_nLam_f();
    Vector w; w.zero_dense(nl);
    for (int i = 0; i < nl; ++i) w.dense[i] = 2.0 * u01(probe_seed, 1, i) - 1.0;
    Vector Pw, a1, FPw, PFPw, a2, MPw, PMPw, a3;
    cluster.Projection(w, Pw, a1);
    cluster.mult_Ff(Pw, FPw);
    cluster.Projection(FPw, PFPw, a2);
    cluster.Preconditioning(Pw, MPw);
    cluster.Projection(MPw, PMPw, a3);
    FILE *fp = std::fopen((out + "/probe.txt").c_str(), "w");
    dump_vec(fp, "w", w.dense);
    dump_vec(fp, "Pw", Pw.dense);
    dump_vec(fp, "PFPw", PFPw.dense);
    dump_vec(fp, "PMPw", PMPw.dense);
    std::fclose(fp);

    // element matrices: an axis-aligned box and a distorted hexahedron
    FILE *fe = std::fopen((out + "/elem.txt").c_str(), "w");
    const double box[8][3] = {{0,0,0},{1,0,0},{1,1,0},{0,1,0},{0,0,1},{1,0,1},{1,1,1},{0,1,1}};
    for (int variant = 0; variant < 2; ++variant) {
        std::vector<Point> X(8, Point(0, 0, 0));
        std::vector<double> xs;
        for (int j = 0; j < 8; ++j) {
            double s[3];
            for (int c = 0; c < 3; ++c) {
                s[c] = 0.25 * box[j][c];
                if (variant == 1) s[c] += 0.025 * (2.0 * u01(99, 2, 3 * j + c) - 1.0);
            }
            X[j].set(s[0], s[1], s[2]);
            xs.push_back(s[0]); xs.push_back(s[1]); xs.push_back(s[2]);
        }
        local_K_f lk;
        cluster.data.stf_mtrx_solid45(lk, X, 2.1e5, 0.3);
        std::vector<double> K, f;
        for (int j = 0; j < 24; ++j)
            for (int i = 0; i < 24; ++i) K.push_back(lk.get_val_K(i, j));
        for (int i = 0; i < 24; ++i) f.push_back(lk.get_val_f(i));
        dump_vec(fe, "coords", xs);
        dump_vec(fe, "Ke_colmajor", K);
        dump_vec(fe, "fe", f);
    }
    std::fclose(fe);
    return 0;
}
