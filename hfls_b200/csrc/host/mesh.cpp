// Structured hexahedral cube mesh, generalised from Mesh::createMesh
// (Mesh.cpp:69-289): clusters x subdomains x elements per axis, optional
// non-uniform subdomain slabs, seeded jitter of interior nodes, materials,
// boundary conditions and surface tractions of the benchmark configurations.
#include <cmath>
#include <cstring>
#include <sstream>

#include "problem.hpp"

namespace htf {

uint64_t mix64(uint64_t z) {
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    return z ^ (z >> 31);
}

double u01(uint64_t seed, uint64_t stream, uint64_t i) {
    uint64_t z = mix64(seed * 0x9E3779B97F4A7C15ULL + stream * 0xD1B54A32D192ED03ULL + i +
                       0x632BE59BD9B4E019ULL);
    return double(z >> 11) * (1.0 / 9007199254740992.0);
}

namespace {
struct Axes {
    int NS[3];                    // subdomain slabs per axis (all clusters)
    int NE[3];                    // elements per axis
    std::vector<int> slab_of[3];  // element index -> slab
    std::vector<int> bound[3];    // slab boundaries (node indices), NS+1 entries
};

int make_axes(const htf_mesh_spec &s, Axes &ax, std::string &err) {
    for (int a = 0; a < 3; ++a) {
        if (s.clusters[a] < 1 || s.subs[a] < 1) { err = "clusters and subs must be >= 1"; return HTF_EINVAL; }
        ax.NS[a] = s.clusters[a] * s.subs[a];
        ax.bound[a].assign(1, 0);
        for (int k = 0; k < ax.NS[a]; ++k) {
            int w = s.widths[a] ? s.widths[a][k] : s.elems[a];
            if (w < 1) { err = "element counts must be >= 1"; return HTF_EINVAL; }
            ax.bound[a].push_back(ax.bound[a].back() + w);
        }
        ax.NE[a] = ax.bound[a].back();
        ax.slab_of[a].resize(ax.NE[a]);
        for (int k = 0; k < ax.NS[a]; ++k)
            for (int e = ax.bound[a][k]; e < ax.bound[a][k + 1]; ++e) ax.slab_of[a][e] = k;
    }
    long long nn = (long long)(ax.NE[0] + 1) * (ax.NE[1] + 1) * (ax.NE[2] + 1);
    if (nn * 3 > 0x7fffffffLL) { err = "mesh too large for 32-bit DOF ids"; return HTF_EINVAL; }
    return HTF_OK;
}
}  // namespace

int mesh_sizes(const htf_mesh_spec &s, int *nn, int *ne, int *ns, int *nc, int *nd, int *ncr,
               std::string &err) {
    Axes ax;
    int rc = make_axes(s, ax, err);
    if (rc) return rc;
    int NX = ax.NE[0] + 1, NY = ax.NE[1] + 1, NZ = ax.NE[2] + 1;
    if (nn) *nn = NX * NY * NZ;
    if (ne) *ne = ax.NE[0] * ax.NE[1] * ax.NE[2];
    if (ns) *ns = ax.NS[0] * ax.NS[1] * ax.NS[2];
    if (nc) *nc = s.clusters[0] * s.clusters[1] * s.clusters[2];
    if (nd) {
        int face = NY * NZ;          // nodes with x = 0
        if (s.bc == HTF_BC_CLAMP_X0) *nd = 3 * face;
        else *nd = NY * NZ + NX * NZ + NX * NY;
    }
    if (ncr) *ncr = 3 * ((ax.NS[0] + 1) * (ax.NS[1] + 1) * (ax.NS[2] + 1) - 8);
    return HTF_OK;
}

int generate_mesh(const htf_mesh_spec &s, Mesh &m, std::string &err) {
    Axes ax;
    int rc = make_axes(s, ax, err);
    if (rc) return rc;
    const int NEx = ax.NE[0], NEy = ax.NE[1], NEz = ax.NE[2];
    const int NX = NEx + 1, NY = NEy + 1, NZ = NEz + 1;
    m.n_nodes = NX * NY * NZ;
    m.coords.assign(3 * size_t(m.n_nodes), 0.0);
    const double dx = 1.0 / NEx, dy = 1.0 / NEy, dz = 1.0 / NEz;
    // Mesh.cpp:152-171 (radius warp off): x = (i dx - 0.5) + 0.5, z = k dz + 0
    for (int k = 0, n = 0; k < NZ; ++k)
        for (int j = 0; j < NY; ++j)
            for (int i = 0; i < NX; ++i, ++n) {
                double x = (i * dx - 0.5) + 0.5;
                double y = (j * dy - 0.5) + 0.5;
                double z = k * dz + 0.0;
                bool interior = i > 0 && j > 0 && k > 0 && i < NEx && j < NEy && k < NEz;
                if (interior && s.jitter != 0.0) {
                    x += s.jitter * dx * (2.0 * u01(s.seed, 0, 3 * uint64_t(n) + 0) - 1.0);
                    y += s.jitter * dy * (2.0 * u01(s.seed, 0, 3 * uint64_t(n) + 1) - 1.0);
                    z += s.jitter * dz * (2.0 * u01(s.seed, 0, 3 * uint64_t(n) + 2) - 1.0);
                }
                m.coords[3 * size_t(n) + 0] = x;
                m.coords[3 * size_t(n) + 1] = y;
                m.coords[3 * size_t(n) + 2] = z;
            }
    // elements (Mesh.cpp:243-264) and partition (Mesh.cpp:271-288), cluster-major
    const int CX = s.clusters[0], CY = s.clusters[1], CZ = s.clusters[2];
    const int SX = s.subs[0], SY = s.subs[1], SZ = s.subs[2];
    const int per_cluster = SX * SY * SZ;
    const int ne = NEx * NEy * NEz;
    m.elems.resize(8 * size_t(ne));
    m.elem_sub.resize(ne);
    const int nxy = NX * NY;
    for (int k = 0, e = 0; k < NEz; ++k)
        for (int j = 0; j < NEy; ++j)
            for (int i = 0; i < NEx; ++i, ++e) {
                int f0 = i + j * NX, f1 = i + 1 + j * NX, f2 = i + 1 + (j + 1) * NX, f3 = i + (j + 1) * NX;
                int *q = &m.elems[8 * size_t(e)];
                q[0] = f0 + k * nxy; q[1] = f1 + k * nxy; q[2] = f2 + k * nxy; q[3] = f3 + k * nxy;
                q[4] = f0 + (k + 1) * nxy; q[5] = f1 + (k + 1) * nxy; q[6] = f2 + (k + 1) * nxy; q[7] = f3 + (k + 1) * nxy;
                int gx = ax.slab_of[0][i], gy = ax.slab_of[1][j], gz = ax.slab_of[2][k];
                int cx = gx / SX, cy = gy / SY, cz = gz / SZ;
                int c = cx + CX * (cy + CY * cz);
                int l = (gx % SX) + SX * ((gy % SY) + SY * (gz % SZ));
                m.elem_sub[e] = c * per_cluster + l;
            }
    const int nsub = CX * CY * CZ * per_cluster;
    m.sub_cluster.resize(nsub);
    m.sub_E.resize(nsub);
    m.sub_nu.assign(nsub, s.nu);
    for (int d = 0; d < nsub; ++d) {
        m.sub_cluster[d] = d / per_cluster;
        double E = s.E;
        if (s.material == HTF_MAT_CHECKER) {
            // material id = remainder(partition, 2); id 0 gets E * ratio
            if (std::remainder(double(d), 2.0) == 0.0) E = s.E * s.E_hi;
        } else if (s.material == HTF_MAT_LOGUNIFORM) {
            double lo = std::log(s.E), hi = std::log(s.E_hi);
            E = std::exp(lo + u01(s.seed, 1, uint64_t(d)) * (hi - lo));
        }
        m.sub_E[d] = E;
    }
    // Dirichlet DOFs (Mesh.cpp:221-239)
    m.dirichlet.clear();
    const double eps0 = 1e-8;
    for (int n = 0; n < m.n_nodes; ++n) {
        double x = m.coords[3 * size_t(n)], y = m.coords[3 * size_t(n) + 1], z = m.coords[3 * size_t(n) + 2];
        if (s.bc == HTF_BC_CLAMP_X0) {
            if (std::fabs(x) < eps0)
                for (int c = 0; c < 3; ++c) m.dirichlet.push_back(3 * n + c);
        } else {
            if (std::fabs(x) < eps0) m.dirichlet.push_back(3 * n + 0);
            if (std::fabs(y) < eps0) m.dirichlet.push_back(3 * n + 1);
            if (std::fabs(z) < eps0) m.dirichlet.push_back(3 * n + 2);
        }
    }
    // corner DOFs: subdomain-grid vertices except the 8 cube corners (Mesh.cpp:175-208)
    m.corner.clear();
    for (int kk : ax.bound[2])
        for (int jj : ax.bound[1])
            for (int ii : ax.bound[0]) {
                bool cube_corner = (ii == 0 || ii == NEx) && (jj == 0 || jj == NEy) && (kk == 0 || kk == NEz);
                if (cube_corner) continue;
                int n = ii + NX * (jj + NY * kk);
                for (int c = 0; c < 3; ++c) m.corner.push_back(3 * n + c);
            }
    for (int a = 0; a < 3; ++a) m.body_force[a] = s.body_force[a];
    return HTF_OK;
}

int mesh_traction(const htf_mesh_spec &s, uint64_t seed, int n_rhs, double scale, double *f,
                  std::string &err) {
    Axes ax;
    int rc = make_axes(s, ax, err);
    if (rc) return rc;
    const int NX = ax.NE[0] + 1, NY = ax.NE[1] + 1, NZ = ax.NE[2] + 1;
    const size_t ndof = 3 * size_t(NX) * NY * NZ;
    const double two_pi = 6.283185307179586;
    for (int r = 0; r < n_rhs; ++r)
        for (int k = 0; k < NZ; ++k)
            for (int j = 0; j < NY; ++j) {
                int n = (NX - 1) + NX * (j + NY * k);     // node on x = 1
                for (int c = 0; c < 3; ++c) {
                    uint64_t idx = 2 * (3 * uint64_t(n) + c);
                    double u1 = u01(seed, 16 + uint64_t(r), idx), u2 = u01(seed, 16 + uint64_t(r), idx + 1);
                    double g = std::sqrt(-2.0 * std::log(1.0 - u1)) * std::cos(two_pi * u2);  // Box-Muller
                    f[size_t(r) * ndof + 3 * size_t(n) + c] += scale * g;
                }
            }
    return HTF_OK;
}

int parse_options(const char *s, Options &o, std::string &err) {
    if (!s) return HTF_OK;
    std::stringstream ss(s);
    std::string item;
    while (std::getline(ss, item, ';')) {
        if (item.empty()) continue;
        size_t eq = item.find('=');
        if (eq == std::string::npos) { err = "option without '=': " + item; return HTF_EINVAL; }
        std::string k = item.substr(0, eq), v = item.substr(eq + 1);
        if (k == "typeBc") {
            if (v == "all") v = "cor";     // Cluster.cpp:744-747: "all" behaves like "cor"
            if (v != "cor" && v != "ker") { err = "typeBc must be cor|ker|all"; return HTF_EINVAL; }
            o.typeBc = v;
        } else if (k == "preconditioner") {
            if (v != "Dirichlet_explicit" && v != "Dirichlet_implicit" && v != "lumped") {
                err = "preconditioner must be Dirichlet_explicit|Dirichlet_implicit|lumped";
                return HTF_EINVAL;
            }
            o.preconditioner = v;
        } else if (k == "eps_iter") o.eps_iter = std::atof(v.c_str());
        else if (k == "mixed_eps_factor") {
            o.mixed_eps_factor = std::atof(v.c_str());
            if (!(o.mixed_eps_factor > 0.0 && o.mixed_eps_factor <= 1.0)) {
                err = "mixed_eps_factor must be in (0, 1]";
                return HTF_EINVAL;
            }
        }
        else if (k == "max_iter") o.max_iter = std::atoi(v.c_str());
        else if (k == "print_matrices") o.print_matrices = std::atoi(v.c_str());
        else if (k == "precision") {
            if (v != "fp64" && v != "mixed") { err = "precision must be fp64|mixed"; return HTF_EINVAL; }
            o.mixed = (v == "mixed");
        } else if (k == "device") o.device = std::atoi(v.c_str());
        else if (k == "check_every") o.check_every = std::max(1, std::atoi(v.c_str()));
        else if (k == "verbose") o.verbose = std::atoi(v.c_str());
        else if (k == "autotune") o.autotune = std::atoi(v.c_str());
        else if (k == "tune_file") o.tune_file = v;
        else if (k == "S_fp64") {
            if (v != "0" && v != "1") { err = "S_fp64 must be 0 or 1"; return HTF_EINVAL; }
            o.S_fp64 = (v == "1");
        } else if (k == "admit_oversize") {
            if (v != "0" && v != "1") { err = "admit_oversize must be 0 or 1"; return HTF_EINVAL; }
            o.admit_oversize = (v == "1");
        } else if (k == "factor_wave_gb") {
            o.factor_wave_gb = std::atof(v.c_str());
            if (!(o.factor_wave_gb >= 0.0)) { err = "factor_wave_gb must be >= 0"; return HTF_EINVAL; }
        }
        else if (k == "batch") {
            o.batch = std::atoi(v.c_str());
            if (o.batch != 16 && o.batch != 32) { err = "batch must be 16 or 32"; return HTF_EINVAL; }
        }
        // reference keys without effect on this path (kept for drop-in option maps)
        else if (k == "vtkWithinIter" || k == "metis" || k == "Ac_clust_explicit" || k == "path2data" ||
                 k == "young_modulus" || k == "ratio_mat" || k == "poissons_ratio" || k == "linear_solver" ||
                 k == "Ac_extended_by_kerGc" || k == "GcTGc_assembl_block_by_block" ||
                 k == "Bc_fullRank" || k == "create_analytic_ker_K" || k == "Nx" || k == "Ny" || k == "Nz" ||
                 k == "nx" || k == "ny" || k == "nz" || k == "nparts") {
        } else {
            err = "unknown option: " + k;
            return HTF_EINVAL;
        }
    }
    return HTF_OK;
}

}  // namespace htf
