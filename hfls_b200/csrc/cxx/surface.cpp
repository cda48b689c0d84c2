// The reference's C++ class surface (Driver, Cluster, Solver, Mesh, Vector;
// ostravaTokyo/hfls src/*.hpp) over this library's C ABI, so that a main
// written against the reference's headers (its htfeti.cpp: an options map,
// Driver driver(options); driver.initialization();) compiles against
// include/hfls/ and runs the solve on the GPU.  Headers: include/hfls/*.hpp.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "htfeti.h"
#include "hfls/Driver.hpp"

namespace {

double opt_num(map<string, string> &o, const char *key, double dflt) {
    auto it = o.find(key);
    return it == o.end() || it->second.empty() ? dflt : std::atof(it->second.c_str());
}

int opt_int(map<string, string> &o, const char *key, int dflt) {
    auto it = o.find(key);
    return it == o.end() || it->second.empty() ? dflt : std::atoi(it->second.c_str());
}

// rho * a of the reference's element load (Data.cpp:315-318)
const double kBodyForce[3] = {0.0, 0.0, 2.0 * 98.1};

}  // namespace

// ---- Mesh (Mesh.cpp:69-289 createMesh, 292-351 SaveVTK, 352-... ddm_metis) -
void Mesh::createMesh(map<string, string> &o) {
    htf_mesh_spec s;
    std::memset(&s, 0, sizeof(s));
    s.clusters[0] = s.clusters[1] = s.clusters[2] = 1;
    s.subs[0] = opt_int(o, "Nx", 2);
    s.subs[1] = opt_int(o, "Ny", 2);
    s.subs[2] = opt_int(o, "Nz", 2);
    s.elems[0] = opt_int(o, "nx", 5);
    s.elems[1] = opt_int(o, "ny", 5);
    s.elems[2] = opt_int(o, "nz", 5);
    s.bc = HTF_BC_ROLLERS;
    s.material = HTF_MAT_CHECKER;
    s.E = opt_num(o, "young_modulus", 1000.0);
    s.E_hi = opt_num(o, "ratio_mat", 1.0);
    s.nu = opt_num(o, "poissons_ratio", 0.3);
    for (int a = 0; a < 3; ++a) s.body_force[a] = kBodyForce[a];
    int nn = 0, ne = 0, ns = 0, nc = 0, nd = 0, ncr = 0;
    int rc = htf_mesh_sizes(&s, &nn, &ne, &ns, &nc, &nd, &ncr);
    if (rc) throw hfls::Error(rc, "Mesh::createMesh: bad subdomain / element counts");
    std::vector<double> xyz(3 * (size_t)nn);
    std::vector<int> el(8 * (size_t)ne), part(ne), dir(nd), cor(ncr);
    rc = htf_mesh_fill(&s, xyz.data(), el.data(), part.data(), nullptr, nullptr, nullptr, dir.data(), cor.data());
    if (rc) throw hfls::Error(rc, "Mesh::createMesh: htf_mesh_fill failed");
    points.clear();
    points.reserve(nn);
    for (int i = 0; i < nn; ++i) points.emplace_back(xyz[3 * i], xyz[3 * i + 1], xyz[3 * i + 2]);
    elements.assign(ne, Element());
    nElementsSub.assign(ns, 0);
    for (int e = 0; e < ne; ++e) {
        for (int j = 0; j < 8; ++j) elements[e].setInd(j, el[8 * (size_t)e + j]);
        elements[e].setPartitionId(part[e]);
        elements[e].setMaterialId(int(std::remainder(double(part[e]), 2.0)));   // Mesh.cpp:280-281
        ++nElementsSub[part[e]];
    }
    DirichletDOFs = dir;
    cornerDOFs = cor;
    cornerNodes.clear();
    for (size_t i = 0; i < cor.size(); i += 3) cornerNodes.push_back(cor[i] / 3);
    nPoints = nn;
    nElementsClst = ne;
    nSubClst = nSub = ns;
    for (int a = 0; a < 3; ++a) {
        nSubXYZ[a] = s.subs[a];
        nElSubXYZ[a] = s.elems[a];
    }
    material.young_modulus = s.E;
    material.poissons_ratio = s.nu;
}

void Mesh::ddm_metis(map<string, string> &o) {
    auto it = o.find("metis");
    if (it != o.end() && it->second == "false") return;
    throw hfls::Error(HTF_EINVAL, "Mesh::ddm_metis: METIS repartitioning is not part of this library; "
                                  "set metis=false to keep the structured decomposition");
}

void Mesh::SaveVTK(vector<double> u, string folder, int it) {
    char path[1024];
    if (it == -1) std::snprintf(path, sizeof(path), "%s/box.vtk", folder.c_str());
    else std::snprintf(path, sizeof(path), "%s/box%d.vtk", folder.c_str(), it);
    std::vector<double> xyz;
    xyz.reserve(3 * points.size());
    for (auto &p : points) { xyz.push_back(p.get_x()); xyz.push_back(p.get_y()); xyz.push_back(p.get_z()); }
    std::vector<int> el, part, mat;
    for (auto &e : elements) {
        for (int j = 0; j < 8; ++j) el.push_back(e.getInd(j));
        part.push_back(e.getPartitionId());
        mat.push_back(e.getMaterialId());
    }
    const int rc = htf_write_vtk(path, int(points.size()), xyz.data(), int(elements.size()), el.data(), part.data(),
                                 mat.data(), u.data());
    if (rc) throw hfls::Error(rc, std::string("Mesh::SaveVTK: cannot write ") + path);
}

// ---- Cluster --------------------------------------------------------------
Cluster::~Cluster() {
    if (ctx) htf_destroy(ctx);
}

void Cluster::check(int rc, const char *what) {
    if (rc) throw hfls::Error(rc, std::string(what) + ": " + (ctx ? htf_last_error(ctx) : "no context"));
}

void Cluster::initialization(map<string, string> options, Mesh &m) {
    const auto t0 = std::chrono::steady_clock::now();
    options2 = options;
    mesh = &m;
    folder = options2.count("path2data") ? options2["path2data"] : string("data/");
    if (ctx) {
        htf_destroy(ctx);
        ctx = nullptr;
    }
    string opts;
    for (auto &kv : options2) opts += kv.first + "=" + kv.second + ";";
    int rc = htf_create(opts.c_str(), &ctx);
    if (rc) {
        ctx = nullptr;
        throw hfls::Error(rc, "Cluster::initialization: bad options (" + opts + ")");
    }
    // Data::fe_assemb_local_K_f reads the material from the options (Data.cpp:34, 47-48)
    const double E = opt_num(options2, "young_modulus", 1000.0), ratio = opt_num(options2, "ratio_mat", 1.0);
    const double nu = opt_num(options2, "poissons_ratio", 0.3);
    const int nn = int(m.points.size()), ne = int(m.elements.size());
    std::vector<double> xyz;
    xyz.reserve(3 * (size_t)nn);
    for (auto &p : m.points) { xyz.push_back(p.get_x()); xyz.push_back(p.get_y()); xyz.push_back(p.get_z()); }
    std::vector<int> el(8 * (size_t)ne), part(ne);
    int ns = 0;
    for (int e = 0; e < ne; ++e) {
        for (int j = 0; j < 8; ++j) el[8 * (size_t)e + j] = m.elements[e].getInd(j);
        part[e] = m.elements[e].getPartitionId();
        ns = std::max(ns, part[e] + 1);
    }
    std::vector<double> sE(ns, E), snu(ns, nu);
    for (int e = 0; e < ne; ++e)
        if (m.elements[e].getMaterialId() == 0) sE[part[e]] = E * ratio;
    std::vector<int> scl(ns, 0);                      // one cluster (Driver.cpp:29)
    check(htf_set_mesh(ctx, nn, xyz.data(), ne, el.data(), part.data(), ns, scl.data(), sE.data(), snu.data(),
                       int(m.DirichletDOFs.size()), m.DirichletDOFs.data(), int(m.cornerDOFs.size()),
                       m.cornerDOFs.data(), kBodyForce),
          "htf_set_mesh");
    check(htf_setup(ctx), "htf_setup");
    const int print_mat = opt_int(options2, "print_matrices", 0);
    if (print_mat >= 2) check(htf_dump(ctx, folder.c_str(), print_mat), "htf_dump");   // Cluster.cpp:118-358
    int nl = 0, nsub = 0, ncl = 0;
    check(htf_dual_sizes(ctx, &nl, &nsub, &ncl), "htf_dual_sizes");
    nLam_f = nl;
    nSubClst = nsub;
    pcpg();
    time_total = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    std::printf("Solver time:  %3.1f s.\n", time_solver);
    std::printf("Total time:   %3.1f s.\n", time_total);
}

void Cluster::pcpg() {
    if (!ctx || !mesh) throw hfls::Error(HTF_ESTATE, "Cluster::pcpg before Cluster::initialization");
    u.assign(3 * mesh->points.size(), 0.0);
    htf_stats st;
    const auto t0 = std::chrono::steady_clock::now();
    check(htf_pcpg(ctx, u.data(), &st), "htf_pcpg");
    time_solver = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    its = st.iterations[0];
    mesh->SaveVTK(u, folder, -1);                     // Cluster::printVTK(..., -1), Cluster.cpp:1456
}

void Cluster::mult_Ff(Vector const &x, Vector &Fx) {
    if (!ctx) throw hfls::Error(HTF_ESTATE, "Cluster::mult_Ff before Cluster::initialization");
    if (x.get_numel() != nLam_f) throw hfls::Error(HTF_EINVAL, "Cluster::mult_Ff: vector of the wrong length");
    if (Fx.get_numel() == 0) Fx.zero_dense(nLam_f);
    check(htf_mult_Ff(ctx, x.dense.data(), Fx.dense.data(), 1), "htf_mult_Ff");
}

void Cluster::Projection(Vector &x, Vector &Px, Vector &alpha) {
    (void)alpha;
    if (!ctx) throw hfls::Error(HTF_ESTATE, "Cluster::Projection before Cluster::initialization");
    if (x.get_numel() != nLam_f) throw hfls::Error(HTF_EINVAL, "Cluster::Projection: vector of the wrong length");
    if (Px.get_numel() == 0) Px.zero_dense(nLam_f);
    check(htf_projection(ctx, x.dense.data(), Px.dense.data(), 1), "htf_projection");
}

void Cluster::Preconditioning(Vector &x, Vector &Mx) {
    if (!ctx) throw hfls::Error(HTF_ESTATE, "Cluster::Preconditioning before Cluster::initialization");
    if (x.get_numel() != nLam_f) throw hfls::Error(HTF_EINVAL, "Cluster::Preconditioning: vector of the wrong length");
    if (Mx.get_numel() == 0) Mx.zero_dense(nLam_f);
    check(htf_preconditioning(ctx, x.dense.data(), Mx.dense.data(), 1), "htf_preconditioning");
}

// ---- Solver, Driver ---------------------------------------------------------
void Solver::pcpg(map<string, string> options, Cluster &cluster) {
    (void)options;
    const auto t0 = std::chrono::steady_clock::now();
    cluster.pcpg();
    time_solver = cluster.solver_time();
    time_total = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
}

void Driver::initialization() {
    folder = options2.count("path2data") ? options2["path2data"] : string("data/");
    mesh.createMesh(options2);
    mesh.ddm_metis(options2);
    cluster.initialization(options2, mesh);
}
