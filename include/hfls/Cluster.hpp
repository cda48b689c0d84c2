// Cluster of the reference's surface (ostravaTokyo/hfls src/Cluster.hpp:15-138)
// over this library's C ABI (include/htfeti.h): initialization runs the setup
// on the GPU, the PCPG solve and the displacement output, as the
// reference's does (Cluster.cpp:21-385); pcpg, mult_Ff, Projection and
// Preconditioning are the GPU operators on host vectors.  Where the reference
// exits the process (PARDISO errors, Matrix.cpp:1174-1178) these throw
// hfls::Error with the library's code and message.  The per-subdomain Matrix
// members of the reference (K, R, Bf, ...) live on the device and are not
// exposed; print_matrices >= 2 writes them as the reference's dump files.
#ifndef HFLS_CLUSTER_HPP
#define HFLS_CLUSTER_HPP

#include <map>
#include <stdexcept>
#include <string>
#include <vector>

#include "Matrix.hpp"
#include "Mesh.hpp"

struct htf_ctx;

namespace hfls {
class Error : public std::runtime_error {
public:
    Error(int code, const std::string &msg) : std::runtime_error(msg), code(code) {}
    int code;
};
}  // namespace hfls

class Cluster {
public:
    Cluster() {}
    ~Cluster();
    Cluster(const Cluster &) = delete;
    Cluster &operator=(const Cluster &) = delete;
    // setup (Cluster.cpp:21-360), pcpg, box.vtk of u in options["path2data"]
    void initialization(map<string, string> options, Mesh &mesh);
    // PCPG of the load vector with the resident factors (Cluster.cpp:1363-1458)
    // and the displacement field (Cluster.cpp:1648-1678)
    void pcpg();
    void mult_Ff(Vector const &x, Vector &Fx);                 // Cluster.cpp:1114-1188
    void Projection(Vector &x, Vector &Px, Vector &alpha);    // Cluster.cpp:1314-1329 (alpha left empty)
    void Preconditioning(Vector &x, Vector &Mx);              // Cluster.cpp:1043-1112
    int get_nSubClst() { return nSubClst; }
    int get_nLam_f() { return nLam_f; }
    // this library's additions: results of the last pcpg
    const vector<double> &displacements() const { return u; }
    int iterations() const { return its; }
    double solver_time() const { return time_solver; }
    string folder;
    Mesh *mesh = nullptr;

private:
    void check(int rc, const char *what);
    htf_ctx *ctx = nullptr;
    map<string, string> options2;
    vector<double> u;
    int nSubClst = 0, nLam_f = 0, its = 0;
    double time_solver = 0.0, time_total = 0.0;
};

#endif
