// A main in the shape of the reference's htfeti.cpp (options map, Driver,
// initialization), compiled against this library's include/hfls/ headers in
// place of the reference's src/*.hpp.  Options come as key=value arguments
// on top of the reference's defaults for a solve.
#include <cstdio>
#include <iostream>
#include <map>
#include <string>

#include "Cluster.hpp"
#include "Driver.hpp"

using namespace std;

int main(int argc, char *argv[]) {
    map<string, string> options2;
    options2["eps_iter"] = "1e-8";
    options2["max_iter"] = "500";
    options2["vtkWithinIter"] = "false";
    options2["metis"] = "false";
    options2["preconditioner"] = "Dirichlet_explicit";
    options2["path2data"] = "data/";
    options2["young_modulus"] = "1000";
    options2["ratio_mat"] = "1";
    options2["poissons_ratio"] = "0.3";
    options2["typeBc"] = "ker";
    options2["Nx"] = "2";
    options2["Ny"] = "2";
    options2["Nz"] = "2";
    options2["nx"] = "5";
    options2["ny"] = "5";
    options2["nz"] = "5";
    for (int i = 1; i < argc; ++i) {
        string a = argv[i];
        size_t eq = a.find('=');
        if (eq != string::npos) options2[a.substr(0, eq)] = a.substr(eq + 1);
    }
    try {
        Driver driver(options2);
        driver.initialization();
        Cluster &c = driver.get_cluster();
        // the dual operators of the reference's surface on a probe vector
        Vector w, Pw, a, FPw, MPw;
        w.zero_dense(c.get_nLam_f());
        for (int i = 0; i < w.get_numel(); ++i) w.dense[i] = 1.0 / (1.0 + i);
        c.Projection(w, Pw, a);
        c.mult_Ff(Pw, FPw);
        c.Preconditioning(Pw, MPw);
        printf("iterations %d lambda %d subdomains %d |FPw| %.6e |MPw| %.6e\n", c.iterations(), c.get_nLam_f(),
               c.get_nSubClst(), Vector::dot(FPw, FPw), Vector::dot(MPw, MPw));
    } catch (const hfls::Error &e) {
        fprintf(stderr, "hfls error %d: %s\n", e.code, e.what());
        return 3;
    }
    cout << "----------------- done -----------------\n";
    return 0;
}
