// Driver of the reference's surface (ostravaTokyo/hfls src/Driver.hpp:11-24,
// Driver.cpp:14-38): Driver(options); initialization() builds the mesh,
// keeps its structured decomposition and runs the cluster (setup, PCPG and
// box.vtk) on the GPU.  A main written against the reference's headers, like
// its htfeti.cpp, compiles against these and links libhtfeti_b200.so.
#ifndef HFLS_DRIVER_HPP
#define HFLS_DRIVER_HPP

#include <map>
#include <string>

#include "Cluster.hpp"
#include "Mesh.hpp"
#include "Solver.hpp"

class Driver {
public:
    Driver() {}
    Driver(map<string, string> options) : options2(options) {}
    void initialization();
    // this library's addition: the cluster after initialization
    Cluster &get_cluster() { return cluster; }

private:
    Mesh mesh;
    Cluster cluster;
    map<string, string> options2;
    string folder;
    Solver solver;
};

#endif
