// Solver of the reference's surface (ostravaTokyo/hfls src/Solver.hpp:12-20):
// pcpg(options, cluster) solves the cluster's problem again (the reference's
// Solver::pcpg duplicates Cluster::pcpg, Solver.cpp:11-105).
#ifndef HFLS_SOLVER_HPP
#define HFLS_SOLVER_HPP

#include <map>
#include <string>

#include "Cluster.hpp"

class Solver {
public:
    Solver() {}
    void pcpg(map<string, string> options, Cluster &cluster);

private:
    double time_solver = 0.0;
    double time_total = 0.0;
};

#endif
