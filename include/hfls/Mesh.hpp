// Mesh of the reference's surface (ostravaTokyo/hfls src/Mesh.hpp:22-87):
// the same public fields (points, elements, DirichletDOFs, cornerDOFs, the
// per-axis counts) and createMesh / ddm_metis / SaveVTK, built by this
// library's mesh generator (htf_mesh_fill: the reference's structured cube,
// rollers on the faces x = 0, y = 0, z = 0, the checkerboard material of
// young_modulus / ratio_mat) and written by htf_write_vtk.
#ifndef HFLS_MESH_HPP
#define HFLS_MESH_HPP

#include <map>
#include <string>
#include <vector>

using namespace std;

class Element {
public:
    Element() {}
    void setInd(int j, int v) { ind[j] = v; }
    int getInd(int j) { return ind[j]; }
    void setPartitionId(int p) { PartitionId = p; }
    void setMaterialId(int m) { MaterialId = m; }
    int getPartitionId() { return PartitionId; }
    int getMaterialId() { return MaterialId; }

private:
    int ind[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    int PartitionId = 0;
    int MaterialId = 0;
};

class Point {
public:
    Point(double x_, double y_, double z_) : x(x_), y(y_), z(z_) {}
    void set(double a, double b, double c) { x = a; y = b; z = c; }
    void set_x(double a) { x = a; }
    void set_y(double a) { y = a; }
    void set_z(double a) { z = a; }
    double get_x() { return x; }
    double get_y() { return y; }
    double get_z() { return z; }

private:
    double x, y, z;
};

class Material {
public:
    double young_modulus = 0.0;
    double poissons_ratio = 0.0;
};

class Mesh {
public:
    Mesh() {}
    ~Mesh() {}
    int nElementsClst = 0;
    int nSubClst = 0;
    vector<int> nElementsSub;
    int nPoints = 0;
    int nSub = 0;
    vector<Element> elements;
    vector<Point> points;
    vector<int> cornerNodes;
    vector<int> cornerDOFs;
    vector<int> DirichletDOFs;
    Material material;
    int nElSubXYZ[3] = {0, 0, 0};
    int nSubXYZ[3] = {0, 0, 0};
    // options Nx, Ny, Nz (subdomains), nx, ny, nz (elements per subdomain),
    // young_modulus, ratio_mat, poissons_ratio (Mesh.cpp:69-289)
    void createMesh(map<string, string> &options);
    // the structured decomposition of createMesh is kept (metis=false); METIS
    // repartitioning (metis=true) is not part of this library and throws
    void ddm_metis(map<string, string> &options);
    // box.vtk (or box<it>.vtk for it >= 0) of the displacements in folder
    void SaveVTK(vector<double> u, string folder, int it);
};

#endif
