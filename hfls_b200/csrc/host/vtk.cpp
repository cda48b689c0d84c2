// Legacy ASCII VTK output of a displacement field on hex8 elements.
//
// The file is the one Mesh::SaveVTK (Mesh.cpp:292-351) writes as box.vtk at
// the end of the reference's solve (Cluster::printVTK, Cluster.cpp:1648-1678),
// so post-processing written for the reference reads this one unchanged.
// Its layout and number formats are that file's interface and are kept
// exactly: "%f" for coordinates and displacements, one cell line per element
// ("8" and the eight node ids, each printed with "% d"), cell type 12
// (VTK_HEXAHEDRON), the point field "displacements" (3 components) and the
// cell fields "decomposition" (subdomain) and "materialId".
#include <cmath>
#include <cstdio>
#include <vector>

#include "host/problem.hpp"
#include "htfeti.h"

namespace htf {

// Material id of an element of subdomain p when the caller gives none:
// remainder(p, 2) as Mesh.cpp:280-281 computes it (round-to-nearest-even
// quotient), i.e. 0 for even p and +1 / -1 alternately for odd p.
static int reference_material(int p) { return static_cast<int>(std::remainder(static_cast<double>(p), 2.0)); }

int write_vtk(const char *path, int n_nodes, const double *coords, int n_elems, const int *elems,
              const int *elem_sub, const int *elem_mat, const double *u) {
    if (!path || n_nodes < 0 || n_elems < 0 || n_elems > (1 << 30) / 9) return HTF_EINVAL;
    if (n_nodes > 0 && (!coords || !u)) return HTF_EINVAL;
    if (n_elems > 0 && (!elems || !elem_sub)) return HTF_EINVAL;
    for (long long i = 0; i < 8LL * n_elems; ++i)
        if (elems[i] < 0 || elems[i] >= n_nodes) return HTF_EINVAL;
    std::vector<char> buf(1 << 20);          // outlives the stream: fclose below
    FILE *f = std::fopen(path, "w");
    if (!f) return HTF_EIO;
    std::setvbuf(f, buf.data(), _IOFBF, buf.size());

    std::fputs("# vtk DataFile Version 3.0\nvtk output\nASCII\n\nDATASET UNSTRUCTURED_GRID\n", f);
    std::fprintf(f, "POINTS %d float\n", n_nodes);
    for (int i = 0; i < n_nodes; ++i) std::fprintf(f, "%f %f %f\n", coords[3 * i], coords[3 * i + 1], coords[3 * i + 2]);

    std::fprintf(f, "CELLS %d %d\n", n_elems, 9 * n_elems);
    for (int e = 0; e < n_elems; ++e) {
        std::fputs("8 ", f);
        for (int k = 0; k < 8; ++k) std::fprintf(f, "% d", elems[8 * e + k]);
        std::fputc('\n', f);
    }
    std::fprintf(f, "CELL_TYPES %d\n", n_elems);
    for (int e = 0; e < n_elems; ++e) std::fputs("12\n", f);

    std::fprintf(f, "POINT_DATA %d\nSCALARS displacements float 3\nLOOKUP_TABLE my_table\n", n_nodes);
    for (int i = 0; i < n_nodes; ++i) std::fprintf(f, "%f %f %f\n", u[3 * i], u[3 * i + 1], u[3 * i + 2]);

    std::fprintf(f, "\nCELL_DATA %d\nSCALARS decomposition int 1\nLOOKUP_TABLE decomposition\n", n_elems);
    for (int e = 0; e < n_elems; ++e) std::fprintf(f, "%d\n", elem_sub[e]);
    std::fputs("SCALARS materialId int 1\nLOOKUP_TABLE materialId\n", f);
    for (int e = 0; e < n_elems; ++e)
        std::fprintf(f, "%d\n", elem_mat ? elem_mat[e] : reference_material(elem_sub[e]));

    const bool written = !std::ferror(f);
    const bool closed = std::fclose(f) == 0;
    return written && closed ? HTF_OK : HTF_EIO;
}

}  // namespace htf
