// MatrixMarket dumps of a set-up problem in the reference's file layout
// (Matrix::printToFile, Matrix.cpp:556-632: "<folder>/dump_<name>_<index>.txt",
// a "%%MatrixMarket matrix coordinate real general|symmetric" header, a
// "rows<TAB>cols<TAB>nnz" line and one "i<TAB>j<TAB>%.16e" line per entry,
// 1-based), so the reference's Python cross-checks (python/myModul.py)
// read matrices this library built.  Levels follow the reference's
// print_matrices thresholds (Cluster.cpp:118-358): >= 2 K_i, rhs_i, Bc_i,
// Bf_i; >= 3 R_i, Rf_i, Gf_clust, GfTGf, iGfTGf; >= 4 the explicit Dirichlet
// preconditioner S_i.  Dense matrices are written entry by entry with the
// zeros left out.  K_i comes from the copy the set-up kept before the
// factorisation (option print_matrices >= 2).
#include <algorithm>
#include <cstdio>
#include <string>
#include <vector>

#include "../device/engine.hpp"

namespace htf {

namespace {

struct Entry {
    int i, j;
    double v;
};

int write_mm(const std::string &folder, const char *name, int index, int nrow, int ncol, bool symmetric,
             const std::vector<Entry> &e, std::string &err) {
    char path[1024];
    std::snprintf(path, sizeof(path), "%s/dump_%s_%d.txt", folder.c_str(), name, index);
    FILE *fp = std::fopen(path, "w");
    if (!fp) {
        err = std::string("htf_dump: cannot write ") + path;
        return HTF_EIO;
    }
    std::fprintf(fp, "%%%%MatrixMarket matrix coordinate real %s\n", symmetric ? "symmetric" : "general");
    std::fprintf(fp, "%d\t%d\t%d\n", nrow, ncol, int(e.size()));
    for (const Entry &x : e) std::fprintf(fp, "%d\t%d\t%.16e\n", x.i + 1, x.j + 1, x.v);
    if (std::fclose(fp) != 0) {
        err = std::string("htf_dump: error writing ") + path;
        return HTF_EIO;
    }
    return HTF_OK;
}

// column-major dense (n x m) as entries, zeros left out
std::vector<Entry> dense_entries(const double *A, int n, int m, int lda) {
    std::vector<Entry> e;
    for (int i = 0; i < n; ++i)
        for (int j = 0; j < m; ++j)
            if (A[i + size_t(j) * lda] != 0.0) e.push_back({i, j, A[i + size_t(j) * lda]});
    return e;
}

}  // namespace

int Engine::dump(const Problem &p, const std::string &folder, int level, std::string &err) {
    int rc = HTF_OK;
    if (level >= 2 && dumpK_.empty()) {
        err = "htf_dump: K_i is kept only when the context was set up with print_matrices >= 2";
        return HTF_ESTATE;
    }
    std::vector<double> fbody(nfull_);
    if (level >= 2) {
        rc = check(cudaMemcpy(fbody.data(), d_fbody_, nfull_ * sizeof(double), cudaMemcpyDeviceToHost), "htf_dump", err);
        if (rc) return rc;
    }
    std::vector<double> Stiles;
    if (level >= 4 && d_S_ && opt_.preconditioner == "Dirichlet_explicit") {
        Stiles.resize(size_t(ntiles_) * TILE_ELEMS);
        rc = check(cudaMemcpy(Stiles.data(), d_S_, Stiles.size() * sizeof(double), cudaMemcpyDeviceToHost), "htf_dump",
                   err);
        if (rc) return rc;
    }
    for (int d = 0; d < nsub_ && !rc; ++d) {
        const Subdomain &s = p.sub[d];
        const SubDev &h = hs_[d];
        const int n = s.n;
        if (level >= 2) {
            // K_i, upper triangle in local order (Data.cpp:147-273 CSR, symmetric)
            std::vector<Entry> e;
            for (int i = 0; i < n; ++i)
                for (int j = i; j < n; ++j) {
                    const int pi = s.perm[i], pj = s.perm[j];
                    double v = dumpK_[kidx(h, std::max(pi, pj), std::min(pi, pj))];
                    if (pi == pj)
                        for (int q = 0; q < 6; ++q)
                            if (h.fix[q] == pi) v *= 0.5;          // K_reg doubled the fix diagonal
                    if (v != 0.0) e.push_back({i, j, v});
                }
            rc = write_mm(folder, "K", d, n, n, true, e, err);
            // rhs_i: the assembled element load
            e.clear();
            for (int i = 0; i < n && !rc; ++i) {
                const double v = fbody[h.nfull_off + s.perm[i]];
                if (v != 0.0) e.push_back({i, 0, v});
            }
            if (!rc) rc = write_mm(folder, "rhs", d, n, 1, false, e, err);
            // Bc_i: cluster Bc rows x local DOFs
            e.clear();
            for (size_t q = 0; q < s.bc_row.size(); ++q) e.push_back({s.bc_row[q], s.bc_col[q], s.bc_val[q]});
            if (!rc) rc = write_mm(folder, "Bc", d, p.clu[s.cluster].nlam_c, n, false, e, err);
            // Bf_i: global Bf rows x local DOFs
            e.clear();
            for (int r = 0; r < p.n_lam; ++r)
                for (int k = 0; k < 2; ++k)
                    if (p.rows[r].sub[k] == d) {
                        const int l = int(std::lower_bound(s.l2g.begin(), s.l2g.end(), p.rows[r].dof[k]) -
                                          s.l2g.begin());
                        e.push_back({r, l, p.rows[r].sign[k]});
                    }
            if (!rc) rc = write_mm(folder, "Bf", d, p.n_lam, n, false, e, err);
        }
        if (level >= 3 && !rc) {
            rc = write_mm(folder, "R", d, n, 6, false, dense_entries(s.R.data(), n, 6, n), err);
            std::vector<double> Rf(size_t(n) * 6, 0.0);             // Rf_i = R_i H_i (Cluster.cpp:1332-1352)
            for (int i = 0; i < n; ++i)
                for (int q = 0; q < 6; ++q) {
                    double v = 0.0;
                    for (int j = 0; j < 6; ++j) v += s.R[i + size_t(j) * n] * Hd_[d][j * 6 + q];
                    Rf[i + size_t(q) * n] = v;
                }
            if (!rc) rc = write_mm(folder, "Rf", d, n, 6, false, dense_entries(Rf.data(), n, 6, n), err);
        }
        if (level >= 4 && !rc && !Stiles.empty()) {
            // S_i over the Bf column set (j_col_cmpr order), from the packed tiles
            std::vector<Entry> e;
            for (int i = 0; i < s.nb; ++i)
                for (int j = 0; j < s.nb; ++j) {
                    const int a = std::max(i, j), b = std::min(i, j);
                    const int I = a / TILE, J = b / TILE;
                    const double v = Stiles[size_t(h.T_off + (long long)I * (I + 1) / 2 + J) * TILE_ELEMS +
                                            (a % TILE) * TILE + (b % TILE)];
                    if (v != 0.0) e.push_back({i, j, v});
                }
            rc = write_mm(folder, "S", d, s.nb, s.nb, false, e, err);
        }
    }
    if (level >= 3 && !rc) {
        const int m = 6 * ncl_;
        std::vector<Entry> e;
        for (int r = 0; r < nlam_; ++r)
            for (int k = 0; k < 2; ++k) {
                const int c = gcl_[2 * (size_t)r + k];
                if (c < 0) continue;
                for (int q = 0; q < 6; ++q) {
                    const double v = gval_[6 * (2 * (size_t)r + k) + q];
                    if (v != 0.0) e.push_back({r, 6 * c + q, v});
                }
            }
        rc = write_mm(folder, "Gf_clust", 0, nlam_, m, false, e, err);
        if (!rc) rc = write_mm(folder, "GfTGf", 0, m, m, false, dense_entries(gtg_.data(), m, m, m), err);
        if (!rc) rc = write_mm(folder, "iGfTGf", 0, m, m, false, dense_entries(invGtG_.data(), m, m, m), err);
    }
    return rc;
}

}  // namespace htf
