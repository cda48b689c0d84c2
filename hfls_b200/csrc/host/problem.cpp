// Dual layout and subdomain data of the HTFETI path (host side).
//   l2g maps               Data::buildMappingStruct        Data.cpp:111-144
//   interfaces             Cluster::create_cluster_constraints Cluster.cpp:682-727
//   Bf rows and weights    Cluster::create_Bc_or_Bf_in_CSR Cluster.cpp:832-928
//   Bc (cor / ker)         Cluster.cpp:737-747, 772-821
//   b set (Bf columns)     Cluster.cpp:756-765
//   kernel R               Data::create_analytic_ker_K     Data.cpp:61-109
//                          Matrix::GramSchmidtOrtho        Matrix.cpp:2450-2472
//   fix DOFs               Matrix::getNullPivots           Matrix.cpp:835-884
// Sums are written left-to-right so the values match the oracle bit for bit
// (compiled without FMA contraction).
#include <algorithm>
#include <cmath>
#include <cstring>
#include <numeric>

#include "problem.hpp"

namespace htf {

void kernel_of(const Mesh &m, const std::vector<int> &l2g, std::vector<double> &R) {
    const int n = int(l2g.size());
    R.assign(size_t(n) * 6, 0.0);
    for (int i = 0; i < n / 3; ++i) {
        int node = l2g[3 * i] / 3;
        double x = m.coords[3 * size_t(node)], y = m.coords[3 * size_t(node) + 1], z = m.coords[3 * size_t(node) + 2];
        R[3 * i + 0 + size_t(n) * 0] = 1;
        R[3 * i + 1 + size_t(n) * 1] = 1;
        R[3 * i + 2 + size_t(n) * 2] = 1;
        R[3 * i + 0 + size_t(n) * 3] = -y;
        R[3 * i + 1 + size_t(n) * 3] = x;
        R[3 * i + 0 + size_t(n) * 4] = -z;
        R[3 * i + 2 + size_t(n) * 4] = x;
        R[3 * i + 1 + size_t(n) * 5] = -z;
        R[3 * i + 2 + size_t(n) * 5] = y;
    }
    std::vector<double> w(n), coef(6);
    for (int j = 0; j < 6; ++j) {
        std::memcpy(w.data(), &R[size_t(j) * n], sizeof(double) * n);
        for (int i = 0; i < j; ++i) {
            double s = 0.0;
            const double *Ri = &R[size_t(i) * n];
            for (int k = 0; k < n; ++k) s += w[k] * Ri[k];
            coef[i] = s;
        }
        for (int i = 0; i < j; ++i) {
            const double *Ri = &R[size_t(i) * n];
            for (int k = 0; k < n; ++k) w[k] = w[k] - Ri[k] * coef[i];
        }
        double s = 0.0;
        for (int k = 0; k < n; ++k) s += w[k] * w[k];
        double nrm = std::sqrt(s);
        for (int k = 0; k < n; ++k) R[size_t(j) * n + k] = w[k] / nrm;
    }
}

std::vector<int> null_pivots(const std::vector<double> &R, int n, int m) {
    std::vector<double> N(R);
    std::vector<int> piv(n);
    std::iota(piv.begin(), piv.end(), 0);
    std::vector<double> tmp(std::max(n, m));
    auto at = [&](int i, int j) -> double & { return N[i + size_t(j) * n]; };
    for (int j = 0; j < m; ++j) {
        // last maximum of |N| over the first m-j columns, column-major order
        size_t len = size_t(n) * (m - j), I = 0;
        double mx = -1.0;
        for (size_t t = 0; t < len; ++t) {
            double v = std::fabs(N[t]);
            if (v >= mx) { mx = v; I = t; }
        }
        int col = int(I / n), row = int(I - size_t(col) * n);
        int last = n - 1 - j;
        for (int k = 0; k < m - j; ++k) {
            tmp[k] = at(last, k);
            at(last, k) = at(row, k);
            at(row, k) = tmp[k];
        }
        std::swap(piv[row], piv[last]);
        if (m - 1 - j != col)
            for (int i = 0; i < n; ++i) std::swap(at(i, m - 1 - j), at(i, col));
        double p = at(last, m - 1 - j);
        for (int J = 0; J < m - j - 1; ++J)
            for (int i = 0; i < n - j; ++i) at(i, J) -= at(i, m - 1 - j) * at(last, J) / p;
    }
    std::vector<int> out(m);
    for (int i = 0; i < m; ++i) out[i] = piv[n - 1 - i];
    std::sort(out.begin(), out.end());
    return out;
}

// Right-looking Cholesky, column-contiguous updates.
bool chol_lower(int n, double *A, int lda) {
    // a pivot below 1e-12 of its column's original diagonal means the matrix
    // is singular to working precision (a rank-deficient Gram matrix leaves
    // round-off of either sign there), which is reported like a negative one
    std::vector<double> diag(n);
    for (int k = 0; k < n; ++k) diag[k] = A[k + size_t(k) * lda];
    for (int k = 0; k < n; ++k) {
        double *ck = A + size_t(k) * lda;
        const double d = ck[k];
        if (!(d > 1e-12 * diag[k])) return false;
        const double r = std::sqrt(d);
        ck[k] = r;
        for (int i = k + 1; i < n; ++i) ck[i] /= r;
        for (int j = k + 1; j < n; ++j) {
            const double ljk = ck[j];
            if (ljk == 0.0) continue;
            double *cj = A + size_t(j) * lda;
            for (int i = j; i < n; ++i) cj[i] -= ck[i] * ljk;
        }
    }
    return true;
}

// L L^T X = B for nrhs columns; forward in axpy form, backward in dot form,
// both over contiguous columns of L.
void chol_solve(int n, const double *L, int lda, double *B, int ldb, int nrhs) {
    for (int r = 0; r < nrhs; ++r) {
        double *x = B + size_t(r) * ldb;
        for (int k = 0; k < n; ++k) {
            const double *ck = L + size_t(k) * lda;
            const double xk = x[k] / ck[k];
            x[k] = xk;
            if (xk != 0.0)
                for (int i = k + 1; i < n; ++i) x[i] -= ck[i] * xk;
        }
        for (int i = n - 1; i >= 0; --i) {
            const double *ci = L + size_t(i) * lda;
            double s = x[i];
            for (int k = i + 1; k < n; ++k) s -= ci[k] * x[k];
            x[i] = s / ci[i];
        }
    }
}

void sym_eig(int n, std::vector<double> &A, std::vector<double> &w, std::vector<double> &V) {
    V.assign(size_t(n) * n, 0.0);
    for (int i = 0; i < n; ++i) V[i + size_t(i) * n] = 1.0;
    for (int sweep = 0; sweep < 100; ++sweep) {
        double off = 0.0, tot = 0.0;
        for (int j = 0; j < n; ++j)
            for (int i = 0; i < n; ++i) {
                double v = A[i + size_t(j) * n] * A[i + size_t(j) * n];
                tot += v;
                if (i != j) off += v;
            }
        if (off == 0.0 || off <= 1e-30 * tot) break;
        for (int p = 0; p < n - 1; ++p)
            for (int q = p + 1; q < n; ++q) {
                double apq = A[p + size_t(q) * n];
                if (apq == 0.0) continue;
                double app = A[p + size_t(p) * n], aqq = A[q + size_t(q) * n];
                double theta = (aqq - app) / (2.0 * apq);
                double t = (theta >= 0 ? 1.0 : -1.0) / (std::fabs(theta) + std::sqrt(theta * theta + 1.0));
                double c = 1.0 / std::sqrt(t * t + 1.0), s = t * c;
                for (int k = 0; k < n; ++k) {
                    double akp = A[k + size_t(p) * n], akq = A[k + size_t(q) * n];
                    A[k + size_t(p) * n] = c * akp - s * akq;
                    A[k + size_t(q) * n] = s * akp + c * akq;
                }
                for (int k = 0; k < n; ++k) {
                    double apk = A[p + size_t(k) * n], aqk = A[q + size_t(k) * n];
                    A[p + size_t(k) * n] = c * apk - s * aqk;
                    A[q + size_t(k) * n] = s * apk + c * aqk;
                }
                for (int k = 0; k < n; ++k) {
                    double vkp = V[k + size_t(p) * n], vkq = V[k + size_t(q) * n];
                    V[k + size_t(p) * n] = c * vkp - s * vkq;
                    V[k + size_t(q) * n] = s * vkp + c * vkq;
                }
            }
    }
    w.resize(n);
    for (int i = 0; i < n; ++i) w[i] = A[i + size_t(i) * n];
}

namespace {
// Matrix::test_of_Bc_constraints (Matrix.cpp:1538-1571): singular values of
// A A^T (6x6 PSD, so its eigenvalues), a jump below 1e-4 means rank defect.
bool bc_rank_full(const std::vector<double> &A, int rows, int cols) {
    std::vector<double> G(size_t(rows) * rows, 0.0), w, V;
    for (int i = 0; i < rows; ++i)
        for (int j = 0; j < rows; ++j) {
            double s = 0.0;
            for (int k = 0; k < cols; ++k) s += A[i + size_t(k) * rows] * A[j + size_t(k) * rows];
            G[i + size_t(j) * rows] = s;
        }
    sym_eig(rows, G, w, V);
    for (double &x : w) x = std::fabs(x);
    std::sort(w.begin(), w.end(), [](double a, double b) { return a > b; });
    for (int i = 0; i + 1 < rows; ++i)
        if (std::fabs(w[i + 1] / w[i]) < 1e-4) return false;
    return true;
}
}  // namespace

// l2g, interface groups, Bf rows and weights, b sets and Bf CSR on the host
// (the inspection entry points; frontend_on_device restates it on the GPU);
// node_ptr / node_subs: the sorted subdomains of every node
static int frontend_host(Problem &p, std::vector<int> &node_ptr, std::vector<int> &node_subs, std::string &err) {
    Mesh &m = p.mesh;
    const int ns = m.n_sub();
    // l2g (Data.cpp:111-144)
    for (int d = 0; d < ns; ++d)
        if (p.sub[d].elems.empty()) { err = "subdomain without elements"; return HTF_EINVAL; }
#pragma omp parallel for schedule(dynamic, 4)
    for (int d = 0; d < ns; ++d) {
        Subdomain &s = p.sub[d];
        std::vector<int> &l = s.l2g;
        l.reserve(s.elems.size() * 24);
        for (int e : s.elems)
            for (int c = 0; c < 3; ++c)
                for (int j = 0; j < 8; ++j) l.push_back(3 * m.elems[8 * size_t(e) + j] + c);
        std::sort(l.begin(), l.end());
        l.erase(std::unique(l.begin(), l.end()), l.end());
        s.n = int(l.size());
    }
    // interfaces: sorted (dof, sub) pairs
    std::vector<std::pair<int, int>> ds;
    for (int d = 0; d < ns; ++d)
        for (int g : p.sub[d].l2g) ds.emplace_back(g, d);
    std::sort(ds.begin(), ds.end());
    // per subdomain: shared DOFs (ascending) with the group of subdomains sharing them
    std::vector<std::vector<std::pair<int, int>>> iface(ns);   // (dof, group start in grp)
    std::vector<int> grp, grp_len_at;                            // concatenated groups
    std::vector<int> grp_ptr;
    for (size_t i = 0; i < ds.size();) {
        size_t j = i;
        while (j < ds.size() && ds[j].first == ds[i].first) ++j;
        if (j - i >= 2) {
            int gi = int(grp_ptr.size());
            grp_ptr.push_back(int(grp.size()));
    node_ptr.assign(size_t(m.n_nodes) + 1, 0);
    node_subs.clear();
    for (const auto &x : ds)
        if (x.first % 3 == 0) ++node_ptr[x.first / 3 + 1];
    for (int v = 0; v < m.n_nodes; ++v) node_ptr[v + 1] += node_ptr[v];
    for (const auto &x : ds)
        if (x.first % 3 == 0) node_subs.push_back(x.second);
            for (size_t k = i; k < j; ++k) grp.push_back(ds[k].second);
            for (size_t k = i; k < j; ++k) iface[ds[k].second].emplace_back(ds[i].first, gi);
        }
        i = j;
    }
    grp_ptr.push_back(int(grp.size()));
    node_ptr.assign(size_t(m.n_nodes) + 1, 0);
    node_subs.clear();
    for (const auto &x : ds)
        if (x.first % 3 == 0) ++node_ptr[x.first / 3 + 1];
    for (int v = 0; v < m.n_nodes; ++v) node_ptr[v + 1] += node_ptr[v];
    for (const auto &x : ds)
        if (x.first % 3 == 0) node_subs.push_back(x.second);
    std::vector<char> is_dir(3 * size_t(m.n_nodes), 0);
    for (int g : m.dirichlet) {
        if (g < 0 || g >= 3 * m.n_nodes) { err = "Dirichlet DOF out of range"; return HTF_EINVAL; }
        is_dir[g] = 1;
    }
    auto local_of = [&](int d, int g) {
        const std::vector<int> &l = p.sub[d].l2g;
        return int(std::lower_bound(l.begin(), l.end(), g) - l.begin());
    };
    // Bf (Cluster.cpp:846-924)
    p.rows.clear();
    p.weight.clear();
    for (int d = 0; d < ns; ++d)
        for (auto &it : iface[d]) {
            int g = it.first;
            if (is_dir[g]) continue;
            int a = grp_ptr[it.second], b = grp_ptr[it.second + 1];
            int others = b - a - 1;
            for (int k = a; k < b; ++k) {
                int nb = grp[k];
                if (nb > d) {
                    p.rows.push_back(BfRow{{d, nb}, {g, g}, {1.0, -1.0}});
                    p.weight.push_back(1. / ((double)others + 1));
                }
            }
        }
    {
        // Dirichlet rows in the order (subdomain, position in the Dirichlet list)
        std::vector<std::vector<int>> drows(ns);
        std::vector<int> dpos(3 * size_t(m.n_nodes), -1);    // position in the Dirichlet list
        bool dup = false;
        for (size_t i = 0; i < m.dirichlet.size(); ++i) {
            int &q = dpos[m.dirichlet[i]];
            if (q >= 0) dup = true;
            else q = int(i);
        }
#pragma omp parallel for schedule(dynamic, 4)
        for (int d = 0; d < ns; ++d) {
            const std::vector<int> &l = p.sub[d].l2g;
            if (dup) {                 // a DOF listed twice gives two rows, as the reference's scan does
                for (int g : m.dirichlet)
                    if (std::binary_search(l.begin(), l.end(), g)) drows[d].push_back(g);
            } else {
                std::vector<std::pair<int, int>> hit;
                for (int g : l)
                    if (dpos[g] >= 0) hit.push_back({dpos[g], g});
                std::sort(hit.begin(), hit.end());
                for (auto &h : hit) drows[d].push_back(h.second);
            }
        }
        for (int d = 0; d < ns; ++d)
            for (int g : drows[d]) {
                p.rows.push_back(BfRow{{d, -1}, {g, -1}, {1.0, 0.0}});
                p.weight.push_back(1);
            }
    }
    p.n_lam = int(p.rows.size());
    if (p.n_lam == 0) { err = "no dual rows (no interface and no Dirichlet DOF)"; return HTF_EINVAL; }
    // b sets, permutation and Bf gather CSR
    {
        std::vector<std::vector<std::pair<int, std::pair<int, double>>>> ent(ns);   // (local, (row, sign))
        for (int r = 0; r < p.n_lam; ++r)
            for (int k = 0; k < 2; ++k) {
                int d = p.rows[r].sub[k];
                if (d < 0) continue;
                ent[d].push_back({local_of(d, p.rows[r].dof[k]), {r, p.rows[r].sign[k]}});
            }
        int few = -1;
#pragma omp parallel for schedule(dynamic, 4)
        for (int d = 0; d < ns; ++d) {
            Subdomain &s = p.sub[d];
            std::sort(ent[d].begin(), ent[d].end());
            s.b.clear();
            for (auto &e : ent[d])
                if (s.b.empty() || s.b.back() != e.first) s.b.push_back(e.first);
            s.nb = int(s.b.size());
            s.nr = s.n - s.nb;
            s.perm.assign(s.n, -1);
            for (int i = 0; i < s.nb; ++i) s.perm[s.b[i]] = s.nr + i;
            int c = 0;
            for (int l = 0; l < s.n; ++l)
                if (s.perm[l] < 0) s.perm[l] = c++;
            s.bf_ptr.assign(s.nb + 1, 0);
            s.bf_lam.clear();
            s.bf_sign.clear();
            int bi = 0;
            for (auto &e : ent[d]) {
                while (s.b[bi] != e.first) ++bi;
                s.bf_ptr[bi + 1]++;
                s.bf_lam.push_back(e.second.first);
                s.bf_sign.push_back(e.second.second);
            }
            for (int i = 0; i < s.nb; ++i) s.bf_ptr[i + 1] += s.bf_ptr[i];
            if (s.nb < 6) {
#pragma omp critical
                few = (few < 0 || d < few) ? d : few;
            }
        }
        if (few >= 0) { err = "subdomain with fewer than 6 interface/Dirichlet DOFs"; return HTF_EINVAL; }
    }
    return HTF_OK;
}

int build_problem(Problem &p, std::string &err, bool on_device) {
    Mesh &m = p.mesh;
    const int ns = m.n_sub(), ne = m.n_elems();
    if (ns < 1 || ne < 1) { err = "empty mesh"; return HTF_EINVAL; }
    for (int e = 0; e < ne; ++e)
        if (m.elem_sub[e] < 0 || m.elem_sub[e] >= ns) { err = "elem_sub out of range"; return HTF_EINVAL; }
    for (int v : m.elems)
        if (v < 0 || v >= m.n_nodes) { err = "element node id out of range"; return HTF_EINVAL; }
    p.sub.assign(ns, Subdomain());
    int ncl = 0;
    for (int d = 0; d < ns; ++d) {
        if (m.sub_cluster[d] < 0) { err = "negative cluster id"; return HTF_EINVAL; }
        ncl = std::max(ncl, m.sub_cluster[d] + 1);
    }
    p.clu.assign(ncl, Cluster());
    for (int d = 0; d < ns; ++d) {
        Subdomain &s = p.sub[d];
        s.id = d;
        s.cluster = m.sub_cluster[d];
        s.cl_index = int(p.clu[s.cluster].subs.size());
        p.clu[s.cluster].subs.push_back(d);
    }
    for (int c = 0; c < ncl; ++c)
        if (p.clu[c].subs.empty()) { err = "cluster without subdomains"; return HTF_EINVAL; }
    for (int e = 0; e < ne; ++e) p.sub[m.elem_sub[e]].elems.push_back(e);
    for (int d = 0; d < ns; ++d)
        if (p.sub[d].elems.empty()) { err = "subdomain without elements"; return HTF_EINVAL; }
    // l2g, Bf rows, b sets: on the device for a set-up (frontend.cu), on the
    // host for the inspection entry points, for Dirichlet lists with repeated
    // DOFs and without a device (the set-up then fails at its first device
    // step), bit for bit the same
    std::vector<int> node_ptr, node_subs;
    p.context_ms = p.frontend_ms = p.kernel_ms = 0.0;
    int frc = on_device ? frontend_on_device(p, node_ptr, node_subs, err) : HTF_ESTATE;
    if (frc == HTF_ESTATE || frc == HTF_ENODEV) frc = frontend_host(p, node_ptr, node_subs, err);
    if (frc) return frc;
    std::vector<char> is_corner(3 * size_t(m.n_nodes), 0);
    for (int g : m.corner)
        if (g >= 0 && g < 3 * m.n_nodes) is_corner[g] = 1;
    auto local_of = [&](int d, int g) {
        const std::vector<int> &l = p.sub[d].l2g;
        return int(std::lower_bound(l.begin(), l.end(), g) - l.begin());
    };
    // kernels and fix DOFs: on the device for a set-up (kernel_fix.cu), on the
    // host for the layout inspection entry points, bit for bit the same
    if (on_device) {
        double t[2] = {0.0, 0.0};
        const int rc = kernels_fix_on_device(m, p.sub, p.opt.device, err, t);
        p.context_ms += t[0];
        p.kernel_ms = t[1];
        if (rc) return rc;
    } else {
#pragma omp parallel for schedule(dynamic, 4)
    for (int d = 0; d < ns; ++d) {
        Subdomain &s = p.sub[d];
        kernel_of(m, s.l2g, s.R);
        std::vector<double> Rb(size_t(s.nb) * 6);
        for (int j = 0; j < 6; ++j)
            for (int i = 0; i < s.nb; ++i) Rb[i + size_t(j) * s.nb] = s.R[s.b[i] + size_t(j) * s.n];
        std::vector<int> pv = null_pivots(Rb, s.nb, 6);
        s.fix.resize(6);
        for (int i = 0; i < 6; ++i) s.fix[i] = s.b[pv[i]];
        std::sort(s.fix.begin(), s.fix.end());
    }
    }
    // neighbour lists (subdomains sharing at least one node)
    std::vector<std::vector<int>> neigh(ns);
    for (int v = 0; v < m.n_nodes; ++v)
        for (int a = node_ptr[v]; a < node_ptr[v + 1]; ++a)
            for (int b = node_ptr[v]; b < node_ptr[v + 1]; ++b)
                if (a != b) neigh[node_subs[a]].push_back(node_subs[b]);
    for (auto &v : neigh) {
        std::sort(v.begin(), v.end());
        v.erase(std::unique(v.begin(), v.end()), v.end());
    }
    // Bc per cluster
    for (int ci = 0; ci < ncl; ++ci) {
        Cluster &cl = p.clu[ci];
        int cnt = 0;
        if (p.opt.typeBc == "cor") {             // Cluster.cpp:846-903 with full rank
            for (int d : cl.subs)
                for (int g : p.sub[d].l2g) {          // the shared DOFs of d, ascending
                    const int v = g / 3;
                    if (node_ptr[v + 1] - node_ptr[v] < 2 || !is_corner[g]) continue;
                    for (int k = node_ptr[v]; k < node_ptr[v + 1]; ++k) {
                        int nb = node_subs[k];
                        if (nb > d && m.sub_cluster[nb] == ci) {
                            Subdomain &a = p.sub[d], &b = p.sub[nb];
                            a.bc_row.push_back(cnt); a.bc_col.push_back(local_of(d, g)); a.bc_val.push_back(1.0);
                            b.bc_row.push_back(cnt); b.bc_col.push_back(local_of(nb, g)); b.bc_val.push_back(-1.0);
                            ++cnt;
                            break;
                        }
                    }
                }
        } else {                                  // Cluster.cpp:772-821
            for (int i : cl.subs)
                for (int j : neigh[i]) {
                    if (j <= i || m.sub_cluster[j] != ci) continue;
                    Subdomain &a = p.sub[i], &b = p.sub[j];
                    std::vector<int> com;
                    std::set_intersection(a.l2g.begin(), a.l2g.end(), b.l2g.begin(), b.l2g.end(),
                                          std::back_inserter(com));
                    int nc = int(com.size());
                    if (nc == 0) continue;
                    std::vector<double> A(6 * size_t(nc));
                    std::vector<int> li(nc), lj(nc);
                    for (int k = 0; k < nc; ++k) {
                        li[k] = local_of(i, com[k]);
                        lj[k] = local_of(j, com[k]);
                        for (int l = 0; l < 6; ++l) A[l + 6 * size_t(k)] = a.R[li[k] + size_t(l) * a.n];
                    }
                    if (!bc_rank_full(A, 6, nc)) continue;
                    for (int k = 0; k < 6; ++k) {
                        for (int l = 0; l < nc; ++l) {
                            double v = A[k + 6 * size_t(l)];
                            a.bc_row.push_back(cnt); a.bc_col.push_back(li[l]); a.bc_val.push_back(v);
                            b.bc_row.push_back(cnt); b.bc_col.push_back(lj[l]); b.bc_val.push_back(-v);
                        }
                        ++cnt;
                    }
                }
        }
        cl.nlam_c = cnt;
        for (int d : cl.subs) {
            Subdomain &s = p.sub[d];
            s.bc_rows = s.bc_row;
            std::sort(s.bc_rows.begin(), s.bc_rows.end());
            s.bc_rows.erase(std::unique(s.bc_rows.begin(), s.bc_rows.end()), s.bc_rows.end());
            // Bc columns must lie in the b set (corner / face DOFs are interface DOFs)
            for (int l : s.bc_col)
                if (s.perm[l] < s.nr) { err = "Bc entry outside the Bf column set"; return HTF_EINVAL; }
        }
    }
    return HTF_OK;
}

}  // namespace htf
