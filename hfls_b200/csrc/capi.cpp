// C ABI of the HTFETI path (declared in include/htfeti.h).
#include <chrono>
#include <cstring>
#include <memory>
#include <new>
#include <string>

#include "device/engine.hpp"
#include "host/problem.hpp"
#include "htfeti.h"

struct htf_ctx {
    htf::Problem p;
    std::unique_ptr<htf::Engine> eng;
    std::string err;
    bool has_mesh = false, is_setup = false;
};

namespace {
int fail(htf_ctx *c, int rc, const std::string &msg) {
    if (c) c->err = msg;
    return rc;
}
}  // namespace

extern "C" {

int htf_mesh_sizes(const htf_mesh_spec *spec, int *n_nodes, int *n_elems, int *n_sub, int *n_clusters,
                   int *n_dirichlet, int *n_corner) {
    if (!spec) return HTF_EINVAL;
    std::string err;
    return htf::mesh_sizes(*spec, n_nodes, n_elems, n_sub, n_clusters, n_dirichlet, n_corner, err);
}

int htf_mesh_fill(const htf_mesh_spec *spec, double *coords, int *elems, int *elem_sub, int *sub_cluster,
                  double *sub_E, double *sub_nu, int *dirichlet, int *corner) {
    if (!spec) return HTF_EINVAL;
    std::string err;
    htf::Mesh m;
    int rc = htf::generate_mesh(*spec, m, err);
    if (rc) return rc;
    if (coords) std::memcpy(coords, m.coords.data(), m.coords.size() * sizeof(double));
    if (elems) std::memcpy(elems, m.elems.data(), m.elems.size() * sizeof(int));
    if (elem_sub) std::memcpy(elem_sub, m.elem_sub.data(), m.elem_sub.size() * sizeof(int));
    if (sub_cluster) std::memcpy(sub_cluster, m.sub_cluster.data(), m.sub_cluster.size() * sizeof(int));
    if (sub_E) std::memcpy(sub_E, m.sub_E.data(), m.sub_E.size() * sizeof(double));
    if (sub_nu) std::memcpy(sub_nu, m.sub_nu.data(), m.sub_nu.size() * sizeof(double));
    if (dirichlet) std::memcpy(dirichlet, m.dirichlet.data(), m.dirichlet.size() * sizeof(int));
    if (corner) std::memcpy(corner, m.corner.data(), m.corner.size() * sizeof(int));
    return HTF_OK;
}

int htf_mesh_traction(const htf_mesh_spec *spec, uint64_t seed, int n_rhs, double scale, double *f) {
    if (!spec || !f || n_rhs < 1) return HTF_EINVAL;
    std::string err;
    return htf::mesh_traction(*spec, seed, n_rhs, scale, f, err);
}

int htf_write_vtk(const char *path, int n_nodes, const double *coords, int n_elems, const int *elems,
                  const int *elem_sub, const int *elem_mat, const double *u) {
    return htf::write_vtk(path, n_nodes, coords, n_elems, elems, elem_sub, elem_mat, u);
}

int htf_create(const char *options, htf_ctx **ctx) {
    if (!ctx) return HTF_EINVAL;
    *ctx = nullptr;
    htf_ctx *c = new (std::nothrow) htf_ctx();
    if (!c) return HTF_ENOMEM;
    int rc = htf::parse_options(options, c->p.opt, c->err);
    if (rc) {
        delete c;
        return rc;
    }
    *ctx = c;
    return HTF_OK;
}

int htf_destroy(htf_ctx *ctx) {
    delete ctx;
    return HTF_OK;
}

const char *htf_last_error(const htf_ctx *ctx) { return ctx ? ctx->err.c_str() : "null context"; }

int htf_status_sub(const htf_ctx *ctx) { return ctx && ctx->eng ? ctx->eng->status_sub : -1; }

int htf_set_mesh(htf_ctx *ctx, int n_nodes, const double *coords, int n_elems, const int *elems,
                 const int *elem_sub, int n_sub, const int *sub_cluster, const double *sub_E,
                 const double *sub_nu, int n_dirichlet, const int *dirichlet, int n_corner, const int *corner,
                 const double body_force[3]) {
    if (!ctx) return HTF_EINVAL;
    if (ctx->is_setup) return fail(ctx, HTF_ESTATE, "mesh already set up; create a new context");
    if (n_nodes < 1 || n_elems < 1 || n_sub < 1 || !coords || !elems || !elem_sub || !sub_cluster || !sub_E ||
        !sub_nu || (n_dirichlet > 0 && !dirichlet) || (n_corner > 0 && !corner))
        return fail(ctx, HTF_EINVAL, "htf_set_mesh: bad sizes or null arrays");
    htf::Mesh &m = ctx->p.mesh;
    m.n_nodes = n_nodes;
    m.coords.assign(coords, coords + 3 * (size_t)n_nodes);
    m.elems.assign(elems, elems + 8 * (size_t)n_elems);
    m.elem_sub.assign(elem_sub, elem_sub + n_elems);
    m.sub_cluster.assign(sub_cluster, sub_cluster + n_sub);
    m.sub_E.assign(sub_E, sub_E + n_sub);
    m.sub_nu.assign(sub_nu, sub_nu + n_sub);
    m.dirichlet.assign(dirichlet, dirichlet + std::max(n_dirichlet, 0));
    m.corner.assign(corner, corner + std::max(n_corner, 0));
    for (int a = 0; a < 3; ++a) m.body_force[a] = body_force ? body_force[a] : 0.0;
    ctx->has_mesh = true;
    return HTF_OK;
}

int htf_set_loads(htf_ctx *ctx, int n_rhs, const double *f_nodal) {
    if (!ctx) return HTF_EINVAL;
    if (!ctx->has_mesh) return fail(ctx, HTF_ESTATE, "htf_set_loads before htf_set_mesh");
    if (ctx->is_setup) return fail(ctx, HTF_ESTATE, "htf_set_loads after htf_setup");
    if (n_rhs < 1 || !f_nodal) return fail(ctx, HTF_EINVAL, "htf_set_loads: bad arguments");
    ctx->p.nrhs = n_rhs;
    ctx->p.f_nodal.assign(f_nodal, f_nodal + 3 * (size_t)ctx->p.mesh.n_nodes * n_rhs);
    return HTF_OK;
}

int htf_setup(htf_ctx *ctx) {
    if (!ctx) return HTF_EINVAL;
    if (!ctx->has_mesh) return fail(ctx, HTF_ESTATE, "htf_setup before htf_set_mesh");
    if (ctx->is_setup) return fail(ctx, HTF_ESTATE, "htf_setup called twice");
    const auto t0 = std::chrono::steady_clock::now();
    int rc = htf::build_problem(ctx->p, ctx->err, true);
    if (rc) return rc;
    ctx->eng.reset(new (std::nothrow) htf::Engine(ctx->p.opt));
    if (!ctx->eng) return fail(ctx, HTF_ENOMEM, "engine allocation failed");
    // phase 0 without the device context creation, which the kernel detection
    // triggers and which belongs to phase 1
    ctx->eng->phase_ms[0] =
        std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count() - ctx->p.context_ms;
    ctx->eng->kernel_detection_ms = ctx->p.kernel_ms;
    ctx->eng->frontend_ms = ctx->p.frontend_ms;
    rc = ctx->eng->setup(ctx->p, ctx->err);
    if (rc) return rc;
    ctx->eng->phase_ms[1] += ctx->p.context_ms;
    ctx->is_setup = true;
    return HTF_OK;
}

int htf_pcpg(htf_ctx *ctx, double *u, htf_stats *stats) {
    if (!ctx) return HTF_EINVAL;
    if (!ctx->is_setup) return fail(ctx, HTF_ESTATE, "htf_pcpg before htf_setup");
    if (stats) std::memset(stats, 0, sizeof(*stats));
    const double *fn = ctx->p.f_nodal.empty() ? nullptr : ctx->p.f_nodal.data();
    return ctx->eng->solve(ctx->p, ctx->p.nrhs, fn, u, stats, ctx->err);
}

int htf_solve(htf_ctx *ctx, int n_rhs, const double *f_nodal, double *u, htf_stats *stats) {
    if (!ctx) return HTF_EINVAL;
    if (!ctx->is_setup) return fail(ctx, HTF_ESTATE, "htf_solve before htf_setup");
    if (n_rhs < 1) return fail(ctx, HTF_EINVAL, "htf_solve: n_rhs < 1");
    if (stats) std::memset(stats, 0, sizeof(*stats));
    return ctx->eng->solve(ctx->p, n_rhs, f_nodal, u, stats, ctx->err);
}

int htf_profile(htf_ctx *ctx, int reps, htf_profile_info *info) {
    if (!ctx) return HTF_EINVAL;
    if (!ctx->is_setup) return fail(ctx, HTF_ESTATE, "htf_profile before htf_setup");
    return ctx->eng->profile(reps, info, ctx->err);
}

static int apply_op(htf_ctx *ctx, int op, const double *x, double *y, int nrhs) {
    if (!ctx) return HTF_EINVAL;
    if (!ctx->is_setup) return fail(ctx, HTF_ESTATE, "operator before htf_setup");
    if (!x || !y || nrhs < 1) return fail(ctx, HTF_EINVAL, "operator: bad arguments");
    return ctx->eng->apply(op, x, y, nrhs, ctx->err);
}

int htf_mult_Ff(htf_ctx *ctx, const double *w, double *Fw, int nrhs) { return apply_op(ctx, 0, w, Fw, nrhs); }
int htf_projection(htf_ctx *ctx, const double *x, double *Px, int nrhs) { return apply_op(ctx, 1, x, Px, nrhs); }
int htf_preconditioning(htf_ctx *ctx, const double *x, double *Mx, int nrhs) { return apply_op(ctx, 2, x, Mx, nrhs); }

int htf_projection_noalloc(htf_ctx *ctx, const double *x_dev, double *Px_dev, void *stream) {
    if (!ctx) return HTF_EINVAL;
    if (!ctx->is_setup) return fail(ctx, HTF_ESTATE, "htf_projection_noalloc before htf_setup");
    if (!x_dev || !Px_dev) return fail(ctx, HTF_EINVAL, "htf_projection_noalloc: null vector");
    int prev = -1;
    if (cudaGetDevice(&prev) != cudaSuccess) return fail(ctx, HTF_ECUDA, "cudaGetDevice failed");
    if (prev != ctx->eng->device() && cudaSetDevice(ctx->eng->device()) != cudaSuccess)
        return fail(ctx, HTF_ECUDA, "cudaSetDevice failed");
    // both vectors must be device (or managed) memory of the context's device: a host pointer or a
    // pointer on another GPU would reach the kernels as an invalid address
    for (const void *ptr : {static_cast<const void *>(x_dev), static_cast<const void *>(Px_dev)}) {
        cudaPointerAttributes a;
        if (cudaPointerGetAttributes(&a, ptr) != cudaSuccess) {
            cudaGetLastError();
            if (prev != ctx->eng->device()) cudaSetDevice(prev);
            return fail(ctx, HTF_EINVAL, "htf_projection_noalloc: a vector is not CUDA memory");
        }
        if ((a.type != cudaMemoryTypeDevice && a.type != cudaMemoryTypeManaged) || a.device != ctx->eng->device()) {
            if (prev != ctx->eng->device()) cudaSetDevice(prev);
            return fail(ctx, HTF_EINVAL,
                        "htf_projection_noalloc: both vectors must be device memory of the context's device");
        }
    }
    int rc = ctx->eng->project_noalloc(x_dev, Px_dev, static_cast<cudaStream_t>(stream), ctx->err);
    if (prev != ctx->eng->device()) cudaSetDevice(prev);
    return rc;
}

int htf_residual_history(htf_ctx *ctx, int rhs, double *hist, int cap) {
    if (!ctx) return HTF_EINVAL;
    if (!ctx->is_setup) return fail(ctx, HTF_ESTATE, "htf_residual_history before htf_setup");
    return ctx->eng->history(rhs, hist, cap, ctx->err);
}

int htf_dump(htf_ctx *ctx, const char *folder, int level) {
    if (!ctx) return HTF_EINVAL;
    if (!ctx->is_setup) return fail(ctx, HTF_ESTATE, "htf_dump before htf_setup");
    if (!folder) return fail(ctx, HTF_EINVAL, "htf_dump: null folder");
    return ctx->eng->dump(ctx->p, folder, level, ctx->err);
}

int htf_dual_sizes(htf_ctx *ctx, int *n_lambda, int *n_sub, int *n_clusters) {
    if (!ctx) return HTF_EINVAL;
    if (ctx->p.rows.empty()) {
        if (!ctx->has_mesh) return fail(ctx, HTF_ESTATE, "htf_dual_sizes before htf_set_mesh");
        int rc = htf::build_problem(ctx->p, ctx->err);
        if (rc) return rc;
    }
    if (n_lambda) *n_lambda = ctx->p.n_lam;
    if (n_sub) *n_sub = int(ctx->p.sub.size());
    if (n_clusters) *n_clusters = int(ctx->p.clu.size());
    return HTF_OK;
}

int htf_dual_layout(htf_ctx *ctx, int *row_sub, int *row_dof, double *row_sign, double *weight) {
    int rc = htf_dual_sizes(ctx, nullptr, nullptr, nullptr);
    if (rc) return rc;
    const auto &p = ctx->p;
    for (int r = 0; r < p.n_lam; ++r)
        for (int k = 0; k < 2; ++k) {
            if (row_sub) row_sub[2 * r + k] = p.rows[r].sub[k];
            if (row_dof) row_dof[2 * r + k] = p.rows[r].dof[k];
            if (row_sign) row_sign[2 * r + k] = p.rows[r].sign[k];
        }
    if (weight) std::memcpy(weight, p.weight.data(), p.n_lam * sizeof(double));
    return HTF_OK;
}

int htf_fix_dofs(htf_ctx *ctx, int *fix_global) {
    int rc = htf_dual_sizes(ctx, nullptr, nullptr, nullptr);
    if (rc) return rc;
    if (!fix_global) return fail(ctx, HTF_EINVAL, "null output");
    const auto &p = ctx->p;
    for (size_t d = 0; d < p.sub.size(); ++d)
        for (int q = 0; q < 6; ++q) fix_global[6 * d + q] = p.sub[d].l2g[p.sub[d].fix[q]];
    return HTF_OK;
}

}  // extern "C"
