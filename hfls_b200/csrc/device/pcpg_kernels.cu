// PCPG kernels of the HTFETI path (sm_100a).  All reductions are
// deterministic (fixed-order trees, no floating-point atomics), so a solve
// gives the same bits alone and inside a batch.
//
//  F w = Bf K_HT^+ Bf^T w   (Cluster::mult_Ff, Cluster.cpp:1114-1188):
//    k_gather_b        x_b = Bf_d^T w             signed gather over the b slots
//    k_symv_units      y_b = F_d x_b              packed 32x32 lower tiles, one pass, in work
//                      t_d = V_d^T x_b            units; V = [F Bc_b^T, -R_b]
//    k_gc              gc  = sum_d t_d            per cluster (gather map)
//    k_coarse          s   = M gc                 M = Ac^{-1} restricted
//    k_reduce_correct  y_b = sum of the unit partials - V_d s_d
//    k_rows            Fw  = Bf y                 <= 2 entries per row
//  Preconditioner (Cluster::Preconditioning, Cluster.cpp:1043-1112):
//    k_gather_b(weighted) -> k_symv_units(S_d or K_bb) -> k_reduce_correct -> k_rows(weighted)
//  Projector (Cluster::Projection, Cluster.cpp:1314-1329):
//    k_gft_partial (Gf^T x partials per chunk) -> k_gf_apply_fused (sums, (Gf^T Gf)^{-1}, x - Gf a)
#include <cuda_runtime.h>
#include <cstdint>

#include "device.cuh"

namespace htf {

constexpr unsigned FULL = 0xffffffffu;

// ---------------------------------------------------------------------------
// signed gather: x[slot] = sum_e sign_e * (weight[lam_e]) * w[lam_e]
// ent = 2*lam + (sign < 0)
// ---------------------------------------------------------------------------
__global__ void k_gather_b(int nslots, const int *__restrict__ ptr, const int *__restrict__ ent,
                           const double *__restrict__ w, const double *__restrict__ weight,
                           double *__restrict__ x, const PcpgState *__restrict__ st) {
    if (st && st->done) return;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nslots) return;
    double v = 0.0;
    for (int e = ptr[i]; e < ptr[i + 1]; ++e) {
        const int q = ent[e];
        const int lam = q >> 1;
        double a = w[lam];
        if (weight) a *= weight[lam];
        v += (q & 1) ? -a : a;
    }
    x[i] = v;
}

// ---------------------------------------------------------------------------
// y_b = A x_b for packed symmetric tiles; one CTA per subdomain, 4 warps,
// per-warp partial sums in shared memory summed in fixed order.
// ---------------------------------------------------------------------------
__device__ __forceinline__ void reduce_scatter32(double (&p)[32], int lane) {
#pragma unroll
    for (int s = 16; s >= 1; s >>= 1) {
        const bool upper = lane & s;
#pragma unroll
        for (int q = 0; q < s; ++q) {
            const double send = upper ? p[q] : p[q + s];
            const double keep = upper ? p[q + s] : p[q];
            p[q] = keep + __shfl_xor_sync(FULL, send, s);
        }
    }
}



// SYMV over work units (kinds 0 and 2) and V^T x (kind 1) in one launch; the
// partial y of a unit over its row window -> ypart[y_off, y_off + rows),
// summed later in unit order.  Shared memory: x and one partial y per warp
// over the unit's window.
template <typename T>
__global__ void __launch_bounds__(SYMV_WARPS * 32) k_symv_units(const SymvUnit *__restrict__ units,
                                                                const SubDev *__restrict__ subs,
                                                                const T *__restrict__ tiles,
                                                                const double *__restrict__ Vbuf,
                                                                const double *__restrict__ xb,
                                                                double *__restrict__ ypart,
                                                                double *__restrict__ t,
                                                                const PcpgState *__restrict__ st) {
    if (st && st->done) return;
    extern __shared__ double sm[];
    const SymvUnit u = units[blockIdx.x];
    const SubDev &sd = subs[u.d];
    const int lane = threadIdx.x % 32, warp = threadIdx.x / 32;
    const double *x = xb + sd.xb_off;
    if (u.kind == 1) {                      // t_d = V_d^T x_b
        for (int col = warp; col < sd.c + 6; col += SYMV_WARPS) {
            const double *V = Vbuf + sd.V_off + (size_t)col * sd.nbp;
            double a = 0.0;
            for (int i = lane; i < sd.nb; i += 32) a += V[i] * x[i];
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) a += __shfl_xor_sync(FULL, a, o);
            if (lane == 0) t[sd.t_off + col] = a;
        }
        return;
    }
    const int rows = u.rows, r0 = u.row0;
    // kind 0: window = rows [r0, r0 + rows); kind 2: rows [r0, r0 + seg) of the
    // column blocks, then the 32 rows of the unit's tile row at rowI
    const int seg = u.kind == 2 ? rows - TILE : rows;
    double *yp = sm + rows;                 // SYMV_WARPS x rows
    for (int i = threadIdx.x; i < rows; i += blockDim.x) sm[i] = x[i < seg ? r0 + i : u.rowI + (i - seg)];
    for (int i = threadIdx.x; i < SYMV_WARPS * rows; i += blockDim.x) yp[i] = 0.0;
    __syncthreads();
    const double *xs = sm - r0;             // x of column block J at xs + 32 J
    double *ys = yp + warp * rows;          // this warp's partial y over the window
    double *my = ys - r0;                   // column block J at my + 32 J
    const T *base = tiles + sd.T_off * TILE_ELEMS;
    for (long long tt = u.t0 + warp; tt < u.t1; tt += SYMV_WARPS) {
        int I = (int)((sqrt(8.0 * (double)tt + 1.0) - 1.0) * 0.5);
        while ((long long)(I + 1) * (I + 2) / 2 <= tt) ++I;
        while ((long long)I * (I + 1) / 2 > tt) --I;
        const int J = (int)(tt - (long long)I * (I + 1) / 2);
        const T *tp = base + tt * TILE_ELEMS;
        double v[32];
#pragma unroll
        for (int r = 0; r < 32; ++r) v[r] = (double)tp[r * TILE + lane];
        const double xJ = xs[TILE * J + lane];
        const double *xI = u.kind == 2 ? sm + seg : xs + TILE * I;      // x of row block I
        double *yI = u.kind == 2 ? ys + seg : my + TILE * I;             // partial y of row block I
        double p[32];
        double col = 0.0;
#pragma unroll
        for (int r = 0; r < 32; ++r) {
            p[r] = v[r] * xJ;
            col += v[r] * xI[r];
        }
        reduce_scatter32(p, lane);
        yI[lane] += p[0];
        if (I != J) my[TILE * J + lane] += col;
    }
    __syncthreads();
    double *out = ypart + u.y_off;
    for (int i = threadIdx.x; i < rows; i += blockDim.x) {
        double a = 0.0;
#pragma unroll
        for (int q = 0; q < SYMV_WARPS; ++q) a += yp[q * rows + i];
        out[i] = a;
    }
}

template __global__ void k_symv_units<double>(const SymvUnit *, const SubDev *, const double *, const double *,
                                              const double *, double *, double *, const PcpgState *);
template __global__ void k_symv_units<float>(const SymvUnit *, const SubDev *, const float *, const double *,
                                             const double *, double *, double *, const PcpgState *);

// y_b = sum of the unit partials (in unit order: only the units covering the
// row's 32-row block, listed per block) [- V_d s_d when s != null];
// grid (subdomain, chunk of 256 b rows)
__global__ void k_reduce_correct(const SubDev *__restrict__ subs, const SymvUnit *__restrict__ units,
                                 const int *__restrict__ rbptr, const int *__restrict__ rbunit,
                                 const double *__restrict__ ypart, const ClusterDev *__restrict__ cl,
                                 const double *__restrict__ Vbuf, const int *__restrict__ bcrows,
                                 const double *__restrict__ s, double *__restrict__ yb,
                                 const PcpgState *__restrict__ st) {
    if (st && st->done) return;
    __shared__ double sd_s[256];
    const SubDev &sd = subs[blockIdx.x];
    const int i = blockIdx.y * blockDim.x + threadIdx.x;
    const int nc = sd.c + 6;
    if (s) {
        const ClusterDev &c = cl[sd.cluster];
        for (int q = threadIdx.x; q < nc; q += blockDim.x) {
            const int pos = (q < sd.c) ? bcrows[sd.bcr_off + q] : sd.alpha_pos + (q - sd.c);
            sd_s[q] = s[c.gc_off + pos];
        }
        __syncthreads();
    }
    if (blockIdx.y * blockDim.x >= sd.nbp || i >= sd.nbp) return;
    double a = 0.0;
    const int R = i / TILE;                  // the units covering this row's block, in unit order
    for (int q = rbptr[sd.rb_off + R]; q < rbptr[sd.rb_off + R + 1]; ++q) {
        const SymvUnit &u = units[rbunit[q]];
        const int seg = u.kind == 2 ? u.rows - TILE : u.rows;
        if (i >= u.row0 && i < u.row0 + seg) a += ypart[u.y_off + (i - u.row0)];
        if (u.kind == 2 && i >= u.rowI && i < u.rowI + TILE) a += ypart[u.y_off + seg + (i - u.rowI)];
    }
    if (s && i < sd.nb) {
        const double *V = Vbuf + sd.V_off + i;
        for (int q = 0; q < nc; ++q) a -= V[(size_t)q * sd.nbp] * sd_s[q];
    }
    yb[sd.xb_off + i] = a;
}

// gc[q] = sum of the t entries listed for q (fixed order)
__global__ void k_gc(int ngc_total, const int *__restrict__ gptr, const int *__restrict__ gidx,
                     const double *__restrict__ t, double *__restrict__ gc, const PcpgState *__restrict__ st) {
    if (st && st->done) return;
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= ngc_total) return;
    double s = 0.0;
    for (int e = gptr[q]; e < gptr[q + 1]; ++e) s += t[gidx[e]];
    gc[q] = s;
}

// s = M gc per cluster; one warp per row
__global__ void k_coarse(const ClusterDev *__restrict__ cl, const double *__restrict__ Mbuf,
                         const double *__restrict__ gc, double *__restrict__ s, const PcpgState *__restrict__ st) {
    if (st && st->done) return;
    const ClusterDev c = cl[blockIdx.x];
    const int lane = threadIdx.x % 32, warp = threadIdx.x / 32, nw = blockDim.x / 32;
    const int row = blockIdx.y * nw + warp;
    if (row >= c.ngc) return;
    const double *M = Mbuf + c.M_off + (size_t)row * c.ngc;     // symmetric: column = row
    const double *g = gc + c.gc_off;
    double a = 0.0;
    for (int p = lane; p < c.ngc; p += 32) a += M[p] * g[p];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) a += __shfl_xor_sync(FULL, a, o);
    if (lane == 0) s[c.gc_off + row] = a;
}

// y_b -= V_d s_d  with s_d = (s at the Bc rows of d, alpha_d)
__global__ void k_correct(const SubDev *__restrict__ subs, const ClusterDev *__restrict__ cl,
                          const double *__restrict__ Vbuf, const int *__restrict__ bcrows,
                          const double *__restrict__ s, double *__restrict__ yb, const PcpgState *__restrict__ st) {
    if (st && st->done) return;
    __shared__ double sd_s[256];
    const SubDev &sd = subs[blockIdx.x];
    const ClusterDev &c = cl[sd.cluster];
    const int nc = sd.c + 6;
    for (int q = threadIdx.x; q < nc; q += blockDim.x) {
        const int pos = (q < sd.c) ? bcrows[sd.bcr_off + q] : sd.alpha_pos + (q - sd.c);
        sd_s[q] = s[c.gc_off + pos];
    }
    __syncthreads();
    const double *V = Vbuf + sd.V_off;
    double *y = yb + sd.xb_off;
    for (int i = threadIdx.x; i < sd.nb; i += blockDim.x) {
        double a = y[i];
        for (int q = 0; q < nc; ++q) a -= V[i + (size_t)q * sd.nbp] * sd_s[q];
        y[i] = a;
    }
}

// out[r] = wt[r] * sum_k sign_k * y[slot_k]; optional fused dot partial with `dotv`
__global__ void k_rows(int nlam, const int *__restrict__ rslot, const double *__restrict__ rsign,
                       const double *__restrict__ yb, const double *__restrict__ weight,
                       double *__restrict__ out, const double *__restrict__ dotv,
                       double *__restrict__ partial, const PcpgState *__restrict__ st) {
    if (st && st->done) return;
    __shared__ double red[256];
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    double prod = 0.0;
    if (r < nlam) {
        double v = 0.0;
        const int s0 = rslot[2 * r], s1 = rslot[2 * r + 1];
        if (s0 >= 0) v += rsign[2 * r] * yb[s0];
        if (s1 >= 0) v += rsign[2 * r + 1] * yb[s1];
        if (weight) v *= weight[r];
        out[r] = v;
        if (dotv) prod = v * dotv[r];
    }
    if (!partial) return;
    red[threadIdx.x] = prod;
    __syncthreads();
    for (int o = blockDim.x / 2; o > 0; o >>= 1) {
        if (threadIdx.x < o) red[threadIdx.x] += red[threadIdx.x + o];
        __syncthreads();
    }
    if (threadIdx.x == 0) partial[blockIdx.x] = red[0];
}

__device__ double block_sum_fixed(const double *partial, int np) {
    __shared__ double red[256];
    double s = 0.0;
    for (int i = threadIdx.x; i < np; i += blockDim.x) s += partial[i];
    red[threadIdx.x] = s;
    __syncthreads();
    for (int o = blockDim.x / 2; o > 0; o >>= 1) {
        if (threadIdx.x < o) red[threadIdx.x] += red[threadIdx.x + o];
        __syncthreads();
    }
    const double r = red[0];
    __syncthreads();
    return r;
}

// ---------------------------------------------------------------------------
// projector: a = (Gf^T Gf)^{-1} Gf^T x ; Px = x - Gf a
// Gf stored per cluster as a list of (row, 6 values); per row as up to two
// (cluster, 6 values) entries.
// ---------------------------------------------------------------------------
__global__ void k_gft_partial(const int *__restrict__ chunk_cl, const int *__restrict__ chunk_beg,
                              const int *__restrict__ chunk_end, const int *__restrict__ crow,
                              const double *__restrict__ cval, const double *__restrict__ x,
                              double *__restrict__ partial, const PcpgState *__restrict__ st) {
    if (st && st->done) return;
    __shared__ double red[6][256];
    const int ch = blockIdx.x;
    double s[6] = {0, 0, 0, 0, 0, 0};
    for (int e = chunk_beg[ch] + threadIdx.x; e < chunk_end[ch]; e += blockDim.x) {
        const double xv = x[crow[e]];
#pragma unroll
        for (int q = 0; q < 6; ++q) s[q] += cval[6 * (size_t)e + q] * xv;
    }
#pragma unroll
    for (int q = 0; q < 6; ++q) red[q][threadIdx.x] = s[q];
    __syncthreads();
    for (int o = blockDim.x / 2; o > 0; o >>= 1) {
        if (threadIdx.x < o)
#pragma unroll
            for (int q = 0; q < 6; ++q) red[q][threadIdx.x] += red[q][threadIdx.x + o];
        __syncthreads();
    }
    if (threadIdx.x < 6) partial[6 * (size_t)ch + threadIdx.x] = red[threadIdx.x][0];
}

// Px = x - Gf a with a = invGtG * (chunk partials summed per cluster)
// computed by every CTA (the coarse dimension 6*ncl is small); CTA 0 also
// writes a and -a (alpha) to global memory.
__global__ void k_gf_apply_fused(int nlam, int ncl, const int *__restrict__ cl_chunk_ptr,
                                 const double *__restrict__ gpart, const double *__restrict__ invGtG,
                                 const int *__restrict__ gcl, const double *__restrict__ gval,
                                 const double *__restrict__ x, double *__restrict__ a_out,
                                 double *__restrict__ alpha_out, double *__restrict__ Px,
                                 const double *__restrict__ dotv, double *__restrict__ partial,
                                 const PcpgState *__restrict__ st) {
    if (st && st->done) return;
    extern __shared__ double sh[];
    double *gt = sh;                 // 6*ncl
    double *a = sh + 6 * ncl;        // 6*ncl
    __shared__ double red[256];
    const int m = 6 * ncl;
    for (int q = threadIdx.x; q < m; q += blockDim.x) {
        const int c = q / 6, i = q % 6;
        double s = 0.0;
        for (int ch = cl_chunk_ptr[c]; ch < cl_chunk_ptr[c + 1]; ++ch) s += gpart[6 * (size_t)ch + i];
        gt[q] = s;
    }
    __syncthreads();
    for (int q = threadIdx.x; q < m; q += blockDim.x) {
        double s = 0.0;
        for (int p = 0; p < m; ++p) s += invGtG[q + (size_t)p * m] * gt[p];
        a[q] = s;
        if (blockIdx.x == 0) {
            if (a_out) a_out[q] = s;
            if (alpha_out) alpha_out[q] = -s;
        }
    }
    __syncthreads();
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    double prod = 0.0;
    if (r < nlam) {
        double v = 0.0;
#pragma unroll
        for (int k = 0; k < 2; ++k) {
            const int c = gcl[2 * r + k];
            if (c < 0) continue;
            const double *g = gval + 6 * (size_t)(2 * r + k);
#pragma unroll
            for (int q = 0; q < 6; ++q) v += g[q] * a[6 * c + q];
        }
        const double pv = x[r] - v;
        Px[r] = pv;
        if (dotv) prod = pv * dotv[r];
    }
    if (!partial) return;
    red[threadIdx.x] = prod;
    __syncthreads();
    for (int o = blockDim.x / 2; o > 0; o >>= 1) {
        if (threadIdx.x < o) red[threadIdx.x] += red[threadIdx.x + o];
        __syncthreads();
    }
    if (threadIdx.x == 0) partial[blockIdx.x] = red[0];
}

// a = invGtG * (chunk partials summed per cluster), once (one CTA): the
// coefficient that k_gf_apply_fused recomputes in every CTA, with the same sums
// in the same order; a_out gets a, alpha_out (if given) -a.
__global__ void k_gf_coef(int ncl, const int *__restrict__ cl_chunk_ptr, const double *__restrict__ gpart,
                          const double *__restrict__ invGtG, double *__restrict__ a_out,
                          double *__restrict__ alpha_out, const PcpgState *__restrict__ st) {
    if (st && st->done) return;
    extern __shared__ double sh[];
    double *gt = sh;                 // 6*ncl
    const int m = 6 * ncl;
    for (int q = threadIdx.x; q < m; q += blockDim.x) {
        const int c = q / 6, i = q % 6;
        double s = 0.0;
        for (int ch = cl_chunk_ptr[c]; ch < cl_chunk_ptr[c + 1]; ++ch) s += gpart[6 * (size_t)ch + i];
        gt[q] = s;
    }
    __syncthreads();
    for (int q = threadIdx.x; q < m; q += blockDim.x) {
        double s = 0.0;
        for (int p = 0; p < m; ++p) s += invGtG[q + (size_t)p * m] * gt[p];
        a_out[q] = s;
        if (alpha_out) alpha_out[q] = -s;
    }
}

// Px = x - Gf a for the coefficient a of k_gf_coef (and the partials of Px.dotv)
__global__ void k_gf_apply(int nlam, int ncl, const double *__restrict__ acoef, const int *__restrict__ gcl,
                           const double *__restrict__ gval, const double *__restrict__ x, double *__restrict__ Px,
                           const double *__restrict__ dotv, double *__restrict__ partial,
                           const PcpgState *__restrict__ st) {
    if (st && st->done) return;
    extern __shared__ double sh[];
    double *a = sh;                  // 6*ncl
    __shared__ double red[256];
    for (int q = threadIdx.x; q < 6 * ncl; q += blockDim.x) a[q] = acoef[q];
    __syncthreads();
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    double prod = 0.0;
    if (r < nlam) {
        double v = 0.0;
#pragma unroll
        for (int k = 0; k < 2; ++k) {
            const int c = gcl[2 * r + k];
            if (c < 0) continue;
            const double *g = gval + 6 * (size_t)(2 * r + k);
#pragma unroll
            for (int q = 0; q < 6; ++q) v += g[q] * a[6 * c + q];
        }
        const double pv = x[r] - v;
        Px[r] = pv;
        if (dotv) prod = pv * dotv[r];
    }
    if (!partial) return;
    red[threadIdx.x] = prod;
    __syncthreads();
    for (int o = blockDim.x / 2; o > 0; o >>= 1) {
        if (threadIdx.x < o) red[threadIdx.x] += red[threadIdx.x + o];
        __syncthreads();
    }
    if (threadIdx.x == 0) partial[blockIdx.x] = red[0];
}

// lambda = G a  (initial lambda0 = Gf (GfTGf)^{-1} e)
__global__ void k_gf_mult(int nlam, const int *__restrict__ gcl, const double *__restrict__ gval,
                          const double *__restrict__ a, double *__restrict__ out) {
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= nlam) return;
    double v = 0.0;
    for (int k = 0; k < 2; ++k) {
        const int c = gcl[2 * r + k];
        if (c < 0) continue;
        const double *g = gval + 6 * (size_t)(2 * r + k);
        for (int q = 0; q < 6; ++q) v += g[q] * a[6 * c + q];
    }
    out[r] = v;
}

// ---------------------------------------------------------------------------
// PCPG scalar / vector updates (Cluster::pcpg, Cluster.cpp:1422-1450)
// ---------------------------------------------------------------------------
// after Fw and the partials of w.Fw: rho = -gPz / wFw ; lam += rho w ; g += rho Fw
__global__ void k_update_lam_g(int n, const double *__restrict__ partial, int np, const double *__restrict__ w,
                               const double *__restrict__ Fw, double *__restrict__ lam, double *__restrict__ g,
                               PcpgState *__restrict__ st) {
    if (st->done) return;
    __shared__ double rho_s;
    const double wFw = block_sum_fixed(partial, np);
    if (threadIdx.x == 0) {
        double rho = -st->gPz / wFw;
        if (!(wFw > 0.0) || !isfinite(rho)) rho = 0.0;
        rho_s = rho;
        if (blockIdx.x == 0) {
            st->wFw = wFw;
            st->rho = rho;
        }
    }
    __syncthreads();
    const double rho = rho_s;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        lam[i] += rho * w[i];
        g[i] += rho * Fw[i];
    }
}

// after Pz and the partials of g.Pz: gamma, w = Pz + gamma w, convergence test
__global__ void k_update_w(int n, const double *__restrict__ partial, int np, const double *__restrict__ Pz,
                           double *__restrict__ w, PcpgState *__restrict__ st) {
    if (st->done) return;
    __shared__ double gam_s;
    const double gPz = block_sum_fixed(partial, np);
    if (threadIdx.x == 0) gam_s = gPz / st->gPz;
    __syncthreads();
    const double gam = gam_s;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) w[i] = Pz[i] + gam * w[i];
    // st->gPz is committed by k_finish_iter, launched after this kernel
}

// end of one iteration: commit gPz/gamma, count it, test convergence; the
// relative residual sqrt(g'Pz)/sqrt(g0'Pz0) of iteration it goes to hist[it]
// (hist holds max_iter + 1 entries)
__global__ void k_finish_iter(const double *__restrict__ partial, int np, PcpgState *__restrict__ st,
                              double *__restrict__ hist) {
    if (st->done) return;
    const double gPz = block_sum_fixed(partial, np);
    if (threadIdx.x == 0) {
        st->gamma = gPz / st->gPz;
        st->gPz_prev = st->gPz;
        st->gPz = gPz;
        st->it += 1;
        st->rel = sqrt(gPz) / st->norm0;
        if (hist && st->it <= st->max_iter) hist[st->it] = st->rel;
        if (!(st->wFw > 0.0) || !isfinite(gPz)) st->done = 2;          // breakdown
        else if (sqrt(gPz) < st->eps * st->norm0) st->done = 1;        // converged
        else if (st->it >= st->max_iter) st->done = 3;                  // max_iter
    }
}

// initial state: norm0 = sqrt(g0.Pz0)
__global__ void k_init_state(const double *__restrict__ partial, int np, PcpgState *__restrict__ st, double eps,
                             int max_iter) {
    const double gPz = block_sum_fixed(partial, np);
    if (threadIdx.x == 0) {
        st->gPz = gPz;
        st->gPz_prev = gPz;
        st->norm0 = sqrt(gPz);
        st->rel = 1.0;
        st->it = 0;
        st->eps = eps;
        st->max_iter = max_iter;
        st->wFw = 1.0;
        st->done = (gPz > 0.0 && isfinite(gPz)) ? ((max_iter <= 0) ? 3 : 0) : (gPz == 0.0 ? 1 : 2);
    }
}

// generic: y = a*x + b*y on n entries
__global__ void k_axpby(int n, double a, const double *__restrict__ x, double b, double *__restrict__ y) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) y[i] = a * x[i] + b * y[i];
}

// ---------------------------------------------------------------------------
// Dirichlet preconditioner without the dense S_d (preconditioner =
// Dirichlet_implicit, the reference's Cluster.cpp:1082-1104 variant that
// keeps no explicit S_d): the factor of K_reg,d eliminates the interior
// first, so its trailing b-set columns hold L_bb with L_bb L_bb^T = S_reg =
// S_d + D_fix (D_fix = the original diagonal at the 6 fix DOFs).  y_b =
// S_d x_b = L_bb (L_bb^T x_b) - D_fix x_b, two passes over the b-set
// column panels of the resident factor, no S_d stored.
//   k_lbt_x: t = L_bb^T x_b, one CTA per (subdomain, 32-column block p):
//            4 warps over the 32-row blocks R >= p, lane l row 32 R + l,
//            32 column sums per lane, reduce-scatter, warps added in order;
//   k_lb_t:  y = L_bb t - D_fix x_b, one CTA per (subdomain, 32-row block R):
//            4 warps over the column blocks p <= R, warps added in order.
// Each block of L_bb is read once per pass, 32 contiguous rows of a column
// per warp load.  `blk` lists (subdomain, block) pairs.
// ---------------------------------------------------------------------------
__global__ void k_lbt_x(const int2 *__restrict__ blk, const SubDev *__restrict__ subs, const double *__restrict__ K,
                        const double *__restrict__ xb, double *__restrict__ tb, const PcpgState *__restrict__ st) {
    if (st && st->done) return;
    __shared__ double part[4][32];
    const int2 b = blk[blockIdx.x];
    const SubDev sd = subs[b.x];
    const int p = b.y, warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int cb = sd.nr + 32 * p;
    double acc[32];
#pragma unroll
    for (int j = 0; j < 32; ++j) acc[j] = 0.0;
    // the 32 columns are one factor panel: (r, cb + j) at pbase + j * ld + r
    const double *pbase = K + kcol(sd, cb);
    const long long ld = kld(sd, cb);
    for (int R = p + warp; R < sd.nt; R += 4) {
        const int r = sd.nr + 32 * R + lane;
        const double xr = xb[sd.xb_off + 32 * R + lane];
        const double *col = pbase + r;
#pragma unroll
        for (int j = 0; j < 32; ++j) {
            const double l = (R > p || lane >= j) ? col[j * ld] : 0.0;
            acc[j] += l * xr;
        }
    }
    reduce_scatter32(acc, lane);
    part[warp][lane] = acc[0];
    __syncthreads();
    if (warp == 0)
        tb[sd.xb_off + 32 * p + lane] = ((part[0][lane] + part[1][lane]) + part[2][lane]) + part[3][lane];
}

__global__ void k_lb_t(const int2 *__restrict__ blk, const SubDev *__restrict__ subs, const double *__restrict__ K,
                       const double *__restrict__ tb, const double *__restrict__ xb, double *__restrict__ yb,
                       const PcpgState *__restrict__ st) {
    if (st && st->done) return;
    __shared__ double part[4][32];
    const int2 b = blk[blockIdx.x];
    const SubDev sd = subs[b.x];
    const int R = b.y, warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int r = sd.nr + 32 * R + lane;
    double z = 0.0;
    for (int p = warp; p <= R; p += 4) {
        const int cb = sd.nr + 32 * p;
        const double tl = tb[sd.xb_off + 32 * p + lane];
        const double *col = K + kcol(sd, cb) + r;      // (r, cb + j) at col + j * ld
        const long long ld = kld(sd, cb);
#pragma unroll
        for (int j = 0; j < 32; ++j) {
            const double tj = __shfl_sync(FULL, tl, j);
            const double l = (p < R || lane >= j) ? col[j * ld] : 0.0;
            z += l * tj;
        }
    }
    part[warp][lane] = z;
    __syncthreads();
    if (warp == 0) {
        double y = ((part[0][lane] + part[1][lane]) + part[2][lane]) + part[3][lane];
#pragma unroll
        for (int k = 0; k < 6; ++k)
            if (sd.fix[k] == r) y -= sd.fix_diag[k] * xb[sd.xb_off + 32 * R + lane];
        yb[sd.xb_off + 32 * R + lane] = y;
    }
}

// ---------------------------------------------------------------------------
// Coarse solve s = M gc with the symmetric M stored once, as packed lower
// 32x32 tiles (tile (I, J), J <= I, at MT_off + I (I + 1) / 2 + J, row-major
// inside, diagonal tiles full): half the bytes of the dense M every F apply
// reads.  `mt` lists (cluster, tile row) pairs.
//   k_pack_M:      tiles of tile row I from the dense M (set-up);
//   k_msym_rows:   CTA (cluster, I), 4 warps over the tiles of row I: the
//                  direct product M_IJ x_J summed per warp then in warp
//                  order into D[I]; the transposed M_IJ^T x_I (J < I) of each
//                  tile into its own 32-value slot P[(I, J)];
//   k_msym_reduce: s_J = D[J] + sum over I > J of P[(I, J)], in I order.
// Every tile is read once and every sum has a fixed order.
// ---------------------------------------------------------------------------
__global__ void k_pack_M(const int2 *__restrict__ mt, const ClusterDev *__restrict__ cl,
                         const double *__restrict__ M, double *__restrict__ T) {
    const int2 b = mt[blockIdx.x];
    const ClusterDev c = cl[b.x];
    const int I = b.y;
    double *row = T + (c.MT_off + (long long)I * (I + 1) / 2) * TILE_ELEMS;
    for (int idx = threadIdx.x; idx < (I + 1) * TILE_ELEMS; idx += blockDim.x) {
        const int J = idx / TILE_ELEMS, e = idx % TILE_ELEMS, r = e / TILE, j = e % TILE;
        const int gr = TILE * I + r, gcn = TILE * J + j;
        row[idx] = (gr < c.ngc && gcn < c.ngc) ? M[c.M_off + gr + (size_t)gcn * c.ngc] : 0.0;
    }
}

__global__ void k_msym_rows(const int2 *__restrict__ mt, const ClusterDev *__restrict__ cl,
                            const double *__restrict__ T, const double *__restrict__ gc, double *__restrict__ D,
                            double *__restrict__ P, const PcpgState *__restrict__ st) {
    if (st && st->done) return;
    __shared__ double xI[TILE];
    __shared__ double part[4][TILE];
    const int2 b = mt[blockIdx.x];
    const ClusterDev c = cl[b.x];
    const int I = b.y, warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const double *g = gc + c.gc_off;
    if (threadIdx.x < TILE) xI[threadIdx.x] = (TILE * I + threadIdx.x < c.ngc) ? g[TILE * I + threadIdx.x] : 0.0;
    __syncthreads();
    const long long t0 = c.MT_off + (long long)I * (I + 1) / 2;
    double dir = 0.0;
    for (int J = warp; J <= I; J += 4) {
        const double *tp = T + (t0 + J) * TILE_ELEMS;
        double v[32];
#pragma unroll
        for (int r = 0; r < 32; ++r) v[r] = tp[r * TILE + lane];
        const double xJ = (TILE * J + lane < c.ngc) ? g[TILE * J + lane] : 0.0;
        double p[32];
        double col = 0.0;
#pragma unroll
        for (int r = 0; r < 32; ++r) {
            p[r] = v[r] * xJ;
            col += v[r] * xI[r];
        }
        reduce_scatter32(p, lane);
        dir += p[0];
        if (J < I) P[(t0 + J) * TILE + lane] = col;
    }
    part[warp][lane] = dir;
    __syncthreads();
    if (warp == 0)
        D[((long long)c.mt_row_off + I) * TILE + lane] = ((part[0][lane] + part[1][lane]) + part[2][lane]) + part[3][lane];
}

__global__ void k_msym_reduce(const int2 *__restrict__ mt, const ClusterDev *__restrict__ cl,
                              const double *__restrict__ D, const double *__restrict__ P, double *__restrict__ s,
                              const PcpgState *__restrict__ st) {
    if (st && st->done) return;
    const int2 b = mt[blockIdx.x];
    const ClusterDev c = cl[b.x];
    const int J = b.y, lane = threadIdx.x;
    double y = D[((long long)c.mt_row_off + J) * TILE + lane];
    for (int I = J + 1; I < c.mt; ++I) y += P[(c.MT_off + (long long)I * (I + 1) / 2 + J) * TILE + lane];
    if (TILE * J + lane < c.ngc) s[c.gc_off + TILE * J + lane] = y;
}

}  // namespace htf
