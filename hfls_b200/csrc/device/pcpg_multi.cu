// Batched PCPG kernels: K load cases at once, vectors RHS-interleaved
// (entry (row, j) at row*K + j), one PcpgState per load case.  Each load
// case follows Cluster::pcpg (Cluster.cpp:1363-1458) independently; the
// matrices are read once per iteration for all K.  Reductions are
// fixed-order (deterministic).
#include <cuda_fp16.h>
#include <cuda_runtime.h>
#include <cstdint>

#include "device.cuh"

namespace htf {

// D += A B on the FP64 tensor path: one 8x8x4 product per warp.  Fragments:
// a = A[g][t4], b = B[t4][g], (d0, d1) = D[g][2 t4], D[g][2 t4 + 1] with
// g = lane / 4, t4 = lane % 4.
__device__ __forceinline__ void dmma_8x8x4(double &d0, double &d1, double a, double b) {
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};"
                 : "+d"(d0), "+d"(d1)
                 : "d"(a), "d"(b));
}

// x_b = Bf^T w (optionally weighted; x_b itself only when xb != nullptr) for
// all K columns; also writes the X slabs of the tensor-core product: every
// column scaled by 2^EX_j (EX_j from the column's largest |w| times the bound
// xbound >= |x_b| / max|w|) as FP16 hi + lo, the hi plane (K rows x 64 B)
// then the lo plane, SWIZZLE_64B K-major.  One CTA per 32 consecutive slots
// (one K slab of one subdomain: b offsets and padded sizes are multiples of
// 32); the values go through shared memory so both outputs are written
// coalesced.
__global__ void k_gather_multi(int nslots, int K, const int *__restrict__ ptr, const int *__restrict__ ent,
                               const double *__restrict__ w, const double *__restrict__ weight,
                               double *__restrict__ xb, float *__restrict__ Xs, const unsigned *__restrict__ xmax,
                               float xbound) {
    __shared__ double vs[32 * 33];
    __shared__ int ex[32];
    const int i0 = blockIdx.x * 32;
    for (int o = threadIdx.x; o < 32 * K; o += blockDim.x) {
        const int il = o / K, j = o % K, i = i0 + il;
        double v = 0.0;
        if (i < nslots)
            for (int e = ptr[i]; e < ptr[i + 1]; ++e) {
                const int q = ent[e];
                const int lam = q >> 1;
                double a = w[(size_t)lam * K + j];
                if (weight) a *= weight[lam];
                v += (q & 1) ? -a : a;
            }
        if (xb && i < nslots) xb[(size_t)i * K + j] = v;
        vs[il * 33 + j] = v;
    }
    if (!Xs) return;
    if (threadIdx.x < K) ex[threadIdx.x] = tc_scale_exp(xmax[threadIdx.x], xbound);
    __syncthreads();
    // row j (load case) of each plane holds the 32 slots of this chunk, 64 bytes
    __half *hi = reinterpret_cast<__half *>(Xs + (size_t)i0 * K);
    __half *lo = hi + 32 * K;
    for (int o = threadIdx.x; o < 32 * K; o += blockDim.x) {
        const int j = o / 32, c = o % 32;
        const double v = ldexp(vs[c * 33 + j], ex[j]);
        const __half vh = __double2half(v);
        const uint32_t b = uint32_t(j * 64 + c * 2);
        const uint32_t bs = b ^ (((b >> 7) & 3u) << 4);
        hi[bs / 2] = vh;
        lo[bs / 2] = __double2half(v - (double)__half2float(vh));
    }
}

// Partial V_d^T x_b over the 128-row chunk ch of subdomain d:
// tpart[(t_off + q) * nch + ch][j] = sum_{i in chunk} V_d[i][q] x_b[i][j]
// for q < c + 6 (QN >= c + 6 columns computed).  32-row pieces of V (stored
// q-major in shared memory) and x_b are staged, the next piece prefetched
// into registers; the products run on the FP64 tensor path, warp w owning
// the 8x8 output tiles w, w + 8, ... (q band = tile % (QN/8)).  Row strides
// of 36 and K + 4 doubles keep the fragment loads free of bank conflicts.
// CTA (subdomain, chunk), 256 threads.
template <int K, int QN>
__global__ void __launch_bounds__(256) k_vt_multi(int nch, const SubDev *__restrict__ subs,
                                                  const double *__restrict__ Vbuf, const double *__restrict__ xb,
                                                  double *__restrict__ tpart) {
    constexpr int VS = 36, XS = K + 4;
    constexpr int T = QN * K / 512;                 // 8x8 tiles per warp
    constexpr int UX = 32 * K / 256, UV = QN / 8;   // staged values per thread
    __shared__ double Vs[QN * VS];                  // [q][ii]
    __shared__ double Xs[32 * XS];                  // [ii][j]
    const SubDev &sd = subs[blockIdx.x];
    const int ch = blockIdx.y;
    const int ncol = sd.c + 6;
    const int r_end = min(sd.nb, ch * 128 + 128);
    const double *V = Vbuf + sd.V_off;
    const double *x = xb + (size_t)sd.xb_off * K;
    const int warp = threadIdx.x / 32, lane = threadIdx.x % 32;
    const int g = lane >> 2, t4 = lane & 3;
    double acc[T][2];
#pragma unroll
    for (int u = 0; u < T; ++u) acc[u][0] = acc[u][1] = 0.0;
    double xr[UX], vr[UV];
    auto fetch = [&](int i0) {
#pragma unroll
        for (int u = 0; u < UX; ++u) {
            const int o = threadIdx.x + 256 * u, ii = o / K;
            xr[u] = (i0 + ii < r_end) ? x[(size_t)(i0 + ii) * K + (o % K)] : 0.0;
        }
#pragma unroll
        for (int u = 0; u < UV; ++u) {
            const int o = threadIdx.x + 256 * u, q = o / 32, ii = o % 32;
            vr[u] = (q < ncol && i0 + ii < r_end) ? V[(size_t)q * sd.nbp + i0 + ii] : 0.0;
        }
    };
    if (ch * 128 < r_end) fetch(ch * 128);
    for (int i0 = ch * 128; i0 < r_end; i0 += 32) {
#pragma unroll
        for (int u = 0; u < UX; ++u) {
            const int o = threadIdx.x + 256 * u;
            Xs[(o / K) * XS + o % K] = xr[u];
        }
#pragma unroll
        for (int u = 0; u < UV; ++u) {
            const int o = threadIdx.x + 256 * u;
            Vs[(o / 32) * VS + o % 32] = vr[u];
        }
        __syncthreads();
        if (i0 + 32 < r_end) fetch(i0 + 32);        // next piece in flight during the products
#pragma unroll
        for (int kk = 0; kk < 8; ++kk) {
#pragma unroll
            for (int u = 0; u < T; ++u) {
                const int tile = warp + 8 * u, qb = tile % (QN / 8), jb = tile / (QN / 8);
                const double av = Vs[(8 * qb + g) * VS + 4 * kk + t4];
                const double bv = Xs[(4 * kk + t4) * XS + 8 * jb + g];
                dmma_8x8x4(acc[u][0], acc[u][1], av, bv);
            }
        }
        __syncthreads();
    }
#pragma unroll
    for (int u = 0; u < T; ++u) {
        const int tile = warp + 8 * u, qb = tile % (QN / 8), jb = tile / (QN / 8);
        const int q = 8 * qb + g, j = 8 * jb + 2 * t4;
        if (q < ncol) {
            double *o = tpart + (((size_t)sd.t_off + q) * nch + ch) * K + j;
            o[0] = acc[u][0];
            o[1] = acc[u][1];
        }
    }
}
#define HTF_VT(K, QN) \
    template __global__ void k_vt_multi<K, QN>(int, const SubDev *, const double *, const double *, double *);
HTF_VT(16, 32)
HTF_VT(16, 64)
HTF_VT(16, 128)
HTF_VT(32, 32)
HTF_VT(32, 64)
#undef HTF_VT

// gc[q][j] = sum over the t entries of coarse row q and their row chunks
__global__ void k_gc_multi(int ngc_total, int K, int nch, const int *__restrict__ gptr, const int *__restrict__ gidx,
                           const double *__restrict__ tpart, double *__restrict__ gc) {
    const long long id = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (id >= (long long)ngc_total * K) return;
    const int q = int(id / K), j = int(id % K);
    double s = 0.0;
    for (int e = gptr[q]; e < gptr[q + 1]; ++e)
        for (int ch = 0; ch < nch; ++ch) s += tpart[((size_t)gidx[e] * nch + ch) * K + j];
    gc[(size_t)q * K + j] = s;
}

// S = M G per cluster (M symmetric ngc x ngc, G = gc ngc x K): CTA
// (cluster, 32-row block) of 128 threads; 32 x 64 tiles of M and 64-row
// tiles of G staged in shared memory, the next pair prefetched into
// registers.  Products on the FP64 tensor path: warp w owns rows
// 8w .. 8w + 7 and all K columns (K / 8 tiles sharing one A fragment).
template <int K>
__global__ void __launch_bounds__(128) k_coarse_multi(const ClusterDev *__restrict__ cl,
                                                      const double *__restrict__ Mbuf, const double *__restrict__ gc,
                                                      double *__restrict__ s) {
    constexpr int PK = 64, MS = PK + 4, GS = K + 4, NT = K / 8;
    constexpr int UM = 32 * PK / 128, UG = PK * K / 128;
    __shared__ double Ms[32 * MS];                  // [r][p]
    __shared__ double Gs[PK * GS];                  // [p][j]
    const ClusterDev c = cl[blockIdx.x];
    const int row0 = blockIdx.y * 32;
    if (row0 >= c.ngc) return;
    const double *M = Mbuf + c.M_off;
    const double *G = gc + (size_t)c.gc_off * K;
    const int warp = threadIdx.x / 32, lane = threadIdx.x % 32;
    const int g = lane >> 2, t4 = lane & 3;
    double acc[NT][2];
#pragma unroll
    for (int u = 0; u < NT; ++u) acc[u][0] = acc[u][1] = 0.0;
    double mr[UM], gr[UG];
    auto fetch = [&](int p0) {
#pragma unroll
        for (int u = 0; u < UM; ++u) {
            const int o = threadIdx.x + 128 * u, r = o / PK, pp = o % PK;
            mr[u] = (row0 + r < c.ngc && p0 + pp < c.ngc) ? M[(size_t)(row0 + r) * c.ngc + p0 + pp] : 0.0;
        }
#pragma unroll
        for (int u = 0; u < UG; ++u) {
            const int o = threadIdx.x + 128 * u, pp = o / K;
            gr[u] = (p0 + pp < c.ngc) ? G[(size_t)(p0 + pp) * K + (o % K)] : 0.0;
        }
    };
    fetch(0);
    for (int p0 = 0; p0 < c.ngc; p0 += PK) {
#pragma unroll
        for (int u = 0; u < UM; ++u) {
            const int o = threadIdx.x + 128 * u;
            Ms[(o / PK) * MS + o % PK] = mr[u];
        }
#pragma unroll
        for (int u = 0; u < UG; ++u) {
            const int o = threadIdx.x + 128 * u;
            Gs[(o / K) * GS + o % K] = gr[u];
        }
        __syncthreads();
        if (p0 + PK < c.ngc) fetch(p0 + PK);        // next tiles in flight during the products
#pragma unroll
        for (int kk = 0; kk < PK / 4; ++kk) {
            const double av = Ms[(8 * warp + g) * MS + 4 * kk + t4];
#pragma unroll
            for (int u = 0; u < NT; ++u)
                dmma_8x8x4(acc[u][0], acc[u][1], av, Gs[(4 * kk + t4) * GS + 8 * u + g]);
        }
        __syncthreads();
    }
    const int row = row0 + 8 * warp + g;
    if (row < c.ngc)
#pragma unroll
        for (int u = 0; u < NT; ++u) {
            double *o = s + ((size_t)c.gc_off + row) * K + 8 * u + 2 * t4;
            o[0] = acc[u][0];
            o[1] = acc[u][1];
        }
}
template __global__ void k_coarse_multi<16>(const ClusterDev *, const double *, const double *, double *);
template __global__ void k_coarse_multi<32>(const ClusterDev *, const double *, const double *, double *);

// per-block, per-column tree sum of prod over the block's rows (256 / K rows,
// threads j, j+K, ...) -> partial[block][j]
__device__ __forceinline__ void block_col_partial(double prod, int K, double *__restrict__ partial) {
    __shared__ double red[256];
    const int rows_per_block = 256 / K;
    const int lr = threadIdx.x / K, j = threadIdx.x % K;
    red[threadIdx.x] = prod;
    __syncthreads();
    for (int o = rows_per_block / 2; o > 0; o >>= 1) {
        if (lr < o) red[threadIdx.x] += red[threadIdx.x + o * K];
        __syncthreads();
    }
    if (lr == 0) partial[(size_t)blockIdx.x * K + j] = red[j];
}

// out[r][j] = wt[r] * sum_k sign * y[slot][j]; partial dot with dotv per
// (block, j).  Blocks stride over groups of 256 / K rows (fixed assignment,
// so the partials and their sums are the same on every run); each thread
// has the loads of two of its rows in flight and adds them in row order.
__device__ __forceinline__ double row_value(int r, int K, int j, const int *__restrict__ rslot,
                                            const double *__restrict__ rsign, const double *__restrict__ yb,
                                            const double *__restrict__ weight) {
    const int2 sl = reinterpret_cast<const int2 *>(rslot)[r];
    const double2 sg = reinterpret_cast<const double2 *>(rsign)[r];
    double v = 0.0;
    if (sl.x >= 0) v += sg.x * yb[(size_t)sl.x * K + j];
    if (sl.y >= 0) v += sg.y * yb[(size_t)sl.y * K + j];
    if (weight) v *= weight[r];
    return v;
}

// y_b -= V_d s_d for all K load cases of a batch vector: the coarse
// correction of the F apply (Cluster.cpp:1114-1188, y = F_d x_b - V_d s_d
// with V_d = [F_d Bc_d^T, -R_d], s_d the cluster coarse solution at the
// subdomain's Bc rows and alpha slot), after the tensor-core product so the
// product's CTAs end without an FP64 epilogue.  CTA (subdomain, 128-row
// chunk), a 128 x K by (c + 6) x K product: s_d staged in shared memory
// ((c + 6) K <= 2048 doubles, checked at set-up), V in chunks of 16 columns
// (coalesced column reads); thread (row group, case group) keeps 128 K / 256
// outputs in registers (rows rg + RG i, cases jg + JG c: conflict-free
// shared-memory reads), summed over the columns in order.
template <int K>
__global__ void __launch_bounds__(256, 2) k_correct_multi(const SubDev *__restrict__ subs,
                                                       const ClusterDev *__restrict__ cl,
                                                       const double *__restrict__ V, const int *__restrict__ bcr,
                                                       const double *__restrict__ s, double *__restrict__ yb) {
    constexpr int QC = 16;                            // V columns per shared-memory chunk
    constexpr int JG = K / 4;                         // case groups (4 cases per thread)
    constexpr int RG = 256 / JG;                      // row groups
    constexpr int RPT = 128 / RG;                     // rows per thread
    __shared__ double ss[2048];
    __shared__ double vs[QC][128];
    const SubDev &sd = subs[blockIdx.x];
    const int r0 = blockIdx.y * 128;
    if (r0 >= sd.nb) return;
    const int nc = sd.c + 6;
    const int gc_off = cl[sd.cluster].gc_off;
    for (int o = threadIdx.x; o < nc * K; o += blockDim.x) {
        const int q = o / K, j = o % K;
        const int pos = q < sd.c ? bcr[sd.bcr_off + q] : sd.alpha_pos + (q - sd.c);
        ss[o] = s[((size_t)gc_off + pos) * K + j];
    }
    const int rend = min(128, sd.nb - r0);
    const int jg = threadIdx.x % JG, rg = threadIdx.x / JG;
    const double *Vd = V + sd.V_off + r0;
    double acc[RPT][4];
#pragma unroll
    for (int i = 0; i < RPT; ++i)
#pragma unroll
        for (int c = 0; c < 4; ++c) acc[i][c] = 0.0;
    // the next V chunk is loaded into registers while the current one multiplies
    constexpr int VPT = QC * 128 / 256;               // V values per thread and chunk
    double vr[VPT];
    auto fetch = [&](int q0) {
#pragma unroll
        for (int u = 0; u < VPT; ++u) {
            const int o = threadIdx.x + 256 * u, q = o >> 7, r = o & 127;
            vr[u] = (q0 + q < nc && r < rend) ? Vd[(size_t)(q0 + q) * sd.nbp + r] : 0.0;
        }
    };
    fetch(0);
    // this thread's y entries, read now so their latency overlaps the products
    double yv[RPT][4];
#pragma unroll
    for (int i = 0; i < RPT; ++i) {
        const int row = rg + RG * i;
#pragma unroll
        for (int c = 0; c < 4; ++c)
            yv[i][c] = row < rend ? yb[((size_t)sd.xb_off + r0 + row) * K + jg + JG * c] : 0.0;
    }
    for (int q0 = 0; q0 < nc; q0 += QC) {
        const int qn = min(QC, nc - q0);
        __syncthreads();                              // s_d staged, the previous chunk consumed
#pragma unroll
        for (int u = 0; u < VPT; ++u) {
            const int o = threadIdx.x + 256 * u;
            vs[o >> 7][o & 127] = vr[u];
        }
        __syncthreads();
        if (q0 + QC < nc) fetch(q0 + QC);
        for (int q = 0; q < qn; ++q) {
            const double *sq = ss + (q0 + q) * K + jg;
            double sv[4];
#pragma unroll
            for (int c = 0; c < 4; ++c) sv[c] = sq[JG * c];
#pragma unroll
            for (int i = 0; i < RPT; ++i) {
                const double v = vs[q][rg + RG * i];
#pragma unroll
                for (int c = 0; c < 4; ++c) acc[i][c] += v * sv[c];
            }
        }
    }
#pragma unroll
    for (int i = 0; i < RPT; ++i) {
        const int row = rg + RG * i;
        if (row < rend) {
            double *y = yb + ((size_t)sd.xb_off + r0 + row) * K + jg;
#pragma unroll
            for (int c = 0; c < 4; ++c) y[JG * c] = yv[i][c] - acc[i][c];
        }
    }
}

template __global__ void k_correct_multi<16>(const SubDev *, const ClusterDev *, const double *, const int *,
                                             const double *, double *);
template __global__ void k_correct_multi<32>(const SubDev *, const ClusterDev *, const double *, const int *,
                                             const double *, double *);

__global__ void k_rows_multi(int nlam, int K, const int *__restrict__ rslot, const double *__restrict__ rsign,
                             const double *__restrict__ yb, const double *__restrict__ weight,
                             double *__restrict__ out, const double *__restrict__ dotv,
                             double *__restrict__ partial) {
    const int rows_per_block = 256 / K;
    const int lr = threadIdx.x / K, j = threadIdx.x % K;
    const int stride = gridDim.x * rows_per_block;
    double prod = 0.0;
    if (lr < rows_per_block)
        for (int r0 = blockIdx.x * rows_per_block; r0 < nlam; r0 += 2 * stride) {
            const int ra = r0 + lr, rb = r0 + stride + lr;
            const bool ha = ra < nlam, hb = rb < nlam;
            double va = 0.0, vb = 0.0, da = 0.0, db = 0.0;
            if (ha) va = row_value(ra, K, j, rslot, rsign, yb, weight);
            if (hb) vb = row_value(rb, K, j, rslot, rsign, yb, weight);
            if (dotv) {
                if (ha) da = dotv[(size_t)ra * K + j];
                if (hb) db = dotv[(size_t)rb * K + j];
            }
            if (ha) {
                out[(size_t)ra * K + j] = va;
                if (dotv) prod += va * da;
            }
            if (hb) {
                out[(size_t)rb * K + j] = vb;
                if (dotv) prod += vb * db;
            }
        }
    if (partial) block_col_partial(prod, K, partial);
}

// Gf^T x per chunk and column: partial[ch][q][j].  The chunk's row indices
// and Gf values are staged in shared memory 256 entries at a time; thread
// (lr, j) walks every (256/K)-th entry with eight x loads in flight, adding
// its entries in the order lr, lr + 256/K, ...; the 6 sums are then reduced
// over lr in one pass through shared memory.
__global__ void __launch_bounds__(256) k_gft_partial_multi(int K, const int *__restrict__ chunk_beg,
                                                           const int *__restrict__ chunk_end,
                                                           const int *__restrict__ crow,
                                                           const double *__restrict__ cval,
                                                           const double *__restrict__ x,
                                                           double *__restrict__ partial) {
    __shared__ double red[6 * 256];
    __shared__ double cs[6 * 256];
    __shared__ int rs[256];
    const int ch = blockIdx.x;
    const int j = threadIdx.x % K, nl = 256 / K, lr = threadIdx.x / K;
    const int beg = chunk_beg[ch], end = chunk_end[ch];
    double s[6] = {0, 0, 0, 0, 0, 0};
    for (int e0 = beg; e0 < end; e0 += 256) {
        const int n = min(256, end - e0);
        __syncthreads();                            // the previous stage is consumed
        if (threadIdx.x < n) rs[threadIdx.x] = crow[e0 + threadIdx.x];
        for (int o = threadIdx.x; o < 6 * n; o += 256) cs[o] = cval[6 * (size_t)e0 + o];
        __syncthreads();
        int e = lr;
        for (; e + 7 * nl < n; e += 8 * nl) {
            double xv[8];
#pragma unroll
            for (int u = 0; u < 8; ++u) xv[u] = x[(size_t)rs[e + u * nl] * K + j];
#pragma unroll
            for (int u = 0; u < 8; ++u) {
                const double *cv = cs + 6 * (e + u * nl);
#pragma unroll
                for (int q = 0; q < 6; ++q) s[q] += cv[q] * xv[u];
            }
        }
        for (; e < n; e += nl) {
            const double xv = x[(size_t)rs[e] * K + j];
#pragma unroll
            for (int q = 0; q < 6; ++q) s[q] += cs[6 * e + q] * xv;
        }
    }
#pragma unroll
    for (int q = 0; q < 6; ++q) red[q * 256 + threadIdx.x] = s[q];
    __syncthreads();
    for (int o = nl / 2; o > 0; o >>= 1) {
        if (lr < o)
#pragma unroll
            for (int q = 0; q < 6; ++q) red[q * 256 + threadIdx.x] += red[q * 256 + threadIdx.x + o * K];
        __syncthreads();
    }
    if (lr == 0)
#pragma unroll
        for (int q = 0; q < 6; ++q) partial[((size_t)ch * 6 + q) * K + j] = red[q * 256 + j];
}

// gt[c][i][j] = sum of the chunk partials of cluster c (fixed order); CTA per
// cluster, thread (i, j)
__global__ void k_gt_sum_multi(int K, const int *__restrict__ cl_chunk_ptr, const double *__restrict__ gpart,
                               double *__restrict__ gt) {
    const int c = blockIdx.x;
    for (int o = threadIdx.x; o < 6 * K; o += blockDim.x) {
        const int i = o / K, j = o % K;
        double s = 0.0;
        for (int chk = cl_chunk_ptr[c]; chk < cl_chunk_ptr[c + 1]; ++chk) s += gpart[((size_t)chk * 6 + i) * K + j];
        gt[((size_t)c * 6 + i) * K + j] = s;
    }
}

// a = (Gf^T Gf)^{-1} gt per column (gt = Gf^T x from k_gt_sum_multi); one
// CTA; alpha_out = -a when requested.
__global__ void k_gf_coef_multi(int K, int ncl, const double *__restrict__ invGtG, const double *__restrict__ gt,
                                double *__restrict__ a, double *__restrict__ alpha_out) {
    const int m = 6 * ncl;
    for (int o = threadIdx.x; o < m * K; o += blockDim.x) {
        const int q = o / K, j = o % K;
        double s = 0.0;
        for (int p = 0; p < m; ++p) s += invGtG[q + (size_t)p * m] * gt[p * K + j];
        a[o] = s;
        if (alpha_out) alpha_out[o] = -s;
    }
}

// Px = x - Gf a; partial dot with dotv per (block, j); blocks stride over
// row groups like k_rows_multi
__global__ void k_gf_apply_multi(int nlam, int K, const double *__restrict__ a, const int *__restrict__ gcl,
                                 const double *__restrict__ gval, const double *__restrict__ x,
                                 double *__restrict__ Px, const double *__restrict__ dotv,
                                 double *__restrict__ partial) {
    const int rows_per_block = 256 / K;
    const int lr = threadIdx.x / K, j = threadIdx.x % K;
    double prod = 0.0;
    for (int r0 = blockIdx.x * rows_per_block; r0 < nlam; r0 += gridDim.x * rows_per_block) {
        const int r = r0 + lr;
        if (lr < rows_per_block && r < nlam) {
            double v = 0.0;
            for (int k = 0; k < 2; ++k) {
                const int c = gcl[2 * r + k];
                if (c < 0) continue;
                const double *g = gval + 6 * (size_t)(2 * r + k);
#pragma unroll
                for (int q = 0; q < 6; ++q) v += g[q] * a[(6 * c + q) * K + j];
            }
            const double pv = x[(size_t)r * K + j] - v;
            Px[(size_t)r * K + j] = pv;
            if (dotv) prod += pv * dotv[(size_t)r * K + j];
        }
    }
    if (partial) block_col_partial(prod, K, partial);
}

// sum of partials of column j (fixed order), one CTA per column
__device__ double col_sum(const double *partial, int np, int K, int j) {
    __shared__ double red[256];
    double s = 0.0;
    for (int i = threadIdx.x; i < np; i += blockDim.x) s += partial[(size_t)i * K + j];
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

// per column: scalar = sum of partials -> out[j]
__global__ void k_colsum(const double *__restrict__ partial, int np, int K, double *__restrict__ out) {
    const double s = col_sum(partial, np, K, blockIdx.x);
    if (threadIdx.x == 0) out[blockIdx.x] = s;
}

// rho_j = -gPz_j / wFw_j ; lam += rho w ; g += rho Fw  (skips finished columns)
__global__ void k_update_lam_g_multi(int n, int K, const double *__restrict__ wFw, const double *__restrict__ gw,
                                     const double *__restrict__ w, const double *__restrict__ Fw,
                                     double *__restrict__ lam, double *__restrict__ g, PcpgState *__restrict__ st) {
    const long long id = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (id >= (long long)n * K) return;
    const int j = int(id % K);
    if (st[j].done) return;
    // step length -g'w / w'Fw: equal to -g'Pz / w'Fw in exact arithmetic, and
    // still the exact line minimum along w after the residual g has been
    // replaced by the FP64 one
    const double d = wFw[j];
    double rho = -gw[j] / d;
    if (!(d > 0.0) || !isfinite(rho)) rho = 0.0;
    lam[id] += rho * w[id];
    g[id] += rho * Fw[id];
}

// partial[blk][j] = sum over the rows of block blk of a[r][j] * b[r][j]
// (row groups of 256 / K rows, strided like k_rows_multi)
__global__ void k_dot_multi(int nlam, int K, const double *__restrict__ a, const double *__restrict__ b,
                            double *__restrict__ partial) {
    const int rows_per_block = 256 / K;
    const int lr = threadIdx.x / K, j = threadIdx.x % K;
    double prod = 0.0;
    for (int r0 = blockIdx.x * rows_per_block; r0 < nlam; r0 += gridDim.x * rows_per_block) {
        const int r = r0 + lr;
        if (lr < rows_per_block && r < nlam) prod += a[(size_t)r * K + j] * b[(size_t)r * K + j];
    }
    block_col_partial(prod, K, partial);
}

__global__ void k_update_w_multi(int n, int K, const double *__restrict__ gPz_new, const double *__restrict__ Pz,
                                 double *__restrict__ w, const PcpgState *__restrict__ st) {
    const long long id = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (id >= (long long)n * K) return;
    const int j = int(id % K);
    if (st[j].done) return;
    w[id] = Pz[id] + (gPz_new[j] / st[j].gPz) * w[id];
}

__global__ void k_finish_multi(int K, const double *__restrict__ wFw, const double *__restrict__ gPz_new,
                               PcpgState *__restrict__ st) {
    const int j = threadIdx.x;
    if (j >= K || st[j].done) return;
    const double gPz = gPz_new[j];
    st[j].wFw = wFw[j];
    st[j].gamma = gPz / st[j].gPz;
    st[j].gPz_prev = st[j].gPz;
    st[j].gPz = gPz;
    st[j].it += 1;
    st[j].rel = sqrt(gPz) / st[j].norm0;
    if (!(wFw[j] > 0.0) || !isfinite(gPz)) st[j].done = 2;   // hand back to the FP64 residual check
    else if (sqrt(gPz) < st[j].eps * st[j].norm0) st[j].done = 1;
    else if (st[j].it >= st[j].max_iter) st[j].done = 3;
}

// strided column copy between a batch vector (stride K) and a plain vector
__global__ void k_col_get(int n, int K, int j, const double *__restrict__ B, double *__restrict__ v) {
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r < n) v[r] = B[(size_t)r * K + j];
}
__global__ void k_col_set(int n, int K, int j, const double *__restrict__ v, double *__restrict__ B) {
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r < n) B[(size_t)r * K + j] = v[r];
}

}  // namespace htf

namespace htf {

// ---------------------------------------------------------------------------
// FP64 residual of several load cases at once (the reliable-update step of
// the batched form): y_b(:, j) = A_d x_b(:, j) from the packed FP64 tiles for
// the K columns of a batch vector.  One CTA per (subdomain, 32-row block I)
// sums the tiles of block row I and, transposed, of block column I, so each
// output row is written once and no partial sums are needed.  The products
// run on the FP64 tensor path (mma.sync m8n8k4 .f64): warp w owns the 8-row
// band w mod 4 and K/16 column bands of 8; shared-memory row strides keep
// both operand loads free of bank conflicts.  With s given (the F apply),
// the coarse correction y_b -= V_d s_d is applied before the store.
// ---------------------------------------------------------------------------

template <int K>
__global__ void __launch_bounds__(256) k_symv_rows_multi(const int2 *__restrict__ rowblk,
                                                         const SubDev *__restrict__ subs,
                                                         const double *__restrict__ tiles,
                                                         const double *__restrict__ xb, double *__restrict__ yb,
                                                         const ClusterDev *__restrict__ cl,
                                                         const double *__restrict__ Vbuf,
                                                         const int *__restrict__ bcrows,
                                                         const double *__restrict__ s) {
    constexpr int NT = K / 16;                      // 8x8 output tiles per warp
    constexpr int TS = 36, XS = K + 4;              // row strides (doubles): conflict-free fragment loads
    __shared__ double Ts[32 * TS];
    __shared__ double Xs[32 * XS];
    const int2 rb = rowblk[blockIdx.x];
    const SubDev &sd = subs[rb.x];
    const int I = rb.y;
    const int warp = threadIdx.x / 32, lane = threadIdx.x % 32;
    const int g = lane >> 2, t4 = lane & 3;         // fragment row / column groups
    const int band = warp & 3, cb0 = (warp >> 2) * NT;
    const double *base = tiles + sd.T_off * TILE_ELEMS;
    double acc[NT][2];
#pragma unroll
    for (int q = 0; q < NT; ++q) acc[q][0] = acc[q][1] = 0.0;
    for (int J = 0; J < sd.nt; ++J) {
        const bool lower = J <= I;
        const double *tp = base + (lower ? (long long)I * (I + 1) / 2 + J : (long long)J * (J + 1) / 2 + I) * TILE_ELEMS;
        for (int e = threadIdx.x; e < TILE_ELEMS; e += blockDim.x) {
            const int rr = e / TILE, cc = e % TILE;
            const double v = tp[e];                 // stored tile, row rr, column cc
            if (lower) Ts[rr * TS + cc] = v;        // A[32I + rr][32J + cc]
            else Ts[cc * TS + rr] = v;              // tile (J, I): A[32I + cc][32J + rr]
        }
        for (int e = threadIdx.x; e < TILE * K; e += blockDim.x) {
            const int c = e / K, j = e % K;
            Xs[c * XS + j] = xb[(size_t)(sd.xb_off + TILE * J + c) * K + j];
        }
        __syncthreads();
#pragma unroll
        for (int kk = 0; kk < TILE / 4; ++kk) {
            const double a = Ts[(8 * band + g) * TS + 4 * kk + t4];
#pragma unroll
            for (int q = 0; q < NT; ++q) {
                const double b = Xs[(4 * kk + t4) * XS + 8 * (cb0 + q) + g];
                dmma_8x8x4(acc[q][0], acc[q][1], a, b);
            }
        }
        __syncthreads();
    }
    const int row = TILE * I + 8 * band + g;        // this thread's output row
    if (s && row < sd.nb) {
        const int gc_off = cl[sd.cluster].gc_off;
        const double *Vr = Vbuf + sd.V_off + row;
        for (int q = 0; q < sd.c + 6; ++q) {
            const double v = Vr[(size_t)q * sd.nbp];
            const int pos = q < sd.c ? bcrows[sd.bcr_off + q] : sd.alpha_pos + (q - sd.c);
            const double *sq = s + ((size_t)gc_off + pos) * K;
#pragma unroll
            for (int u = 0; u < NT; ++u) {
                const int col = 8 * (cb0 + u) + 2 * t4;
                acc[u][0] -= v * sq[col];
                acc[u][1] -= v * sq[col + 1];
            }
        }
    }
    double *y = yb + (size_t)(sd.xb_off + row) * K;
#pragma unroll
    for (int u = 0; u < NT; ++u) {
        const int col = 8 * (cb0 + u) + 2 * t4;
        y[col] = acc[u][0];
        y[col + 1] = acc[u][1];
    }
}
template __global__ void k_symv_rows_multi<16>(const int2 *, const SubDev *, const double *, const double *, double *,
                                               const ClusterDev *, const double *, const int *, const double *);
template __global__ void k_symv_rows_multi<32>(const int2 *, const SubDev *, const double *, const double *, double *,
                                               const ClusterDev *, const double *, const int *, const double *);

// B(:, j) = A(:, j) for the columns j with mask[j] (n rows, K-interleaved)
__global__ void k_cols_copy(long long n, int K, const int *__restrict__ mask, const double *__restrict__ A,
                            double *__restrict__ B) {
    for (long long o = blockIdx.x * (long long)blockDim.x + threadIdx.x; o < n * K;
         o += (long long)gridDim.x * blockDim.x)
        if (mask[o % K]) B[o] = A[o];
}

// per-column alpha (m values per column, column-major) of the columns with
// mask[j] from the projector's K-interleaved output
__global__ void k_alpha_cols(int m, int K, const int *__restrict__ mask, const double *__restrict__ a,
                             double *__restrict__ alpha) {
    for (int o = threadIdx.x; o < m * K; o += blockDim.x) {
        const int q = o / K, j = o % K;
        if (mask[j]) alpha[(size_t)j * m + q] = a[o];
    }
}

}  // namespace htf
