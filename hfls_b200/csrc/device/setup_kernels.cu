// Setup kernels of the HTFETI path (FP64, sm_100a).
//
//  k_assemble        hex8 element stiffness (2x2x2 Gauss) and body-force
//                    load, scattered into the dense permuted K_d; elements of
//                    one colour share no node, so no atomics are needed.
//                    Restates Data::stf_mtrx_solid45 (Data.cpp:297-490) with
//                    the standard J^{-T} gradient and Data::feti_numeric
//                    (Data.cpp:231-273).
//  k_potrf_diag /    step-synchronous batched right-looking Cholesky: one
//  k_trsm_panel /    launch per 32-column step covers every subdomain that
//  k_syrk_update     still has that step (replaces the PARDISO factorisation
//                    of K_reg, Matrix.cpp:1115-1202).
//  k_snapshot        copies S_reg - D_fix (Dirichlet) or K_bb (lumped) of the
//                    trailing block into packed tiles (Matrix.cpp:1708-1871).
//  k_trtri_step      X = L_bb^{-1}, one launch per 32-row block.
//  k_lauum_tiles     F = X^T X = (K_reg^{-1})_bb into packed tiles.
//  k_build_V/Fc      V = [F Bc_b^T, -R_b] and Fc_d = Bc_b F Bc_b^T
//                    (Cluster.cpp:150-185).
//  k_trsv_fwd/bwd    batched dense triangular solves with the full factor.
#include <cuda_runtime.h>
#include <cstdint>

#include "device.cuh"

namespace htf {

// ---------------------------------------------------------------------------
// assembly
// ---------------------------------------------------------------------------
__constant__ double c_gp[8][3];      // Gauss points (Data.cpp:363-386 order)

// Gauss points +-0.577350269189626 (the reference's literal, Data.cpp:344)
cudaError_t set_gauss_points(cudaStream_t s) {
    const double pt = 0.577350269189626;
    const double gr[8] = {-pt, -pt, -pt, -pt, pt, pt, pt, pt}, gs[8] = {-pt, -pt, pt, pt, -pt, -pt, pt, pt},
                 gt[8] = {-pt, pt, -pt, pt, -pt, pt, -pt, pt};
    double gp[8][3];
    for (int g = 0; g < 8; ++g) { gp[g][0] = gr[g]; gp[g][1] = gs[g]; gp[g][2] = gt[g]; }
    return cudaMemcpyToSymbolAsync(c_gp, gp, sizeof(gp), 0, cudaMemcpyHostToDevice, s);
}

__global__ void k_assemble(const int *__restrict__ elist, int count, const double *__restrict__ ecoord,
                           const int *__restrict__ esub, const int *__restrict__ eperm,
                           const double *__restrict__ subE, const double *__restrict__ subnu,
                           const SubDev *__restrict__ subs, double *__restrict__ Kbuf,
                           double *__restrict__ fbuf, double bfx, double bfy, double bfz) {
    __shared__ double G[8][8][3];    // dN_a/dx_k at Gauss point g
    __shared__ double Nw[8][8];      // N_a * detJ
    __shared__ double W[8];          // detJ
    __shared__ int P[24];
    __shared__ double X[8][3];
    const int e = elist[blockIdx.x];
    const int t = threadIdx.x;
    if (t < 24) {
        X[t / 3][t % 3] = ecoord[24 * (size_t)e + t];
        P[t] = eperm[24 * (size_t)e + t];
    }
    __syncthreads();
    if (t < 8) {
        const double r = c_gp[t][0], s = c_gp[t][1], q = c_gp[t][2];
        const double rn[8] = {-1, 1, 1, -1, -1, 1, 1, -1};
        const double sn[8] = {-1, -1, 1, 1, -1, -1, 1, 1};
        const double tn[8] = {-1, -1, -1, -1, 1, 1, 1, 1};
        double dNr[8], dNs[8], dNt[8], N[8];
        for (int a = 0; a < 8; ++a) {
            dNr[a] = 0.125 * rn[a] * (1. + sn[a] * s) * (1. + tn[a] * q);
            dNs[a] = 0.125 * sn[a] * (1. + rn[a] * r) * (1. + tn[a] * q);
            dNt[a] = 0.125 * tn[a] * (1. + rn[a] * r) * (1. + sn[a] * s);
            N[a] = 0.125 * (1. + rn[a] * r) * (1. + sn[a] * s) * (1. + tn[a] * q);
        }
        // M[i][j] = d x_i / d r_j
        double M[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
        for (int a = 0; a < 8; ++a)
            for (int i = 0; i < 3; ++i) {
                M[i][0] += dNr[a] * X[a][i];
                M[i][1] += dNs[a] * X[a][i];
                M[i][2] += dNt[a] * X[a][i];
            }
        const double det = M[0][0] * (M[1][1] * M[2][2] - M[1][2] * M[2][1]) -
                           M[0][1] * (M[1][0] * M[2][2] - M[1][2] * M[2][0]) +
                           M[0][2] * (M[1][0] * M[2][1] - M[1][1] * M[2][0]);
        const double id = 1.0 / det;
        // Mi = M^{-1}: Mi[j][i] = d r_j / d x_i
        double Mi[3][3];
        Mi[0][0] = (M[1][1] * M[2][2] - M[1][2] * M[2][1]) * id;
        Mi[0][1] = -(M[0][1] * M[2][2] - M[0][2] * M[2][1]) * id;
        Mi[0][2] = (M[0][1] * M[1][2] - M[0][2] * M[1][1]) * id;
        Mi[1][0] = -(M[1][0] * M[2][2] - M[1][2] * M[2][0]) * id;
        Mi[1][1] = (M[0][0] * M[2][2] - M[0][2] * M[2][0]) * id;
        Mi[1][2] = -(M[0][0] * M[1][2] - M[0][2] * M[1][0]) * id;
        Mi[2][0] = (M[1][0] * M[2][1] - M[1][1] * M[2][0]) * id;
        Mi[2][1] = -(M[0][0] * M[2][1] - M[0][1] * M[2][0]) * id;
        Mi[2][2] = (M[0][0] * M[1][1] - M[0][1] * M[1][0]) * id;
        for (int a = 0; a < 8; ++a) {
            for (int i = 0; i < 3; ++i)      // dN/dx_i = sum_j dN/dr_j * dr_j/dx_i
                G[t][a][i] = dNr[a] * Mi[0][i] + dNs[a] * Mi[1][i] + dNt[a] * Mi[2][i];
            Nw[t][a] = N[a] * det;
        }
        W[t] = det;
    }
    __syncthreads();
    const int d = esub[e];
    const SubDev sd = subs[d];
    const double E = subE[d], nu = subnu[d];
    const double lam = E * nu / ((1. + nu) * (1. - 2. * nu));
    const double mu = E / (2. * (1. + nu));
    for (int idx = t; idx < 576; idx += blockDim.x) {
        const int I = idx % 24, J = idx / 24;
        const int pI = P[I], pJ = P[J];
        if (pI < pJ) continue;                      // lower triangle in permuted order
        const int i = I >> 3, a = I & 7, j = J >> 3, b = J & 7;
        double v = 0.0;
        for (int g = 0; g < 8; ++g) {
            double s = lam * G[g][a][i] * G[g][b][j] + mu * G[g][a][j] * G[g][b][i];
            if (i == j) s += mu * (G[g][a][0] * G[g][b][0] + G[g][a][1] * G[g][b][1] + G[g][a][2] * G[g][b][2]);
            v += s * W[g];
        }
        Kbuf[kidx(sd, pI, pJ)] += v;
    }
    if (fbuf && t < 24) {             // no fbuf: a re-assembly of the factor alone
        const int i = t >> 3, a = t & 7;
        const double bf = (i == 0) ? bfx : (i == 1) ? bfy : bfz;
        double v = 0.0;
        for (int g = 0; g < 8; ++g) v += bf * Nw[g][a];
        fbuf[sd.nfull_off + P[t]] += v;
    }
}

// K_reg = K + D_fix: double the diagonal at the fix DOFs (Matrix.cpp:1029-1057)
// and put the identity on the padded rows.
__global__ void k_regularize(SubDev *subs, int nsub, double *Kbuf) {
    const int d = blockIdx.x;
    if (d >= nsub) return;
    SubDev &sd = subs[d];
    if (threadIdx.x < 6) {
        const int f = sd.fix[threadIdx.x];
        const long long a = kidx(sd, f, f);
        const double v = Kbuf[a];
        sd.fix_diag[threadIdx.x] = v;
        Kbuf[a] = 2.0 * v;
    }
    for (int r = sd.nr + sd.nb + threadIdx.x; r < sd.N; r += blockDim.x) Kbuf[kidx(sd, r, r)] = 1.0;
}

// ---------------------------------------------------------------------------
// batched Cholesky steps of up to CHOL_STEP = 64 columns (two 32-column factor
// panels): the diagonal block in one CTA, the panel below it one row per
// thread, the trailing update keeping one accumulator per 32-column panel and
// subtracting them in turn in registers, so each trailing tile is read and
// written once per 64 columns.  The arithmetic is that of two successive
// 32-column right-looking steps (per panel: Cholesky of the diagonal block,
// row-wise substitution with division by the pivot, block update subtracting
// a 32-term sum), operation for operation.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(CHOL_STEP) k_potrf_diag(const StepDesc *__restrict__ st,
                                                          const SubDev *__restrict__ subs,
                                                          double *__restrict__ Kbuf, int *__restrict__ status) {
    __shared__ double A[CHOL_STEP][CHOL_STEP + 1];
    __shared__ int bad;
    const StepDesc s = st[blockIdx.x];
    const SubDev &sd = subs[s.d];
    const int k = s.k, nb = s.nb, t = threadIdx.x;
    if (t == 0) bad = 0;
    for (int c = 0; c < nb; ++c) {
        const double *col = Kbuf + kcol(sd, k + c);
        A[t][c] = (t < nb && t >= c) ? col[k + t] : 0.0;
    }
    __syncthreads();
    // Cholesky of the 32-column diagonal block starting at column o (rows o .. e-1)
    auto potrf32 = [&](int o, int e) {
        for (int j = o; j < e; ++j) {
            if (t == j) {
                double dj = A[j][j];
                if (!(dj > 0.0)) {
                    if (!bad) bad = k + j + 1;
                    dj = 1.0;
                }
                A[j][j] = sqrt(dj);
            }
            __syncthreads();
            const double dj = A[j][j];
            if (t > j && t < e) A[t][j] /= dj;
            __syncthreads();
            if (t > j && t < e) {
                const double lj = A[t][j];
                for (int c = j + 1; c <= t; ++c) A[t][c] -= lj * A[c][j];
            }
            __syncthreads();
        }
    };
    const int n1 = min(nb, TILE);
    potrf32(0, n1);
    if (nb > TILE) {
        if (t >= TILE && t < nb) {              // rows of the second panel: substitution with the first
            for (int j = 0; j < TILE; ++j) {
                double v = A[t][j];
                for (int i = 0; i < j; ++i) v -= A[t][i] * A[j][i];
                A[t][j] = v / A[j][j];
            }
        }
        __syncthreads();
        if (t >= TILE && t < nb) {              // block update of the second diagonal block
            for (int c = TILE; c <= t; ++c) {
                double acc = 0.0;
                for (int i = 0; i < TILE; ++i) acc += A[t][i] * A[c][i];
                A[t][c] -= acc;
            }
        }
        __syncthreads();
        potrf32(TILE, nb);
    }
    if (t == 0 && bad) atomicCAS(&status[s.d], 0, bad);
    for (int c = 0; c < nb; ++c) {
        double *col = Kbuf + kcol(sd, k + c);
        if (t < nb && t >= c) col[k + t] = A[t][c];
    }
}

// rows below the diagonal block: x = x L_kk^{-T}, one row per thread
// grid: the step's row blocks of 128 (flattened over its entries)
__global__ void __launch_bounds__(128) k_trsm_panel(const StepDesc *__restrict__ st, int cnt,
                                                    const SubDev *__restrict__ subs, double *__restrict__ Kbuf,
                                                    const int *__restrict__ hint) {
    __shared__ double L[CHOL_STEP][CHOL_STEP + 1];
    const int e = step_entry(st, cnt, int(blockIdx.x), [](const StepDesc &x) { return x.rb0; }, hint);
    const StepDesc s = st[e];
    const int rb = int(blockIdx.x) - s.rb0;
    const SubDev &sd = subs[s.d];
    const int N = sd.N, k = s.k, nb = s.nb;
    for (int i = threadIdx.x; i < CHOL_STEP * CHOL_STEP; i += blockDim.x) {
        const int r = i % CHOL_STEP, c = i / CHOL_STEP;
        L[r][c] = (r < nb && c < nb && c <= r) ? Kbuf[kidx(sd, k + r, k + c)] : 0.0;
    }
    __syncthreads();
    const int row = k + nb + rb * blockDim.x + threadIdx.x;
    if (row >= N) return;
    const long long c0 = kcol(sd, k), c1 = kcol(sd, k + TILE);     // the step's two panels
    const long long ld0 = kld(sd, k), ld1 = kld(sd, k + TILE);
    double x[CHOL_STEP];
#pragma unroll
    for (int j = 0; j < CHOL_STEP; ++j)
        x[j] = (j < nb) ? Kbuf[(j < TILE ? c0 + (long long)j * ld0 : c1 + (long long)(j - TILE) * ld1) + row] : 0.0;
#pragma unroll
    for (int j = 0; j < TILE; ++j) {
        if (j < nb) {
            double v = x[j];
#pragma unroll
            for (int i = 0; i < j; ++i) v -= x[i] * L[j][i];
            x[j] = v / L[j][j];
        }
    }
    if (nb > TILE) {
#pragma unroll
        for (int j = TILE; j < CHOL_STEP; ++j) {       // block update by the first panel
            if (j < nb) {
                double acc = 0.0;
#pragma unroll
                for (int i = 0; i < TILE; ++i) acc += x[i] * L[j][i];
                x[j] -= acc;
            }
        }
#pragma unroll
        for (int j = TILE; j < CHOL_STEP; ++j) {
            if (j < nb) {
                double v = x[j];
#pragma unroll
                for (int i = TILE; i < j; ++i) v -= x[i] * L[j][i];
                x[j] = v / L[j][j];
            }
        }
    }
#pragma unroll
    for (int j = 0; j < CHOL_STEP; ++j)
        if (j < nb) Kbuf[(j < TILE ? c0 + (long long)j * ld0 : c1 + (long long)(j - TILE) * ld1) + row] = x[j];
}

// C(64x64 block, lower part of the trailing matrix) -= P_i P_j^T, P = the
// step's panel rows; 32 columns of P at a time, one accumulator per panel,
// C read and written once.  The products run on the FP64 tensor path
// (mma.sync m8n8k4 .f64): warp w owns rows 32 (w / 4) .. +31 and columns
// 16 (w % 4) .. +15 of the block, 4 x 2 tiles of 8 x 8, so per k-group of 4
// a warp loads 6 operand fragments for 8 MMAs (the CUDA-core form loaded 8
// values per 16 FMAs per thread and was bound by shared-memory loads).  A
// row stride of 68 doubles keeps both fragment loads free of bank
// conflicts.  All loads are cp.async into shared memory, issued at the start
// in three groups (panel 0, panel 1, the C block), so panel 1 and C land
// while panel 0 multiplies.  grid: the step's trailing tiles (flattened);
// dynamic shared memory SYRK_SMEM.
__device__ __forceinline__ void dmma_syrk(double &d0, double &d1, double a, double b) {
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};"
                 : "+d"(d0), "+d"(d1)
                 : "d"(a), "d"(b));
}

// 8-byte asynchronous copy global -> shared; src_bytes 0 writes a zero
__device__ __forceinline__ void cp_async8(double *dst, const double *src, int src_bytes) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;" ::"r"(
                     static_cast<unsigned>(__cvta_generic_to_shared(dst))),
                 "l"(src), "r"(src_bytes)
                 : "memory");
}

__global__ void __launch_bounds__(256) k_syrk_update(const StepDesc *__restrict__ st, int cnt,
                                                     const SubDev *__restrict__ subs,
                                                     double *__restrict__ Kbuf, const int *__restrict__ hint) {
    constexpr int LDP = 68, LDC = 65;
    extern __shared__ double syrk_sm[];
    double(*Pa)[32][LDP] = reinterpret_cast<double(*)[32][LDP]>(syrk_sm);                 // [2][32][LDP]
    double(*Pb)[32][LDP] = reinterpret_cast<double(*)[32][LDP]>(syrk_sm + 2 * 32 * LDP);  // [2][32][LDP]
    double *Cs = syrk_sm + 4 * 32 * LDP;                                                    // [64 cols][LDC]
    const int e = step_entry(st, cnt, int(blockIdx.x), [](const StepDesc &x) { return x.tri0; }, hint);
    const StepDesc s = st[e];
    const SubDev &sd = subs[s.d];
    const int N = sd.N, k = s.k, nb = s.nb;
    const int t0 = k + nb;                  // first trailing row/col
    const int m = N - t0;
    const int nbr = (m + 63) / 64;
    const int tri = int(blockIdx.x) - s.tri0;
    if (tri >= nbr * (nbr + 1) / 2) return;
    int bi = (int)((sqrt(8.0 * tri + 1.0) - 1.0) * 0.5);
    while ((bi + 1) * (bi + 2) / 2 <= tri) ++bi;
    while (bi * (bi + 1) / 2 > tri) --bi;
    const int bj = tri - bi * (bi + 1) / 2;
    const int i0 = t0 + 64 * bi, j0 = t0 + 64 * bj;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int g = lane >> 2, t4 = lane & 3;
    const int wr = 32 * (warp >> 2), wc = 16 * (warp & 3);
    const int nq = (nb + TILE - 1) / TILE;
    // groups 0, 1: the panels of the step's 32-column halves (zero outside)
#pragma unroll
    for (int q = 0; q < CHOL_STEP / TILE; ++q) {
        if (q >= nq) break;
        const int kc = TILE * q;
        const int kn = min(TILE, nb - kc);
        const double *P = Kbuf + kidx(sd, k + kc, k + kc);    // panel of columns k+kc..: entry (k+kc+i, k+kc+j) at P[i + j*ld]
        const long long ld = kld(sd, k + kc);
        for (int idx = threadIdx.x; idx < 32 * 64; idx += 256) {
            const int r = idx % 64, kk = idx / 64;
            const bool oka = kk < kn && i0 + r < N, okb = kk < kn && j0 + r < N;
            cp_async8(&Pa[q][kk][r], oka ? P + (i0 + r - k - kc) + kk * ld : Kbuf, oka ? 8 : 0);
            cp_async8(&Pb[q][kk][r], okb ? P + (j0 + r - k - kc) + kk * ld : Kbuf, okb ? 8 : 0);
        }
        asm volatile("cp.async.commit_group;" ::: "memory");
    }
    // last group: the lower part of the C block (rows >= columns, inside the
    // matrix), needed only after the products
    for (int idx = threadIdx.x; idx < 64 * 64; idx += 256) {
        const int r = idx % 64, c = idx / 64;
        const int row = i0 + r, col = j0 + c;
        const bool ok = row < N && col < N && row >= col;
        cp_async8(&Cs[c * LDC + r], ok ? Kbuf + kcol(sd, col) + row : Kbuf, ok ? 8 : 0);
    }
    asm volatile("cp.async.commit_group;" ::: "memory");
    double acc[CHOL_STEP / TILE][4][2][2];
#pragma unroll
    for (int q = 0; q < CHOL_STEP / TILE; ++q)
#pragma unroll
        for (int a = 0; a < 4; ++a)
#pragma unroll
            for (int b = 0; b < 2; ++b) acc[q][a][b][0] = acc[q][a][b][1] = 0.0;
#pragma unroll
    for (int q = 0; q < CHOL_STEP / TILE; ++q) {
        if (q >= nq) break;
        // panel q (and everything committed before it) has landed; the later
        // panel and the C block may still be in flight
        if (q + 1 < nq) asm volatile("cp.async.wait_group 2;" ::: "memory");
        else asm volatile("cp.async.wait_group 1;" ::: "memory");
        __syncthreads();
        const int kn = min(TILE, nb - TILE * q);
        const int kgs = (kn + 3) >> 2;
        for (int kg = 0; kg < kgs; ++kg) {
            const int kr = 4 * kg + t4;
            double av[4], bv[2];
#pragma unroll
            for (int a = 0; a < 4; ++a) av[a] = Pa[q][kr][wr + 8 * a + g];
#pragma unroll
            for (int b = 0; b < 2; ++b) bv[b] = Pb[q][kr][wc + 8 * b + g];
#pragma unroll
            for (int a = 0; a < 4; ++a)
#pragma unroll
                for (int b = 0; b < 2; ++b) dmma_syrk(acc[q][a][b][0], acc[q][a][b][1], av[a], bv[b]);
        }
    }
    asm volatile("cp.async.wait_group 0;" ::: "memory");    // the C block
    __syncthreads();
#pragma unroll
    for (int b = 0; b < 2; ++b)
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            const int cl = wc + 8 * b + 2 * t4 + h, col = j0 + cl;
            if (col >= N) continue;
            double *C = Kbuf + kcol(sd, col);
#pragma unroll
            for (int a = 0; a < 4; ++a) {
                const int rl = wr + 8 * a + g, row = i0 + rl;
                if (row >= N || row < col) continue;
                double c = Cs[cl * LDC + rl];
#pragma unroll
                for (int q = 0; q < CHOL_STEP / TILE; ++q)
                    if (q < nq) c -= acc[q][a][b][h];
                C[row] = c;
            }
        }
}

// Copy the trailing nbp x nbp block into packed tiles, minus the fix diagonal.
__global__ void k_snapshot(const int *__restrict__ dlist, const SubDev *__restrict__ subs,
                           const double *__restrict__ Kbuf, double *__restrict__ Sbuf, long long t0) {
    const SubDev &sd = subs[dlist[blockIdx.x]];
    const int tile = blockIdx.y;
    if (tile >= sd.nt * (sd.nt + 1) / 2) return;
    int I = (int)((sqrt(8.0 * tile + 1.0) - 1.0) * 0.5);
    while ((I + 1) * (I + 2) / 2 <= tile) ++I;
    while (I * (I + 1) / 2 > tile) --I;
    const int J = tile - I * (I + 1) / 2;
    double *T = Sbuf + (sd.T_off - t0 + tile) * TILE_ELEMS;     // Sbuf holds the tiles from t0 on
    for (int idx = threadIdx.x; idx < TILE_ELEMS; idx += blockDim.x) {
        const int r = idx / TILE, c = idx % TILE;
        int gr = sd.nr + TILE * I + r, gc = sd.nr + TILE * J + c;
        if (gr < gc) { int tmp = gr; gr = gc; gc = tmp; }
        double v = Kbuf[kidx(sd, gr, gc)];
        if (gr == gc)
            for (int q = 0; q < 6; ++q)
                if (sd.fix[q] == gr) v -= sd.fix_diag[q];
        T[idx] = v;
    }
}

// acc(32 x 32) += A Xs on the FP64 tensor path (mma.sync m8n8k4): A = Ls
// (TR = false) or Ls^T (TR = true); warp w owns the 8-row tile w / 2 and the
// 8-column tiles 2 (w % 2), 2 (w % 2) + 1 (d[ct][h]: row 8 (w / 2) + lane / 4,
// column 8 (2 (w % 2) + ct) + 2 (lane % 4) + h).  Row stride 36 doubles: the
// fragment loads are conflict-free.
template <bool TR>
__device__ __forceinline__ void trsm_block_mma(const double (*Ls)[36], const double (*Xs)[36], int w, int lane,
                                               double (&d)[2][2]) {
    const int g = lane >> 2, t4 = lane & 3, rt = w >> 1, ct0 = 2 * (w & 1);
#pragma unroll
    for (int kg = 0; kg < 8; ++kg) {
        const int kr = 4 * kg + t4;
        const double a = TR ? Ls[kr][8 * rt + g] : Ls[8 * rt + g][kr];
#pragma unroll
        for (int ct = 0; ct < 2; ++ct) {
            const double b = Xs[kr][8 * (ct0 + ct) + g];
            asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};"
                         : "+d"(d[ct][0]), "+d"(d[ct][1])
                         : "d"(a), "d"(b));
        }
    }
}

// the block products' fragments into acc[q] = row lane, column 4 w + q (T: 32 x 36 scratch)
__device__ __forceinline__ void trsm_gather(double (*T)[36], const double (&d)[2][2], int w, int lane,
                                            double (&acc)[4]) {
    const int g = lane >> 2, t4 = lane & 3, rt = w >> 1, ct0 = 2 * (w & 1);
#pragma unroll
    for (int ct = 0; ct < 2; ++ct)
#pragma unroll
        for (int h = 0; h < 2; ++h) T[8 * rt + g][8 * (ct0 + ct) + 2 * t4 + h] = d[ct][h];
    __syncthreads();
#pragma unroll
    for (int q = 0; q < 4; ++q) acc[q] = T[lane][4 * w + q];
    __syncthreads();
}

// ---------------------------------------------------------------------------
// X = L_bb^{-1}: block row i of X, all block columns j <= i
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256) k_trtri_step(int i, const int *__restrict__ dlist,
                                                    const SubDev *__restrict__ subs,
                                                    const double *__restrict__ Kbuf,
                                                    double *__restrict__ Xbuf) {
    __shared__ double La[32][36];
    __shared__ double Xb[32][36];
    __shared__ double T[32][36];
    const SubDev &sd = subs[dlist[blockIdx.x]];
    const int j = blockIdx.y;
    if (i >= sd.nt || j > i) return;
    const int N = sd.N, nbp = sd.nbp, base = sd.nr;
    double *X = Xbuf + sd.X_off;
    const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
    const int r = tid % 32, c0 = (tid / 32) * 4;
    (void)N;
    // sum_kb L_i,kb X_kb,j on the FP64 tensor path, then T = I - sum (block j = i) or -sum
    double d[2][2] = {{0.0, 0.0}, {0.0, 0.0}};
    for (int kb = j; kb < i; ++kb) {
        for (int idx = tid; idx < 1024; idx += 256) {
            const int rr = idx % 32, cc = idx / 32;
            La[rr][cc] = Kbuf[kidx(sd, base + 32 * i + rr, base + 32 * kb + cc)];
            Xb[rr][cc] = X[(32 * kb + rr) + (size_t)(32 * j + cc) * nbp];
        }
        __syncthreads();
        trsm_block_mma<false>(La, Xb, w, lane, d);
        __syncthreads();
    }
    double acc[4];
    trsm_gather(T, d, w, lane, acc);
#pragma unroll
    for (int cc = 0; cc < 4; ++cc) T[r][c0 + cc] = ((i == j && r == c0 + cc) ? 1.0 : 0.0) - acc[cc];
    for (int idx = tid; idx < 1024; idx += 256) {
        const int rr = idx % 32, cc = idx / 32;
        La[rr][cc] = (cc <= rr) ? Kbuf[kidx(sd, base + 32 * i + rr, base + 32 * i + cc)] : 0.0;
    }
    __syncthreads();
    if (tid < 32) {                        // forward substitution, one column per thread
        const int col = tid;
        for (int rr = 0; rr < 32; ++rr) {
            double v = T[rr][col];
            for (int q = 0; q < rr; ++q) v -= La[rr][q] * T[q][col];
            T[rr][col] = v / La[rr][rr];
        }
    }
    __syncthreads();
    for (int idx = tid; idx < 1024; idx += 256) {
        const int rr = idx % 32, cc = idx / 32;
        X[(32 * i + rr) + (size_t)(32 * j + cc) * nbp] = T[rr][cc];
    }
}

// F tile (I,J) = sum_{k >= I} X_kI^T X_kJ  (X lower triangular)
__global__ void __launch_bounds__(256) k_lauum_tiles(const int *__restrict__ dlist,
                                                     const SubDev *__restrict__ subs,
                                                     const double *__restrict__ Xbuf,
                                                     double *__restrict__ Fbuf) {
    __shared__ double A[32][36];
    __shared__ double B[32][36];
    const SubDev &sd = subs[dlist[blockIdx.x]];
    const int tile = blockIdx.y;
    if (tile >= sd.nt * (sd.nt + 1) / 2) return;
    int I = (int)((sqrt(8.0 * tile + 1.0) - 1.0) * 0.5);
    while ((I + 1) * (I + 2) / 2 <= tile) ++I;
    while (I * (I + 1) / 2 > tile) --I;
    const int J = tile - I * (I + 1) / 2;
    const double *X = Xbuf + sd.X_off;
    const int nbp = sd.nbp;
    const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
    // sum_kb X_kb,I^T X_kb,J on the FP64 tensor path (A = X_kb,I read transposed)
    double d[2][2] = {{0.0, 0.0}, {0.0, 0.0}};
    for (int kb = I; kb < sd.nt; ++kb) {
        for (int idx = tid; idx < 1024; idx += 256) {
            const int q = idx % 32, cc = idx / 32;
            A[q][cc] = X[(32 * kb + q) + (size_t)(32 * I + cc) * nbp];
            B[q][cc] = X[(32 * kb + q) + (size_t)(32 * J + cc) * nbp];
        }
        __syncthreads();
        trsm_block_mma<true>(A, B, w, lane, d);
        __syncthreads();
    }
    double *T = Fbuf + (sd.T_off + tile) * TILE_ELEMS;
    const int g = lane >> 2, t4 = lane & 3, rt = w >> 1, ct0 = 2 * (w & 1);
#pragma unroll
    for (int ct = 0; ct < 2; ++ct)
#pragma unroll
        for (int h = 0; h < 2; ++h) T[(8 * rt + g) * TILE + 8 * (ct0 + ct) + 2 * t4 + h] = d[ct][h];
}

// ---------------------------------------------------------------------------
// V = [F Bc_b^T, -R_b] and Fc_d = Bc_b V(:, 0:c)
// ---------------------------------------------------------------------------
__device__ __forceinline__ double tile_at(const double *F, const SubDev &sd, int i, int p) {
    int I = i / TILE, P = p / TILE;
    if (I >= P) return F[(sd.T_off + (long long)I * (I + 1) / 2 + P) * TILE_ELEMS + (i % TILE) * TILE + (p % TILE)];
    return F[(sd.T_off + (long long)P * (P + 1) / 2 + I) * TILE_ELEMS + (p % TILE) * TILE + (i % TILE)];
}

__global__ void k_build_V(const SubDev *__restrict__ subs, const double *__restrict__ Fbuf,
                          const int *__restrict__ bce_ptr, const int *__restrict__ bce_pos,
                          const double *__restrict__ bce_val, const double *__restrict__ Rbuf,
                          double *__restrict__ Vbuf) {
    const SubDev &sd = subs[blockIdx.x];
    const int col = blockIdx.y;
    if (col >= sd.c + 6) return;
    double *V = Vbuf + sd.V_off + (size_t)col * sd.nbp;
    if (col < sd.c) {
        const int e0 = bce_ptr[sd.bce_off + col], e1 = bce_ptr[sd.bce_off + col + 1];
        for (int i = threadIdx.x; i < sd.nbp; i += blockDim.x) {
            double v = 0.0;
            if (i < sd.nb)
                for (int e = e0; e < e1; ++e) v += bce_val[e] * tile_at(Fbuf, sd, i, bce_pos[e]);
            V[i] = v;
        }
    } else {
        const double *R = Rbuf + sd.R_off + (size_t)(col - sd.c) * sd.N;
        for (int i = threadIdx.x; i < sd.nbp; i += blockDim.x) V[i] = (i < sd.nb) ? -R[sd.nr + i] : 0.0;
    }
}

__global__ void k_build_Fc(const SubDev *__restrict__ subs, const double *__restrict__ Vbuf,
                           const int *__restrict__ bce_ptr, const int *__restrict__ bce_pos,
                           const double *__restrict__ bce_val, const long long *__restrict__ fc_off,
                           double *__restrict__ Fc) {
    const SubDev &sd = subs[blockIdx.x];
    const int c = sd.c;
    double *out = Fc + fc_off[blockIdx.x];
    for (int idx = threadIdx.x; idx < c * c; idx += blockDim.x) {
        const int r = idx % c, q = idx / c;
        const double *V = Vbuf + sd.V_off + (size_t)q * sd.nbp;
        double v = 0.0;
        for (int e = bce_ptr[sd.bce_off + r]; e < bce_ptr[sd.bce_off + r + 1]; ++e) v += bce_val[e] * V[bce_pos[e]];
        out[idx] = v;
    }
}

// ---------------------------------------------------------------------------
// batched dense triangular solves with the full factor (N x N, lower)
// v: full vectors (N per subdomain at nfull_off, nrhs columns of length ldv)
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256) k_trsv_fwd(const SubDev *__restrict__ subs,
                                                  const double *__restrict__ Kbuf, double *__restrict__ v,
                                                  long long ldv) {
    __shared__ double part[8][32];
    __shared__ double xs[32];
    const SubDev &sd = subs[blockIdx.x];
    double *x = v + sd.nfull_off + (size_t)blockIdx.y * ldv;
    const int N = sd.N, lane = threadIdx.x % 32, w = threadIdx.x / 32;
    for (int kb = 0; kb < N; kb += 32) {
        const int nrow = min(32, N - kb);
        double acc = 0.0;
        const int row = kb + lane;
        if (lane < nrow)
            for (int c = w; c < kb; c += 8) acc += Kbuf[kidx(sd, row, c)] * x[c];
        part[w][lane] = acc;
        __syncthreads();
        if (w == 0) {
            double a = (lane < nrow) ? x[row] : 0.0;
            for (int q = 0; q < 8; ++q) a -= part[q][lane];
            for (int q = 0; q < nrow; ++q) {
                double xq = 0.0;
                if (lane == q) xq = a / Kbuf[kidx(sd, row, row)];
                xq = __shfl_sync(0xffffffffu, xq, q);
                if (lane == q) xs[q] = xq;
                if (lane > q && lane < nrow) a -= Kbuf[kidx(sd, row, kb + q)] * xq;
            }
            __syncwarp();
            if (lane < nrow) x[row] = xs[lane];
        }
        __syncthreads();
    }
}

__global__ void __launch_bounds__(256) k_trsv_bwd(const SubDev *__restrict__ subs,
                                                  const double *__restrict__ Kbuf, double *__restrict__ v,
                                                  long long ldv) {
    __shared__ double acc_s[32];
    const SubDev &sd = subs[blockIdx.x];
    double *x = v + sd.nfull_off + (size_t)blockIdx.y * ldv;
    const int N = sd.N, lane = threadIdx.x % 32, w = threadIdx.x / 32;
    const int nblk = (N + 31) / 32;
    for (int b = nblk - 1; b >= 0; --b) {
        const int kb = 32 * b, nrow = min(32, N - kb);
        // acc[r] = x[kb+r] - sum_{c >= kb+nrow} L[c][kb+r] x[c]
        for (int r = w; r < nrow; r += 8) {
            const double *col = Kbuf + kcol(sd, kb + r);
            double s = 0.0;
            for (int c = kb + nrow + lane; c < N; c += 32) s += col[c] * x[c];
            for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
            if (lane == 0) acc_s[r] = x[kb + r] - s;
        }
        __syncthreads();
        if (w == 0) {
            double a = (lane < nrow) ? acc_s[lane] : 0.0;
            for (int q = nrow - 1; q >= 0; --q) {
                double xq = 0.0;
                if (lane == q) xq = a / Kbuf[kidx(sd, kb + q, kb + q)];
                xq = __shfl_sync(0xffffffffu, xq, q);
                if (lane == q) acc_s[q] = xq;
                if (lane < q) a -= Kbuf[kidx(sd, kb + q, kb + lane)] * xq;
            }
            __syncwarp();
            if (lane < nrow) x[kb + lane] = acc_s[lane];
        }
        __syncthreads();
    }
}

}  // namespace htf

namespace htf {

// ---------------------------------------------------------------------------
// batched dense triangular solves with the full factor for up to 32
// right-hand sides at once (the load cases of a batch): the factor is read
// once per call instead of once per load case.  Column j of subdomain d lives
// at v + nfull_off + j*ld (ld = ldv, or N when ldv <= 0).  One CTA of 8 warps
// per (subdomain, chunk of 32 columns = blockIdx.y); warp w owns columns
// 4w..4w+3 of the chunk, lane = row inside the current 32-row block.  The
// chunk has nrhs columns, or min(32, ncols[d] - 32*blockIdx.y) when ncols is
// given.  The next 32x32 block of L and of X is loaded into registers while
// the current one is multiplied out of shared memory.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256) k_trsm_fwd_multi(const SubDev *__restrict__ subs,
                                                        const double *__restrict__ Kbuf, double *__restrict__ v,
                                                        long long ldv, int nrhs, const int *__restrict__ ncols) {
    __shared__ double Ls[32][36];
    __shared__ double Xs[32][36];
    __shared__ double rinv[32];
    const SubDev &sd = subs[blockIdx.x];
    const long long ld = ldv > 0 ? ldv : sd.N;
    const int c0 = 32 * blockIdx.y;
    if (ncols) nrhs = min(32, ncols[blockIdx.x] - c0);
    if (nrhs <= 0) return;
    double *x = v + sd.nfull_off + (size_t)c0 * ld;
    const int N = sd.N, lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int nblk = (N + 31) / 32;
    for (int b = 0; b < nblk; ++b) {
        const int kb = 32 * b, nrow = min(32, N - kb);
        double acc[4] = {0.0, 0.0, 0.0, 0.0};
        double d[2][2] = {{0.0, 0.0}, {0.0, 0.0}};
        double lr[4], xr[4];
        // chunk cb: L rows kb.., columns 32cb.. (all < kb <= N); X rows 32cb..
        auto load = [&](int cb) {
#pragma unroll
            for (int i = 0; i < 4; ++i) {
                const int c = w + 8 * i;
                lr[i] = (lane < nrow) ? Kbuf[kidx(sd, kb + lane, 32 * cb + c)] : 0.0;
                xr[i] = (c < nrhs) ? x[(32 * cb + lane) + (size_t)c * ld] : 0.0;
            }
        };
        if (b > 0) load(0);
        for (int cb = 0; cb < b; ++cb) {
#pragma unroll
            for (int i = 0; i < 4; ++i) {
                Ls[lane][w + 8 * i] = lr[i];
                Xs[lane][w + 8 * i] = xr[i];
            }
            __syncthreads();
            if (cb + 1 < b) load(cb + 1);
            trsm_block_mma<false>(Ls, Xs, w, lane, d);
            __syncthreads();
        }
        if (b > 0) trsm_gather(Xs, d, w, lane, acc);
        // diagonal block: forward substitution, one shuffle per row
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            const int c = w + 8 * i;
            Ls[lane][c] = (lane < nrow && c <= lane) ? Kbuf[kidx(sd, kb + lane, kb + c)] : 0.0;
        }
        __syncthreads();
        if (threadIdx.x < 32) rinv[lane] = (lane < nrow) ? 1.0 / Ls[lane][lane] : 0.0;
        __syncthreads();
        double a[4];
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const int j = 4 * w + q;
            a[q] = (lane < nrow && j < nrhs) ? x[(kb + lane) + (size_t)j * ld] - acc[q] : 0.0;
        }
        for (int p = 0; p < nrow; ++p) {
            const double rp = rinv[p], lp = Ls[lane][p];
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                const double y = __shfl_sync(0xffffffffu, a[q] * rp, p);
                if (lane == p) a[q] = y;
                else if (lane > p) a[q] -= lp * y;
            }
        }
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const int j = 4 * w + q;
            if (lane < nrow && j < nrhs) x[(kb + lane) + (size_t)j * ld] = a[q];
        }
        __syncthreads();
    }
}

__global__ void __launch_bounds__(256) k_trsm_bwd_multi(const SubDev *__restrict__ subs,
                                                        const double *__restrict__ Kbuf, double *__restrict__ v,
                                                        long long ldv, int nrhs, const int *__restrict__ ncols) {
    __shared__ double Ls[32][36];
    __shared__ double Xs[32][36];
    __shared__ double rinv[32];
    const SubDev &sd = subs[blockIdx.x];
    const long long ld = ldv > 0 ? ldv : sd.N;
    const int c0 = 32 * blockIdx.y;
    if (ncols) nrhs = min(32, ncols[blockIdx.x] - c0);
    if (nrhs <= 0) return;
    double *x = v + sd.nfull_off + (size_t)c0 * ld;
    const int N = sd.N, lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int nblk = (N + 31) / 32;
    for (int b = nblk - 1; b >= 0; --b) {
        const int kb = 32 * b, nrow = min(32, N - kb);
        double acc[4] = {0.0, 0.0, 0.0, 0.0};
        double d[2][2] = {{0.0, 0.0}, {0.0, 0.0}};
        double lr[4], xr[4];
        // chunk cb > b: rows c = 32cb + lane of L's columns kb.. (L^T), X rows c
        auto load = [&](int cb) {
            const int c = 32 * cb + lane;
#pragma unroll
            for (int i = 0; i < 4; ++i) {
                const int r = w + 8 * i;
                lr[i] = (c < N && r < nrow) ? Kbuf[kidx(sd, c, kb + r)] : 0.0;
                xr[i] = (c < N && r < nrhs) ? x[c + (size_t)r * ld] : 0.0;
            }
        };
        if (b + 1 < nblk) load(b + 1);
        for (int cb = b + 1; cb < nblk; ++cb) {
#pragma unroll
            for (int i = 0; i < 4; ++i) {
                Ls[lane][w + 8 * i] = lr[i];          // Ls[c][r] = L[32cb + c][kb + r]
                Xs[lane][w + 8 * i] = xr[i];
            }
            __syncthreads();
            if (cb + 1 < nblk) load(cb + 1);
            trsm_block_mma<true>(Ls, Xs, w, lane, d);
            __syncthreads();
        }
        if (b + 1 < nblk) trsm_gather(Xs, d, w, lane, acc);
        // diagonal block: Ls[p][r] = L[kb + p][kb + r], r <= p; back substitution with L^T
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            const int r = w + 8 * i;
            Ls[lane][r] = (lane < nrow && r <= lane) ? Kbuf[kidx(sd, kb + lane, kb + r)] : 0.0;
        }
        __syncthreads();
        if (threadIdx.x < 32) rinv[lane] = (lane < nrow) ? 1.0 / Ls[lane][lane] : 0.0;
        __syncthreads();
        double a[4];
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const int j = 4 * w + q;
            a[q] = (lane < nrow && j < nrhs) ? x[(kb + lane) + (size_t)j * ld] - acc[q] : 0.0;
        }
        for (int p = nrow - 1; p >= 0; --p) {
            const double rp = rinv[p], lp = Ls[p][lane];
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                const double y = __shfl_sync(0xffffffffu, a[q] * rp, p);
                if (lane == p) a[q] = y;
                else if (lane < p) a[q] -= lp * y;
            }
        }
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const int j = 4 * w + q;
            if (lane < nrow && j < nrhs) x[(kb + lane) + (size_t)j * ld] = a[q];
        }
        __syncthreads();
    }
}

}  // namespace htf
