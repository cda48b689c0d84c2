// Multi-right-hand-side F_i / S_i apply on the 5th-generation tensor cores.
//
// Y_b(:, 0:k) = A_i X_b(:, 0:k) for every subdomain i, with A_i the
// symmetric F_i (or S_i) stored in FP32 and the products formed as 3xTF32
// (A_hi X_hi + A_hi X_lo + A_lo X_hi) on the tensor cores
// (Cluster::mult_Ff's local solves, Cluster.cpp:1125-1126, applied to k
// load cases at once).
//
// Storage: the lower triangle of A_i at 128-row block granularity, cut into
// 128 x 32 slabs (128 rows of an M block, 32 columns of a K slab), each
// 16 KB and already in the SWIZZLE_128B K-major layout the MMA reads from
// shared memory (byte b of the logical row-major slab lives at
// b ^ (((b >> 7) & 7) << 4)), so one cp.async.bulk per slab lands it ready
// for tcgen05.mma.  Block m keeps its slabs up to and including its
// diagonal 128 x 128 block; the K steps right of it read the transpose of
// the blocks below, 32 rows of four stored slabs (4 x 4 KB bulk copies),
// which the splitting warps transpose in shared memory.  Each off-diagonal
// slab is thus read from HBM by its own block and, through L2, by the block
// its columns belong to: half the bytes of full symmetric storage.  X is
// written by the gather kernel in the same layout as k x 32 slabs (one
// 128-byte row per load case), already split into its TF32 part and the
// TF32 remainder.
//
// One CTA of 10 warps per (subdomain, 128-row block), two CTAs per SM:
//   * warp 0, one thread: bulk-copy producer (A slab or its four transposed
//     pieces, X_hi, X_lo per stage);
//   * warps 2-9 (two per TMEM lane quarter, taking alternate K steps, so
//     two K steps are split at once): form A_lo = rna_tf32(A - trunc_tf32(A)) of every landed A
//     slab and store it into one of TC_LO 32-column TMEM buffers
//     (tcgen05.st; the MMA reads the FP32 slab itself as A_hi: a TF32
//     operand's low 13 mantissa bits do not take part in the product; a
//     transposed step is first transposed in place, each warp inside its own
//     4 KB), then hand the stage to the MMA issuer;
//     at the end they read the accumulators out of TMEM (warp w owns TMEM
//     lanes 32 (w mod 4) .. +31, and half of the load cases) and write y in
//     FP64;
//   * warp 1, one thread: issues the MMAs (M=128, N=k, K=8 per instruction,
//     4 per slab).
// Products per K step of 8: A_hi [X_hi | X_lo] as one N = 2k MMA (A_hi read
// from shared memory once) and A_lo X_hi (A from TMEM).  Accumulation: K slab
// kk goes to accumulator group kk mod 2 (hi-hi columns, and hi-lo + lo-hi
// columns: the two correction terms are ~2^-11 of the product and share one
// FP32 accumulator), so every FP32 accumulator in TMEM sums half of the K
// range; the groups are added in FP64 in the epilogue.  Every mbarrier wait is bounded; on time-out the
// CTA records HTF_ETIMEDOUT in err and stops issuing work.
#include <cuda_runtime.h>
#include <cstdint>

#include "device.cuh"
#include "htfeti.h"

namespace htf {

constexpr int TC_SLAB_A = 128 * 32;          // floats per A slab (16 KB)
// bounded waits on mbarriers: TC_WAIT_LIMIT tries of up to TC_WAIT_HINT_NS
// each (a waiting thread is suspended until the phase completes or the hint
// runs out, so waiting warps leave the issue slots to the working ones);
// at most ~10 s in all before the wait reports a time-out
constexpr unsigned TC_WAIT_LIMIT = 1u << 20;
constexpr unsigned TC_WAIT_HINT_NS = 10000;

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t *bar, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count));
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, unsigned bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes));
}

// returns false on time-out
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, unsigned parity) {
    uint32_t done = 0;
    for (unsigned it = 0; it < TC_WAIT_LIMIT; ++it) {
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}"
            : "=r"(done)
            : "r"(smem_u32(bar)), "r"(parity), "r"(TC_WAIT_HINT_NS)
            : "memory");
        if (done) return true;
    }
    return false;
}

__device__ __forceinline__ void bulk_g2s(void *dst, const void *src, unsigned bytes, uint64_t *bar) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(smem_u32(dst)),
        "l"(src), "r"(bytes), "r"(smem_u32(bar))
        : "memory");
}

__device__ __forceinline__ uint64_t sw128_desc(const void *smem) {
    const uint64_t addr = smem_u32(smem);
    return ((addr >> 4) & 0x3FFFull) | (1ull << 16) /* LBO (ignored for swizzled K-major) */ |
           (64ull << 32) /* SBO = 1024 B */ | (1ull << 46) /* version */ | (2ull << 61) /* SWIZZLE_128B */;
}

__device__ __forceinline__ uint32_t tf32_idesc(int M, int N) {
    return (1u << 4)            // D format F32
           | (2u << 7)          // A format TF32
           | (2u << 10)         // B format TF32
           | (uint32_t(N >> 3) << 17) | (uint32_t(M >> 4) << 24);   // A, B K-major
}

// A_lo = rna_tf32(a - trunc_tf32(a)) of one row of 32 values into 32
// consecutive TMEM columns of this thread's lane (taddr: the warp's lane
// quarter and the first column), where the MMA reads it as its A operand.
__device__ __forceinline__ void store_lo_row(const float (&v)[32], uint32_t taddr) {
    uint32_t r[32];
#pragma unroll
    for (int j = 0; j < 32; ++j) r[j] = __float_as_uint(tf32_rna(v[j] - tf32_trunc(v[j])));
    asm volatile(
        "tcgen05.st.sync.aligned.32x32b.x32.b32 [%0], {%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,%16,"
        "%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31,%32};" ::"r"(taddr),
        "r"(r[0]), "r"(r[1]), "r"(r[2]), "r"(r[3]), "r"(r[4]), "r"(r[5]), "r"(r[6]), "r"(r[7]), "r"(r[8]),
        "r"(r[9]), "r"(r[10]), "r"(r[11]), "r"(r[12]), "r"(r[13]), "r"(r[14]), "r"(r[15]), "r"(r[16]),
        "r"(r[17]), "r"(r[18]), "r"(r[19]), "r"(r[20]), "r"(r[21]), "r"(r[22]), "r"(r[23]), "r"(r[24]),
        "r"(r[25]), "r"(r[26]), "r"(r[27]), "r"(r[28]), "r"(r[29]), "r"(r[30]), "r"(r[31])
        : "memory");
    asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory");
}

// A stored slab: this thread's row (its TMEM lane) of the SWIZZLE_128B slab
// at a, A_lo of it into TMEM.  Out of line so its live values do not compete
// with the epilogue's registers.
__device__ __noinline__ void split_direct(const float *a, int row, uint32_t taddr) {
    float v[32];
#pragma unroll
    for (int g4 = 0; g4 < 8; ++g4) {
        const float4 h = *reinterpret_cast<const float4 *>(a + row * 32 + ((g4 ^ (row & 7)) * 4));
        v[4 * g4] = h.x; v[4 * g4 + 1] = h.y; v[4 * g4 + 2] = h.z; v[4 * g4 + 3] = h.w;
    }
    store_lo_row(v, taddr);
}

// One warp's 4 KB of a transposed K step: pa holds 32 rows x 32 columns of
// a stored slab (SWIZZLE_128B rows), whose column `lane` becomes row `lane`
// of the same 4 KB in the K-major slab the MMA reads (A_hi, in place); the
// row's A_lo goes to TMEM.
__device__ __noinline__ void split_transposed(float *pa, int lane, uint32_t taddr) {
    float v[32];
#pragma unroll
    for (int j = 0; j < 32; ++j) v[j] = pa[j * 32 + (lane ^ ((j & 7) << 2))];
    __syncwarp();
    float *hrow = pa + lane * 32;
#pragma unroll
    for (int g4 = 0; g4 < 8; ++g4) {
        const int ph = (g4 ^ (lane & 7)) * 4;     // SWIZZLE_128B position of granule g4 in this row
        *reinterpret_cast<float4 *>(hrow + ph) = make_float4(v[4 * g4], v[4 * g4 + 1], v[4 * g4 + 2], v[4 * g4 + 3]);
    }
    store_lo_row(v, taddr);
}

// tcgen05.mma with A from TMEM (a_tmem: lanes = the 128 rows, 8 columns of K)
__device__ __forceinline__ void mma_tf32_ts(uint32_t d, uint32_t a_tmem, uint64_t b, uint32_t idesc, uint32_t acc) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::tf32 [%0], [%1], %2, %3, p;\n\t}" ::"r"(d),
        "r"(a_tmem), "l"(b), "r"(idesc), "r"(acc)
        : "memory");
}

constexpr int TC_NACC = 2;                   // rotating accumulator groups

__device__ __forceinline__ void mbar_arrive(uint64_t *bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

__device__ __forceinline__ void mma_tf32(uint32_t d, uint64_t a, uint64_t b, uint32_t idesc, uint32_t acc) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}" ::"r"(d),
        "l"(a), "l"(b), "r"(idesc), "r"(acc)
        : "memory");
}

// 8, 16 or 32 consecutive FP32 columns of this warp's 32 TMEM lanes, added into acc
template <int N>
__device__ __forceinline__ void tmem_add(uint32_t taddr, double *acc) {
    uint32_t r[N];
    if constexpr (N == 8) {
        asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
                     : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
                       "=r"(r[7])
                     : "r"(taddr));
    } else if constexpr (N == 16) {
        asm volatile(
            "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
            : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
              "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
            : "r"(taddr));
    } else {
        asm volatile(
            "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
            "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
            : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
              "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]),
              "=r"(r[15]), "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]),
              "=r"(r[22]), "=r"(r[23]), "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]),
              "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
            : "r"(taddr));
    }
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int j = 0; j < N; ++j) acc[j] += (double)__uint_as_float(r[j]);
}

// which = 0: F product (A = the set's F slabs; its coarse correction
// y_b -= V_d s_d runs afterwards in k_correct_multi); which = 1: S product
// (A = the set's S slabs).
template <int K>
__global__ void __launch_bounds__(TC_THREADS, 2) k_tc_gemm(const GemmBlock *__restrict__ blocks,
                                                           const TcSet *__restrict__ sets, int which,
                                                           int *__restrict__ err) {
    static_assert(K == 16 || K == 32, "N of the MMA");
    constexpr int SLAB_B = K * 32;                        // floats per X slab
    constexpr unsigned STAGE_TX = (TC_SLAB_A + 2 * SLAB_B) * 4;
    constexpr int GW = 2 * K;                              // TMEM columns per accumulator group
    // TMEM: the accumulator groups (TC_NACC x GW columns: A_hi X_hi, then
    // A_hi X_lo + A_lo X_hi, the two small terms sharing one FP32 accumulator),
    // then TC_LO A_lo buffers of 32 columns each (A_lo of K slab kk in buffer
    // kk mod TC_LO)
    constexpr uint32_t LO_COL = TC_NACC * GW;
    constexpr uint32_t TMEM_COLS = 256;                   // power of two >= LO_COL + 32 TC_LO
    static_assert(LO_COL + 32 * TC_LO <= TMEM_COLS, "TMEM columns");
    extern __shared__ __align__(1024) unsigned char smem_raw[];
    // 1024-byte aligned buffers: stage s holds A (FP32) and X_hi, X_lo (copied from HBM)
    unsigned char *base = reinterpret_cast<unsigned char *>(
        (reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    float *sA = reinterpret_cast<float *>(base);                          // TC_STAGES x 16 KB
    float *sB = reinterpret_cast<float *>(base + TC_STAGES * TC_SLAB_A * 4);
    __shared__ __align__(8) uint64_t full[TC_STAGES], split[TC_STAGES], empty[TC_STAGES], lo_empty[TC_LO], done;
    __shared__ uint32_t tmem_base;
    __shared__ volatile int abort_flag;

    const GemmBlock g = blocks[blockIdx.x];
    const TcSet &ts = sets[g.set];
    const float *__restrict__ A = which == 0 ? ts.AF : ts.AS;
    const float *__restrict__ Xs = ts.Xs;
    const long long xlo_off = ts.xlo;
    double *__restrict__ yb = ts.yb;
    const int warp = threadIdx.x / 32, lane = threadIdx.x % 32;

    if (threadIdx.x == 0) {
        for (int s = 0; s < TC_STAGES; ++s) {
            mbar_init(&full[s], 1);
            mbar_init(&split[s], 4);                      // one arrival per splitting warp of the stage
            mbar_init(&empty[s], 1);
        }
        for (int s = 0; s < TC_LO; ++s) mbar_init(&lo_empty[s], 1);
        mbar_init(&done, 1);
        abort_flag = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tmem_base)),
                     "r"(TMEM_COLS)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = tmem_base;

    if (warp == 0) {
        if (lane == 0) {                                  // producer
            int issued = 0;
            // first stored slab of the subdomain: block m' starts 2 m' (m' + 1) slabs after it
            const long long a0 = g.a_off - 2LL * g.m * (g.m + 1) * TC_SLAB_A;
            for (int kk = 0; kk < g.ks; ++kk) {
                const int s = kk % TC_STAGES;
                if (kk >= TC_STAGES && !mbar_wait(&empty[s], ((kk / TC_STAGES) - 1) & 1)) {
                    atomicExch(err, HTF_ETIMEDOUT);
                    abort_flag = 1;
                    break;
                }
                if (abort_flag) break;
                mbar_expect_tx(&full[s], STAGE_TX);
                if (kk < g.kd) {
                    bulk_g2s(sA + s * TC_SLAB_A, A + g.a_off + (long long)kk * TC_SLAB_A, TC_SLAB_A * 4, &full[s]);
                } else {
                    // above the diagonal block: rows [32 kk, 32 kk + 32) of the stored slabs
                    // (kk / 4, 4 m + p), p = 0..3, i.e. 32 rows x 128 columns of the transpose;
                    // each 32-row piece is 4 KB contiguous (8-row swizzle groups of 1 KB)
                    const int mp = kk >> 2, q = kk & 3;
                    const float *src = A + a0 + (2LL * mp * (mp + 1) + 4LL * g.m) * TC_SLAB_A + q * 1024;
#pragma unroll
                    for (int p = 0; p < 4; ++p)
                        bulk_g2s(sA + s * TC_SLAB_A + p * 1024, src + (long long)p * TC_SLAB_A, 4096, &full[s]);
                }
                bulk_g2s(sB + s * 2 * SLAB_B, Xs + g.x_off + (long long)kk * SLAB_B, SLAB_B * 4, &full[s]);
                bulk_g2s(sB + (s * 2 + 1) * SLAB_B, Xs + xlo_off + g.x_off + (long long)kk * SLAB_B, SLAB_B * 4,
                         &full[s]);
                ++issued;
            }
            // before the CTA may exit: the last copy into every stage has landed (bounded)
            for (int kk = (issued > TC_STAGES ? issued - TC_STAGES : 0); kk < issued; ++kk)
                if (!mbar_wait(&full[kk % TC_STAGES], (kk / TC_STAGES) & 1)) atomicExch(err, HTF_ETIMEDOUT);
        }
    } else if (warp == 1) {
        if (lane == 0) {                                  // MMA issuer
            const uint32_t idesc = tf32_idesc(128, K), idesc2 = tf32_idesc(128, 2 * K);
            for (int kk = 0; kk < g.ks; ++kk) {
                const int s = kk % TC_STAGES;
                if (abort_flag || !mbar_wait(&split[s], (kk / TC_STAGES) & 1)) {
                    atomicExch(err, HTF_ETIMEDOUT);
                    abort_flag = 1;
                    break;
                }
                asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
                const uint32_t d = tmem + uint32_t((kk % TC_NACC) * GW);   // [hi-hi | hi-lo + lo-hi]
                const uint64_t da = sw128_desc(sA + s * TC_SLAB_A);
                const uint32_t tal = tmem + LO_COL + 32u * uint32_t(kk % TC_LO);   // A_lo in TMEM
                const uint64_t db = sw128_desc(sB + s * 2 * SLAB_B);      // X_hi, X_lo: 2k rows
#pragma unroll
                for (int q = 0; q < 4; ++q) {              // 4 x K=8 (32 bytes) per slab
                    const uint32_t acc = (kk >= TC_NACC || q > 0) ? 1u : 0u;
                    mma_tf32(d, da + 2ull * q, db + 2ull * q, idesc2, acc);
                    // issued after the first, which initialised these columns
                    mma_tf32_ts(d + K, tal + 8u * q, db + 2ull * q, idesc, 1u);
                }
                asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                                 smem_u32(&empty[s]))
                             : "memory");
                asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                                 smem_u32(&lo_empty[kk % TC_LO]))
                             : "memory");
            }
            asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                             smem_u32(&done))
                         : "memory");
        }
    } else if (warp >= 2) {
        // warps 2-9: split the A slab of every stage, then the epilogue.  Warp w
        // may access TMEM lanes 32 (w mod 4) .. +31 (its quarter); the two warps
        // of a quarter take alternate K steps (h = (w - 2) / 4: steps kk with
        // kk mod 2 = h), so a stage is always split by the same four warps
        const int quarter = warp & 3, h = (warp - 2) >> 2;
        for (int kk = h; kk < g.ks; kk += 2) {
            const int s = kk % TC_STAGES, lb = kk % TC_LO;
            // the A_lo buffer of slab kk - TC_LO is free once its MMAs completed; the A slab has landed
            bool ok = kk < TC_LO || mbar_wait(&lo_empty[lb], ((kk / TC_LO) - 1) & 1);
            ok = __all_sync(0xffffffffu, ok && mbar_wait(&full[s], (kk / TC_STAGES) & 1));
            if (!__all_sync(0xffffffffu, ok && !abort_flag)) {          // warp-uniform exit
                if (lane == 0 && !ok) atomicExch(err, HTF_ETIMEDOUT);
                abort_flag = 1;
                break;
            }
            const uint32_t taddr = tmem + (uint32_t(quarter * 32) << 16) + LO_COL + 32u * uint32_t(lb);
            if (kk < g.kd) {                              // stored slab: A_lo of this warp's rows
                split_direct(sA + s * TC_SLAB_A, quarter * 32 + lane, taddr);
            } else {
                // transposed pieces: the warp owns piece p = quarter (4 KB at p * 1024 floats), whose
                // column l is row 32 p + l of this K step's A; the output rows 32 p .. 32 p + 31
                // of the K-major slab occupy the same 4 KB, so the transpose stays inside the warp
                split_transposed(sA + s * TC_SLAB_A + quarter * 1024, lane, taddr);
            }
            // generic-proxy writes become visible to the tensor core's async proxy, TMEM stores
            // are ordered before the hand-off
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
            __syncwarp();
            if (lane == 0) mbar_arrive(&split[s]);
        }
        __syncwarp();
        // epilogue: this warp's 32 rows x the K/2 load cases of half h
        constexpr int KH = K / 2;
        const bool have = __all_sync(0xffffffffu, mbar_wait(&done, 0));   // warp-uniform before the .sync.aligned loads
        __syncwarp();
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        double acc[KH];
#pragma unroll
        for (int j = 0; j < KH; ++j) acc[j] = 0.0;
        const bool go = __all_sync(0xffffffffu, have && !abort_flag);
        if (!have) {
            if (lane == 0) atomicExch(err, HTF_ETIMEDOUT);
        } else if (go) {
            const uint32_t taddr = tmem + (uint32_t(quarter * 32) << 16) + uint32_t(h * KH);
            const int nacc = g.ks < TC_NACC ? g.ks : TC_NACC;
            for (int a = 0; a < nacc; ++a) {
                tmem_add<KH>(taddr + uint32_t(a * GW), acc);
                tmem_add<KH>(taddr + uint32_t(a * GW + K), acc);
            }
            // the warp's 32 rows x KH columns through shared memory (row stride KH + 1
            // doubles; the stage buffers are idle: every copy landed before the last
            // MMA completed), stored as 32 segments of KH contiguous doubles
            double *st = reinterpret_cast<double *>(base) + (warp - 2) * 32 * (KH + 1);
#pragma unroll
            for (int j = 0; j < KH; ++j) st[lane * (KH + 1) + j] = acc[j];
            __syncwarp();
            const int r0 = quarter * 32;
            const int nrow = min(32, g.rows - r0);
            double *y = yb + (g.y_row0 + r0) * K + h * KH;
            for (int e = lane; e < nrow * KH; e += 32) y[(e / KH) * K + (e % KH)] = st[(e / KH) * (KH + 1) + (e % KH)];
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 0) {
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TMEM_COLS) : "memory");
    }
}

template __global__ void k_tc_gemm<16>(const GemmBlock *, const TcSet *, int, int *);
template __global__ void k_tc_gemm<32>(const GemmBlock *, const TcSet *, int, int *);

// FP32 slabs of the lower triangle (at 128-row block granularity) of a packed
// symmetric FP64 tile matrix: slab (m, kk), kk < kd, of subdomain d holds
// rows [128m, 128m+128) x columns [32kk, 32kk+32) of the symmetric block,
// swizzled for SWIZZLE_128B K-major.  tiles holds the packed tiles from tile
// t0 on.  grid (block, kk).
__global__ void k_make_slabs(const GemmBlock *__restrict__ blocks, const SubDev *__restrict__ subs,
                             const double *__restrict__ tiles, float *__restrict__ A, long long t0) {
    const GemmBlock g = blocks[blockIdx.x];
    const int kk = blockIdx.y;
    if (kk >= g.kd) return;
    const SubDev &sd = subs[g.d];
    float *slab = A + g.a_off + (long long)kk * TC_SLAB_A;
    for (int idx = threadIdx.x; idx < TC_SLAB_A; idx += blockDim.x) {
        const int r = idx / 32, c = idx % 32;
        const int gr = 128 * g.m + r, gc = 32 * kk + c;
        float v = 0.f;
        if (gr < sd.nbp && gc < sd.nbp) {
            int i = gr, j = gc;
            if (i < j) { int t = i; i = j; j = t; }
            const int I = i / TILE, J = j / TILE;
            const double *T = tiles + (sd.T_off - t0 + (long long)I * (I + 1) / 2 + J) * TILE_ELEMS;
            v = (float)T[(i % TILE) * TILE + (j % TILE)];
        }
        const uint32_t b = uint32_t(r * 128 + c * 4);
        const uint32_t bs = b ^ (((b >> 7) & 7u) << 4);
        slab[bs / 4] = v;
    }
}

}  // namespace htf
