// Multi-right-hand-side F_i / S_i apply on the 5th-generation tensor cores.
//
// Y_b(:, 0:k) = A_i X_b(:, 0:k) for every subdomain i, with A_i the
// symmetric F_i (or S_i) (Cluster::mult_Ff's local solves,
// Cluster.cpp:1125-1126, applied to k load cases at once).
//
// Number format: every operand is held as a pair of FP16 values, hi + lo,
// of one power-of-two scaled copy: A_i scaled by 2^EA (one exponent per
// subdomain and matrix), each column of X by 2^EX_j, so that every scaled
// value is below 2^14; hi = rn_f16(v), lo = rn_f16(v - hi).  The pair costs 4
// bytes per entry, as FP32 does, and carries 22 significant bits.  Products
// per K step of 16: A_hi [X_hi | X_lo] as one N = 2k MMA and A_lo X_hi as a
// second N = k MMA (`tcgen05.mma.kind::f16`, FP16 products are exact in the
// FP32 accumulator); the dropped A_lo X_lo term is ~2^-22 of the product.
// The epilogue multiplies by 2^-(EA + EX_j) in FP64.  EA and EX_j come from
// maxima kept on the device (k_slab_amax, k_colmax), so nothing waits on the
// host.  Unlike the 3xTF32 form, no A_lo has to be made inside the kernel:
// the CTA only streams copies into the tensor cores.
//
// Storage: the lower triangle of A_i at 128-row block granularity, cut into
// 128 x 32 slabs (128 rows of an M block, 32 columns of a K slab), each 16 KB:
// the hi plane (128 rows x 64 B) then the lo plane, each already in the
// SWIZZLE_64B K-major layout the MMA reads (byte b of a plane's logical
// row-major layout lives at b ^ (((b >> 7) & 3) << 4)), so one
// cp.async.bulk lands a slab ready for tcgen05.mma.  Block m keeps its slabs
// up to and including its diagonal 128 x 128 block; the K steps right of it
// read 32 rows of the four slabs below that hold their transpose (eight 2 KB
// bulk copies: four pieces per plane) and give them to the MMA through an
// MN-major descriptor: a K-major 64-byte row of a stored slab is, read
// transposed, the 32-element MN row of an MN-major SWIZZLE_64B atom, so no
// data moves.  Each off-diagonal slab is thus read from HBM by its own block
// and, through L2, by the block its columns belong to: half the bytes of
// full symmetric storage.  X is written by the gather kernel as k x 32 slabs
// per 32 b-space slots, the same two planes of k rows x 64 B.
//
// One CTA of 10 warps per (subdomain, 128-row block), two CTAs per SM:
//   * warp 0, one thread: bulk-copy producer (A slab or its eight transposed
//     pieces, the X slab per stage);
//   * warp 1, one thread: issues the MMAs (M=128, K=16 per instruction, two
//     K steps per 32-column slab);
//   * warps 2-9: the epilogue (warp w owns TMEM lanes 32 (w mod 4) .. +31 and
//     half of the load cases), y written in FP64.
// Accumulation: K slab kk goes to accumulator group kk mod 2 ([hi-hi | hi-lo +
// lo-hi] columns), so every FP32 accumulator sums half of the K range; the
// groups are added in FP64 in the epilogue.  Every mbarrier wait is bounded;
// on time-out the CTA records HTF_ETIMEDOUT in err and stops issuing work.
#include <cuda_fp16.h>
#include <cuda_runtime.h>
#include <cstdint>

#include "device.cuh"
#include "htfeti.h"

namespace htf {

constexpr int TC_SLAB_A = 128 * 32;          // 4-byte words per A slab (16 KB: hi plane, lo plane)
constexpr int TC_PLANE_A = TC_SLAB_A / 2;    // words per A plane (8 KB)
constexpr int TC_PIECE = 512;                // words of 32 stored rows of one plane (2 KB)
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

// SWIZZLE_64B shared-memory descriptors (sm100 layout type 4, version 1).
// K-major: 8-row groups of 64-byte rows, SBO = 512 B between groups (LBO
// unused).  MN-major: 64-byte rows of 32 consecutive M elements, one per K
// index; LBO = the byte distance between 32-element M groups, SBO = 512 B
// between groups of 8 K indices.
__device__ __forceinline__ uint64_t sw64_kmajor(const void *smem) {
    const uint64_t addr = smem_u32(smem);
    return ((addr >> 4) & 0x3FFFull) | (1ull << 16) | (32ull << 32) | (1ull << 46) | (4ull << 61);
}

__device__ __forceinline__ uint64_t sw64_mnmajor(const void *smem, uint32_t lbo_bytes) {
    const uint64_t addr = smem_u32(smem);
    return ((addr >> 4) & 0x3FFFull) | (uint64_t((lbo_bytes >> 4) & 0x3FFFu) << 16) | (32ull << 32) |
           (1ull << 46) | (4ull << 61);
}

// kind::f16 instruction descriptor: D F32, A and B F16, B K-major, A K-major
// or (a_mn) MN-major
__device__ __forceinline__ uint32_t f16_idesc(int M, int N, bool a_mn) {
    return (1u << 4) | (a_mn ? (1u << 15) : 0u) | (uint32_t(N >> 3) << 17) | (uint32_t(M >> 4) << 24);
}

__device__ __forceinline__ void mma_f16(uint32_t d, uint64_t a, uint64_t b, uint32_t idesc, uint32_t acc) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(d),
        "l"(a), "l"(b), "r"(idesc), "r"(acc)
        : "memory");
}

constexpr int TC_NACC = 2;                   // rotating accumulator groups

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
    constexpr int SLAB_B = K * 32;                        // words per X slab: hi plane, lo plane (k x 64 B each)
    constexpr unsigned STAGE_TX = (TC_SLAB_A + SLAB_B) * 4;
    constexpr int GW = 2 * K;                              // TMEM columns per accumulator group
    // TMEM: TC_NACC accumulator groups of GW columns (A_hi X_hi, then
    // A_hi X_lo + A_lo X_hi, the two small terms sharing one FP32 accumulator)
    constexpr uint32_t TMEM_COLS = TC_NACC * GW <= 64 ? 64 : 128;   // power of two >= 32
    static_assert(TC_NACC * GW <= int(TMEM_COLS), "TMEM columns");
    extern __shared__ __align__(1024) unsigned char smem_raw[];
    // 1024-byte aligned buffers: stage s holds the A slab (or its transposed pieces) and the X slab
    unsigned char *base = reinterpret_cast<unsigned char *>(
        (reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    float *sA = reinterpret_cast<float *>(base);                          // TC_STAGES x 16 KB
    float *sB = reinterpret_cast<float *>(base + TC_STAGES * TC_SLAB_A * 4);
    __shared__ __align__(8) uint64_t full[TC_STAGES], empty[TC_STAGES], done;
    __shared__ uint32_t tmem_base;
    __shared__ volatile int abort_flag;

    const GemmBlock g = blocks[blockIdx.x];
    const TcSet &ts = sets[g.set];
    const float *__restrict__ A = which == 0 ? ts.AF : ts.AS;
    const float *__restrict__ Xs = ts.Xs;
    double *__restrict__ yb = ts.yb;
    const int warp = threadIdx.x / 32, lane = threadIdx.x % 32;

    if (threadIdx.x == 0) {
        for (int s = 0; s < TC_STAGES; ++s) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], 1);
        }
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
                float *dA = sA + s * TC_SLAB_A;
                if (kk < g.kd) {
                    bulk_g2s(dA, A + g.a_off + (long long)kk * TC_SLAB_A, TC_SLAB_A * 4, &full[s]);
                } else {
                    // above the diagonal block: rows [32 q, 32 q + 32), q = kk mod 4, of the stored
                    // slabs (kk / 4, 4 m + p), p = 0..3, i.e. the transpose of this K step's
                    // 128 x 32 block; per plane each 32-row piece is 2 KB contiguous (8-row
                    // swizzle groups of 512 B), piece p lands at p x 2 KB of the stage's plane
                    const int mp = kk >> 2, q = kk & 3;
                    const float *src = A + a0 + (2LL * mp * (mp + 1) + 4LL * g.m) * TC_SLAB_A + q * TC_PIECE;
#pragma unroll
                    for (int p = 0; p < 4; ++p) {
                        bulk_g2s(dA + p * TC_PIECE, src + (long long)p * TC_SLAB_A, TC_PIECE * 4, &full[s]);
                        bulk_g2s(dA + TC_PLANE_A + p * TC_PIECE, src + (long long)p * TC_SLAB_A + TC_PLANE_A,
                                 TC_PIECE * 4, &full[s]);
                    }
                }
                bulk_g2s(sB + s * SLAB_B, Xs + g.x_off + (long long)kk * SLAB_B, SLAB_B * 4, &full[s]);
                ++issued;
            }
            // before the CTA may exit: the last copy into every stage has landed (bounded)
            for (int kk = (issued > TC_STAGES ? issued - TC_STAGES : 0); kk < issued; ++kk)
                if (!mbar_wait(&full[kk % TC_STAGES], (kk / TC_STAGES) & 1)) atomicExch(err, HTF_ETIMEDOUT);
        }
    } else if (warp == 1) {
        if (lane == 0) {                                  // MMA issuer
            const uint32_t id2_k = f16_idesc(128, 2 * K, false), id1_k = f16_idesc(128, K, false);
            const uint32_t id2_t = f16_idesc(128, 2 * K, true), id1_t = f16_idesc(128, K, true);
            for (int kk = 0; kk < g.ks; ++kk) {
                const int s = kk % TC_STAGES;
                if (abort_flag || !mbar_wait(&full[s], (kk / TC_STAGES) & 1)) {
                    atomicExch(err, HTF_ETIMEDOUT);
                    abort_flag = 1;
                    break;
                }
                asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
                const uint32_t d = tmem + uint32_t((kk % TC_NACC) * GW);   // [hi-hi | hi-lo + lo-hi]
                const float *pA = sA + s * TC_SLAB_A;
                const bool tr = kk >= g.kd;
                // A_hi and A_lo planes; a K step of 16 is 32 bytes along a K-major row, or two
                // 8-row groups (1 KB) of an MN-major piece
                const uint64_t ahi = tr ? sw64_mnmajor(pA, TC_PIECE * 4) : sw64_kmajor(pA);
                const uint64_t alo = tr ? sw64_mnmajor(pA + TC_PLANE_A, TC_PIECE * 4) : sw64_kmajor(pA + TC_PLANE_A);
                const uint64_t astep = tr ? 64ull : 2ull;                    // descriptor units of 16 bytes
                const uint64_t db = sw64_kmajor(sB + s * SLAB_B);            // X_hi rows, then X_lo rows: 2k rows
                const uint32_t id2 = tr ? id2_t : id2_k, id1 = tr ? id1_t : id1_k;
#pragma unroll
                for (int q = 0; q < 2; ++q) {              // 2 x K=16 (32 bytes) per slab
                    const uint32_t acc = (kk >= TC_NACC || q > 0) ? 1u : 0u;
                    mma_f16(d, ahi + astep * q, db + 2ull * q, id2, acc);
                    // issued after the first, which initialised these columns
                    mma_f16(d + K, alo + astep * q, db + 2ull * q, id1, 1u);
                }
                asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                                 smem_u32(&empty[s]))
                             : "memory");
            }
            asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                             smem_u32(&done))
                         : "memory");
        }
    } else if (warp >= 2) {
        // warps 2-9: the epilogue.  Warp w may access TMEM lanes 32 (w mod 4) .. +31
        // (its quarter); the two warps of a quarter take half of the load cases each
        const int quarter = warp & 3, h = (warp - 2) >> 2;
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
            // undo the scales: 2^-(EA + EX_j)
            const unsigned *amax = which == 0 ? ts.amaxF : ts.amaxS;
            const int ea = tc_scale_exp(amax[g.d], 1.0f);
#pragma unroll
            for (int j = 0; j < KH; ++j) acc[j] = ldexp(acc[j], -(ea + tc_scale_exp(ts.xmax[h * KH + j], ts.xbound)));
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

// The value of the packed symmetric FP64 tile matrix of subdomain d at
// (i, j) of its b-block, 0 outside it (padding rows and columns).  tiles
// holds the packed tiles from tile t0 on.
__device__ __forceinline__ double packed_at(const SubDev &sd, const double *tiles, long long t0, int i, int j) {
    if (i >= sd.nbp || j >= sd.nbp) return 0.0;
    if (i < j) { const int t = i; i = j; j = t; }
    const int I = i / TILE, J = j / TILE;
    const double *T = tiles + (sd.T_off - t0 + (long long)I * (I + 1) / 2 + J) * TILE_ELEMS;
    return T[(i % TILE) * TILE + (j % TILE)];
}

// Largest |A| of every subdomain over its stored slabs (the whole symmetric
// block), as FP32 bits (atomicMax; amax starts at zero): the scale exponent
// of the subdomain's slabs.  grid (block, kk) as k_make_slabs.
__global__ void k_slab_amax(const GemmBlock *__restrict__ blocks, const SubDev *__restrict__ subs,
                            const double *__restrict__ tiles, long long t0, unsigned *__restrict__ amax) {
    const GemmBlock g = blocks[blockIdx.x];
    const int kk = blockIdx.y;
    if (kk >= g.kd) return;
    const SubDev &sd = subs[g.d];
    float m = 0.f;
    for (int idx = threadIdx.x; idx < TC_SLAB_A; idx += blockDim.x)
        m = fmaxf(m, (float)fabs(packed_at(sd, tiles, t0, 128 * g.m + idx / 32, 32 * kk + idx % 32)));
    __shared__ float red[32];
    for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = m;
    __syncthreads();
    if (threadIdx.x < 32) {
        m = threadIdx.x < (blockDim.x >> 5) ? red[threadIdx.x] : 0.f;
        for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
        if (threadIdx.x == 0 && m > 0.f) atomicMax(amax + g.d, __float_as_uint(m));
    }
}

// FP16-pair slabs of the lower triangle (at 128-row block granularity) of a
// packed symmetric FP64 tile matrix: slab (m, kk), kk < kd, of subdomain d
// holds rows [128m, 128m+128) x columns [32kk, 32kk+32) of the symmetric
// block, scaled by 2^EA (EA from amax[d]), as the hi plane then the lo plane
// (SWIZZLE_64B K-major, 128 rows x 64 B each).  tiles holds the packed tiles
// from tile t0 on.  grid (block, kk).
__global__ void k_make_slabs(const GemmBlock *__restrict__ blocks, const SubDev *__restrict__ subs,
                             const double *__restrict__ tiles, float *__restrict__ A, long long t0,
                             const unsigned *__restrict__ amax) {
    const GemmBlock g = blocks[blockIdx.x];
    const int kk = blockIdx.y;
    if (kk >= g.kd) return;
    const SubDev &sd = subs[g.d];
    const int ea = tc_scale_exp(amax[g.d], 1.0f);
    __half *hi = reinterpret_cast<__half *>(A + g.a_off + (long long)kk * TC_SLAB_A);
    __half *lo = hi + 2 * TC_PLANE_A;
    for (int idx = threadIdx.x; idx < TC_SLAB_A; idx += blockDim.x) {
        const int r = idx / 32, c = idx % 32;
        const double v = ldexp(packed_at(sd, tiles, t0, 128 * g.m + r, 32 * kk + c), ea);
        const __half vh = __double2half(v);
        const __half vl = __double2half(v - (double)__half2float(vh));
        const uint32_t b = uint32_t(r * 64 + c * 2);
        const uint32_t bs = b ^ (((b >> 7) & 3u) << 4);
        hi[bs / 2] = vh;
        lo[bs / 2] = vl;
    }
}

// Largest |w| of every column of an RHS-interleaved batch vector (n rows x
// K), as FP32 bits (atomicMax; xmax starts at zero).  blockDim a multiple of
// K and a grid stride that is too, so each thread stays on one column.
__global__ void k_colmax(int n, int K, const double *__restrict__ w, unsigned *__restrict__ xmax) {
    __shared__ float red[256];
    const long long nk = (long long)n * K;
    const long long stride = (long long)gridDim.x * blockDim.x;
    float m = 0.f;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < nk; i += stride)
        m = fmaxf(m, (float)fabs(w[i]));
    red[threadIdx.x] = m;
    __syncthreads();
    if ((int)threadIdx.x < K) {
        for (int t = threadIdx.x + K; t < (int)blockDim.x; t += K) m = fmaxf(m, red[t]);
        if (m > 0.f) atomicMax(xmax + threadIdx.x, __float_as_uint(m));
    }
}

}  // namespace htf
