// Device-side data layout of the HTFETI path (shared by the kernels and the
// host engine).
//
// Per subdomain d (n local DOFs, nb of them touched by Bf = the "b set"):
//   * local DOFs are permuted to [interior (nr) | b set (nb)], the b set
//     padded with identity rows to nbp = 32*ceil(nb/32);
//   * K_d (lower triangle) is stored as column panels, one per 32-column
//     step of the factorisation: interior steps start at 0, 32, ..; b-set
//     steps at nr, nr+32, ..; the panel of the step starting at column cb
//     holds rows [cb, N) of its columns, column-major with ld = N - cb
//     (kidx below).  It is assembled and factored in place: the interior
//     columns are eliminated first, the trailing block then holds
//     S_reg = K_bb - K_bi K_ii^{-1} K_ib;
//   * F_d = (K_reg^{-1})_bb and the preconditioner block (S_d = S_reg - D_fix
//     for Dirichlet, K_bb for lumped) are stored as packed lower-triangular
//     32x32 tiles, tile (I,J) with J<=I at index I(I+1)/2+J, row-major inside
//     the tile, diagonal tiles stored full;
//   * b-space vectors (x_b, y_b) are concatenated with per-subdomain offsets
//     xb_off (multiples of 32).
#pragma once
#include <vector>
#include <cstdint>

namespace htf {

#ifdef __CUDACC__
// Power-of-two scale exponent of a tensor-core operand: values of magnitude
// up to m * mult (m given as FP32 bits) times 2^E stay below 2^14, a quarter
// of the FP16 range, so the hi + lo FP16 pair of a scaled value keeps 22
// significant bits.  m * mult = f 2^e, f in [0.5, 1): E = 14 - e; 0 for zero.
__device__ __forceinline__ int tc_scale_exp(unsigned m_bits, float mult) {
    const float m = __uint_as_float(m_bits) * mult;
    if (!(m > 0.f)) return 0;
    int e;
    frexpf(m, &e);
    return 14 - e;
}
#endif

constexpr int TILE = 32;                  // packed tile edge
constexpr int CHOL_STEP = 64;             // columns per batched Cholesky step (two factor panels)
// dynamic shared memory of k_syrk_update: two 32-column panels of 64 rows for
// each operand (row stride 68) and the 64 x 64 C block (column stride 65)
constexpr int SYRK_SMEM = (4 * 32 * 68 + 64 * 65) * 8;
constexpr int TC_STAGES = 5;              // pipeline stages of the tensor-core product (2 CTAs per SM)
constexpr int TC_THREADS = 320;           // threads of the tensor-core product: producer, MMA, 8 epilogue warps
constexpr int TILE_ELEMS = TILE * TILE;

struct SubDev {
    int n, nr, nb, nbp, nt;               // nt = nbp / 32
    int N;                                // nr + nbp (order of the factor)
    long long K_off;                      // factor panels (doubles)
    long long K_bset;                     // offset of the first b-set panel from K_off;
                                          // < 0: plain column-major N x N (ld = N)
    long long T_off;                      // packed tiles: first tile index (F and S/Kbb share it)
    long long X_off;                      // nbp x nbp scratch (L_bb^{-1}) during setup
    int xb_off;                           // offset of the b block in b-space vectors
    int nfull_off;                        // offset of the N-vector block in full vectors
    int c;                                // Bc rows of this subdomain
    int cluster;                          // cluster index
    int alpha_pos;                        // index of alpha_d in the cluster coarse vector
    long long V_off;                      // V = [F Bc_b^T, -R_b]: nbp x (c+6), col-major
    int t_off;                            // offset of V^T x (c+6 values) in the t vector
    int bcr_off;                          // offset of this subdomain's Bc row ids (c entries)
    int bce_off;                          // Bc entries (CSR by compressed Bc row): ptr offset
    long long R_off;                      // R in permuted local order, N x 6 (padded rows 0)
    int u0, u1;                           // SYMV work units of this subdomain [u0, u1)
    int rb_off;                           // its nt + 1 pointers into the units covering each 32-row block
    int fix[6];                           // fix DOFs (positions in permuted order)
    double fix_diag[6];                   // original diagonal at the fix DOFs
};

struct ClusterDev {
    int nlam_c, ngc;                      // ngc = nlam_c + 6*nsub
    long long M_off;                      // M = (Ac^{-1}) restricted, ngc x ngc (col-major)
    int gc_off;                           // offset in the concatenated coarse vectors
    int gmap_off;                         // gather map: ptr array offset (ngc+1 entries)
    long long MT_off;                     // M as packed lower 32x32 tiles (the plain form's copy): first tile
    int mt;                               // tile rows, ceil(ngc / 32)
    int mt_row_off;                       // first tile row of this cluster in the per-row arrays
};

#ifdef __CUDACC__
#define HTF_HD __host__ __device__ __forceinline__
#else
#define HTF_HD inline
#endif

// doubles of the factor panels of a subdomain with nr interior DOFs and
// nbp padded b-set DOFs, and the offset of its first b-set panel
HTF_HD long long kpanel_interior(int nr, int N) {
    const long long nI = (nr + 31) / 32;
    if (nI == 0) return 0;
    const long long last = nI - 1, wl = nr - 32 * last;
    return 32 * last * N - 512 * last * (last - 1) + wl * (N - 32 * last);
}
HTF_HD long long kpanel_doubles(int nr, int nbp) {
    const long long nt = nbp / 32;
    return kpanel_interior(nr, nr + nbp) + 512 * nt * (nt + 1);
}

// Address of factor entry (r, c), r >= c, of subdomain s
HTF_HD long long kcol(const SubDev &s, int c) {     // address of (0, c) if it were stored: add r
    if (s.K_bset < 0) return s.K_off + (long long)c * s.N;     // plain column-major N x N
    long long base;
    int cb;
    if (c < s.nr) {
        const long long b = c >> 5;
        cb = int(b << 5);
        base = 32 * b * s.N - 512 * b * (b - 1);
    } else {
        const long long j = (c - s.nr) >> 5;
        cb = s.nr + int(j << 5);
        base = s.K_bset + 32 * j * s.nbp - 512 * j * (j - 1);
    }
    return s.K_off + base + (long long)(c - cb) * (s.N - cb) - cb;
}
HTF_HD long long kidx(const SubDev &s, int r, int c) { return kcol(s, c) + r; }
// leading dimension of the panel of the step starting at column k
HTF_HD long long kld(const SubDev &s, int k) { return s.K_bset < 0 ? s.N : s.N - k; }

// One SYMV work unit of subdomain d: packed tiles [t0, t1) (kind 0 and 2), or
// the V^T x_b product (kind 1).  Units write partial y sums over the rows
// their tiles touch (the unit's window) to scratch at y_off; they are summed
// in unit order.  Kind 0 (whole tile rows): window rows [row0, row0 + rows).
// Kind 2 (part of one tile row I, rowI = 32 I): window = rows [row0, row0 +
// rows - 32) for the column blocks, then rows [rowI, rowI + 32).
struct SymvUnit {
    int d, kind;
    long long t0, t1;
    long long y_off;
    int rows;
    int row0;
    int rowI;
    int pad;
};

// SYMV schedule: subdomains with nt tile rows fall in bucket b, the first
// with nt <= SYMV_BUCKET_NT[b]; their tiles are cut into units of tiles[b].
constexpr int SYMV_BUCKETS = 5;
constexpr int SYMV_BUCKET_NT[SYMV_BUCKETS] = {8, 16, 32, 64, 1 << 30};
constexpr int SYMV_DEFAULT_TILES = 48;
constexpr int SYMV_WARPS = 4;                 // warps of a SYMV work-unit CTA
constexpr int SYMV_ROW_DOUBLES = 1 + SYMV_WARPS;   // shared doubles per window row: x + the warps' partials

// One CTA of the tensor-core multi-RHS product: 128-row block m of
// subdomain d.  The symmetric A_d is stored as its lower triangle at 128-row
// block granularity: block m holds the slabs (m, 0 .. kd-1), kd =
// min(4 (m + 1), ks), contiguous at a_off, and the subdomain's blocks follow
// one another, so block m' starts 2 m' (m' + 1) slabs after block 0.  Column
// slabs kk >= kd of block m (above the diagonal block) are read transposed
// from the blocks below.  X slabs at x_off.  `set` names the TcSet (problem)
// the block belongs to: one launch can cover the blocks of several problems.
struct GemmBlock {
    int d;                                // subdomain within its problem
    int m;                                // 128-row block index
    long long a_off;                      // first stored slab (floats) of this block in the set's A arrays
    int ks;                               // K slabs (32 columns each) of the full row
    int rows;                             // valid rows of the block
    long long x_off;                      // first X slab (floats)
    long long y_row0;                     // first output row (b-space slot)
    int set;
    int kd;                               // slabs stored in this block row (the rest are read transposed)
};

// Operands of the tensor-core products of one problem.
struct TcSet {
    const float *AF, *AS;                 // FP16-pair slabs of F_i and S_i (4 bytes per entry)
    const float *Xs;                      // FP16-pair X slabs (k x 32 words per 32 b-space slots)
    double *yb;                           // b-space output, RHS-interleaved
    const unsigned *amaxF, *amaxS;        // largest |F_i|, |S_i| per subdomain (FP32 bits): scale of A
    const unsigned *xmax;                 // largest |w_j| of the gathered batch vector (FP32 bits)
    float xbound;                         // |x_b| <= xbound * max|w_j|: scale of X
};

// One step of the batched Cholesky for one subdomain: columns [k, k + nb),
// nb <= CHOL_STEP, starting at a factor panel and covering at most two.
// tri0 / rb0: first trailing 64x64 tile / first 128-row block of this entry
// in the step's flattened SYRK / panel-solve grid (prefix sums over the step's
// entries, so the grids have no idle CTAs whatever the subdomain sizes).
struct StepDesc {
    int d;      // subdomain
    int k;      // first column of the step
    int nb;     // columns in the step
    int tri0;
    int rb0;
};

// CTAs of a step's flattened grid per entry hint
constexpr int STEP_HINT = 256;

// hints of one step's grid of `total` CTAs: out gets, for every range of
// STEP_HINT CTAs, the entry of its first CTA, then the last entry (so the
// entry of CTA b lies between hint[b / STEP_HINT] and hint[b / STEP_HINT + 1])
inline void step_hints(const std::vector<StepDesc> &v, int total, bool tri, std::vector<int> &out) {
    const int nh = (total + STEP_HINT - 1) / STEP_HINT;
    int e = 0;
    for (int h = 0; h < nh; ++h) {
        const int b = h * STEP_HINT;
        while (e + 1 < int(v.size()) && (tri ? v[e + 1].tri0 : v[e + 1].rb0) <= b) ++e;
        out.push_back(e);
    }
    out.push_back(int(v.size()) - 1);
}

#ifdef __CUDACC__
// entry of a step whose flattened range holds block b (the last one starting at
// or before b); hint (step_hints) narrows the search to the entries of b's range
template <typename F>
__device__ __forceinline__ int step_entry(const StepDesc *st, int cnt, int b, F start, const int *hint) {
    int lo = 0, hi = cnt - 1;
    if (hint) {
        lo = hint[b / STEP_HINT];
        hi = hint[b / STEP_HINT + 1];
    }
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (start(st[mid]) <= b) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}
#endif

// PCPG state in device memory (one per load case).
struct PcpgState {
    double gPz, gPz_prev, wFw, norm0, rho, gamma, rel;
    int it, done, max_iter, pad;
    double eps;
};

}  // namespace htf
