// Problem build on the GPU: the subdomains' DOF maps (l2g, Data.cpp:111-144),
// the interface groups, the Bf rows and weights (Cluster.cpp:846-924) and the
// per-subdomain b sets with their Bf CSR — the integer front-end of a set-up,
// bit for bit the same as the host code that the inspection entry points keep
// (problem.cpp).  Every ordering the host defines by a sort or a sequential
// loop is restated as a sort of unique integer keys, so the result does not
// depend on the order in which threads run:
//   1. (node, subdomain) incidences bucketed by node (counting sort), each
//      bucket sorted and made unique: the subdomains sharing every node;
//   2. the nodes of every subdomain, sorted: l2g (3 DOFs per node);
//   3. interface rows: subdomain d, its shared non-Dirichlet DOFs ascending,
//      the neighbours nb > d ascending (row offsets by prefix sums over the
//      subdomains and, inside one, over its nodes); then the Dirichlet rows,
//      per subdomain in the order of the Dirichlet list;
//   4. Bf entries (local DOF, row) per subdomain, sorted: the b set, its
//      permutation and the Bf CSR.
// Segments of more than FE_SORT_CAP keys are sorted on the host (subdomains
// far larger than the configurations').
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <climits>
#include <string>
#include <vector>

#include "../host/problem.hpp"

namespace htf {
namespace {

constexpr int FE_SORT_CAP = 8192;          // 64-bit keys one CTA sorts in shared memory (64 KB)
constexpr int FE_SCAN_ITEMS = 4096;        // elements per block of the scan
typedef unsigned long long ull;

// ---------------------------------------------------------------------------
// exclusive scan of n ull counts in place (3 passes)
// ---------------------------------------------------------------------------
__device__ __forceinline__ ull block_excl_scan(ull v, ull *warp_tot, ull &total) {
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
    ull x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const ull y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) warp_tot[w] = x;
    __syncthreads();
    if (w == 0) {
        ull t = lane < nw ? warp_tot[lane] : 0;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const ull y = __shfl_up_sync(0xffffffffu, t, o);
            if (lane >= o) t += y;
        }
        if (lane < nw) warp_tot[lane] = t;
    }
    __syncthreads();
    total = warp_tot[nw - 1];
    const ull before = (w > 0 ? warp_tot[w - 1] : 0) + x - v;
    __syncthreads();
    return before;
}

// pass 1: each block scans FE_SCAN_ITEMS elements (4 per thread), block totals to bsum
__global__ void __launch_bounds__(1024) k_scan_local(ull *a, long long n, ull *bsum) {
    __shared__ ull wt[32];
    const long long base = (long long)blockIdx.x * FE_SCAN_ITEMS + 4LL * threadIdx.x;
    ull v[4], s = 0;
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        v[i] = base + i < n ? a[base + i] : 0;
        s += v[i];
    }
    ull total;
    ull run = block_excl_scan(s, wt, total);
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        if (base + i < n) a[base + i] = run;
        run += v[i];
    }
    if (threadIdx.x == 0) bsum[blockIdx.x] = total;
}

// pass 2: one block scans the block totals (in chunks, with a carry)
__global__ void __launch_bounds__(1024) k_scan_sums(ull *bsum, long long nb, ull *grand) {
    __shared__ ull wt[32];
    ull carry = 0;
    for (long long c0 = 0; c0 < nb; c0 += blockDim.x) {
        const long long i = c0 + threadIdx.x;
        const ull v = i < nb ? bsum[i] : 0;
        ull total;
        const ull ex = block_excl_scan(v, wt, total);
        if (i < nb) bsum[i] = carry + ex;
        carry += total;
    }
    if (threadIdx.x == 0) *grand = carry;
}

// pass 3: block offsets added
__global__ void k_scan_add(ull *a, long long n, const ull *bsum) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) a[i] += bsum[i / FE_SCAN_ITEMS];
}

// ---------------------------------------------------------------------------
// bitonic sort of segments of ull keys, one CTA per segment, in shared memory
// (segments longer than FE_SORT_CAP are skipped: the host sorts them)
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(1024) k_sort_segments(ull *keys, const ull *off, int nseg) {
    extern __shared__ ull sk[];
    const int sgm = blockIdx.x;
    if (sgm >= nseg) return;
    const long long b = (long long)off[sgm], n = (long long)off[sgm + 1] - b;
    if (n <= 1 || n > FE_SORT_CAP) return;
    int P = 1;
    while (P < n) P <<= 1;
    for (int i = threadIdx.x; i < P; i += blockDim.x) sk[i] = i < n ? keys[b + i] : ULLONG_MAX;
    __syncthreads();
    for (int k = 2; k <= P; k <<= 1)
        for (int j = k >> 1; j > 0; j >>= 1) {
            for (int i = threadIdx.x; i < P; i += blockDim.x) {
                const int l = i ^ j;
                if (l > i) {
                    const ull x = sk[i], y = sk[l];
                    const bool up = (i & k) == 0;
                    if ((x > y) == up) { sk[i] = y; sk[l] = x; }
                }
            }
            __syncthreads();
        }
    for (int i = threadIdx.x; i < n; i += blockDim.x) keys[b + i] = sk[i];
}


// ---------------------------------------------------------------------------
// front-end kernels
// ---------------------------------------------------------------------------
// incidences (node, subdomain) counted per node
__global__ void k_fe_count_inc(long long ninc, const int *__restrict__ elems, ull *__restrict__ ncnt) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < ninc) atomicAdd(&ncnt[elems[i]], 1ull);
}

__global__ void k_fe_fill_inc(long long ninc, const int *__restrict__ elems, const int *__restrict__ elem_sub,
                              ull *__restrict__ cur, int *__restrict__ bucket) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < ninc) bucket[atomicAdd(&cur[elems[i]], 1ull)] = elem_sub[i / 8];
}

// each node's bucket sorted and made unique in place; ucnt = distinct subdomains
__global__ void k_fe_node_unique(int nn, const ull *__restrict__ off, int *__restrict__ bucket,
                                 ull *__restrict__ ucnt) {
    const int v = blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= nn) return;
    int *a = bucket + off[v];
    const int n = int(off[v + 1] - off[v]);
    for (int i = 1; i < n; ++i) {
        const int x = a[i];
        int j = i - 1;
        while (j >= 0 && a[j] > x) { a[j + 1] = a[j]; --j; }
        a[j + 1] = x;
    }
    int u = 0;
    for (int i = 0; i < n; ++i)
        if (u == 0 || a[i] != a[u - 1]) a[u++] = a[i];
    ucnt[v] = ull(u);
}

__global__ void k_fe_node_compact(int nn, const ull *__restrict__ off, const int *__restrict__ bucket,
                                  const ull *__restrict__ nptr, int *__restrict__ nsub, ull *__restrict__ scnt) {
    const int v = blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= nn) return;
    const int u = int(nptr[v + 1] - nptr[v]);
    for (int i = 0; i < u; ++i) {
        const int s = bucket[off[v] + i];
        nsub[nptr[v] + i] = s;
        atomicAdd(&scnt[s], 1ull);
    }
}

// the nodes of every subdomain (keys; sorted per subdomain afterwards)
__global__ void k_fe_sub_fill(int nn, const ull *__restrict__ nptr, const int *__restrict__ nsub,
                              ull *__restrict__ scur, ull *__restrict__ snodes) {
    const int v = blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= nn) return;
    for (ull i = nptr[v]; i < nptr[v + 1]; ++i) snodes[atomicAdd(&scur[nsub[i]], 1ull)] = ull(v);
}

// per subdomain: interface rows of every node (rc: per sorted node, in
// subdomain order), the subdomain's interface and Dirichlet row counts
__global__ void __launch_bounds__(256) k_fe_row_count(int ns, const ull *__restrict__ soff,
                                                      const ull *__restrict__ snodes, const ull *__restrict__ nptr,
                                                      const int *__restrict__ nsub, const int *__restrict__ dpos,
                                                      int *__restrict__ rc, ull *__restrict__ icnt,
                                                      ull *__restrict__ dcnt) {
    __shared__ ull wt[32];
    const int d = blockIdx.x;
    if (d >= ns) return;
    ull si = 0, sd = 0;
    for (ull i = soff[d] + threadIdx.x; i < soff[d + 1]; i += blockDim.x) {
        const int v = int(snodes[i]);
        const int k = int(nptr[v + 1] - nptr[v]);
        int gt = 0;
        if (k >= 2)
            for (ull q = nptr[v]; q < nptr[v + 1]; ++q) gt += nsub[q] > d;
        int r = 0;
        for (int c = 0; c < 3; ++c) {
            const bool dir = dpos[3 * v + c] >= 0;
            if (!dir) r += gt;
            else ++sd;
        }
        rc[i] = r;
        si += ull(r);
    }
    ull total;
    block_excl_scan(si, wt, total);
    if (threadIdx.x == 0) icnt[d] = total;
    block_excl_scan(sd, wt, total);
    if (threadIdx.x == 0) dcnt[d] = total;
}

// interface rows of subdomain d from ibase[d], in (node, component, neighbour) order
__global__ void __launch_bounds__(256) k_fe_row_fill(int ns, const ull *__restrict__ soff,
                                                     const ull *__restrict__ snodes, const ull *__restrict__ nptr,
                                                     const int *__restrict__ nsub, const int *__restrict__ dpos,
                                                     const int *__restrict__ rc, const ull *__restrict__ ibase,
                                                     int *__restrict__ rsub, int *__restrict__ rdof,
                                                     double *__restrict__ weight) {
    __shared__ ull wt[32];
    const int d = blockIdx.x;
    if (d >= ns) return;
    ull carry = ibase[d];
    for (ull i0 = soff[d]; i0 < soff[d + 1]; i0 += blockDim.x) {
        const ull i = i0 + threadIdx.x;
        const bool in = i < soff[d + 1];
        const int r = in ? rc[i] : 0;
        ull total;
        ull at = carry + block_excl_scan(ull(r), wt, total);
        if (in && r > 0) {
            const int v = int(snodes[i]);
            const int k = int(nptr[v + 1] - nptr[v]);
            const double w = 1. / ((double)(k - 1) + 1);
            for (int c = 0; c < 3; ++c) {
                if (dpos[3 * v + c] >= 0) continue;
                for (ull q = nptr[v]; q < nptr[v + 1]; ++q) {
                    const int nb = nsub[q];
                    if (nb <= d) continue;
                    rsub[2 * at] = d;
                    rsub[2 * at + 1] = nb;
                    rdof[at] = 3 * v + c;
                    weight[at] = w;
                    ++at;
                }
            }
        }
        carry += total;
    }
}

// Dirichlet DOFs of every subdomain as keys (position in the Dirichlet list, DOF)
__global__ void __launch_bounds__(256) k_fe_dir_fill(int ns, const ull *__restrict__ soff,
                                                     const ull *__restrict__ snodes, const int *__restrict__ dpos,
                                                     const ull *__restrict__ dbase, ull *__restrict__ dcur,
                                                     ull *__restrict__ dkeys) {
    const int d = blockIdx.x;
    if (d >= ns) return;
    for (ull i = soff[d] + threadIdx.x; i < soff[d + 1]; i += blockDim.x) {
        const int v = int(snodes[i]);
        for (int c = 0; c < 3; ++c) {
            const int q = dpos[3 * v + c];
            if (q >= 0) dkeys[dbase[d] + atomicAdd(&dcur[d], 1ull)] = (ull(q) << 32) | ull(3 * v + c);
        }
    }
}

// Dirichlet rows after the ni interface rows, per subdomain in list order (keys sorted)
__global__ void k_fe_dir_rows(int ns, const ull *__restrict__ dbase, const ull *__restrict__ dkeys, long long ni,
                              int *__restrict__ rsub, int *__restrict__ rdof, double *__restrict__ weight) {
    const int d = blockIdx.x;
    if (d >= ns) return;
    for (ull i = dbase[d] + threadIdx.x; i < dbase[d + 1]; i += blockDim.x) {
        const long long r = ni + (long long)i;
        rsub[2 * r] = d;
        rsub[2 * r + 1] = -1;
        rdof[r] = int(dkeys[i] & 0xffffffffull);
        weight[r] = 1.0;
    }
}

// Bf entries of every row, counted per subdomain
__global__ void k_fe_ent_count(long long nl, const int *__restrict__ rsub, ull *__restrict__ ecnt) {
    const long long r = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= nl) return;
    atomicAdd(&ecnt[rsub[2 * r]], 1ull);
    if (rsub[2 * r + 1] >= 0) atomicAdd(&ecnt[rsub[2 * r + 1]], 1ull);
}

// entry keys (local DOF, row): the local DOF of global DOF g in subdomain d is
// 3 x (position of node g / 3 among d's sorted nodes) + g mod 3
__global__ void k_fe_ent_fill(long long nl, const int *__restrict__ rsub, const int *__restrict__ rdof,
                              const ull *__restrict__ soff, const ull *__restrict__ snodes,
                              const ull *__restrict__ eoff, ull *__restrict__ ecur, ull *__restrict__ ekeys) {
    const long long r = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= nl) return;
    const int g = rdof[r], v = g / 3;
    for (int k = 0; k < 2; ++k) {
        const int d = rsub[2 * r + k];
        if (d < 0) continue;
        ull lo = soff[d], hi = soff[d + 1];
        while (lo < hi) {
            const ull mid = (lo + hi) >> 1;
            if (snodes[mid] < ull(v)) lo = mid + 1;
            else hi = mid;
        }
        const ull local = 3 * (lo - soff[d]) + ull(g % 3);
        ekeys[eoff[d] + atomicAdd(&ecur[d], 1ull)] = (local << 32) | ull(r);
    }
}


// device scratch released at scope exit
struct FeMem {
    std::vector<void *> p;
    ~FeMem() {
        for (void *q : p) cudaFree(q);
    }
    template <typename T> T *get(size_t n, cudaError_t &e) {
        void *q = nullptr;
        if (e == cudaSuccess) e = cudaMalloc(&q, std::max<size_t>(n, 1) * sizeof(T));
        if (e == cudaSuccess) p.push_back(q);
        return static_cast<T *>(q);
    }
};

int blocks_for(long long n, int t) { return int(std::max<long long>(1, (n + t - 1) / t)); }

// exclusive scan of a[0..n) in place; total = sum of the n inputs
cudaError_t scan(ull *a, long long n, ull &total, FeMem &mem) {
    cudaError_t e = cudaSuccess;
    const long long nb = std::max<long long>(1, (n + FE_SCAN_ITEMS - 1) / FE_SCAN_ITEMS);
    ull *bsum = mem.get<ull>(nb, e), *grand = mem.get<ull>(1, e);
    if (e != cudaSuccess) return e;
    k_scan_local<<<int(nb), 1024>>>(a, n, bsum);
    k_scan_sums<<<1, 1024>>>(bsum, nb, grand);
    k_scan_add<<<blocks_for(n, 256), 256>>>(a, n, bsum);
    e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaMemcpy(&total, grand, sizeof(ull), cudaMemcpyDeviceToHost);
    return e;
}

// sorts the nseg segments [off[i], off[i+1]) of keys (host offsets hoff)
cudaError_t sort_segments(ull *keys, const ull *off, const std::vector<ull> &hoff) {
    const int nseg = int(hoff.size()) - 1;
    if (nseg <= 0) return cudaSuccess;
    k_sort_segments<<<nseg, 1024, FE_SORT_CAP * sizeof(ull)>>>(keys, off, nseg);
    cudaError_t e = cudaGetLastError();
    std::vector<ull> tmp;
    for (int i = 0; i < nseg && e == cudaSuccess; ++i) {
        const size_t n = size_t(hoff[i + 1] - hoff[i]);
        if (n <= size_t(FE_SORT_CAP)) continue;          // long segments on the host
        tmp.resize(n);
        e = cudaMemcpy(tmp.data(), keys + hoff[i], n * sizeof(ull), cudaMemcpyDeviceToHost);
        std::sort(tmp.begin(), tmp.end());
        if (e == cudaSuccess) e = cudaMemcpy(keys + hoff[i], tmp.data(), n * sizeof(ull), cudaMemcpyHostToDevice);
    }
    return e;
}

template <typename T> cudaError_t down(std::vector<T> &h, const T *d, size_t n) {
    h.resize(n);
    return n ? cudaMemcpy(h.data(), d, n * sizeof(T), cudaMemcpyDeviceToHost) : cudaSuccess;
}

}  // namespace

int frontend_on_device(Problem &p, std::vector<int> &node_ptr, std::vector<int> &node_subs, std::string &err) {
    const Mesh &m = p.mesh;
    const int ns = m.n_sub(), nn = m.n_nodes;
    const long long ninc = 8LL * m.n_elems();
    // Dirichlet positions (the list is checked and free of repeats: the caller's host path handles repeats)
    std::vector<int> dpos(3 * size_t(nn), -1);
    for (size_t i = 0; i < m.dirichlet.size(); ++i) {
        const int g = m.dirichlet[i];
        if (g < 0 || g >= 3 * nn) { err = "Dirichlet DOF out of range"; return HTF_EINVAL; }
        if (dpos[g] >= 0) return HTF_ESTATE;            // repeated DOF: the host front-end builds this mesh
        dpos[g] = int(i);
    }
    const auto t0 = std::chrono::steady_clock::now();     // runtime initialisation and context creation
    cudaGetLastError();
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0) {
        cudaGetLastError();
        return HTF_ENODEV;                               // the host front-end runs (and the set-up fails later)
    }
    if (cudaSetDevice(p.opt.device) != cudaSuccess || cudaFree(nullptr) != cudaSuccess) {
        err = "front-end: cudaSetDevice failed";
        return HTF_ECUDA;
    }
    const auto t1 = std::chrono::steady_clock::now();
    p.context_ms += std::chrono::duration<double, std::milli>(t1 - t0).count();
    if (cudaFuncSetAttribute(k_sort_segments, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             int(FE_SORT_CAP * sizeof(ull))) != cudaSuccess) {
        err = "front-end: shared memory opt-in failed";
        return HTF_ECUDA;
    }
    FeMem mem;
    cudaError_t e = cudaSuccess;
    const char *step = "upload";
    auto fail = [&]() {
        err = std::string("front-end: ") + step + ": " + cudaGetErrorString(e);
        return e == cudaErrorMemoryAllocation ? HTF_ENOMEM : HTF_ECUDA;
    };
    int *d_el = mem.get<int>(ninc, e), *d_es = mem.get<int>(m.n_elems(), e), *d_dpos = mem.get<int>(dpos.size(), e);
    if (e == cudaSuccess) e = cudaMemcpy(d_el, m.elems.data(), ninc * sizeof(int), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(d_es, m.elem_sub.data(), m.n_elems() * sizeof(int), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(d_dpos, dpos.data(), dpos.size() * sizeof(int), cudaMemcpyHostToDevice);
    if (e != cudaSuccess) return fail();
    // 1. incidences bucketed by node, made unique: the subdomains of every node
    step = "node buckets";
    ull *off = mem.get<ull>(nn + 1, e), *cur = mem.get<ull>(nn + 1, e), *nptr = mem.get<ull>(nn + 1, e);
    int *bucket = mem.get<int>(ninc, e);
    if (e == cudaSuccess) e = cudaMemset(off, 0, (nn + 1) * sizeof(ull));
    if (e != cudaSuccess) return fail();
    k_fe_count_inc<<<blocks_for(ninc, 256), 256>>>(ninc, d_el, off);
    ull tot = 0;
    if ((e = scan(off, nn + 1, tot, mem)) != cudaSuccess) return fail();
    if ((e = cudaMemcpy(cur, off, (nn + 1) * sizeof(ull), cudaMemcpyDeviceToDevice)) != cudaSuccess) return fail();
    k_fe_fill_inc<<<blocks_for(ninc, 256), 256>>>(ninc, d_el, d_es, cur, bucket);
    if ((e = cudaMemset(nptr, 0, (nn + 1) * sizeof(ull))) != cudaSuccess) return fail();
    k_fe_node_unique<<<blocks_for(nn, 256), 256>>>(nn, off, bucket, nptr);
    ull nU = 0;
    if ((e = scan(nptr, nn + 1, nU, mem)) != cudaSuccess) return fail();
    if (nU > 0x7fffffffull) { err = "front-end: too many (node, subdomain) pairs"; return HTF_EINVAL; }
    // 2. the nodes of every subdomain, sorted
    step = "subdomain nodes";
    int *nsub = mem.get<int>(nU, e);
    ull *soff = mem.get<ull>(ns + 1, e), *scur = mem.get<ull>(ns + 1, e);
    if (e == cudaSuccess) e = cudaMemset(soff, 0, (ns + 1) * sizeof(ull));
    if (e != cudaSuccess) return fail();
    k_fe_node_compact<<<blocks_for(nn, 256), 256>>>(nn, off, bucket, nptr, nsub, soff);
    ull nS = 0;
    if ((e = scan(soff, ns + 1, nS, mem)) != cudaSuccess) return fail();
    ull *snodes = mem.get<ull>(nS, e);
    if (e == cudaSuccess) e = cudaMemcpy(scur, soff, (ns + 1) * sizeof(ull), cudaMemcpyDeviceToDevice);
    if (e != cudaSuccess) return fail();
    k_fe_sub_fill<<<blocks_for(nn, 256), 256>>>(nn, nptr, nsub, scur, snodes);
    std::vector<ull> hsoff;
    if ((e = down(hsoff, soff, size_t(ns) + 1)) != cudaSuccess) return fail();
    if ((e = sort_segments(snodes, soff, hsoff)) != cudaSuccess) return fail();
    // 3. interface rows, then Dirichlet rows
    step = "Bf rows";
    int *rc = mem.get<int>(nS, e);
    ull *ibase = mem.get<ull>(ns + 1, e), *dbase = mem.get<ull>(ns + 1, e), *dcur = mem.get<ull>(ns + 1, e);
    if (e == cudaSuccess) e = cudaMemset(ibase, 0, (ns + 1) * sizeof(ull));
    if (e == cudaSuccess) e = cudaMemset(dbase, 0, (ns + 1) * sizeof(ull));
    if (e == cudaSuccess) e = cudaMemset(dcur, 0, (ns + 1) * sizeof(ull));
    if (e != cudaSuccess) return fail();
    k_fe_row_count<<<ns, 256>>>(ns, soff, snodes, nptr, nsub, d_dpos, rc, ibase, dbase);
    ull nI = 0, nD = 0;
    if ((e = scan(ibase, ns + 1, nI, mem)) != cudaSuccess) return fail();
    if ((e = scan(dbase, ns + 1, nD, mem)) != cudaSuccess) return fail();
    const long long nl = (long long)(nI + nD);
    if (nl == 0) { err = "no dual rows (no interface and no Dirichlet DOF)"; return HTF_EINVAL; }
    if (nl > 0x7fffffffLL) { err = "too many dual rows"; return HTF_EINVAL; }
    int *rsub = mem.get<int>(2 * nl, e), *rdof = mem.get<int>(nl, e);
    double *wgt = mem.get<double>(nl, e);
    ull *dkeys = mem.get<ull>(nD, e);
    if (e != cudaSuccess) return fail();
    k_fe_row_fill<<<ns, 256>>>(ns, soff, snodes, nptr, nsub, d_dpos, rc, ibase, rsub, rdof, wgt);
    k_fe_dir_fill<<<ns, 256>>>(ns, soff, snodes, d_dpos, dbase, dcur, dkeys);
    std::vector<ull> hdbase;
    if ((e = down(hdbase, dbase, size_t(ns) + 1)) != cudaSuccess) return fail();
    if ((e = sort_segments(dkeys, dbase, hdbase)) != cudaSuccess) return fail();
    k_fe_dir_rows<<<ns, 256>>>(ns, dbase, dkeys, (long long)nI, rsub, rdof, wgt);
    // 4. Bf entries per subdomain, sorted by (local DOF, row)
    step = "Bf entries";
    ull *eoff = mem.get<ull>(ns + 1, e), *ecur = mem.get<ull>(ns + 1, e);
    if (e == cudaSuccess) e = cudaMemset(eoff, 0, (ns + 1) * sizeof(ull));
    if (e != cudaSuccess) return fail();
    k_fe_ent_count<<<blocks_for(nl, 256), 256>>>(nl, rsub, eoff);
    ull nE = 0;
    if ((e = scan(eoff, ns + 1, nE, mem)) != cudaSuccess) return fail();
    ull *ekeys = mem.get<ull>(nE, e);
    if (e == cudaSuccess) e = cudaMemset(ecur, 0, (ns + 1) * sizeof(ull));
    if (e != cudaSuccess) return fail();
    k_fe_ent_fill<<<blocks_for(nl, 256), 256>>>(nl, rsub, rdof, soff, snodes, eoff, ecur, ekeys);
    std::vector<ull> heoff;
    if ((e = down(heoff, eoff, size_t(ns) + 1)) != cudaSuccess) return fail();
    if ((e = sort_segments(ekeys, eoff, heoff)) != cudaSuccess) return fail();
    // results to the host
    step = "copy back";
    std::vector<ull> hnptr, hsn, hek;
    std::vector<int> hnsub, hrsub, hrdof;
    std::vector<double> hw;
    if ((e = down(hnptr, nptr, size_t(nn) + 1)) != cudaSuccess) return fail();
    if ((e = down(hnsub, nsub, size_t(nU))) != cudaSuccess) return fail();
    if ((e = down(hsn, snodes, size_t(nS))) != cudaSuccess) return fail();
    if ((e = down(hrsub, rsub, size_t(2 * nl))) != cudaSuccess) return fail();
    if ((e = down(hrdof, rdof, size_t(nl))) != cudaSuccess) return fail();
    if ((e = down(hw, wgt, size_t(nl))) != cudaSuccess) return fail();
    if ((e = down(hek, ekeys, size_t(nE))) != cudaSuccess) return fail();
    node_ptr.resize(size_t(nn) + 1);
    for (int v = 0; v <= nn; ++v) node_ptr[v] = int(hnptr[v]);
    node_subs.swap(hnsub);
    p.n_lam = int(nl);
    p.rows.resize(nl);
    p.weight.swap(hw);
    for (long long r = 0; r < nl; ++r) {
        const int s0 = hrsub[2 * r], s1 = hrsub[2 * r + 1], g = hrdof[r];
        p.rows[r] = s1 >= 0 ? BfRow{{s0, s1}, {g, g}, {1.0, -1.0}} : BfRow{{s0, -1}, {g, -1}, {1.0, 0.0}};
    }
    int few = -1;
#pragma omp parallel for schedule(dynamic, 4)
    for (int d = 0; d < ns; ++d) {
        Subdomain &s = p.sub[d];
        const size_t a = size_t(hsoff[d]), b = size_t(hsoff[d + 1]);
        s.l2g.resize(3 * (b - a));
        for (size_t i = a; i < b; ++i)
            for (int c = 0; c < 3; ++c) s.l2g[3 * (i - a) + c] = 3 * int(hsn[i]) + c;
        s.n = int(s.l2g.size());
        s.b.clear();
        s.bf_lam.clear();
        s.bf_sign.clear();
        const size_t e0 = size_t(heoff[d]), e1 = size_t(heoff[d + 1]);
        for (size_t q = e0; q < e1; ++q) {
            const int local = int(hek[q] >> 32);
            if (s.b.empty() || s.b.back() != local) s.b.push_back(local);
        }
        s.nb = int(s.b.size());
        s.nr = s.n - s.nb;
        s.perm.assign(s.n, -1);
        for (int i = 0; i < s.nb; ++i) s.perm[s.b[i]] = s.nr + i;
        int c = 0;
        for (int l = 0; l < s.n; ++l)
            if (s.perm[l] < 0) s.perm[l] = c++;
        s.bf_ptr.assign(s.nb + 1, 0);
        int bi = 0;
        for (size_t q = e0; q < e1; ++q) {
            const int local = int(hek[q] >> 32), r = int(hek[q] & 0xffffffffull);
            while (s.b[bi] != local) ++bi;
            s.bf_ptr[bi + 1]++;
            s.bf_lam.push_back(r);
            s.bf_sign.push_back(p.rows[r].sub[0] == d ? p.rows[r].sign[0] : p.rows[r].sign[1]);
        }
        for (int i = 0; i < s.nb; ++i) s.bf_ptr[i + 1] += s.bf_ptr[i];
        if (s.nb < 6) {
#pragma omp critical
            few = (few < 0 || d < few) ? d : few;
        }
    }
    if (few >= 0) { err = "subdomain with fewer than 6 interface/Dirichlet DOFs"; return HTF_EINVAL; }
    p.frontend_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t1).count();
    return HTF_OK;
}

}  // namespace htf
