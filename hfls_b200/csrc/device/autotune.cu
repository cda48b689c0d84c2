// SYMV schedules and their autotuner.
//
// The FP64 F / S applies (k_symv_units) read every packed tile once; a
// subdomain's tiles are cut, in storage order, into work units of a fixed
// number of tiles that depends on the subdomain's size bucket (its number of
// 32-row tile rows nt).  Small units give more CTAs per SM (less shared
// memory for the unit's row window) and more partial sums to reduce; large
// units the reverse.  The tuner times the F launch on the problem's own tiles
// for each candidate unit size, first the same size in every bucket (the
// largest window of the launch sets every CTA's shared memory), then bucket
// by bucket (coordinate descent from the best uniform schedule), keeps the
// fastest schedule per (device, problem class) for the
// life of the process, and reads / extends an optional JSON file of tuned
// schedules:
//   {"schedules": [{"key": "<device>|<class>", "tiles": [t0, t1, t2, t3, t4]}, ...]}
// The reference has no counterpart (its local solves are PARDISO calls).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <fstream>
#include <map>
#include <mutex>
#include <sstream>
#include <string>
#include <vector>

#include "engine.hpp"

namespace htf {

template <typename T>
__global__ void k_symv_units(const SymvUnit *, const SubDev *, const T *, const double *, const double *, double *,
                             double *, const PcpgState *);

#define CKE(call)                                                          \
    do {                                                                   \
        int _rc = check((call), #call, err, "autotune.cu", __LINE__);      \
        if (_rc) return _rc;                                               \
    } while (0)

namespace {

constexpr long long SYMV_TUNE_MIN_TILES = 1LL << 17;   // 1 GiB of FP64 tiles
const int CANDIDATES[] = {8, 12, 16, 24, 32, 48, 64, 96};

std::mutex g_mu;
std::map<std::string, std::vector<int>> g_cache;   // tuned schedules of this process
std::map<std::string, bool> g_files_read;

int bucket_of(int nt) {
    for (int b = 0; b < SYMV_BUCKETS; ++b)
        if (nt <= SYMV_BUCKET_NT[b]) return b;
    return SYMV_BUCKETS - 1;
}

// Work units of one subdomain with nt tile rows for a unit size of ut tiles,
// in tile storage order: a tile row I of at least ut tiles is split into
// ceil(len / ut) units of balanced length, tiles J in [j0, j1) (kind 2:
// window 32 (j1 - j0) + 32 rows); shorter rows are grouped while the group
// stays within ut tiles (kind 0: window rows 0 .. 32 (last row + 1), at most
// 32 ut).  fn(t0, t1, kind, row0, rows, rowI).
template <typename Fn>
void partition(int nt, long long ut, Fn fn) {
    long long I = 0;
    while (I < nt) {
        const long long len = I + 1, first = I * (I + 1) / 2;
        if (len >= ut) {
            const long long k = (len + ut - 1) / ut;
            for (long long q = 0; q < k; ++q) {
                const long long j0 = q * len / k, j1 = (q + 1) * len / k;
                fn(first + j0, first + j1, 2, int(TILE * j0), int(TILE * (j1 - j0 + 1)), int(TILE * I));
            }
            ++I;
        } else {
            long long I1 = I, tiles = len;
            while (I1 + 1 < nt && I1 + 2 < ut && tiles + (I1 + 2) <= ut) {
                ++I1;
                tiles += I1 + 1;
            }
            fn(first, (I1 + 1) * (I1 + 2) / 2, 0, 0, int(TILE * (I1 + 1)), 0);
            I = I1 + 1;
        }
    }
}

// units, partial rows and largest row window of one subdomain
void unit_stats(int nt, long long ut, long long &nu, long long &yrows, int &maxrows) {
    nu = 0;
    yrows = 0;
    maxrows = 0;
    partition(nt, ut, [&](long long, long long, int, int, int rows, int) {
        ++nu;
        yrows += rows;
        maxrows = std::max(maxrows, rows);
    });
}

void read_file(const std::string &path) {
    if (path.empty() || g_files_read[path]) return;
    g_files_read[path] = true;
    std::ifstream f(path);
    if (!f) return;
    std::stringstream ss;
    ss << f.rdbuf();
    const std::string s = ss.str();
    size_t pos = 0;
    while ((pos = s.find("\"key\"", pos)) != std::string::npos) {
        const size_t q0 = s.find('"', s.find(':', pos) + 1);
        const size_t q1 = s.find('"', q0 + 1);
        const size_t a0 = s.find('[', q1), a1 = s.find(']', a0);
        if (q0 == std::string::npos || q1 == std::string::npos || a0 == std::string::npos ||
            a1 == std::string::npos)
            break;
        const std::string key = s.substr(q0 + 1, q1 - q0 - 1);
        std::vector<int> t;
        std::stringstream arr(s.substr(a0 + 1, a1 - a0 - 1));
        std::string tok;
        while (std::getline(arr, tok, ',')) t.push_back(std::atoi(tok.c_str()));
        if (int(t.size()) == SYMV_BUCKETS && !g_cache.count(key)) g_cache[key] = t;
        pos = a1;
    }
}

void write_file(const std::string &path) {
    if (path.empty()) return;
    std::ofstream f(path, std::ios::trunc);
    if (!f) return;
    f << "{\"schedules\": [";
    bool first = true;
    for (auto &kv : g_cache) {
        f << (first ? "\n" : ",\n") << "  {\"key\": \"" << kv.first << "\", \"tiles\": [";
        for (int b = 0; b < SYMV_BUCKETS; ++b) f << (b ? ", " : "") << kv.second[b];
        f << "]}";
        first = false;
    }
    f << "\n]}\n";
}

}  // namespace

// Units of the given schedule (host side): sets u0 / u1 of every subdomain.
void Engine::build_units(const std::vector<int> &tiles, std::vector<SymvUnit> &units, long long &yoff,
                         int &smem, std::vector<int> &rbptr, std::vector<int> &rbunit) {
    units.clear();
    rbptr.assign(1, 0);
    rbunit.clear();
    yoff = 0;
    int max_rows = 0;
    std::vector<std::vector<int>> cover;
    for (int d = 0; d < nsub_; ++d) {
        SubDev &h = hs_[d];
        h.u0 = int(units.size());
        partition(h.nt, tiles[bucket_of(h.nt)], [&](long long t0, long long t1, int kind, int row0, int rows, int rowI) {
            units.push_back(SymvUnit{d, kind, t0, t1, yoff, rows, row0, rowI, 0});
            yoff += rows;
            max_rows = std::max(max_rows, rows);
        });
        h.u1 = int(units.size());
        // the units covering each 32-row block, in unit order (the order of the partial sums)
        cover.assign(h.nt, std::vector<int>());
        for (int k = h.u0; k < h.u1; ++k) {
            const SymvUnit &u = units[k];
            const int seg = u.kind == 2 ? u.rows - TILE : u.rows;
            for (int R = u.row0 / TILE; R < (u.row0 + seg + TILE - 1) / TILE && R < h.nt; ++R) cover[R].push_back(k);
            if (u.kind == 2) {
                const int R = u.rowI / TILE;
                if (R < h.nt && (cover[R].empty() || cover[R].back() != k)) cover[R].push_back(k);
            }
        }
        h.rb_off = int(rbptr.size()) - 1;
        for (int R = 0; R < h.nt; ++R) {
            rbunit.insert(rbunit.end(), cover[R].begin(), cover[R].end());
            rbptr.push_back(int(rbunit.size()));
        }
    }
    for (int d = 0; d < nsub_; ++d) units.push_back(SymvUnit{d, 1, 0, 0, 0, 0, 0, 0, 0});   // V^T x units
    smem = SYMV_ROW_DOUBLES * max_rows * int(sizeof(double));
}

// Uploads a schedule into the unit buffers (allocated for the largest
// candidate); with subs_on_device the subdomain table is refreshed from the
// device first (set-up kernels write to it), its u0 / u1 replaced.
int Engine::apply_schedule(const std::vector<int> &tiles, bool subs_on_device, std::string &err) {
    std::vector<SymvUnit> units;
    long long yoff = 0;
    int smem = 0;
    if (subs_on_device) {
        CKE(cudaMemcpyAsync(hs_.data(), d_subs_, nsub_ * sizeof(SubDev), cudaMemcpyDeviceToHost, s_));
        CKE(cudaStreamSynchronize(s_));
    }
    std::vector<int> rbptr, rbunit;
    build_units(tiles, units, yoff, smem, rbptr, rbunit);
    if ((long long)units.size() > units_cap_ || yoff > ypart_cap_ || smem > symv_smem_cap_ ||
        (long long)rbptr.size() > rbptr_cap_ || (long long)rbunit.size() > rbunit_cap_) {
        err = "SYMV schedule exceeds its buffers";
        return HTF_EINVAL;
    }
    nunits_ = int(units.size()) - nsub_;
    symv_smem_ = smem;
    schedule_ = tiles;
    CKE(cudaMemcpyAsync(d_units_, units.data(), units.size() * sizeof(SymvUnit), cudaMemcpyHostToDevice, s_));
    CKE(cudaMemcpyAsync(d_rbptr_, rbptr.data(), rbptr.size() * sizeof(int), cudaMemcpyHostToDevice, s_));
    if (!rbunit.empty())
        CKE(cudaMemcpyAsync(d_rbunit_, rbunit.data(), rbunit.size() * sizeof(int), cudaMemcpyHostToDevice, s_));
    // (pageable copies: the host vectors may go out of scope once the calls return)
    if (subs_on_device)
        CKE(cudaMemcpyAsync(d_subs_, hs_.data(), nsub_ * sizeof(SubDev), cudaMemcpyHostToDevice, s_));
    return HTF_OK;
}

// Unit buffers sized for every schedule the tuner may try (each bucket at
// its most demanding candidate; only the default without autotuning), and
// the default schedule.
int Engine::alloc_units(std::string &err) {
    int rc = HTF_OK;
    std::vector<int> cands(1, SYMV_DEFAULT_TILES);
    if (opt_.autotune) cands.assign(std::begin(CANDIDATES), std::end(CANDIDATES));
    // every unit's row window is at most 32 (ut + 1) rows of 5 doubles: the
    // largest candidate (96 tiles) needs 124 KB, within the 227 KB opt-in limit
    long long bu[SYMV_BUCKETS][8] = {}, by[SYMV_BUCKETS][8] = {};
    int scap = 0;
    for (auto &h : hs_) {
        const int b = bucket_of(h.nt);
        for (size_t c = 0; c < cands.size(); ++c) {
            long long nu = 0, yr = 0;
            int mr = 0;
            unit_stats(h.nt, cands[c], nu, yr, mr);
            bu[b][c] += nu;
            by[b][c] += yr;
            scap = std::max(scap, SYMV_ROW_DOUBLES * mr * int(sizeof(double)));
        }
    }
    long long ucap = nsub_, ycap = 0;
    for (int b = 0; b < SYMV_BUCKETS; ++b) {
        long long mu = 0, my = 0;
        for (size_t c = 0; c < cands.size(); ++c) { mu = std::max(mu, bu[b][c]); my = std::max(my, by[b][c]); }
        ucap += mu;
        ycap += my;
    }
    units_cap_ = ucap;
    ypart_cap_ = ycap;
    symv_smem_cap_ = scap;
    // row-block lists: a unit covers at most rows / 32 + 1 blocks (its window and its tile row)
    long long ntsum = 0;
    for (auto &h : hs_) ntsum += h.nt;
    rbptr_cap_ = ntsum + 1;
    rbunit_cap_ = ycap / TILE + 2 * ucap;
    d_units_ = alloc<SymvUnit>(ucap, err, rc);
    d_ypart_ = alloc<double>(ycap, err, rc);
    d_rbptr_ = alloc<int>(rbptr_cap_, err, rc);
    d_rbunit_ = alloc<int>(rbunit_cap_, err, rc);
    if (rc) return rc;
    if (scap > 48 * 1024) {
        CKE(cudaFuncSetAttribute(k_symv_units<double>, cudaFuncAttributeMaxDynamicSharedMemorySize, scap));
        CKE(cudaFuncSetAttribute(k_symv_units<float>, cudaFuncAttributeMaxDynamicSharedMemorySize, scap));
    }
    return apply_schedule(std::vector<int>(SYMV_BUCKETS, SYMV_DEFAULT_TILES), false, err);
}

// Problem class of the schedule cache: the device and the number of
// subdomains in each size bucket, rounded to a power of two.
std::string Engine::schedule_key() const {
    cudaDeviceProp prop;
    std::string dev = "device";
    if (cudaGetDeviceProperties(&prop, opt_.device) == cudaSuccess) dev = prop.name;
    int cnt[SYMV_BUCKETS] = {0, 0, 0, 0, 0};
    for (auto &h : hs_) cnt[bucket_of(h.nt)]++;
    std::string k = dev + "|";
    for (int b = 0; b < SYMV_BUCKETS; ++b) {
        int l = 0;
        while ((1 << l) < cnt[b]) ++l;
        k += (b ? "," : "") + std::to_string(cnt[b] ? l + 1 : 0);
    }
    return k;
}

// After set-up (F tiles resident): the cached or tuned schedule.  With
// autotune=1 only problems of at least SYMV_TUNE_MIN_TILES tiles are tuned:
// below that the F apply takes tens of microseconds and the default schedule
// keeps small problems' arithmetic fixed from run to run (a tuned schedule
// is chosen by timing, and the summation order follows the schedule).
// autotune=2 tunes every problem.
int Engine::autotune_symv(std::string &err) {
    if (!opt_.autotune || (opt_.autotune == 1 && ntiles_ < SYMV_TUNE_MIN_TILES)) return HTF_OK;
    const std::string key = schedule_key();
    {
        std::lock_guard<std::mutex> lk(g_mu);
        read_file(opt_.tune_file);
        auto it = g_cache.find(key);
        if (it != g_cache.end()) {
            tuned_ = true;
            return apply_schedule(it->second, true, err);
        }
    }
    bool present[SYMV_BUCKETS] = {false, false, false, false, false};
    for (auto &h : hs_) present[bucket_of(h.nt)] = true;
    cudaEvent_t e0, e1;
    CKE(cudaEventCreate(&e0));
    CKE(cudaEventCreate(&e1));
    auto time_of = [&](const std::vector<int> &t, double &ms) -> int {
        int rc = apply_schedule(t, true, err);
        if (rc) return rc;
        auto launch = [&] {
            k_symv_units<double><<<nunits_, SYMV_WARPS * 32, symv_smem_, s_>>>(d_units_, d_subs_, d_F_, d_V_, d_xb_, d_ypart_,
                                                                  d_t_, nullptr);
        };
        launch();
        cudaEventRecord(e0, s_);
        for (int r = 0; r < 3; ++r) launch();
        cudaEventRecord(e1, s_);
        CKE(cudaEventSynchronize(e1));
        float f = 0.f;
        CKE(cudaEventElapsedTime(&f, e0, e1));
        ms = f / 3.0;
        return HTF_OK;
    };
    // the launch's shared memory (and so its CTAs per SM) follows the largest
    // window of any bucket, which one-bucket steps cannot lower: uniform
    // schedules first, then coordinate descent per bucket from the best one
    std::vector<int> best(SYMV_BUCKETS, SYMV_DEFAULT_TILES);
    double best_ms = 0.0;
    int rc = time_of(best, best_ms);
    for (int c : CANDIDATES) {
        if (rc || c == SYMV_DEFAULT_TILES) continue;
        std::vector<int> t(SYMV_BUCKETS, c);
        double ms = 0.0;
        if ((rc = time_of(t, ms))) break;
        if (ms < best_ms) { best_ms = ms; best = t; }
    }
    for (int b = 0; !rc && b < SYMV_BUCKETS; ++b) {
        if (!present[b]) continue;
        for (int c : CANDIDATES) {
            if (c == best[b]) continue;
            std::vector<int> t = best;
            t[b] = c;
            double ms = 0.0;
            if ((rc = time_of(t, ms))) break;
            if (ms < best_ms) { best_ms = ms; best = t; }
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (rc) return rc;
    rc = apply_schedule(best, true, err);
    if (rc) return rc;
    tuned_ = true;
    std::lock_guard<std::mutex> lk(g_mu);
    g_cache[key] = best;
    write_file(opt_.tune_file);
    return HTF_OK;
}

}  // namespace htf
