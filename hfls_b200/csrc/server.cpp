// Continuous-batching solve server (htf_server_* in include/htfeti.h).
//
// Requests (a mesh spec and 1..batch load cases) are queued as they arrive.
// A setup thread admits them in order while the estimated device footprint
// of factors, F_i / S_i and vectors fits the HBM budget and a slot is free,
// and runs their setup on each request's own stream, overlapping the
// iterations of the requests already running.  With admit_oversize, a
// request whose factor panels do not fit beside the rest holds them a wave of
// subdomains at a time and has them assembled and factorised again for its
// start solve and its reconstruction.  A run thread advances every
// live request one batched mixed-precision PCPG iteration at a time: the
// FP64 phases of the requests run side by side, each on its own stream forked
// from and joined back to the server stream, around ONE tensor-core launch
// for the F products of all live requests and one for their S products (the
// F applies of all requests are batched together).
// The sequence is captured as a CUDA graph, re-captured whenever the live set
// changes; requests join and leave only between groups of check_every
// iterations, so each request sees the same iteration cadence, and the same
// arithmetic, alone or in a mix.  Between groups every request's FP64
// residual replacements and convergence checks run; a converged request gets
// its displacements reconstructed and copied to the caller's buffer, frees
// its memory and leaves.  The reference has no counterpart (it solves one
// problem per process, htfeti.cpp:8-21).
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "device/engine.hpp"
#include "host/problem.hpp"
#include "htfeti.h"

namespace htf {

struct Request {
    long long id = 0;
    htf_mesh_spec spec{};
    std::vector<int> widths[3];
    int nrhs = 1;
    std::vector<double> f;          // nodal loads, 3 n_nodes x nrhs (empty: body force only)
    double *u_out = nullptr;        // caller-owned, 3 n_nodes x nrhs
    htf_request_info info{};
    std::string err;
    size_t bytes = 0;               // accounted device bytes (estimate, then actual)
    std::unique_ptr<Problem> p;
    std::unique_ptr<Engine> eng;
    htf_stats stats{};
    cudaStream_t rs = nullptr;      // this request's stream while it iterates
    cudaEvent_t joined = nullptr;   // marks the end of its phase on rs (graph capture)
};

class Server {
public:
    Server(const Options &o, double budget, int max_live) : opt_(o), budget_(budget), max_live_(max_live) {
        t0_ = std::chrono::steady_clock::now();
    }
    ~Server();
    int start(std::string &err);
    int submit(const htf_mesh_spec &spec, int nrhs, const double *f, double *u, long long *ticket,
               std::string &err);
    int info(long long ticket, htf_request_info *out, std::string *err_msg);
    int wait(long long ticket, double timeout_ms, htf_request_info *out);

private:
    double now_ms() const {
        return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0_).count();
    }
    void setup_loop();
    void run_loop();
    int prepare(Request &r, std::string &err);
    size_t estimate(const Problem &p, int nrhs, double wave_gb, bool s_fp64) const;
    int rebuild_graph(std::string &err);
    void finish(Request *r, int rc, const std::string &msg);
    void release_graph();

    Options opt_;
    double budget_;
    int max_live_;
    std::chrono::steady_clock::time_point t0_;
    std::mutex mu_;
    std::condition_variable cv_;
    std::deque<Request *> queue_;               // submitted, not admitted
    std::vector<Request *> ready_;              // set up, waiting to join
    std::vector<Request *> live_;               // iterating
    std::map<long long, std::unique_ptr<Request>> all_;
    long long next_id_ = 1;
    double in_use_ = 0.0;
    int admitted_ = 0;                          // ready + live
    int outstanding_ = 0;                       // submitted, not finished
    bool stop_ = false, started_ = false;
    std::thread t_setup_, t_run_;
    // run-thread state
    cudaStream_t stream_ = nullptr;
    cudaEvent_t fork_ = nullptr;               // start of a phase on the server stream (graph capture)
    cudaGraphExec_t graph_ = nullptr;
    bool dirty_ = true;
    GemmBlock *d_blocks_ = nullptr;
    TcSet *d_sets_ = nullptr;
    int *d_err_ = nullptr;
    size_t cap_blocks_ = 0, cap_sets_ = 0;
    int nblocks_ = 0;
};

static int ck(cudaError_t e, const char *what, std::string &err) {
    if (e == cudaSuccess) return HTF_OK;
    err = std::string(what) + ": " + cudaGetErrorString(e);
    return HTF_ECUDA;
}

// Destruction stops new submissions, lets every submitted request finish,
// then joins the threads.
int Server::start(std::string &err) {
    if (opt_.batch != 16 && opt_.batch != 32) { err = "batch width must be 16 or 32"; return HTF_EINVAL; }
    int rc = ck(cudaSetDevice(opt_.device), "cudaSetDevice", err);
    if (!rc) rc = ck(cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking), "cudaStreamCreate", err);
    if (!rc) rc = ck(cudaEventCreateWithFlags(&fork_, cudaEventDisableTiming), "cudaEventCreate", err);
    if (!rc) rc = ck(cudaMalloc(&d_err_, sizeof(int)), "cudaMalloc", err);
    if (!rc) rc = ck(cudaMemset(d_err_, 0, sizeof(int)), "cudaMemset", err);
    if (rc) return rc;
    if (budget_ <= 0.0) {
        size_t fr = 0, tot = 0;
        if ((rc = ck(cudaMemGetInfo(&fr, &tot), "cudaMemGetInfo", err))) return rc;
        budget_ = 0.85 * double(fr);
    }
    t_setup_ = std::thread([this] { setup_loop(); });
    t_run_ = std::thread([this] { run_loop(); });
    started_ = true;
    return HTF_OK;
}

Server::~Server() {
    {
        std::lock_guard<std::mutex> lk(mu_);
        stop_ = true;
    }
    cv_.notify_all();
    if (t_setup_.joinable()) t_setup_.join();
    if (t_run_.joinable()) t_run_.join();
    release_graph();
    all_.clear();
    if (d_blocks_) cudaFree(d_blocks_);
    if (d_sets_) cudaFree(d_sets_);
    if (d_err_) cudaFree(d_err_);
    if (fork_) cudaEventDestroy(fork_);
    if (stream_) cudaStreamDestroy(stream_);
}

int Server::submit(const htf_mesh_spec &spec, int nrhs, const double *f, double *u, long long *ticket,
                   std::string &err) {
    if (nrhs < 1 || nrhs > opt_.batch) {
        err = "a request carries 1..batch load cases";
        return HTF_EINVAL;
    }
    int nn = 0, ne = 0, ns = 0, nc = 0, nd = 0, ncr = 0;
    int rc = mesh_sizes(spec, &nn, &ne, &ns, &nc, &nd, &ncr, err);
    if (rc) return rc;
    auto r = std::make_unique<Request>();
    r->spec = spec;
    for (int a = 0; a < 3; ++a)
        if (spec.widths[a]) {
            r->widths[a].assign(spec.widths[a], spec.widths[a] + spec.clusters[a] * spec.subs[a]);
            r->spec.widths[a] = r->widths[a].data();
        }
    r->nrhs = nrhs;
    if (f) r->f.assign(f, f + (size_t)3 * nn * nrhs);
    r->u_out = u;
    r->info.status = HTF_REQ_QUEUED;
    r->info.n_rhs = nrhs;
    std::lock_guard<std::mutex> lk(mu_);
    if (stop_) { err = "server is stopping"; return HTF_ESTATE; }
    r->id = next_id_++;
    r->info.t_submit_ms = now_ms();
    *ticket = r->id;
    ++outstanding_;
    queue_.push_back(r.get());
    all_[r->id] = std::move(r);
    cv_.notify_all();
    return HTF_OK;
}

int Server::info(long long ticket, htf_request_info *out, std::string *err_msg) {
    std::lock_guard<std::mutex> lk(mu_);
    auto it = all_.find(ticket);
    if (it == all_.end()) return HTF_EINVAL;
    if (out) *out = it->second->info;
    if (err_msg) *err_msg = it->second->err;
    return HTF_OK;
}

int Server::wait(long long ticket, double timeout_ms, htf_request_info *out) {
    std::unique_lock<std::mutex> lk(mu_);
    auto it = all_.find(ticket);
    if (it == all_.end()) return HTF_EINVAL;
    Request *r = it->second.get();
    auto done = [&] { return r->info.status == HTF_REQ_DONE || r->info.status == HTF_REQ_FAILED; };
    if (timeout_ms < 0) cv_.wait(lk, done);
    else if (!cv_.wait_for(lk, std::chrono::duration<double, std::milli>(timeout_ms), done)) {
        if (out) *out = r->info;
        return HTF_ETIMEDOUT;
    }
    if (out) *out = r->info;
    return r->info.status == HTF_REQ_DONE ? HTF_OK : r->info.rc;
}

// device bytes of a request during and after setup, from the host-side
// problem (factor panels of all subdomains, or of the largest factor wave when
// wave_gb > 0; F_i tiles; S_i tiles of all subdomains, or of the largest wave
// without s_fp64; setup scratch, V, R, tensor-core slabs, coarse M, vectors), with a
// margin
size_t Server::estimate(const Problem &p, int nrhs, double wave_gb, bool s_fp64) const {
    const double K = opt_.batch;
    double b = 0.0, nslots = 0.0, nfull = 0.0, xs = 0.0;
    // panels (and S tiles) held at once: all, or the largest wave of the engine's partition
    const double cap = wave_gb > 0.0 ? std::max(1.0, wave_gb * 1e9 / 8.0) : 1e300;
    double panels = 0.0, wave = 0.0, stiles = 0.0, swave = 0.0;
    for (const Subdomain &s : p.sub) {
        const double nbp = 32.0 * ((s.nb + 31) / 32), nt = nbp / 32;
        const double kp = double(kpanel_doubles(s.n - s.nb, int(nbp)));
        if (wave > 0.0 && wave + kp > cap) wave = swave = 0.0;
        wave += kp;
        swave += nt * (nt + 1) / 2 * 1024.0;
        panels = std::max(panels, wave);
        stiles = std::max(stiles, swave);
    }
    b += 8.0 * panels;
    if (!s_fp64) b += 8.0 * stiles;
    if (wave_gb > 0.0) b += 296.0 * p.mesh.n_elems();     // element data kept for the re-assembly
    for (const Subdomain &s : p.sub) {
        const double nbp = 32.0 * ((s.nb + 31) / 32), N = (s.n - s.nb) + nbp, nt = nbp / 32;
        const double mb = std::ceil(nbp / 128.0), nks = nbp / 32;
        double stored = 0.0;                              // tensor-core slabs: lower triangle of 128-row blocks
        for (int m = 0; m < int(mb); ++m) stored += std::min(4.0 * (m + 1), nks);
        b += 8.0 * ((s_fp64 ? 2.0 : 1.0) * nt * (nt + 1) / 2 * 1024.0 + nbp * (s.c() + 6) + 6 * N + 2 * nbp);
        xs += nbp * nbp;
        b += 2.0 * stored * 4096.0 * 4.0;
        nslots += nbp;
        nfull += N;
    }
    b += 8.0 * std::min(xs, double(1LL << 29));           // L_bb^{-1} scratch of the set-up (one wave)
    for (const Cluster &c : p.clu) {          // dense M (batched coarse solves) + its packed tiles and partials
        const double mt = std::ceil(c.ngc() / 32.0);
        b += 8.0 * double(c.ngc()) * c.ngc() + 8.0 * mt * (mt + 1) / 2 * (1024.0 + 32.0) + 8.0 * 32.0 * mt;
    }
    const double nl = p.n_lam;
    b += nl * 8.0 * (11.0 * K + 12.0) + nslots * (K * (8.0 * 2 + 4.0 * 2) + 8.0 * 4) + nfull * 8.0 * (nrhs + 3);
    b += 3.0 * p.mesh.n_nodes * 8.0 * 2 * nrhs;
    return size_t(1.1 * b) + (size_t(16) << 20);
}

// host problem and device setup of one request, on its own stream
int Server::prepare(Request &r, std::string &err) {
    r.p = std::make_unique<Problem>();
    Problem &p = *r.p;
    p.opt = opt_;
    int rc = generate_mesh(r.spec, p.mesh, err);
    if (rc) return rc;
    p.nrhs = r.nrhs;
    if (!r.f.empty()) p.f_nodal = r.f;
    if ((rc = build_problem(p, err, true))) return rc;
    // with admit_oversize, factor panels that do not fit beside the rest are
    // held a wave at a time and factorised again for each later K_reg solve
    // (set-up start solve and reconstruction): a wave of half the room left by
    // everything else, at most 16 GB; if that is not enough, S_i is kept only
    // as its tensor-core slabs too
    double wave_gb = opt_.factor_wave_gb;
    bool s_fp64 = opt_.S_fp64;
    size_t est = estimate(p, r.nrhs, wave_gb, s_fp64);
    auto waves = [&] {
        if (opt_.factor_wave_gb > 0.0) return;
        const double rest = double(estimate(p, r.nrhs, 1e-9, s_fp64));
        wave_gb = std::min(16.0, std::max(1e-3, 0.5 * (budget_ - rest) / 1e9));
        est = estimate(p, r.nrhs, wave_gb, s_fp64);
    };
    const size_t resident = est;
    if (opt_.admit_oversize) {
        if (double(est) > budget_) waves();
        if (double(est) > budget_ && s_fp64) {
            s_fp64 = false;
            est = estimate(p, r.nrhs, wave_gb, s_fp64);
            if (double(est) > budget_) waves();
        }
    }
    p.opt.factor_wave_gb = wave_gb;
    p.opt.S_fp64 = s_fp64;
    {
        std::unique_lock<std::mutex> lk(mu_);
        r.info.bytes_estimate = double(est);
        if (double(est) > budget_) {
            err = opt_.admit_oversize
                      ? "request needs about " + std::to_string(est >> 20) +
                            " MiB with its factor panels held a wave at a time and S_i in the tensor-core slabs only, more than the "
                            "server budget"
                      : "request needs about " + std::to_string(resident >> 20) +
                            " MiB, more than the server budget (admit_oversize=1 admits it with its factor panels "
                            "held a wave at a time)";
            return HTF_ENOMEM;
        }
        // admission: waits for memory and a slot (live requests always finish)
        cv_.wait(lk, [&] { return in_use_ + est <= budget_ && admitted_ < max_live_; });
        in_use_ += double(est);
        r.bytes = est;
        r.info.bytes_estimate = double(est);
        ++admitted_;
        r.info.status = HTF_REQ_SETUP;
        r.info.t_admit_ms = now_ms();
    }
    r.eng = std::make_unique<Engine>(p.opt);
    rc = r.eng->setup(p, err);
    if (!rc) rc = r.eng->batch_loads(r.nrhs, r.f.empty() ? nullptr : r.f.data(), err);
    if (!rc) rc = r.eng->batch_begin(0, r.nrhs, err);
    if (!rc) rc = ck(cudaStreamSynchronize(r.eng->stream()), "cudaStreamSynchronize", err);
    const size_t actual = r.eng ? r.eng->device_bytes() : 0;
    {
        std::lock_guard<std::mutex> lk(mu_);
        in_use_ += double(actual) - double(r.bytes);
        r.bytes = actual;
        r.info.bytes = double(actual);
        r.info.setup_ms = r.eng ? r.eng->setup_ms : 0.0;
    }
    return rc;
}

void Server::finish(Request *r, int rc, const std::string &msg) {
    // caller holds no lock; frees the request's device memory
    if (r->eng) {
        r->eng->set_stream(nullptr);
        r->eng.reset();
    }
    if (r->joined) cudaEventDestroy(r->joined);
    if (r->rs && r->rs != stream_) cudaStreamDestroy(r->rs);
    r->joined = nullptr;
    r->rs = nullptr;
    r->p.reset();
    std::lock_guard<std::mutex> lk(mu_);
    if (r->info.status >= HTF_REQ_SETUP) {
        in_use_ -= double(r->bytes);
        --admitted_;
    }
    r->info.rc = rc;
    r->err = msg;
    r->info.status = rc == HTF_OK ? HTF_REQ_DONE : HTF_REQ_FAILED;
    r->info.t_done_ms = now_ms();
    --outstanding_;
    cv_.notify_all();
}

void Server::setup_loop() {
    cudaSetDevice(opt_.device);
    for (;;) {
        Request *r = nullptr;
        {
            std::unique_lock<std::mutex> lk(mu_);
            cv_.wait(lk, [&] { return stop_ || !queue_.empty(); });
            if (queue_.empty()) return;            // stopping and drained
            r = queue_.front();
            queue_.pop_front();
        }
        std::string err;
        const int rc = prepare(*r, err);
        if (rc) {
            finish(r, rc, err);
            continue;
        }
        std::lock_guard<std::mutex> lk(mu_);
        ready_.push_back(r);
        cv_.notify_all();
    }
}

void Server::release_graph() {
    if (graph_) {
        cudaGraphExecDestroy(graph_);
        graph_ = nullptr;
    }
}

// joint block table of the live requests and the captured macro iteration
int Server::rebuild_graph(std::string &err) {
    release_graph();
    std::vector<GemmBlock> blocks;
    std::vector<TcSet> sets;
    for (size_t i = 0; i < live_.size(); ++i) {
        Engine &e = *live_[i]->eng;
        sets.push_back(e.tc_set());
        for (GemmBlock g : e.tc_blocks()) {
            g.set = int(i);
            blocks.push_back(g);
        }
    }
    int rc;
    if (blocks.size() > cap_blocks_) {
        if (d_blocks_) cudaFree(d_blocks_);
        d_blocks_ = nullptr;
        cap_blocks_ = std::max<size_t>(blocks.size(), 2 * cap_blocks_);
        if ((rc = ck(cudaMalloc(&d_blocks_, cap_blocks_ * sizeof(GemmBlock)), "cudaMalloc", err))) return rc;
    }
    if (sets.size() > cap_sets_) {
        if (d_sets_) cudaFree(d_sets_);
        d_sets_ = nullptr;
        cap_sets_ = std::max<size_t>(sets.size(), 2 * cap_sets_);
        if ((rc = ck(cudaMalloc(&d_sets_, cap_sets_ * sizeof(TcSet)), "cudaMalloc", err))) return rc;
    }
    nblocks_ = int(blocks.size());
    if ((rc = ck(cudaMemcpyAsync(d_blocks_, blocks.data(), blocks.size() * sizeof(GemmBlock),
                                 cudaMemcpyHostToDevice, stream_), "cudaMemcpyAsync", err)))
        return rc;
    if ((rc = ck(cudaMemcpyAsync(d_sets_, sets.data(), sets.size() * sizeof(TcSet), cudaMemcpyHostToDevice,
                                 stream_), "cudaMemcpyAsync", err)))
        return rc;
    if ((rc = ck(cudaStreamSynchronize(stream_), "cudaStreamSynchronize", err))) return rc;
    const int smem = tc_smem_bytes(opt_.batch);
    cudaGraph_t g;
    if ((rc = ck(cudaStreamBeginCapture(stream_, cudaStreamCaptureModeThreadLocal), "cudaStreamBeginCapture", err)))
        return rc;
    // each request's phase on its own stream, forked from and joined back to the server stream
    auto phase = [&](void (Engine::*fn)()) -> int {
        int e = ck(cudaEventRecord(fork_, stream_), "cudaEventRecord", err);
        for (Request *r : live_) {
            if (!e) e = ck(cudaStreamWaitEvent(r->rs, fork_, 0), "cudaStreamWaitEvent", err);
            if (!e) ((*r->eng).*fn)();
            if (!e) e = ck(cudaEventRecord(r->joined, r->rs), "cudaEventRecord", err);
            if (!e) e = ck(cudaStreamWaitEvent(stream_, r->joined, 0), "cudaStreamWaitEvent", err);
        }
        return e;
    };
    rc = phase(&Engine::iter_a);
    if (!rc) tc_launch(opt_.batch, d_blocks_, nblocks_, d_sets_, 0, smem, d_err_, stream_);
    if (!rc) rc = phase(&Engine::iter_b);
    if (!rc) tc_launch(opt_.batch, d_blocks_, nblocks_, d_sets_, 1, smem, d_err_, stream_);
    if (!rc) rc = phase(&Engine::iter_c);
    const int rc_end = ck(cudaStreamEndCapture(stream_, &g), "cudaStreamEndCapture", err);
    if (rc) {
        if (!rc_end) cudaGraphDestroy(g);
        return rc;
    }
    if ((rc = rc_end)) return rc;
    rc = ck(cudaGraphInstantiate(&graph_, g, 0), "cudaGraphInstantiate", err);
    cudaGraphDestroy(g);
    dirty_ = false;
    return rc;
}

void Server::run_loop() {
    cudaSetDevice(opt_.device);
    for (;;) {
        {
            std::unique_lock<std::mutex> lk(mu_);
            cv_.wait(lk, [&] { return !ready_.empty() || !live_.empty() || (stop_ && outstanding_ == 0); });
            if (live_.empty() && ready_.empty()) return;     // stopping and drained
            for (Request *r : ready_) {
                if (!r->rs && cudaStreamCreateWithFlags(&r->rs, cudaStreamNonBlocking) != cudaSuccess) r->rs = stream_;
                if (!r->joined && cudaEventCreateWithFlags(&r->joined, cudaEventDisableTiming) != cudaSuccess)
                    r->joined = nullptr;
                r->eng->set_stream(r->rs);
                r->info.status = HTF_REQ_RUNNING;
                r->info.t_start_ms = now_ms();
                live_.push_back(r);
                dirty_ = true;
            }
            ready_.clear();
        }
        std::string err;
        int rc = HTF_OK;
        if (dirty_) rc = rebuild_graph(err);
        // work the requests left on their own streams (residual replacements) comes first
        for (Request *r : live_) {
            if (!rc && r->rs != stream_) rc = ck(cudaEventRecord(r->joined, r->rs), "cudaEventRecord", err);
            if (!rc && r->rs != stream_) rc = ck(cudaStreamWaitEvent(stream_, r->joined, 0), "cudaStreamWaitEvent", err);
        }
        for (int k = 0; !rc && k < opt_.check_every; ++k)
            rc = ck(cudaGraphLaunch(graph_, stream_), "cudaGraphLaunch", err);
        int tcerr = 0;
        if (!rc) rc = ck(cudaStreamSynchronize(stream_), "cudaStreamSynchronize", err);
        if (!rc) rc = ck(cudaMemcpy(&tcerr, d_err_, sizeof(int), cudaMemcpyDeviceToHost), "cudaMemcpy", err);
        if (!rc && tcerr) {
            rc = tcerr;
            err = "tensor-core product timed out on a barrier";
        }
        if (rc) {                                     // the joint work failed: every live request fails
            release_graph();
            std::vector<Request *> failed;
            failed.swap(live_);
            dirty_ = true;
            for (Request *r : failed) finish(r, rc, err);
            cudaMemset(d_err_, 0, sizeof(int));
            continue;
        }
        std::vector<Request *> keep;
        for (Request *r : live_) {
            bool done = false;
            std::string e2;
            int rc2 = r->eng->batch_check(done, e2);
            if (!rc2 && !done) {
                keep.push_back(r);
                continue;
            }
            double ms = 0.0;
            if (!rc2) rc2 = r->eng->batch_finish(&r->stats, ms, e2);
            if (rc2 != HTF_ECUDA && r->u_out) {
                cudaMemcpyAsync(r->u_out, r->eng->u_dev(), (size_t)r->eng->n_dof() * r->nrhs * sizeof(double),
                                cudaMemcpyDeviceToHost, r->eng->stream());
                if (cudaStreamSynchronize(r->eng->stream()) != cudaSuccess && !rc2) {
                    rc2 = HTF_ECUDA;
                    e2 = "copy of the displacements failed";
                }
            }
            int itmax = 0;
            for (int j = 0; j < r->nrhs && j < 64; ++j) itmax = std::max(itmax, r->stats.iterations[j]);
            r->info.iterations_max = itmax;
            r->info.solve_ms = ms;
            dirty_ = true;
            finish(r, rc2, e2);
        }
        live_.swap(keep);
    }
}

}  // namespace htf

// ---------------------------------------------------------------------------
struct htf_server {
    std::unique_ptr<htf::Server> s;
    std::mutex mu;
    std::map<long long, std::string> errs;
    std::string err;
};

extern "C" {

int htf_server_create(const char *options, double hbm_budget_bytes, int max_live, htf_server **srv) {
    if (!srv) return HTF_EINVAL;
    *srv = nullptr;
    htf::Options o;
    std::string err;
    int rc = htf::parse_options(options, o, err);
    if (rc) return rc;
    o.mixed = true;
    auto h = std::make_unique<htf_server>();
    h->s = std::make_unique<htf::Server>(o, hbm_budget_bytes, max_live > 0 ? max_live : 8);
    if ((rc = h->s->start(err))) return rc;
    *srv = h.release();
    return HTF_OK;
}

int htf_server_destroy(htf_server *srv) {
    delete srv;
    return HTF_OK;
}

int htf_server_submit(htf_server *srv, const htf_mesh_spec *spec, int n_rhs, const double *f_nodal, double *u,
                      long long *ticket) {
    if (!srv || !spec || !ticket) return HTF_EINVAL;
    std::string err;
    const int rc = srv->s->submit(*spec, n_rhs, f_nodal, u, ticket, err);
    if (rc) {
        std::lock_guard<std::mutex> lk(srv->mu);
        srv->err = err;
    }
    return rc;
}

int htf_server_wait(htf_server *srv, long long ticket, double timeout_ms, htf_request_info *info) {
    if (!srv) return HTF_EINVAL;
    return srv->s->wait(ticket, timeout_ms, info);
}

int htf_server_info(htf_server *srv, long long ticket, htf_request_info *info) {
    if (!srv) return HTF_EINVAL;
    return srv->s->info(ticket, info, nullptr);
}

const char *htf_server_error(htf_server *srv, long long ticket) {
    if (!srv) return "null server";
    std::lock_guard<std::mutex> lk(srv->mu);
    if (ticket <= 0) return srv->err.c_str();
    std::string m;
    if (srv->s->info(ticket, nullptr, &m) != HTF_OK) return "unknown ticket";
    srv->errs[ticket] = m;
    return srv->errs[ticket].c_str();
}

}  // extern "C"
