// Reconstruction server: 2D-slice and laminography jobs submitted from any
// host thread run concurrently on one GPU.
//
// The reference runs one reconstruction per process (src/recon.cpp:40-118,
// src/mbir2d.cpp:66-100): it builds the polar grid, the right-hand side and
// the point-spread function, then solves.  Here a fixed set of workers, each
// with its own context and stream, takes jobs from one FIFO queue:
//  * admission: the head job starts only when its estimated device footprint
//    fits in the HBM budget next to the jobs already running, so requests
//    that arrive while others run are admitted as workers and memory free up,
//    and their kernels overlap on the device; while the head waits for
//    memory, later jobs that fit start ahead of it (backfill), at most
//    `backfill` of them per head so that it cannot starve;
//  * 2D jobs run on high-priority streams: a slice submitted next to a
//    running laminography volume gets SMs as soon as CTAs of the volume
//    retire, instead of waiting behind its whole launches;
//  * a geometry-keyed cache keeps the FP32 Toeplitz spectra resident: a job on
//    a geometry seen before skips the PSF construction and shares the cached
//    spectrum read-only (only its work buffers are its own);
//  * the solvers replay their iterations as CUDA graphs when asked to;
//  * a failing job records its status and message and leaves the server and
//    the other jobs running.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <cstdio>
#include <cstring>
#include <deque>
#include <list>
#include <map>
#include <set>
#include <thread>
#include <vector>

#include "lc_internal.hpp"

using namespace lc;
using Clock = std::chrono::steady_clock;

namespace lc {
namespace {

double ms_between(Clock::time_point a, Clock::time_point b) {
    return std::chrono::duration<double, std::milli>(b - a).count();
}

struct Job {
    long long id = 0;
    bool three_d = false;
    const float *in = nullptr;    // host input, owned by the caller until the wait
    int d0 = 0, d1 = 0, d2 = 0;   // 2D: ns, ntheta, nradial; 3D: ntheta, nrows, ncols
    std::vector<double> theta, gamma, beta;
    std::vector<float> shifts;
    int recon_dims[3] = {0, 0, 0};
    lc_recon_params p{};
    float *out = nullptr;
    size_t bytes = 0;
    // results
    bool done = false;
    int status = LC_OK;
    std::string err;
    lc_solver_stats stats{};
    bool psf_hit = false;
    int worker = -1;
    Clock::time_point t_submit, t_start, t_end;
};

// Geometry-keyed cache of Toeplitz spectra, LRU-evicted under a byte cap.  A
// miss builds the spectrum on the caller's stream (the construction ends with
// a stream synchronisation, so a stored spectrum is complete before any other
// stream reads it); concurrent misses on one key wait for the first builder.
class PsfCache {
  public:
    explicit PsfCache(size_t cap) : cap_(cap) {}

    std::shared_ptr<Toeplitz> get(Context &ctx, const PolarGeometry &g, const long dims[3],
                                  bool three_d, bool *hit) {
        const std::string key = make_key(g, dims, three_d);
        std::unique_lock<std::mutex> lk(mu_);
        for (;;) {
            auto it = map_.find(key);
            if (it != map_.end()) {
                lru_.splice(lru_.begin(), lru_, it->second.pos);
                std::shared_ptr<Toeplitz> src = it->second.T;
                ++hits_;
                lk.unlock();
                if (hit) *hit = true;
                return std::make_shared<Toeplitz>(ctx, *src, true);
            }
            if (!building_.count(key)) break;
            cv_.wait(lk);
        }
        building_.insert(key);
        ++misses_;
        lk.unlock();
        std::shared_ptr<Toeplitz> T;
        try {
            T = std::make_shared<Toeplitz>(ctx, g, dims, three_d);
            // other workers read the spectrum on their own streams
            LC_CUDA(cudaStreamSynchronize(ctx.stream()));
        } catch (...) {
            lk.lock();
            building_.erase(key);
            cv_.notify_all();
            throw;
        }
        auto entry = std::make_shared<Toeplitz>(ctx, *T, false);
        lk.lock();
        building_.erase(key);
        const size_t b = entry->spectrum_bytes();
        if (b <= cap_) {
            while (used_ + b > cap_ && !lru_.empty()) evict_one();
            lru_.push_front(key);
            map_[key] = Entry{entry, b, lru_.begin()};
            used_ += b;
        }
        cv_.notify_all();
        if (hit) *hit = false;
        return T;
    }

    // drops every entry (jobs holding a spectrum keep their copy) and, with
    // `counters`, zeroes the hit and miss counts
    void clear(bool counters = false) {
        std::lock_guard<std::mutex> lk(mu_);
        map_.clear();
        lru_.clear();
        used_ = 0;
        if (counters) hits_ = misses_ = 0;
    }
    void counters(long &hits, long &misses, size_t &used, long &entries) {
        std::lock_guard<std::mutex> lk(mu_);
        hits = hits_;
        misses = misses_;
        used = used_;
        entries = (long)map_.size();
    }

  private:
    struct Entry {
        std::shared_ptr<Toeplitz> T;
        size_t bytes;
        std::list<std::string>::iterator pos;
    };
    // The PSF depends on the angles, the detector size and the padded volume
    // dims; shifts do not enter it.  The key holds the exact FP64 angles.
    static std::string make_key(const PolarGeometry &g, const long dims[3], bool three_d) {
        std::string k;
        auto put = [&](const void *p, size_t n) { k.append((const char *)p, n); };
        const int hdr[5] = {three_d ? 3 : 2, g.pts.ntheta, g.pts.nr, g.pts.nrows, g.pts.ncols};
        put(hdr, sizeof(hdr));
        put(dims, 3 * sizeof(long));
        put(g.theta.data(), g.theta.size() * sizeof(double));
        put(g.gamma.data(), g.gamma.size() * sizeof(double));
        put(g.beta.data(), g.beta.size() * sizeof(double));
        return k;
    }
    void evict_one() {
        auto it = map_.find(lru_.back());
        used_ -= it->second.bytes;
        map_.erase(it);
        lru_.pop_back();
    }
    size_t cap_, used_ = 0;
    long hits_ = 0, misses_ = 0;
    std::mutex mu_;
    std::condition_variable cv_;
    std::map<std::string, Entry> map_;
    std::list<std::string> lru_;
    std::set<std::string> building_;
};

size_t next23(long n) { return (size_t)next_smooth23(n); }

// Conservative device footprint of a job: inputs, detector lines, NUFFT
// grids, solver vectors, Toeplitz work buffers and a PSF construction.
size_t estimate_bytes(const Job &j) {
    const bool sb = j.p.method == 1;
    const size_t vecs = 2 + 3 + (sb ? 8 : 0);  // rhs, x; r, p, Ap; d[3], b[3], rhs, x_old
    if (!j.three_d) {
        const size_t ns = j.d0, nt = j.d1, nr = j.d2, n = j.recon_dims[1];
        const size_t M = nt * nr, nv = ns * n * n;
        const size_t nf = next23(std::max<long>(2 * (long)n, 8));
        size_t b = 4 * ns * M + 8 * ns * M;   // sinogram, complex detector lines
        b += 4 * M + 3 * 8 * nf * nf * ns;     // point permutation, fine grid and pruned passes
        b += 4 * nv * vecs;
        const long dims[3] = {(long)ns, (long)n, (long)n};
        b += Toeplitz::work_bytes(dims, false) + Toeplitz::build_peak_bytes(dims, false);
        return b + ((size_t)64 << 20);
    }
    const float pf = j.p.pad_factor;
    long N[3];
    for (int d = 0; d < 3; ++d) N[d] = odd_pad(j.recon_dims[d], pf);
    long PR = odd_pad(j.d1, pf), PC = odd_pad(j.d2, pf);
    if (pf - 1.0f < 1e-6f) {
        PR = j.d1;
        PC = j.d2;
    }
    const size_t nt = j.d0, M = nt * PR * PC, nv = (size_t)N[0] * N[1] * N[2];
    const size_t fine = next23(2 * N[0]) * next23(2 * N[1]) * next23(2 * N[2]);
    size_t b = 4 * nt * j.d1 * j.d2 + 4 * M + 8 * M;  // raw and padded projections, complex lines
    b += 4 * M + 3 * 8 * fine;
    b += 4 * nv * vecs;
    b += 4 * (size_t)j.recon_dims[0] * j.recon_dims[1] * j.recon_dims[2];
    b += Toeplitz::work_bytes(N, true) + Toeplitz::build_peak_bytes(N, true);
    return b + ((size_t)64 << 20);
}

}  // namespace
}  // namespace lc

struct lc_server_s {
    lc_server_params prm{};
    std::vector<std::unique_ptr<lc_context_s>> ctxs;
    std::vector<std::thread> workers;
    std::mutex mu;
    std::condition_variable cv_work, cv_done;
    std::deque<std::shared_ptr<Job>> queue;
    std::map<long long, std::shared_ptr<Job>> jobs;
    long long next_id = 1;
    size_t budget = 0, in_use = 0, peak_in_use = 0;
    int running = 0, peak_running = 0;
    int head_bypassed = 0;  // jobs started ahead of the current head
    long backfilled = 0;
    std::vector<cudaStream_t> hi_streams;  // per worker, for 2D jobs
    bool stopping = false;
    std::unique_ptr<PsfCache> cache;
    PsfProvider provider;
    std::string err;
    // finished jobs
    std::vector<double> latencies, lat2d, lat3d;
    long completed = 0, failed = 0;
    bool have_first = false;
    Clock::time_point t_first_submit, t_last_end;

    ~lc_server_s() {
        // the contexts' buffers may be ordered on the high-priority streams
        ctxs.clear();
        for (cudaStream_t x : hi_streams)
            if (x) cudaStreamDestroy(x);
    }
    void worker_loop(int w);
    void run_job(int w, Job &j);
    // the queued job to start now (queue.end() if none), called under mu
    std::deque<std::shared_ptr<Job>>::iterator pick();
};

std::deque<std::shared_ptr<Job>>::iterator lc_server_s::pick() {
    if (queue.empty()) return queue.end();
    // a job alone always starts; the head starts when it fits the budget
    if (running == 0 || in_use + queue.front()->bytes <= budget) return queue.begin();
    // backfill: the first later job that fits, while the head may still be bypassed
    if (head_bypassed >= prm.backfill) return queue.end();
    for (auto it = std::next(queue.begin()); it != queue.end(); ++it)
        if (in_use + (*it)->bytes <= budget) return it;
    return queue.end();
}

void lc_server_s::run_job(int w, Job &j) {
    lc_context c = ctxs[w].get();
    Context &ctx = *c->ctx;
    DeviceGuard dg(ctx.device());
    cudaStream_t s = ctx.stream();
    const PsfProvider *pp = cache ? &provider : nullptr;
    const long nin = (long)j.d0 * j.d1 * j.d2;
    const long nv = (long)j.recon_dims[0] * j.recon_dims[1] * j.recon_dims[2];
    // the job's stream: the worker's high-priority one for 2D jobs
    struct StreamSwap {
        Context &ctx;
        cudaStream_t prev;
        ~StreamSwap() { ctx.set_stream(prev); }
    } swap{ctx, s};
    if (!j.three_d && w < (int)hi_streams.size() && hi_streams[w]) {
        ctx.set_stream(hi_streams[w]);
        s = hi_streams[w];
    }
    DevBuf<float> din, dout(nv, s);
    if (!j.three_d) {
        din.upload(j.in, nin, s);
        mbir2d_core(c, din.get(), j.d0, j.d1, j.d2, j.theta.data(), j.recon_dims, &j.p, dout.get(),
                    &j.stats, pp, &j.psf_hit);
    } else {
        // the projections arrive while the geometry and (on a cache miss) the PSF are built
        din.alloc(nin, s);
        with_overlapped_upload(*c->ctx, din.get(), j.in, nin, [&](const std::function<void()> &load) {
            mbir3d_core(c, din.get(), j.d0, j.d1, j.d2, j.theta.data(), j.gamma.data(), j.beta.data(),
                        j.shifts.empty() ? nullptr : j.shifts.data(), j.recon_dims, &j.p, dout.get(),
                        &j.stats, pp, &j.psf_hit, load);
        });
    }
    LC_CUDA(cudaMemcpyAsync(j.out, dout.get(), nv * sizeof(float), cudaMemcpyDeviceToHost, s));
    LC_CUDA(cudaStreamSynchronize(s));
}

void lc_server_s::worker_loop(int w) {
    for (;;) {
        std::shared_ptr<Job> j;
        {
            std::unique_lock<std::mutex> lk(mu);
            // the head when it fits the budget next to the running jobs (a job
            // alone always starts), else a later job that fits (backfill)
            std::deque<std::shared_ptr<Job>>::iterator it;
            cv_work.wait(lk, [&] {
                if (queue.empty()) return stopping;
                it = pick();
                return it != queue.end();
            });
            if (queue.empty()) return;
            if (it == queue.begin()) {
                head_bypassed = 0;
            } else {
                ++head_bypassed;
                ++backfilled;
            }
            j = *it;
            queue.erase(it);
            in_use += j->bytes;
            peak_in_use = std::max(peak_in_use, in_use);
            ++running;
            peak_running = std::max(peak_running, running);
            j->worker = w;
            j->t_start = Clock::now();
        }
        std::string msg;
        // an error left on this thread by an earlier job must not fail this one
        cudaGetLastError();
        const int rc = run_guarded(msg, [&] { run_job(w, *j); });
        if (rc != LC_OK) {
            // leave the worker's stream idle and its context usable
            cudaStreamSynchronize(ctxs[w]->ctx->stream());
            cudaGetLastError();
        }
        {
            std::lock_guard<std::mutex> lk(mu);
            j->status = rc;
            j->err = msg;
            j->t_end = Clock::now();
            j->done = true;
            in_use -= j->bytes;
            --running;
            if (rc == LC_OK) {
                ++completed;
                const double lat = ms_between(j->t_submit, j->t_end);
                latencies.push_back(lat);
                (j->three_d ? lat3d : lat2d).push_back(lat);
            } else {
                ++failed;
            }
            t_last_end = j->t_end;
        }
        cv_done.notify_all();
        cv_work.notify_all();
    }
}

namespace {

int submit(lc_server sv, const std::shared_ptr<Job> &j, long long *job_id) {
    const int rc = run_guarded(sv->err, [&] {
        LC_REQUIRE(job_id, "NULL job id");
        LC_REQUIRE(j->in && j->out, "NULL input or output buffer");
        LC_REQUIRE(j->d0 > 0 && j->d1 > 0 && j->d2 > 0, "sizes must be positive");
        LC_REQUIRE(j->recon_dims[0] > 0 && j->recon_dims[1] > 0 && j->recon_dims[2] > 0,
                   "recon_dims must be positive");
        LC_REQUIRE(j->p.method == 0 || j->p.method == 1, "method must be 0 (CG) or 1 (Split-Bregman)");
        if (j->three_d)
            LC_REQUIRE(j->p.pad_factor >= 1.0f && j->p.pad_factor < 4.0f, "pad_factor must be in [1, 4)");
        j->bytes = estimate_bytes(*j);
        std::lock_guard<std::mutex> lk(sv->mu);
        LC_REQUIRE(!sv->stopping, "server is shutting down");
        if (j->bytes > sv->budget)
            throw Error(LC_ERR_TOO_LARGE, "job needs about " + std::to_string(j->bytes >> 20) +
                                              " MiB of device memory, above the server's HBM budget");
        j->id = sv->next_id++;
        j->t_submit = Clock::now();
        if (!sv->have_first) {
            sv->have_first = true;
            sv->t_first_submit = j->t_submit;
        }
        sv->jobs[j->id] = j;
        sv->queue.push_back(j);
        *job_id = j->id;
    });
    // wake an idle worker: the new job may be the head of the queue
    if (rc == LC_OK) sv->cv_work.notify_all();
    return rc;
}

// nearest-rank percentile
double percentile(std::vector<double> v, double q) {
    if (v.empty()) return 0.0;
    std::sort(v.begin(), v.end());
    size_t r = (size_t)std::ceil(q * (double)v.size());
    r = std::min(std::max<size_t>(r, 1), v.size());
    return v[r - 1];
}

}  // namespace

extern "C" {

void lc_server_params_default(lc_server_params *p) {
    if (!p) return;
    p->device = 0;
    p->workers = 4;
    p->hbm_budget_bytes = 0;  // 0: 85% of the free device memory at creation
    p->psf_cache_bytes = 0;   // 0: 16 GiB
    p->psf_cache = 1;
    p->backfill = 16;
    p->priority_2d = 1;
}

int lc_server_create(const lc_server_params *prm, lc_server *out) {
    if (!prm || !out) return LC_ERR_INVALID;
    *out = nullptr;
    if (prm->workers < 1 || prm->workers > 64) return LC_ERR_INVALID;
    if (prm->hbm_budget_bytes < 0 || prm->psf_cache_bytes < 0 || prm->backfill < 0) return LC_ERR_INVALID;
    auto sv = std::make_unique<lc_server_s>();
    std::string msg;
    const int rc = run_guarded(msg, [&] {
        sv->prm = *prm;
        DeviceGuard dg(prm->device);
        size_t free_b = 0, total_b = 0;
        LC_CUDA(cudaMemGetInfo(&free_b, &total_b));
        sv->budget = prm->hbm_budget_bytes > 0 ? (size_t)prm->hbm_budget_bytes
                                               : (size_t)(0.85 * (double)free_b);
        const size_t cap = prm->psf_cache_bytes > 0 ? (size_t)prm->psf_cache_bytes : (size_t)16 << 30;
        if (prm->psf_cache) {
            sv->cache = std::make_unique<PsfCache>(cap);
            PsfCache *pc = sv->cache.get();
            sv->provider = [pc](Context &ctx, const PolarGeometry &g, const long dims[3],
                                bool three_d, bool *hit) { return pc->get(ctx, g, dims, three_d, hit); };
        }
        for (int w = 0; w < prm->workers; ++w) {
            auto c = std::make_unique<lc_context_s>();
            c->ctx = std::make_unique<Context>(prm->device, nullptr);
            sv->ctxs.push_back(std::move(c));
        }
        if (prm->priority_2d) {
            int lo = 0, hi = 0;
            LC_CUDA(cudaDeviceGetStreamPriorityRange(&lo, &hi));  // hi: greatest priority
            sv->hi_streams.assign(prm->workers, nullptr);
            for (int w = 0; w < prm->workers; ++w)
                LC_CUDA(cudaStreamCreateWithPriority(&sv->hi_streams[w], cudaStreamNonBlocking, hi));
        }
        lc_server_s *raw = sv.get();
        for (int w = 0; w < prm->workers; ++w) sv->workers.emplace_back([raw, w] { raw->worker_loop(w); });
    });
    if (rc != LC_OK) {
        {
            std::lock_guard<std::mutex> lk(sv->mu);
            sv->stopping = true;
        }
        sv->cv_work.notify_all();
        for (auto &t : sv->workers) t.join();
        return rc;
    }
    *out = sv.release();
    return LC_OK;
}

int lc_server_destroy(lc_server sv) {
    if (!sv) return LC_ERR_INVALID;
    {
        std::lock_guard<std::mutex> lk(sv->mu);
        sv->stopping = true;  // queued jobs still run; new submissions are refused
    }
    sv->cv_work.notify_all();
    for (auto &t : sv->workers) t.join();
    {
        DeviceGuard dg(sv->prm.device);
        if (sv->cache) sv->cache->clear();
        sv->ctxs.clear();
        for (cudaStream_t &x : sv->hi_streams) {
            if (x) cudaStreamDestroy(x);
            x = nullptr;
        }
    }
    delete sv;
    return LC_OK;
}

int lc_server_submit2d(lc_server sv, const float *sino, int ns, int ntheta, int nradial,
                       const double *theta, const int *recon_dims, const lc_recon_params *p,
                       float *recon, long long *job_id) {
    if (!sv) return LC_ERR_INVALID;
    if (!theta || !recon_dims || !p || ntheta <= 0) {
        sv->err = "NULL argument or non-positive ntheta";
        return LC_ERR_INVALID;
    }
    auto j = std::make_shared<Job>();
    j->in = sino;
    j->d0 = ns;
    j->d1 = ntheta;
    j->d2 = nradial;
    j->theta.assign(theta, theta + ntheta);
    std::memcpy(j->recon_dims, recon_dims, sizeof(j->recon_dims));
    j->p = *p;
    j->out = recon;
    return submit(sv, j, job_id);
}

int lc_server_submit3d(lc_server sv, const float *projs, int ntheta, int nrows, int ncols,
                       const double *theta, const double *gamma, const double *beta,
                       const float *shifts, const int *recon_dims, const lc_recon_params *p,
                       float *recon, long long *job_id) {
    if (!sv) return LC_ERR_INVALID;
    if (!theta || !gamma || !beta || !recon_dims || !p || ntheta <= 0) {
        sv->err = "NULL argument or non-positive ntheta";
        return LC_ERR_INVALID;
    }
    auto j = std::make_shared<Job>();
    j->three_d = true;
    j->in = projs;
    j->d0 = ntheta;
    j->d1 = nrows;
    j->d2 = ncols;
    j->theta.assign(theta, theta + ntheta);
    j->gamma.assign(gamma, gamma + ntheta);
    j->beta.assign(beta, beta + ntheta);
    if (shifts) j->shifts.assign(shifts, shifts + 2 * (size_t)ntheta);
    std::memcpy(j->recon_dims, recon_dims, sizeof(j->recon_dims));
    j->p = *p;
    j->out = recon;
    return submit(sv, j, job_id);
}

int lc_server_wait(lc_server sv, long long job_id, double timeout_ms, lc_solver_stats *stats,
                   lc_job_info *info) {
    if (!sv) return LC_ERR_INVALID;
    std::shared_ptr<Job> j;
    {
        std::unique_lock<std::mutex> lk(sv->mu);
        auto it = sv->jobs.find(job_id);
        if (it == sv->jobs.end()) {
            sv->err = "unknown job id (already waited for?)";
            return LC_ERR_INVALID;
        }
        j = it->second;
        if (timeout_ms > 0) {
            const auto until = Clock::now() + std::chrono::duration<double, std::milli>(timeout_ms);
            if (!sv->cv_done.wait_until(lk, until, [&] { return j->done; })) {
                sv->err = "timed out waiting for the job (it stays queued or running)";
                return LC_ERR_TIMEOUT;
            }
        } else {
            sv->cv_done.wait(lk, [&] { return j->done; });
        }
        sv->jobs.erase(job_id);
    }
    if (stats) *stats = j->stats;
    if (info) {
        std::memset(info, 0, sizeof(*info));
        info->queue_ms = ms_between(j->t_submit, j->t_start);
        info->run_ms = ms_between(j->t_start, j->t_end);
        info->latency_ms = ms_between(j->t_submit, j->t_end);
        info->psf_hit = j->psf_hit ? 1 : 0;
        info->worker = j->worker;
        info->device_bytes = (double)j->bytes;
        std::snprintf(info->error, sizeof(info->error), "%s", j->err.c_str());
    }
    return j->status;
}

int lc_server_get_stats(lc_server sv, lc_server_stats *out) {
    if (!sv || !out) return LC_ERR_INVALID;
    std::memset(out, 0, sizeof(*out));
    {
        std::lock_guard<std::mutex> lk(sv->mu);
        out->completed = sv->completed;
        out->failed = sv->failed;
        out->queued = (long)sv->queue.size();
        out->running = sv->running;
        out->peak_running = sv->peak_running;
        out->p50_ms = percentile(sv->latencies, 0.50);
        out->p99_ms = percentile(sv->latencies, 0.99);
        double sum = 0;
        for (double v : sv->latencies) sum += v;
        out->mean_ms = sv->latencies.empty() ? 0.0 : sum / (double)sv->latencies.size();
        if (sv->have_first && sv->completed > 0) {
            out->span_s = ms_between(sv->t_first_submit, sv->t_last_end) / 1e3;
            out->recons_per_s = out->span_s > 0 ? (double)sv->completed / out->span_s : 0.0;
        }
        out->hbm_budget_bytes = (double)sv->budget;
        out->peak_admitted_bytes = (double)sv->peak_in_use;
        out->p50_2d_ms = percentile(sv->lat2d, 0.50);
        out->p99_2d_ms = percentile(sv->lat2d, 0.99);
        out->p50_3d_ms = percentile(sv->lat3d, 0.50);
        out->p99_3d_ms = percentile(sv->lat3d, 0.99);
        out->backfilled = sv->backfilled;
    }
    if (sv->cache) {
        size_t used = 0;
        sv->cache->counters(out->psf_hits, out->psf_misses, used, out->psf_cache_entries);
        out->psf_cache_bytes = (double)used;
    }
    return LC_OK;
}

int lc_server_reset_stats(lc_server sv) {
    if (!sv) return LC_ERR_INVALID;
    std::lock_guard<std::mutex> lk(sv->mu);
    sv->latencies.clear();
    sv->lat2d.clear();
    sv->lat3d.clear();
    sv->backfilled = 0;
    sv->completed = sv->failed = 0;
    sv->have_first = false;
    sv->peak_in_use = sv->in_use;
    sv->peak_running = sv->running;
    return LC_OK;
}

int lc_server_clear_psf_cache(lc_server sv) {
    if (!sv) return LC_ERR_INVALID;
    if (sv->cache) sv->cache->clear(true);
    return LC_OK;
}

const char *lc_server_last_error(lc_server sv) { return sv ? sv->err.c_str() : "NULL server"; }

}  // extern "C"
