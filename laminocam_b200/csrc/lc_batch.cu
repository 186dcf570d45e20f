// Cross-job batching of unregularised 2D CG reconstructions: the jobs of a
// batch (one slice each, any image size n and angle count) iterate in
// lockstep, and every stage of an iteration is ONE launch over all of them.
//
// The reference solves slices one at a time: include/gpu/nufft.h:92-95 runs
// one cuFINUFFT execute per slice, include/gpu/toeplitz2d.h:68-76 one Thrust
// multiply per slice, src/gpu/conjgrad.cu:45-108 a handful of launches and
// host syncs per iteration per job.  Here an iteration is six launches for
// the whole batch:
//   p = r + beta p                     work list of (job, chunk) items
//   Toeplitz x rows (R2C)              AxisFFTBatch: (job, row group) CTAs
//   Toeplitz y columns x spectrum      AxisFFTBatch: (job, column group) CTAs
//   Toeplitz x rows (C2R, scaled)      AxisFFTBatch
//   p.Ap and alpha                     (job, chunk) items
//   x += alpha p, r -= alpha Ap, beta  (job, chunk) items
// Every job keeps its own FP64 scalars (CGState) and stopping tests in device
// memory; a job whose test fired, or whose iteration budget is spent, turns
// the later launches into no-ops for its CTAs.  Each job's reductions are
// per-chunk FP64 partials summed by the job's last CTA (a per-job ticket) in
// chunk order, and the chunking depends on the job's size alone, so a job's
// result is bit-for-bit the same whatever else is in the batch.
//
// The setup of every job (sinogram upload, bin sort, backprojection, FP64
// PSF) runs on a pool of worker contexts, each with its own stream; the
// batched iterations then run on the caller's context, replayed from a CUDA
// graph of eight iterations.
#include <algorithm>
#include <atomic>
#include <cmath>
#include <memory>
#include <thread>
#include <vector>

#include "../../include/laminocam.h"
#include "lc_internal.hpp"
#include "lc_solver.hpp"
#include "lc_toeplitz.hpp"

namespace lc {

namespace {

constexpr int kVecThreads = 256;
constexpr long kChunk = 4096;  // elements of one job's vectors per CTA

struct VecJob {
    float *x, *r, *p, *ap;
    const float *y;
    long n;
    int part0;   // first partial slot (chunk index base) of this job
    int nchunks;
    int max_iters;
    float tol, xtol;
};

// Block reduce of K sums; the job's partial slot `slot` gets them.  Returns
// true in every thread of the CTA that finished the job's chunks last.
template <int K>
__device__ bool job_partials(double (&v)[K], double *part, long slot, unsigned *counter, int nchunks) {
    __shared__ double sh[K][kVecThreads / 32];
    __shared__ bool last;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
    for (int k = 0; k < K; ++k) {
        double s = v[k];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
        if (lane == 0) sh[k][wid] = s;
    }
    __syncthreads();
    if (threadIdx.x < 32) {
#pragma unroll
        for (int k = 0; k < K; ++k) {
            double s = lane < kVecThreads / 32 ? sh[k][lane] : 0.0;
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
            if (lane == 0) part[slot * 4 + k] = s;
        }
    }
    __threadfence();
    if (threadIdx.x == 0) {
        const unsigned t = atomicAdd(counter, 1u);
        last = (t == (unsigned)nchunks - 1);
    }
    __syncthreads();
    return last;
}

// Fixed-order total of partial k over a job's chunks (the last CTA of the job)
__device__ double job_total(const double *part, int part0, int nchunks, int k) {
    __shared__ double sh[kVecThreads / 32];
    __shared__ double res;
    double s = 0.0;
    for (int c = threadIdx.x; c < nchunks; c += blockDim.x) s += part[((long)part0 + c) * 4 + k];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    if (lane == 0) sh[wid] = s;
    __syncthreads();
    if (threadIdx.x < 32) {
        double t = lane < kVecThreads / 32 ? sh[lane] : 0.0;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) t += __shfl_down_sync(0xffffffffu, t, o);
        if (lane == 0) res = t;
    }
    __syncthreads();
    const double out = res;
    __syncthreads();
    return out;
}

// r = y, p = y (x0 = 0); y.y; the job's state starts over
__global__ void __launch_bounds__(kVecThreads) batch_init_kernel(const VecJob *__restrict__ jobs,
                                                                 const int2 *__restrict__ items, CGState *st,
                                                                 double *part, unsigned *counters) {
    const int2 it = items[blockIdx.x];
    const VecJob J = jobs[it.x];
    const long b = (long)it.y * kChunk, e = min(J.n, b + kChunk);
    double v[1] = {0.0};
    for (long i = b + threadIdx.x; i < e; i += kVecThreads) {
        const float yi = J.y[i];
        J.r[i] = yi;
        J.p[i] = yi;
        v[0] += (double)yi * (double)yi;
    }
    if (job_partials<1>(v, part, (long)J.part0 + it.y, counters + it.x, J.nchunks)) {
        const double y2 = job_total(part, J.part0, J.nchunks, 0);
        if (threadIdx.x == 0) {
            CGState &s = st[it.x];
            s.y2 = y2;
            s.rs_old = y2;
            s.beta = 0.0;
            s.iters = 0;
            s.done = J.max_iters <= 0 ? 1 : 0;
            s.reason = 0;
            s.res = 0;
            s.dx = 0;
            counters[it.x] = 0;
        }
    }
}

__global__ void __launch_bounds__(kVecThreads) batch_p_update_kernel(const VecJob *__restrict__ jobs,
                                                                     const int2 *__restrict__ items,
                                                                     const CGState *st) {
    const int2 it = items[blockIdx.x];
    if (st[it.x].done) return;
    const VecJob J = jobs[it.x];
    const float beta = (float)st[it.x].beta;
    const long b = (long)it.y * kChunk, e = min(J.n, b + kChunk);
    for (long i = b + threadIdx.x; i < e; i += kVecThreads) J.p[i] = fmaf(beta, J.p[i], J.r[i]);
}

// p.Ap, then alpha = r.r / p.Ap, or the |p.Ap| < 1e-10 stop (src/conjgrad.cpp:53-56)
__global__ void __launch_bounds__(kVecThreads) batch_dot_kernel(const VecJob *__restrict__ jobs,
                                                                const int2 *__restrict__ items, CGState *st,
                                                                double *part, unsigned *counters) {
    const int2 it = items[blockIdx.x];
    if (st[it.x].done) return;
    const VecJob J = jobs[it.x];
    const long b = (long)it.y * kChunk, e = min(J.n, b + kChunk);
    double v[1] = {0.0};
    for (long i = b + threadIdx.x; i < e; i += kVecThreads) v[0] += (double)J.p[i] * (double)J.ap[i];
    if (job_partials<1>(v, part, (long)J.part0 + it.y, counters + it.x, J.nchunks)) {
        const double pap = job_total(part, J.part0, J.nchunks, 0);
        if (threadIdx.x == 0) {
            CGState &s = st[it.x];
            s.pAp = pap;
            if (fabs(pap) < 1e-10) {
                s.done = 1;
                s.reason = 3;
            } else {
                s.alpha = s.rs_old / pap;
            }
            counters[it.x] = 0;
        }
    }
}

// x += alpha p, r -= alpha Ap; r.r, |alpha p|^2, x.x; beta, the residual and
// step tests (src/gpu/conjgrad.cu:85,97) and the iteration budget
__global__ void __launch_bounds__(kVecThreads) batch_update_kernel(const VecJob *__restrict__ jobs,
                                                                   const int2 *__restrict__ items, CGState *st,
                                                                   double *part, unsigned *counters) {
    const int2 it = items[blockIdx.x];
    if (st[it.x].done) return;
    const VecJob J = jobs[it.x];
    const float a = (float)st[it.x].alpha;
    const long b = (long)it.y * kChunk, e = min(J.n, b + kChunk);
    double v[3] = {0.0, 0.0, 0.0};
    for (long i = b + threadIdx.x; i < e; i += kVecThreads) {
        const float step = a * J.p[i];
        const float xi = J.x[i] + step;
        const float ri = fmaf(-a, J.ap[i], J.r[i]);
        J.x[i] = xi;
        J.r[i] = ri;
        v[0] += (double)ri * (double)ri;
        v[1] += (double)step * (double)step;
        v[2] += (double)xi * (double)xi;
    }
    if (job_partials<3>(v, part, (long)J.part0 + it.y, counters + it.x, J.nchunks)) {
        const double rs = job_total(part, J.part0, J.nchunks, 0);
        const double s2 = job_total(part, J.part0, J.nchunks, 1);
        const double x2 = job_total(part, J.part0, J.nchunks, 2);
        if (threadIdx.x == 0) {
            CGState &s = st[it.x];
            s.beta = rs / s.rs_old;
            s.rs_old = rs;
            s.res = sqrt(rs) / (sqrt(s.y2) + 1e-8);
            s.dx = sqrt(s2) / (sqrt(x2) + 1e-8);
            s.iters += 1;
            if (s.res < (double)J.tol) {
                s.done = 1;
                s.reason = 1;
            } else if (s.dx < (double)J.xtol) {
                s.done = 1;
                s.reason = 2;
            } else if (s.iters >= J.max_iters) {
                s.done = 1;
                s.reason = 0;
            }
            counters[it.x] = 0;
        }
    }
}

}  // namespace

// One lockstep CG over several 2D Toeplitz operators.
class BatchCG2D {
  public:
    struct Job {
        std::shared_ptr<Toeplitz> T;  // 2D, one slice
        const float *y;               // right-hand side (device, n x n)
        float *x;                     // solution (device, n x n); starts at zero
        int max_iters;
        float tol, xtol;
    };

    BatchCG2D(Context &ctx, std::vector<Job> jobs) : jobs_(std::move(jobs)) {
        cudaStream_t s = ctx.stream();
        const int J = (int)jobs_.size();
        LC_REQUIRE(J > 0, "batch: no jobs");
        std::vector<long> voff(J), hoff(J);
        long vtot = 0, htot = 0;
        int chunks = 0;
        for (int j = 0; j < J; ++j) {
            const Toeplitz &T = *jobs_[j].T;
            LC_REQUIRE(!T.three_d() && T.dims()[0] == 1, "batch: 2D operators of one slice only");
            LC_REQUIRE(T.P()[2] % 2 == 0, "batch: the Toeplitz grid must be even");
            const long n = T.nvox();
            voff[j] = vtot;
            vtot += (n + 3) & ~3L;  // 16-byte aligned vectors
            hoff[j] = htot;
            htot += T.dims()[1] * (T.P()[2] / 2 + 1);
            chunks += (int)((n + kChunk - 1) / kChunk);
        }
        vec_.alloc(3 * vtot, s);  // r, p, Ap
        h_.alloc(htot, s);
        st_.alloc(J, s);
        counters_.alloc(J, s);
        counters_.zero(s);
        part_.alloc((size_t)chunks * 4, s);
        std::vector<VecJob> vj(J);
        std::vector<int2> items;
        items.reserve(chunks);
        int part0 = 0;
        for (int j = 0; j < J; ++j) {
            const Toeplitz &T = *jobs_[j].T;
            const long n = T.nvox();
            VecJob &v = vj[j];
            v.x = jobs_[j].x;
            v.y = jobs_[j].y;
            v.r = vec_.get() + voff[j];
            v.p = vec_.get() + vtot + voff[j];
            v.ap = vec_.get() + 2 * vtot + voff[j];
            v.n = n;
            v.part0 = part0;
            v.nchunks = (int)((n + kChunk - 1) / kChunk);
            v.max_iters = jobs_[j].max_iters;
            v.tol = jobs_[j].tol;
            v.xtol = jobs_[j].xtol;
            for (int c = 0; c < v.nchunks; ++c) items.push_back(make_int2(j, c));
            part0 += v.nchunks;
            add_toeplitz(ctx, T, v.p, v.ap, h_.get() + hoff[j], &st_.get()[j].done);
        }
        vjobs_.upload(vj.data(), J, s);
        items_.upload(items.data(), items.size(), s);
        nitems_ = (int)items.size();
        rows_fwd_.finalize(ctx);
        cols_.finalize(ctx);
        rows_inv_.finalize(ctx);
        host_vj_ = std::move(vj);
    }

    // Runs every job to its stopping test or iteration budget.
    void run(Context &ctx, bool use_graph, std::vector<CGState> *out) {
        cudaStream_t s = ctx.stream();
        int maxit = 0;
        bool poll = false;
        for (const Job &j : jobs_) {
            maxit = std::max(maxit, j.max_iters);
            poll = poll || j.tol > 0.f || j.xtol > 0.f;
        }
        batch_init_kernel<<<nitems_, kVecThreads, 0, s>>>(vjobs_.get(), items_.get(), st_.get(), part_.get(),
                                                          counters_.get());
        LC_CHECK_LAUNCH();
        const int chunk = 8;
        CapturedGraph graph;
        for (int done = 0; done < maxit; done += chunk) {
            const int k = std::min(chunk, maxit - done);
            if (use_graph && k == chunk) {
                if (!graph.ready()) {
                    ctx.set_stream(ctx.capture_stream());
                    graph.capture(ctx.capture_stream(), [&] {
                        for (int i = 0; i < chunk; ++i) iteration(ctx);
                    });
                    ctx.set_stream(s);
                }
                graph.launch(s);
            } else {
                for (int i = 0; i < k; ++i) iteration(ctx);
            }
            if (poll && done + k < maxit) {
                std::vector<CGState> hs(jobs_.size());
                LC_CUDA(cudaMemcpyAsync(hs.data(), st_.get(), hs.size() * sizeof(CGState), cudaMemcpyDeviceToHost,
                                        s));
                LC_CUDA(cudaStreamSynchronize(s));
                if (std::all_of(hs.begin(), hs.end(), [](const CGState &c) { return c.done != 0; })) break;
            }
        }
        if (out) {
            out->resize(jobs_.size());
            LC_CUDA(cudaMemcpyAsync(out->data(), st_.get(), out->size() * sizeof(CGState), cudaMemcpyDeviceToHost,
                                    s));
        }
        LC_CUDA(cudaStreamSynchronize(s));
    }

    long launches_per_iteration() const { return 6; }

  private:
    void iteration(Context &ctx) {
        cudaStream_t s = ctx.stream();
        batch_p_update_kernel<<<nitems_, kVecThreads, 0, s>>>(vjobs_.get(), items_.get(), st_.get());
        LC_CHECK_LAUNCH();
        rows_fwd_.launch(ctx);
        cols_.launch(ctx);
        rows_inv_.launch(ctx);
        batch_dot_kernel<<<nitems_, kVecThreads, 0, s>>>(vjobs_.get(), items_.get(), st_.get(), part_.get(),
                                                         counters_.get());
        LC_CHECK_LAUNCH();
        batch_update_kernel<<<nitems_, kVecThreads, 0, s>>>(vjobs_.get(), items_.get(), st_.get(), part_.get(),
                                                            counters_.get());
        LC_CHECK_LAUNCH();
    }

    // the three passes of the 2D Toeplitz apply (lc_toeplitz.cu) as items of
    // the three batched launches
    void add_toeplitz(Context &ctx, const Toeplitz &T, const float *p, float *ap, float2 *h, const int *skip) {
        const long n = T.dims()[1];
        const int P = T.P()[2], Ph = P / 2 + 1;
        AxisFFT a;
        a.in = p;
        a.in_t = E_F32;
        a.out = h;
        a.out_t = E_C64;
        a.n_outer = n;
        a.n_inner = 1;
        a.in_ostride = n;
        a.out_ostride = Ph;
        a.n_in = (int)n;
        a.L = P / 2;
        a.n_out = Ph;
        a.in_map = IN_REAL_PACKED;
        a.out_map = OUT_R2C_UNPACK;
        a.sign = -1;
        rows_fwd_.add(ctx, a, skip);
        AxisFFT b;
        b.in = h;
        b.in_t = E_C64;
        b.out = h;
        b.out_t = E_C64;
        b.n_outer = 1;
        b.n_inner = Ph;
        b.in_ostride = n * Ph;
        b.out_ostride = n * Ph;
        b.n_in = (int)n;
        b.L = P;
        b.n_out = (int)n;
        b.out_map = OUT_WINDOW;
        b.out_off = 0;
        b.sign = -1;
        b.mid = T.spectrum();
        b.mid_ra = Ph;
        b.sign2 = +1;
        cols_.add(ctx, b, skip);
        AxisFFT c;
        c.in = h;
        c.in_t = E_C64;
        c.out = ap;
        c.out_t = E_F32;
        c.n_outer = n;
        c.n_inner = 1;
        c.in_ostride = Ph;
        c.out_ostride = n;
        c.n_in = Ph;
        c.L = P / 2;
        c.n_out = (int)n;
        c.in_map = IN_C2R_PACK;
        c.out_map = OUT_REAL_UNPACK;
        c.out_off = 0;
        c.sign = +1;
        c.scale = T.scale();
        rows_inv_.add(ctx, c, skip);
    }

    std::vector<Job> jobs_;
    std::vector<VecJob> host_vj_;
    DevBuf<float> vec_;
    DevBuf<float2> h_;
    DevBuf<CGState> st_;
    DevBuf<unsigned> counters_;
    DevBuf<double> part_;
    DevBuf<VecJob> vjobs_;
    DevBuf<int2> items_;
    int nitems_ = 0;
    AxisFFTBatch rows_fwd_, cols_, rows_inv_;
};

}  // namespace lc

using namespace lc;

extern "C" int lc_mbir2d_batch(lc_context c, const lc_job2d *jobs, int njobs, const lc_recon_params *p,
                               int setup_workers, lc_solver_stats *stats) {
    return guarded(c, [&] {
        LC_REQUIRE(jobs && p && njobs > 0, "NULL argument or no jobs");
        LC_REQUIRE(p->method == 0, "lc_mbir2d_batch: batched jobs use CG (method 0)");
        LC_REQUIRE(p->solver.max_iters >= 0, "iteration counts must be >= 0");
        LC_REQUIRE(std::isfinite(p->solver.tol) && std::isfinite(p->solver.xtol), "tolerances must be finite");
        for (int j = 0; j < njobs; ++j) {
            const lc_job2d &q = jobs[j];
            LC_REQUIRE(q.sinogram && q.theta && q.recon, "job with a NULL pointer");
            LC_REQUIRE(q.ntheta > 0 && q.nradial > 0 && q.n > 0, "job sizes must be positive");
        }
        Context &ctx = *c->ctx;
        cudaStream_t s = ctx.stream();
        const int nw = std::max(1, std::min(setup_workers > 0 ? setup_workers : 8, njobs));
        // per job: right-hand side and Toeplitz operator, built on the workers
        std::vector<std::unique_ptr<lc_context_s>> wctx(nw);
        for (int w = 0; w < nw; ++w) {
            wctx[w].reset(new lc_context_s);
            wctx[w]->ctx = std::make_shared<Context>(ctx.device(), nullptr);
        }
        std::vector<DevBuf<float>> rhs(njobs), xs(njobs);
        std::vector<std::shared_ptr<Toeplitz>> ops(njobs);
        std::vector<std::string> errs(njobs);
        std::atomic<int> next{0};
        auto work = [&](int w) {
            lc_context wc = wctx[w].get();
            Context &wx = *wc->ctx;
            DeviceGuard dg(wx.device());
            for (int j = next++; j < njobs; j = next++) {
                const lc_job2d &q = jobs[j];
                const int rc = run_guarded(errs[j], [&] {
                    cudaStream_t ws = wx.stream();
                    DevBuf<float> dsino;
                    dsino.upload(q.sinogram, (size_t)q.ntheta * q.nradial, ws);
                    lc_geometry g = nullptr;
                    const int grc = lc_geometry2d_create(wc, q.theta, q.ntheta, q.nradial, &g);
                    if (grc) throw Error(grc == LC_ERR_INVALID ? 1 : 3, wc->err);
                    std::unique_ptr<lc_geometry_s> gown(g);
                    const long nv = (long)q.n * q.n;
                    rhs[j].alloc(nv, ws);
                    xs[j].alloc(nv, ws);
                    LC_CUDA(cudaMemsetAsync(xs[j].get(), 0, nv * sizeof(float), ws));
                    const int brc = lc_backproj2d(wc, g, dsino.get(), 1, q.n, q.n, rhs[j].get(), p->nufft_tol);
                    if (brc) throw Error(brc == LC_ERR_INVALID ? 1 : 3, wc->err);
                    const long dims[3] = {1, q.n, q.n};
                    ops[j] = std::make_shared<Toeplitz>(wx, g->g, dims, false);
                    LC_CUDA(cudaStreamSynchronize(ws));
                });
                if (rc && errs[j].empty()) errs[j] = "setup failed";
            }
        };
        std::vector<std::thread> th;
        for (int w = 1; w < nw; ++w) th.emplace_back(work, w);
        work(0);
        for (auto &t : th) t.join();
        for (int j = 0; j < njobs; ++j)
            if (!errs[j].empty()) throw Error(1, "job " + std::to_string(j) + ": " + errs[j]);
        std::vector<BatchCG2D::Job> bj(njobs);
        for (int j = 0; j < njobs; ++j)
            bj[j] = {ops[j], rhs[j].get(), xs[j].get(), p->solver.max_iters, p->solver.tol, p->solver.xtol};
        std::vector<CGState> fin;
        {
            BatchCG2D batch(ctx, std::move(bj));
            batch.run(ctx, p->solver.use_graph != 0, &fin);
        }
        for (int j = 0; j < njobs; ++j) {
            const long nv = (long)jobs[j].n * jobs[j].n;
            LC_CUDA(cudaMemcpyAsync(jobs[j].recon, xs[j].get(), nv * sizeof(float), cudaMemcpyDeviceToHost, s));
            if (stats) {
                stats[j].iters = fin[j].iters;
                stats[j].cg_iters_total = fin[j].iters;
                stats[j].residual = fin[j].res;
                stats[j].dx = fin[j].dx;
                stats[j].stop_reason = fin[j].reason;
                stats[j].elapsed_ms = 0.0;
            }
        }
        LC_CUDA(cudaStreamSynchronize(s));
        // worker-owned buffers are released in the order of the workers' streams
        for (auto &o : ops) o.reset();
        for (auto &b : rhs) b.release();
        for (auto &b : xs) b.release();
        for (auto &w : wctx) LC_CUDA(cudaStreamSynchronize(w->ctx->stream()));
    });
}
