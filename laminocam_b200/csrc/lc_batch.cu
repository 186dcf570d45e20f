// Cross-job batching of unregularised 2D CG reconstructions: the jobs of a
// batch (one slice each, any image size n and angle count) iterate in
// lockstep, and every stage of an iteration is launched once for the whole
// batch, or once per Toeplitz grid size P for the FFT passes.
//
// The reference solves slices one at a time: include/gpu/nufft.h:92-95 runs
// one cuFINUFFT execute per slice, include/gpu/toeplitz2d.h:68-76 one Thrust
// multiply per slice, src/gpu/conjgrad.cu:45-108 a handful of launches and
// host syncs per iteration per job.  Here an iteration is:
//   per grid size P, in parallel graph branches, over the jobs of that P:
//     Toeplitz x rows (R2C)             one launch, (job, row group) CTAs;
//                                       p = r + beta p on the way in
//     Toeplitz y columns x spectrum     one launch, (job, column group) CTAs
//     Toeplitz x rows (C2R, scaled)     one launch; p.Ap and alpha on the
//                                       way out (per-job partials and ticket)
//   x += alpha p, r -= alpha Ap, beta   one launch, (job, chunk) items
// The FFT passes use the register-plan row and column kernels (batched over
// an item table) where a plan covers P, else the generic shared-memory kernel
// (AxisFFTBatch), whose jobs take the direction update and p.Ap as vector
// launches of their own at the ends of their branch.  A launch per P keeps
// the compile-time plan of those kernels, and the branches run concurrently.
//
// Every job keeps its own FP64 scalars (CGState) and stopping tests in device
// memory; a job whose test fired, or whose iteration budget is spent, turns
// the later launches into no-ops for its CTAs.  Each job's reductions are
// per-chunk FP64 partials summed by the job's last CTA (a per-job ticket) in
// chunk order, and the chunking and FFT kernels depend on the job's size
// alone, so a job's result is bit-for-bit the same whatever else is in the
// batch.
//
// The setup of every job (sinogram upload, bin sort, backprojection, FP64
// PSF) runs on a pool of worker contexts, each with its own stream; the
// batched iterations run on the caller's context, replayed from a CUDA graph
// of eight iterations.  Batches of eight jobs or more run in two waves: the
// larger half (by pixels x angles) iterates while the workers still set up
// the other half, so setup and iterations overlap on the GPU.
#include <algorithm>
#include <atomic>
#include <cmath>
#include <condition_variable>
#include <memory>
#include <mutex>
#include <thread>
#include <vector>

#include "../../include/laminocam.h"
#include "lc_internal.hpp"
#include "lc_reduce.cuh"
#include "lc_solver.hpp"
#include "lc_toeplitz.hpp"

// Host time of the setup phases (geometry, backprojection queued, PSF
// queued, stream drained), summed over jobs, printed to stderr when the
// library is built with -DLC_BATCH_TRACE (a profiling build).
#ifdef LC_BATCH_TRACE
#include <chrono>
#include <cstdio>
static double g_batch_t[4];
static std::mutex g_batch_mu;
#define LC_BATCH_T0() auto lc_bt_prev = std::chrono::steady_clock::now()
#define LC_BATCH_T(k)                                                                          \
    do {                                                                                       \
        auto lc_bt_now = std::chrono::steady_clock::now();                                     \
        std::lock_guard<std::mutex> lc_bt_lk(g_batch_mu);                                      \
        g_batch_t[k] += std::chrono::duration<double, std::milli>(lc_bt_now - lc_bt_prev).count(); \
        lc_bt_prev = lc_bt_now;                                                                \
    } while (0)
#else
#define LC_BATCH_T0() ((void)0)
#define LC_BATCH_T(k) ((void)0)
#endif

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
        std::vector<long> voff(J), hoff(J), roff(J);
        long vtot = 0, htot = 0, rtot = 0;
        int chunks = 0;
        for (int j = 0; j < J; ++j) {
            const Toeplitz &T = *jobs_[j].T;
            LC_REQUIRE(!T.three_d() && T.dims()[0] == 1, "batch: 2D operators of one slice only");
            const long n = T.nvox();
            voff[j] = vtot;
            vtot += (n + 3) & ~3L;  // 16-byte aligned vectors
            hoff[j] = htot;
            htot += T.dims()[1] * (T.P()[2] / 2 + 1);
            roff[j] = rtot;
            rtot += row_fft_ctas(T.dims()[1]);
            chunks += (int)((n + kChunk - 1) / kChunk);
        }
        vec_.alloc(3 * vtot, s);  // r, p, Ap
        h_.alloc(htot, s);
        st_.alloc(J, s);
        counters_.alloc(J, s);
        counters_.zero(s);
        part_.alloc((size_t)chunks * 4, s);
        rpart_.alloc((size_t)rtot * kRedParts, s);  // p.Ap partials of the fused row passes
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
            Group &g = group_for(T.P()[2]);
            CGFusion f;
            f.p = v.p;
            f.r = v.r;
            f.st = st_.get() + j;
            f.part = rpart_.get() + roff[j] * kRedParts;
            f.counter = counters_.get() + j;
            f.fp32 = 0;
            if (!add_toeplitz(ctx, g, T, v.p, v.ap, h_.get() + hoff[j], &st_.get()[j].done, f))
                for (int c = 0; c < v.nchunks; ++c) g.plain.push_back(make_int2(j, c));
        }
        vjobs_.upload(vj.data(), J, s);
        items_.upload(items.data(), items.size(), s);
        nitems_ = (int)items.size();
        for (auto &g : groups_) {
            for (Stage *st : {&g->fwd, &g->col, &g->inv}) st->finalize(ctx);
            if (!g->plain.empty()) g->dplain.upload(g->plain.data(), g->plain.size(), s);
        }
        // side streams of the per-grid branches (created here, outside any capture)
        const int nside = (int)std::min<size_t>(groups_.size(), 8);
        side_.resize(nside, nullptr);
        join_.resize(nside, nullptr);
        for (int i = 0; i < nside; ++i) {
            LC_CUDA(cudaStreamCreateWithFlags(&side_[i], cudaStreamNonBlocking));
            LC_CUDA(cudaEventCreateWithFlags(&join_[i], cudaEventDisableTiming));
        }
        LC_CUDA(cudaEventCreateWithFlags(&fork_, cudaEventDisableTiming));
    }

    ~BatchCG2D() {
        for (cudaStream_t x : side_)
            if (x) {
                cudaStreamSynchronize(x);
                cudaStreamDestroy(x);
            }
        for (cudaEvent_t e : join_)
            if (e) cudaEventDestroy(e);
        if (fork_) cudaEventDestroy(fork_);
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
#ifdef LC_BATCH_TRACE
                    const auto tc = std::chrono::steady_clock::now();
#endif
                    const cudaStream_t cs = ctx.capture_stream();
                    graph.capture(cs, [&] {
                        for (int i = 0; i < chunk; ++i) iteration(cs);
                    });
#ifdef LC_BATCH_TRACE
                    std::fprintf(stderr, "batch graph of %d iterations, %zu grid sizes: captured in %.2f ms\n", chunk,
                                 groups_.size(),
                                 std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - tc)
                                     .count());
#endif
                }
                graph.launch(s);
            } else {
                for (int i = 0; i < k; ++i) iteration(s);
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

  private:
    // one FFT pass of the jobs of one grid size: the register-plan kernels
    // when a plan covers it, else the generic kernel
    struct Stage {
        RegLineBatch reg;
        AxisFFTBatch gen;
        bool generic = false;
        // true when the register kernels took the transform with its fused
        // CG work; the generic kernel takes it without
        bool add(Context &ctx, const AxisFFT &a, const int *skip) {
            if (!generic && reg.add(a, skip)) return true;
            LC_REQUIRE(reg.empty(), "batch: the jobs of one grid size take different kernels");
            generic = true;
            AxisFFT b = a;
            b.cg = nullptr;
            b.cg_parts = 0;
            gen.add(ctx, b, skip);
            return false;
        }
        void finalize(Context &ctx) {
            if (generic) gen.finalize(ctx);
            else reg.finalize(ctx);
        }
        void launch(cudaStream_t st) const {
            if (generic) gen.launch(st);
            else reg.launch(st);
        }
    };
    struct Group {
        int P = 0;
        Stage fwd, col, inv;
        // (job, chunk) items of the jobs whose row passes do not fuse the
        // direction update and p.Ap (the generic kernel)
        std::vector<int2> plain;
        DevBuf<int2> dplain;
    };

    Group &group_for(int P) {
        for (auto &g : groups_)
            if (g->P == P) return *g;
        groups_.emplace_back(new Group);
        groups_.back()->P = P;
        return *groups_.back();
    }

    void iteration(cudaStream_t s) {
        // the grid sizes' Toeplitz passes as parallel branches
        LC_CUDA(cudaEventRecord(fork_, s));
        for (size_t i = 0; i < side_.size(); ++i) LC_CUDA(cudaStreamWaitEvent(side_[i], fork_, 0));
        for (size_t g = 0; g < groups_.size(); ++g) {
            const cudaStream_t b = side_[g % side_.size()];
            const Group &G = *groups_[g];
            const unsigned np = (unsigned)G.plain.size();
            if (np) {
                batch_p_update_kernel<<<np, kVecThreads, 0, b>>>(vjobs_.get(), G.dplain.get(), st_.get());
                LC_CHECK_LAUNCH();
            }
            G.fwd.launch(b);
            G.col.launch(b);
            G.inv.launch(b);
            if (np) {
                batch_dot_kernel<<<np, kVecThreads, 0, b>>>(vjobs_.get(), G.dplain.get(), st_.get(), part_.get(),
                                                            counters_.get());
                LC_CHECK_LAUNCH();
            }
        }
        for (size_t i = 0; i < side_.size(); ++i) {
            LC_CUDA(cudaEventRecord(join_[i], side_[i]));
            LC_CUDA(cudaStreamWaitEvent(s, join_[i], 0));
        }
        batch_update_kernel<<<nitems_, kVecThreads, 0, s>>>(vjobs_.get(), items_.get(), st_.get(), part_.get(),
                                                            counters_.get());
        LC_CHECK_LAUNCH();
    }

    // The three passes of the 2D Toeplitz apply (lc_toeplitz.cu) as items of
    // the group's three launches.  Real rows of an even grid run as complex
    // rows of half the length (even/odd packing), of an odd grid (3^q) as
    // complex rows of the full length.
    // Returns true when the row passes fuse the direction update and p.Ap (f).
    bool add_toeplitz(Context &ctx, Group &g, const Toeplitz &T, const float *p, float *ap, float2 *h,
                      const int *skip, const CGFusion &f) {
        const long n = T.dims()[1];
        const int P = T.P()[2], Ph = P / 2 + 1;
        const bool even = P % 2 == 0;
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
        a.L = even ? P / 2 : P;
        a.n_out = Ph;
        a.in_map = even ? IN_REAL_PACKED : IN_DIRECT;
        a.out_map = even ? OUT_R2C_UNPACK : OUT_DIRECT;
        a.sign = -1;
        a.cg = &f;
        a.cg_parts = kFusedUpdate;
        const bool fwd_fused = g.fwd.add(ctx, a, skip);
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
        g.col.add(ctx, b, skip);
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
        c.L = even ? P / 2 : P;
        c.n_out = (int)n;
        c.in_map = even ? IN_C2R_PACK : IN_HERM;
        c.out_map = even ? OUT_REAL_UNPACK : OUT_WINDOW;
        c.out_off = 0;
        c.sign = +1;
        c.scale = T.scale();
        c.cg = &f;
        c.cg_parts = kFusedDot;
        const bool inv_fused = g.inv.add(ctx, c, skip);
        LC_REQUIRE(fwd_fused == inv_fused, "batch: the row passes of one job take different kernels");
        return fwd_fused;
    }

    std::vector<Job> jobs_;
    DevBuf<float> vec_;
    DevBuf<float2> h_;
    DevBuf<CGState> st_;
    DevBuf<unsigned> counters_;
    DevBuf<double> part_;
    DevBuf<double> rpart_;
    DevBuf<VecJob> vjobs_;
    DevBuf<int2> items_;
    int nitems_ = 0;
    std::vector<std::unique_ptr<Group>> groups_;
    std::vector<cudaStream_t> side_;
    std::vector<cudaEvent_t> join_;
    cudaEvent_t fork_ = nullptr;
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
#ifdef LC_BATCH_TRACE
        const auto lc_t00 = std::chrono::steady_clock::now();
        auto lc_tr = [&](const char *what) {
            std::fprintf(stderr, "batch %s at %.2f ms\n", what,
                         std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - lc_t00).count());
        };
#else
        auto lc_tr = [](const char *) {};
#endif
        const int nw = std::max(1, std::min(setup_workers > 0 ? setup_workers : 8, njobs));
        // per job: right-hand side and Toeplitz operator, built on the workers
        // (contexts kept in the caller's context for later calls)
        auto &wctx = c->batch_workers;
        while ((int)wctx.size() < nw) {
            wctx.emplace_back(new lc_context_s);
            wctx.back()->ctx = std::make_shared<Context>(ctx.device(), nullptr);
        }
        std::vector<DevBuf<float>> rhs(njobs), xs(njobs);
        std::vector<std::shared_ptr<Toeplitz>> ops(njobs);
        std::vector<std::string> errs(njobs);
        // Two waves: the larger jobs (by pixels x angles, about half the
        // setup work) are set up first and iterate on the caller's stream
        // while the workers set up the rest.  A job's result does not depend
        // on the batch it runs in.
        std::vector<int> order(njobs);
        for (int j = 0; j < njobs; ++j) order[j] = j;
        auto cost = [&](int j) { return (double)jobs[j].n * jobs[j].n * (double)jobs[j].ntheta; };
        std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return cost(a) > cost(b); });
        std::vector<int> wave_end;
        if (njobs >= 8) {
            double tot = 0, acc = 0;
            for (int j = 0; j < njobs; ++j) tot += cost(j);
            int h = 0;
            while (h < njobs - 1 && acc < 0.5 * tot) acc += cost(order[h++]);
            wave_end = {h, njobs};
        } else {
            wave_end = {njobs};
        }
        std::mutex mu;
        std::condition_variable cv;
        std::vector<char> ready(njobs, 0);
        std::atomic<int> next{0};
        auto work = [&](int w) {
            lc_context wc = wctx[w].get();
            Context &wx = *wc->ctx;
            DeviceGuard dg(wx.device());
            for (int t = next++; t < njobs; t = next++) {
                const int j = order[t];
                const lc_job2d &q = jobs[j];
                const int rc = run_guarded(errs[j], [&] {
                    LC_BATCH_T0();
                    cudaStream_t ws = wx.stream();
                    DevBuf<float> dsino;
                    dsino.upload(q.sinogram, (size_t)q.ntheta * q.nradial, ws);
                    lc_geometry g = nullptr;
                    const int grc = lc_geometry2d_create(wc, q.theta, q.ntheta, q.nradial, &g);
                    if (grc) throw Error(grc == LC_ERR_INVALID ? 1 : 3, wc->err);
                    std::unique_ptr<lc_geometry_s> gown(g);
                    LC_BATCH_T(0);
                    const long nv = (long)q.n * q.n;
                    rhs[j].alloc(nv, ws);
                    xs[j].alloc(nv, ws);
                    LC_CUDA(cudaMemsetAsync(xs[j].get(), 0, nv * sizeof(float), ws));
                    const int brc = lc_backproj2d(wc, g, dsino.get(), 1, q.n, q.n, rhs[j].get(), p->nufft_tol);
                    if (brc) throw Error(brc == LC_ERR_INVALID ? 1 : 3, wc->err);
                    LC_BATCH_T(1);
                    const long dims[3] = {1, q.n, q.n};
                    ops[j] = std::make_shared<Toeplitz>(wx, g->g, dims, false);
                    LC_BATCH_T(2);
                    LC_CUDA(cudaStreamSynchronize(ws));
                    LC_BATCH_T(3);
                });
                if (rc && errs[j].empty()) errs[j] = "setup failed";
                {
                    std::lock_guard<std::mutex> lk(mu);
                    ready[t] = 1;
                }
                cv.notify_all();
            }
        };
#ifdef LC_BATCH_TRACE
        for (double &v : g_batch_t) v = 0;
        const auto lc_t0 = std::chrono::steady_clock::now();
#endif
        lc_tr("workers start");
        std::vector<std::thread> th;
        for (int w = 0; w < nw; ++w) th.emplace_back(work, w);
        // the workers finish every setup even when a wave fails: on every exit
        // path join them and drain the caller's stream before the buffers go
        struct Joiner {
            std::vector<std::thread> &t;
            cudaStream_t s;
            ~Joiner() {
                for (auto &x : t)
                    if (x.joinable()) x.join();
                cudaStreamSynchronize(s);
            }
        } joiner{th, s};
        int begin = 0;
        for (const int end : wave_end) {
            {
                std::unique_lock<std::mutex> lk(mu);
                cv.wait(lk, [&] {
                    for (int t = begin; t < end; ++t)
                        if (!ready[t]) return false;
                    return true;
                });
            }
#ifdef LC_BATCH_TRACE
            std::fprintf(stderr, "batch wave [%d, %d) set up at %.2f ms\n", begin, end,
                         std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - lc_t0).count());
#endif
            for (int t = begin; t < end; ++t)
                if (!errs[order[t]].empty())
                    throw Error(1, "job " + std::to_string(order[t]) + ": " + errs[order[t]]);
            std::vector<BatchCG2D::Job> bj;
            for (int t = begin; t < end; ++t) {
                const int j = order[t];
                bj.push_back({ops[j], rhs[j].get(), xs[j].get(), p->solver.max_iters, p->solver.tol, p->solver.xtol});
            }
            std::vector<CGState> fin;
            {
                BatchCG2D batch(ctx, std::move(bj));
#ifdef LC_BATCH_TRACE
                std::fprintf(stderr, "batch wave [%d, %d) built at %.2f ms\n", begin, end,
                             std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - lc_t0)
                                 .count());
#endif
                batch.run(ctx, p->solver.use_graph != 0, &fin);
#ifdef LC_BATCH_TRACE
                std::fprintf(stderr, "batch wave [%d, %d) iterated at %.2f ms\n", begin, end,
                             std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - lc_t0)
                                 .count());
#endif
            }
            for (int t = begin; t < end; ++t) {
                const int j = order[t];
                const long nv = (long)jobs[j].n * jobs[j].n;
                LC_CUDA(cudaMemcpyAsync(jobs[j].recon, xs[j].get(), nv * sizeof(float), cudaMemcpyDeviceToHost, s));
                if (stats) {
                    const CGState &f = fin[t - begin];
                    stats[j].iters = f.iters;
                    stats[j].cg_iters_total = f.iters;
                    stats[j].residual = f.res;
                    stats[j].dx = f.dx;
                    stats[j].stop_reason = f.reason;
                    stats[j].elapsed_ms = 0.0;
                }
            }
            lc_tr("results copied");
            begin = end;
        }
        for (auto &t : th) t.join();
#ifdef LC_BATCH_TRACE
        std::fprintf(stderr, "batch setup summed over jobs: geometry %.2f backproj %.2f psf %.2f drain %.2f\n",
                     g_batch_t[0], g_batch_t[1], g_batch_t[2], g_batch_t[3]);
#endif
        LC_CUDA(cudaStreamSynchronize(s));
        lc_tr("joined");
        // worker-owned buffers are released in the order of the workers' streams
        for (auto &o : ops) o.reset();
        for (auto &b : rhs) b.release();
        for (auto &b : xs) b.release();
        for (int w = 0; w < nw; ++w) LC_CUDA(cudaStreamSynchronize(wctx[w]->ctx->stream()));
        lc_tr("released");
    });
}
