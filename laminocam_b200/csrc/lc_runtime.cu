// Host runtime: context, FFT plan cache and twiddle tables.
#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdint>
#include <cstdlib>

#include <nvtx3/nvToolsExt.h>

#include "lc_runtime.hpp"

namespace lc {

static std::atomic<long> g_launches{0};
// launches recorded while this thread captures a graph run only on replay
static thread_local bool t_capturing = false;
long kernel_launch_count() { return g_launches.load(std::memory_order_relaxed); }
void note_kernel_launch() {
    if (!t_capturing) g_launches.fetch_add(1, std::memory_order_relaxed);
}

void CapturedGraph::reset() {
    if (exec_) cudaGraphExecDestroy(exec_);
    exec_ = nullptr;
    kernels_ = 0;
}

void CapturedGraph::capture(cudaStream_t s, const std::function<void()> &body) {
    reset();
    LC_CUDA(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
    t_capturing = true;
    cudaGraph_t g = nullptr;
    try {
        body();
    } catch (...) {
        t_capturing = false;
        cudaStreamEndCapture(s, &g);  // leaves the stream usable again
        if (g) cudaGraphDestroy(g);
        cudaGetLastError();
        throw;
    }
    t_capturing = false;
    LC_CUDA(cudaStreamEndCapture(s, &g));
    size_t nn = 0;
    cudaError_t e = cudaGraphGetNodes(g, nullptr, &nn);
    if (e == cudaSuccess && nn) {
        std::vector<cudaGraphNode_t> nodes(nn);
        e = cudaGraphGetNodes(g, nodes.data(), &nn);
        for (size_t i = 0; e == cudaSuccess && i < nn; ++i) {
            cudaGraphNodeType t;
            if (cudaGraphNodeGetType(nodes[i], &t) == cudaSuccess && t == cudaGraphNodeTypeKernel)
                ++kernels_;
        }
    }
    if (e == cudaSuccess) e = cudaGraphInstantiateWithFlags(&exec_, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) {
        exec_ = nullptr;
        kernels_ = 0;
        LC_CUDA(e);
    }
}

void CapturedGraph::launch(cudaStream_t s) {
    LC_REQUIRE(exec_ != nullptr, "graph launched before capture");
    LC_CUDA(cudaGraphLaunch(exec_, s));
    g_launches.fetch_add(kernels_, std::memory_order_relaxed);
}

bool is_smooth23(long n) {
    if (n < 1) return false;
    while (n % 2 == 0) n /= 2;
    while (n % 3 == 0) n /= 3;
    return n == 1;
}

long next_smooth23(long n) {
    long best = 1;
    while (best < n) best <<= 1;
    for (long q3 = 3; q3 < best; q3 *= 3) {
        long x = q3;
        while (x < n) x <<= 1;
        if (x < best) best = x;
    }
    return best;
}

static void factorise(int L, FFTPlan &pl) {
    LC_REQUIRE(L >= 1 && L < (1 << 20) && fft_factorise(L, pl), "FFT length must be 2^p*3^q");
}

const FFTPlan &PlanCache::get(int L, bool fp64, cudaStream_t s) {
    std::lock_guard<std::mutex> lk(mu_);
    auto key = std::make_pair(L, fp64);
    auto it = plans_.find(key);
    if (it != plans_.end()) return it->second->plan;
    auto e = std::make_unique<PlanEntry>();
    factorise(L, e->plan);
    const double two_pi = 6.283185307179586476925286766559;
    if (fp64) {
        std::vector<double2> h(L);
        for (int m = 0; m < L; ++m) {
            double a = two_pi * (double)m / (double)L;
            h[m] = make_double2(std::cos(a), -std::sin(a));
        }
        e->tw.alloc(sizeof(double2) * L, s);
        LC_CUDA(cudaMemcpyAsync(e->tw.get(), h.data(), sizeof(double2) * L,
                                cudaMemcpyHostToDevice, s));
    } else {
        std::vector<float2> h(L);
        for (int m = 0; m < L; ++m) {
            double a = two_pi * (double)m / (double)L;
            h[m] = make_float2((float)std::cos(a), (float)-std::sin(a));
        }
        e->tw.alloc(sizeof(float2) * L, s);
        LC_CUDA(cudaMemcpyAsync(e->tw.get(), h.data(), sizeof(float2) * L,
                                cudaMemcpyHostToDevice, s));
    }
    // the host vectors die here; make the copy complete first
    LC_CUDA(cudaStreamSynchronize(s));
    e->plan.tw = e->tw.get();
    auto &ref = e->plan;
    plans_[key] = std::move(e);
    return ref;
}

const float2 *PlanCache::dft_twiddles(int n, cudaStream_t s) {
    std::lock_guard<std::mutex> lk(mu_);
    auto it = dft_.find(n);
    if (it != dft_.end()) return it->second->get();
    std::vector<float2> h(n);
    const double two_pi = 6.283185307179586476925286766559;
    for (int m = 0; m < n; ++m) {
        double a = two_pi * (double)m / (double)n;
        h[m] = make_float2((float)std::cos(a), (float)-std::sin(a));
    }
    auto b = std::make_unique<DevBuf<float2>>(n, s);
    LC_CUDA(cudaMemcpyAsync(b->get(), h.data(), sizeof(float2) * n, cudaMemcpyHostToDevice, s));
    LC_CUDA(cudaStreamSynchronize(s));
    const float2 *p = b->get();
    dft_[n] = std::move(b);
    return p;
}

const char *prof_name(int s) {
    static const char *names[PS_COUNT] = {
        "toeplitz_x_fwd", "toeplitz_y_fwd", "toeplitz_z_mid", "toeplitz_y_inv", "toeplitz_x_inv",
        "toeplitz_y_mid", "neg_laplacian", "nufft_spread", "nufft_interp", "nufft_fft",
        "detector_dft", "psf_generate", "psf_fft", "cg_vector", "sb_vector"};
    return (s >= 0 && s < PS_COUNT) ? names[s] : "?";
}

cudaEvent_t Profiler::take() {
    if (!pool.empty()) {
        cudaEvent_t e = pool.back();
        pool.pop_back();
        return e;
    }
    cudaEvent_t e;
    LC_CUDA(cudaEventCreate(&e));
    return e;
}

void Profiler::collect() {
    for (auto &r : recs) {
        LC_CUDA(cudaEventSynchronize(r.b));
        float t = 0;
        LC_CUDA(cudaEventElapsedTime(&t, r.a, r.b));
        ms[r.sec] += t;
        bytes[r.sec] += r.bytes;
        count[r.sec] += 1;
        pool.push_back(r.a);
        pool.push_back(r.b);
    }
    recs.clear();
}

void Profiler::reset() {
    collect();
    for (int i = 0; i < PS_COUNT; ++i) {
        ms[i] = 0;
        bytes[i] = 0;
        count[i] = 0;
    }
}

Profiler::~Profiler() {
    for (auto &r : recs) {
        cudaEventDestroy(r.a);
        cudaEventDestroy(r.b);
    }
    for (auto e : pool) cudaEventDestroy(e);
}

// LC_NVTX=1 names every profiler section with an NVTX range (for example to
// select one section's kernels in a profiler with --nvtx-include)
static bool nvtx_enabled() {
    static const bool on = [] {
        const char *e = std::getenv("LC_NVTX");
        return e && e[0] == '1';
    }();
    return on;
}

ProfScope::ProfScope(Context &ctx, int sec, double bytes) : ctx_(&ctx) {
    if (nvtx_enabled()) {
        nvtxRangePushA(prof_name(sec));
        nvtx_ = true;
    }
    if (!ctx.prof.on) return;
    // bound the number of live events: fold finished records into the totals
    if (ctx.prof.recs.size() >= 50000) ctx.prof.collect();
    Profiler::Rec r{sec, bytes, ctx.prof.take(), ctx.prof.take()};
    LC_CUDA(cudaEventRecord(r.a, ctx.stream()));
    ctx.prof.recs.push_back(r);
    idx_ = (int)ctx.prof.recs.size() - 1;
}

ProfScope::~ProfScope() {
    if (nvtx_) nvtxRangePop();
    if (idx_ < 0) return;
    cudaEventRecord(ctx_->prof.recs[idx_].b, ctx_->stream());
}

Context::Context(int device, cudaStream_t stream) : device_(device) {
    DeviceGuard g(device);
    LC_CUDA(cudaStreamCreateWithFlags(&own_stream_, cudaStreamNonBlocking));
    stream_ = stream ? stream : own_stream_;
    // two attributes (cudaGetDeviceProperties fills the whole table, which
    // takes milliseconds)
    int sms = 0, smem = 0;
    LC_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
    LC_CUDA(cudaDeviceGetAttribute(&smem, cudaDevAttrMaxSharedMemoryPerBlockOptin, device));
    num_sms_ = sms;
    max_smem_ = (size_t)smem;
    // keep freed pool memory cached in the process instead of returning it
    cudaMemPool_t pool;
    if (cudaDeviceGetDefaultMemPool(&pool, device) == cudaSuccess) {
        uint64_t thr = UINT64_MAX;
        // optional: without it freed pool memory returns to the device sooner
        if (cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &thr) != cudaSuccess)
            cudaGetLastError();
    }
}

cudaStream_t Context::copy_stream() {
    if (!copy_stream_) {
        DeviceGuard g(device_);
        LC_CUDA(cudaStreamCreateWithFlags(&copy_stream_, cudaStreamNonBlocking));
    }
    return copy_stream_;
}

void *Context::pinned_scratch(size_t bytes) {
    if (bytes > pinned_bytes_) {
        // pinned allocation and release synchronise the whole device, so the
        // buffer is grown rarely and kept for the context's lifetime
        if (pinned_) cudaFreeHost(pinned_);
        pinned_ = nullptr;
        pinned_bytes_ = 0;
        LC_CUDA(cudaMallocHost(&pinned_, std::max<size_t>(bytes, 4096)));
        pinned_bytes_ = std::max<size_t>(bytes, 4096);
    }
    return pinned_;
}

Context::~Context() {
    cudaSetDevice(device_);
    plans_.clear();
    if (pinned_) cudaFreeHost(pinned_);
    if (copy_stream_) {
        cudaStreamSynchronize(copy_stream_);
        cudaStreamDestroy(copy_stream_);
    }
    if (own_stream_) {
        cudaStreamSynchronize(own_stream_);
        cudaStreamDestroy(own_stream_);
    }
}

}  // namespace lc
