// Host runtime of laminocam_b200: device context, stream-ordered buffers and
// the FFT plan cache.  Everything here is plain C++ over the CUDA runtime.
#pragma once

#include <cuda_runtime.h>

#include <functional>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <utility>
#include <vector>

#include "lc_common.cuh"

namespace lc {

// Device buffer allocated from the stream-ordered pool of the context's device
// (cudaMallocAsync): repeated create/destroy cycles reuse pool memory instead
// of calling the driver allocator.
template <typename T>
class DevBuf {
  public:
    DevBuf() = default;
    DevBuf(size_t n, cudaStream_t s) { alloc(n, s); }
    ~DevBuf() { release(); }
    DevBuf(const DevBuf &) = delete;
    DevBuf &operator=(const DevBuf &) = delete;
    DevBuf(DevBuf &&o) noexcept : p_(o.p_), n_(o.n_), s_(o.s_) {
        o.p_ = nullptr;
        o.n_ = 0;
    }
    DevBuf &operator=(DevBuf &&o) noexcept {
        if (this != &o) {
            release();
            p_ = o.p_;
            n_ = o.n_;
            s_ = o.s_;
            o.p_ = nullptr;
            o.n_ = 0;
        }
        return *this;
    }
    void alloc(size_t n, cudaStream_t s) {
        release();
        s_ = s;
        n_ = n;
        if (n) LC_CUDA(cudaMallocAsync((void **)&p_, n * sizeof(T), s));
    }
    // grow-only: keeps the buffer when it is already large enough
    void ensure(size_t n, cudaStream_t s) {
        if (n > n_) alloc(n, s);
    }
    void release() {
        // a failed free (a leak) must not surface as the error of a later,
        // unrelated call on this thread
        if (p_ && cudaFreeAsync(p_, s_) != cudaSuccess) cudaGetLastError();
        p_ = nullptr;
        n_ = 0;
    }
    void zero(cudaStream_t s) {
        if (n_) LC_CUDA(cudaMemsetAsync(p_, 0, n_ * sizeof(T), s));
    }
    void upload(const T *h, size_t n, cudaStream_t s) {
        ensure(n, s);
        LC_CUDA(cudaMemcpyAsync(p_, h, n * sizeof(T), cudaMemcpyHostToDevice, s));
    }
    T *get() const { return p_; }
    size_t size() const { return n_; }

  private:
    T *p_ = nullptr;
    size_t n_ = 0;
    cudaStream_t s_ = nullptr;
};

// FFT plan: factorisation of L into radices 8/4/2/3 and a twiddle table in
// the requested precision.  Lengths must be 2^p * 3^q.
struct PlanEntry {
    FFTPlan plan{};
    DevBuf<char> tw;
};

bool is_smooth23(long n);
long next_smooth23(long n);  // smallest 2^p 3^q >= n

// Bluestein (chirp-z) tables for a DFT of arbitrary length n and sign s:
// chirp[j] = exp(s i pi j^2 / n) (j < n) and V = FFT_L(conj chirp, wrapped) / L.
struct BluesteinEntry {
    int n = 0, L = 0, sign = 0;
    DevBuf<float2> chirp, V;
};

class Context;

// Per-device cache of FFT plans and twiddle tables.
class PlanCache {
  public:
    const FFTPlan &get(int L, bool fp64, cudaStream_t s);
    // twiddle table exp(-2*pi*i*m/n) for a direct DFT of arbitrary n (float2)
    const float2 *dft_twiddles(int n, cudaStream_t s);
    // cached Bluestein tables (built by the caller on a miss)
    BluesteinEntry *find_bluestein(int n, int sign) {
        std::lock_guard<std::mutex> lk(mu_);
        auto it = blue_.find(std::make_pair(n, sign));
        return it == blue_.end() ? nullptr : it->second.get();
    }
    BluesteinEntry *store_bluestein(std::unique_ptr<BluesteinEntry> e) {
        std::lock_guard<std::mutex> lk(mu_);
        auto key = std::make_pair(e->n, e->sign);
        auto &slot = blue_[key];
        if (!slot) slot = std::move(e);
        return slot.get();
    }
    void clear() {
        std::lock_guard<std::mutex> lk(mu_);
        plans_.clear();
        dft_.clear();
        blue_.clear();
    }

  private:
    std::mutex mu_;
    std::map<std::pair<int, bool>, std::unique_ptr<PlanEntry>> plans_;
    std::map<int, std::unique_ptr<DevBuf<float2>>> dft_;
    std::map<std::pair<int, int>, std::unique_ptr<BluesteinEntry>> blue_;
};

// Optional per-section device timing: sections record a CUDA event pair on
// the context stream; totals are read back (with one synchronisation) later.
enum ProfSection {
    PS_TOEP_X_FWD = 0,
    PS_TOEP_Y_FWD,
    PS_TOEP_Z_MID,
    PS_TOEP_Y_INV,
    PS_TOEP_X_INV,
    PS_TOEP_Y_MID,
    PS_NEG_LAP,
    PS_SPREAD,
    PS_INTERP,
    PS_NUFFT_FFT,
    PS_DFT,
    PS_PSF_GEN,
    PS_PSF_FFT,
    PS_CG_VEC,
    PS_SB_VEC,
    PS_COUNT
};
const char *prof_name(int s);

struct Profiler {
    bool on = false;
    struct Rec {
        int sec;
        double bytes;
        cudaEvent_t a, b;
    };
    std::vector<Rec> recs;
    std::vector<cudaEvent_t> pool;
    double ms[PS_COUNT] = {0};
    double bytes[PS_COUNT] = {0};
    long count[PS_COUNT] = {0};
    cudaEvent_t take();
    void collect();  // synchronises on the events, folds them into the totals
    void reset();
    ~Profiler();
};

class Context;

class ProfScope {
  public:
    ProfScope(Context &ctx, int sec, double bytes);
    ~ProfScope();

  private:
    Context *ctx_;
    int idx_ = -1;
    bool nvtx_ = false;
};

class Context {
  public:
    Context(int device, cudaStream_t stream);
    ~Context();
    int device() const { return device_; }
    cudaStream_t stream() const { return stream_; }
    void set_stream(cudaStream_t s) { stream_ = s ? s : own_stream_; }
    // the context's private stream: graphs are captured there (the caller's
    // stream may be the legacy default stream, which cannot capture)
    cudaStream_t capture_stream() const { return own_stream_; }
    // a second private stream for host-to-device copies that overlap work on
    // stream() (created on first use)
    cudaStream_t copy_stream();
    // A pinned host buffer of at least `bytes`, owned by the context and
    // reused by its solvers for device-to-host copies of small state.  The
    // pointer stays valid until a larger request or the context's end.
    void *pinned_scratch(size_t bytes);
    PlanCache &plans() { return plans_; }
    int num_sms() const { return num_sms_; }
    size_t max_smem() const { return max_smem_; }
    std::string last_error;
    int verbose = 0;
    Profiler prof;

  private:
    int device_;
    cudaStream_t stream_;
    cudaStream_t own_stream_ = nullptr;
    cudaStream_t copy_stream_ = nullptr;
    PlanCache plans_;
    void *pinned_ = nullptr;
    size_t pinned_bytes_ = 0;
    int num_sms_ = 148;
    size_t max_smem_ = 227 * 1024;
};

// A fixed launch sequence captured once from one stream into a CUDA graph and
// replayed.  Launches issued while capturing are not counted; each replay
// counts the graph's kernel nodes instead.  The body must not allocate, copy
// to the host or synchronise.
class CapturedGraph {
  public:
    CapturedGraph() = default;
    CapturedGraph(const CapturedGraph &) = delete;
    CapturedGraph &operator=(const CapturedGraph &) = delete;
    ~CapturedGraph() { reset(); }
    void capture(cudaStream_t s, const std::function<void()> &body);
    void launch(cudaStream_t s);
    bool ready() const { return exec_ != nullptr; }
    long kernels() const { return kernels_; }
    void reset();

  private:
    cudaGraphExec_t exec_ = nullptr;
    long kernels_ = 0;
};

// Raises a kernel's dynamic shared-memory limit to all the device allows
// beside the kernel's static shared memory.  The limit is a property of the
// function shared by every thread of the process: setting it to each launch's
// own size would let a concurrent launch (a server worker) lower it between
// another thread's set and launch.  This value is the same from every thread.
template <typename K>
void allow_max_dynamic_smem(const Context &ctx, K kern) {
    cudaFuncAttributes fa;
    LC_CUDA(cudaFuncGetAttributes(&fa, kern));
    LC_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)(ctx.max_smem() - fa.sharedSizeBytes)));
}

// Makes `dev` current for the lifetime of the guard.
class DeviceGuard {
  public:
    explicit DeviceGuard(int dev) {
        cudaGetDevice(&prev_);
        if (prev_ != dev) LC_CUDA(cudaSetDevice(dev));
    }
    ~DeviceGuard() {
        int cur;
        cudaGetDevice(&cur);
        if (cur != prev_) cudaSetDevice(prev_);
    }

  private:
    int prev_ = 0;
};

}  // namespace lc
