// Axis FFT / DFT kernels.  One CTA transforms C lines held in shared memory;
// global loads and stores are arranged so that consecutive threads touch
// consecutive addresses (along i for contiguous lines, along c otherwise).
#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <map>
#include <memory>
#include <mutex>
#include <tuple>
#include <vector>

#include "lc_fft.hpp"

namespace lc {

namespace {

template <typename T, typename TI>
__device__ __forceinline__ cx<T> ld_elem(const TI *p) {
    if constexpr (std::is_same_v<TI, float> || std::is_same_v<TI, double>) {
        return mk<T>((T)*p, T(0));
    } else {
        TI v = *p;
        return mk<T>((T)v.x, (T)v.y);
    }
}

template <typename T, typename TO>
__device__ __forceinline__ void st_elem(TO *p, cx<T> v) {
    if constexpr (std::is_same_v<TO, float> || std::is_same_v<TO, double>) {
        *p = (TO)v.x;
    } else {
        TO o;
        o.x = v.x;
        o.y = v.y;
        *p = o;
    }
}

struct KArgs {
    const void *in;
    void *out;
    long n_outer, n_inner, in_ostride, out_ostride;
    int n_in, n_out, L;
    int in_map, out_map, out_off, sign, sign2;
    const void *pre, *linefac, *post;
    double scale;
    const float *mid;
    long mid_ra;
    int mid_fold;
    int logC;
    long blocks_per_outer;
};

struct FFTBatchItem {
    KArgs a;
    FFTPlan pl;
    long first_block;
    const int *skip;
};

// One CTA transforms C = 1 << logC lines.  Rows (n_inner == 1) are C
// consecutive lines, each contiguous in memory, walked line by line so that
// consecutive threads touch consecutive addresses; otherwise the CTA takes C
// adjacent inner indices c of one outer index o and consecutive threads walk c.
template <typename T, typename TI, typename TO>
__device__ __forceinline__ void axis_fft_body(const KArgs &a, const FFTPlan &pl, long bid) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    using V = cx<T>;
    const int logC = a.logC;
    const int C = 1 << logC;
    const int L = a.L;
    V *buf = reinterpret_cast<V *>(smem_raw);
    V *alt = buf + ((long)L << logC);
    const TI *in = reinterpret_cast<const TI *>(a.in);
    TO *out = reinterpret_cast<TO *>(a.out);
    const T *pre = reinterpret_cast<const T *>(a.pre);
    const T *linefac = reinterpret_cast<const T *>(a.linefac);
    const T *post = reinterpret_cast<const T *>(a.post);
    const int tid = threadIdx.x, nt = blockDim.x;
    const bool rows = (a.n_inner == 1);
    long o_base, c_base;
    if (rows) {
        o_base = bid << logC;
        c_base = 0;
    } else {
        o_base = bid / a.blocks_per_outer;
        c_base = (bid % a.blocks_per_outer) << logC;
    }
    // lines of this CTA that exist
    const int nlines = rows ? (int)min((long)C, a.n_outer - o_base) : (int)min((long)C, a.n_inner - c_base);

    // ---- zero padding (only the positions the load does not write) ----
    int gap0 = 0, gap1 = 0;
    if (a.in_map == IN_DIRECT) {
        gap0 = a.n_in;
        gap1 = L;
    } else if (a.in_map == IN_MODES) {
        gap0 = a.n_in - a.n_in / 2;
        gap1 = L - a.n_in / 2;
    } else if (a.in_map == IN_REAL_PACKED) {
        gap0 = (a.n_in + 1) / 2;
        gap1 = L;
    }
    const int gap = gap1 - gap0;
    for (int idx = tid; idx < (gap << logC); idx += nt) {
        const int cl = idx & (C - 1);
        buf[((gap0 + (idx >> logC)) << logC) + cl] = mk<T>(T(0), T(0));
    }

    // ---- load ----
    // Each thread issues kBatch independent global loads before it writes any
    // of them to shared memory, so that several loads per thread are in flight.
    constexpr int kBatch = 4;
    const int nh = L / 2 + 1;
    if (rows) {
        const T lf = linefac ? linefac[0] : T(1);
        const int per = (a.in_map == IN_HERM || a.in_map == IN_C2R_PACK)
                            ? L
                            : (a.in_map == IN_REAL_PACKED ? (a.n_in + 1) / 2 : a.n_in);
        const int total = per * nlines;
        const unsigned long long per_magic = fast_div_magic((unsigned)max(per, 1));
        for (int base = tid; base < total; base += kBatch * nt) {
            V v[kBatch];
            int dst[kBatch];
#pragma unroll
            for (int u = 0; u < kBatch; ++u) {
                const int idx = base + u * nt;
                dst[u] = -1;
                if (idx >= total) continue;
                const int cl = (int)fast_div((unsigned)idx, per_magic);
                const int e = idx - cl * per;
                const TI *src = in + (o_base + cl) * a.in_ostride;
                if (a.in_map == IN_HERM) {
                    const int j = e < nh ? e : L - e;
                    v[u] = ld_elem<T, TI>(src + j);
                    if (e >= nh) v[u].y = -v[u].y;
                    dst[u] = (e << logC) + cl;
                } else if (a.in_map == IN_REAL_PACKED) {
                    // z[e] = x[2e] + i x[2e+1]
                    const T re = ld_elem<T, TI>(src + 2 * e).x;
                    const T im = 2 * e + 1 < a.n_in ? ld_elem<T, TI>(src + 2 * e + 1).x : T(0);
                    v[u] = mk<T>(re, im);
                    dst[u] = (e << logC) + cl;
                } else if (a.in_map == IN_C2R_PACK) {
                    // Z[k] = (X[k] + conj X[L-k]) + i exp(i pi k / L) (X[k] - conj X[L-k])
                    const V xa = ld_elem<T, TI>(src + e);
                    const V xb = ld_elem<T, TI>(src + (L - e));
                    const V sm = mk<T>(xa.x + xb.x, xa.y - xb.y);
                    const V df = mk<T>(xa.x - xb.x, xa.y + xb.y);
                    T sn, cs;
                    if constexpr (std::is_same_v<T, double>) sincospi((double)e / (double)L, &sn, &cs);
                    else sincospif((float)e / (float)L, &sn, &cs);
                    const V wd = cmul(mk<T>(cs, sn), df);
                    v[u] = mk<T>(sm.x - wd.y, sm.y + wd.x);
                    dst[u] = (e << logC) + cl;
                } else {
                    v[u] = ld_elem<T, TI>(src + e);
                    if (pre) v[u] = cscale(v[u], pre[e] * lf);
                    else if (linefac) v[u] = cscale(v[u], lf);
                    int f = e;
                    if (a.in_map == IN_MODES) {
                        f = e - a.n_in / 2;
                        if (f < 0) f += L;
                    }
                    dst[u] = (f << logC) + cl;
                }
            }
#pragma unroll
            for (int u = 0; u < kBatch; ++u)
                if (dst[u] >= 0) buf[dst[u]] = v[u];
        }
    } else {
        const TI *src = in + o_base * a.in_ostride + c_base;
        const int total = (a.in_map == IN_HERM ? L : a.n_in) << logC;
        for (int base = tid; base < total; base += kBatch * nt) {
            V v[kBatch];
            int dst[kBatch];
#pragma unroll
            for (int u = 0; u < kBatch; ++u) {
                const int idx = base + u * nt;
                dst[u] = -1;
                if (idx >= total) continue;
                const int cl = idx & (C - 1);
                if (cl >= nlines) continue;
                const int e = idx >> logC;
                if (a.in_map == IN_HERM) {
                    const int j = e < nh ? e : L - e;
                    v[u] = ld_elem<T, TI>(src + (long)j * a.n_inner + cl);
                    if (e >= nh) v[u].y = -v[u].y;
                    dst[u] = idx;
                } else {
                    v[u] = ld_elem<T, TI>(src + (long)e * a.n_inner + cl);
                    if (pre || linefac) {
                        T s = T(1);
                        if (pre) s *= pre[e];
                        if (linefac) s *= linefac[c_base + cl];
                        v[u] = cscale(v[u], s);
                    }
                    int f = e;
                    if (a.in_map == IN_MODES) {
                        f = e - a.n_in / 2;
                        if (f < 0) f += L;
                    }
                    dst[u] = (f << logC) + cl;
                }
            }
#pragma unroll
            for (int u = 0; u < kBatch; ++u)
                if (dst[u] >= 0) buf[dst[u]] = v[u];
        }
    }
    __syncthreads();

    buf = smem_fft<T>(buf, alt, logC, pl, a.sign);
    alt = (buf == reinterpret_cast<V *>(smem_raw)) ? buf + ((long)L << logC) : reinterpret_cast<V *>(smem_raw);

    if (a.mid) {
        // rows mode never carries a spectral multiply (lines are columns here)
        const float *mrow = a.mid + c_base;
        for (int idx = tid; idx < (L << logC); idx += nt) {
            const int cl = idx & (C - 1);
            const int f = idx >> logC;
            if (cl >= nlines) continue;
            const int fr = (a.mid_fold && f > L / 2) ? L - f : f;
            buf[idx] = cscale(buf[idx], (T)__ldg(mrow + (long)fr * a.mid_ra + cl));
        }
        __syncthreads();
        buf = smem_fft<T>(buf, alt, logC, pl, a.sign2);
    }

    // ---- store ----
    const T scale = (T)a.scale;
    auto fidx = [&](int j) {
        int f = j;
        if (a.out_map == OUT_MODES) {
            f = j - a.n_out / 2;
            if (f < 0) f += L;
        } else if (a.out_map == OUT_WINDOW) {
            f = j + a.out_off;
        }
        return f;
    };
    if (rows && a.out_map == OUT_R2C_UNPACK) {
        // X[k] = (Z[k] + conj Z[L-k]) / 2 - (i/2) exp(-i pi k / L) (Z[k] - conj Z[L-k])
        for (int cl = 0; cl < nlines; ++cl) {
            TO *dst = out + (o_base + cl) * a.out_ostride;
            for (int k = tid; k < a.n_out; k += nt) {
                const int k1 = k == L ? 0 : k;
                const int k2 = k == 0 ? 0 : L - k;
                const V za = buf[(k1 << logC) + cl];
                const V zb = buf[(k2 << logC) + cl];
                const V sm = mk<T>(T(0.5) * (za.x + zb.x), T(0.5) * (za.y - zb.y));
                const V df = mk<T>(T(0.5) * (za.x - zb.x), T(0.5) * (za.y + zb.y));
                T sn, cs;
                if constexpr (std::is_same_v<T, double>) sincospi((double)k / (double)L, &sn, &cs);
                else sincospif((float)k / (float)L, &sn, &cs);
                const V wd = cmul(mk<T>(cs, -sn), df);  // exp(-i pi k / L) (Z[k] - conj Z[L-k]) / 2
                T s = scale;
                if (post) s *= post[k];
                st_elem<T, TO>(dst + k, cscale(mk<T>(sm.x + wd.y, sm.y - wd.x), s));
            }
        }
    } else if (rows && a.out_map == OUT_REAL_UNPACK) {
        for (int cl = 0; cl < nlines; ++cl) {
            TO *dst = out + (o_base + cl) * a.out_ostride;
            for (int j = tid; j < a.n_out; j += nt) {
                const V z = buf[((j >> 1) << logC) + cl];
                T s = scale;
                if (post) s *= post[j];
                st_elem<T, TO>(dst + j, mk<T>(((j & 1) ? z.y : z.x) * s, T(0)));
            }
        }
    } else if (rows) {
        for (int cl = 0; cl < nlines; ++cl) {
            TO *dst = out + (o_base + cl) * a.out_ostride;
            for (int j = tid; j < a.n_out; j += nt) {
                T s = scale;
                if (post) s *= post[j];
                st_elem<T, TO>(dst + j, cscale(buf[(fidx(j) << logC) + cl], s));
            }
        }
    } else {
        TO *dst = out + o_base * a.out_ostride + c_base;
        for (int idx = tid; idx < (a.n_out << logC); idx += nt) {
            const int cl = idx & (C - 1);
            const int j = idx >> logC;
            if (cl >= nlines) continue;
            T s = scale;
            if (post) s *= post[j];
            st_elem<T, TO>(dst + (long)j * a.n_inner + cl, cscale(buf[(fidx(j) << logC) + cl], s));
        }
    }
}

template <typename T, typename TI, typename TO>
__global__ void axis_fft_kernel(KArgs a, FFTPlan pl) {
    axis_fft_body<T, TI, TO>(a, pl, (long)blockIdx.x);
}

// One launch over many FP32 transforms: CTA b runs block b - first_block of
// the item whose range holds b (items sorted by first_block); an item whose
// skip flag is set (a finished job) does nothing.
template <typename TI, typename TO>
__global__ void axis_fft_batch_kernel(const FFTBatchItem *__restrict__ items, int nitems) {
    const long b = (long)blockIdx.x;
    int lo = 0, hi = nitems - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (items[mid].first_block <= b) lo = mid;
        else hi = mid - 1;
    }
    const FFTBatchItem &it = items[lo];
    if (it.skip && *it.skip) return;
    axis_fft_body<float, TI, TO>(it.a, it.pl, b - it.first_block);
}

template <typename T, typename TI, typename TO>
void launch_t(Context &ctx, const KArgs &ka, const FFTPlan &pl, int threads, size_t smem,
              long blocks) {
    auto kern = axis_fft_kernel<T, TI, TO>;
    static thread_local int configured_dev = -1;
    if (configured_dev != ctx.device()) {
        LC_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)ctx.max_smem()));
        configured_dev = ctx.device();
    }
    kern<<<(unsigned)blocks, threads, smem, ctx.stream()>>>(ka, pl);
    LC_CHECK_LAUNCH();
}

template <typename T>
void dispatch(Context &ctx, const AxisFFT &a, const KArgs &ka, const FFTPlan &pl, int threads,
              size_t smem, long blocks) {
    using R = T;
    using Cx = cx<T>;
    auto ti = a.in_t, to = a.out_t;
    bool in_real = (ti == E_F32 || ti == E_F64);
    bool out_real = (to == E_F32 || to == E_F64);
    bool in64 = (ti == E_F64 || ti == E_C128);
    bool out64 = (to == E_F64 || to == E_C128);
    constexpr bool t64 = std::is_same_v<T, double>;
    LC_REQUIRE(in64 == t64 && out64 == t64, "axis FFT: element precision must match compute precision");
    if (in_real && out_real) launch_t<T, R, R>(ctx, ka, pl, threads, smem, blocks);
    else if (in_real) launch_t<T, R, Cx>(ctx, ka, pl, threads, smem, blocks);
    else if (out_real) launch_t<T, Cx, R>(ctx, ka, pl, threads, smem, blocks);
    else launch_t<T, Cx, Cx>(ctx, ka, pl, threads, smem, blocks);
}

KArgs make_kargs(const AxisFFT &a, int logC, long &blocks) {
    const int C = 1 << logC;
    KArgs ka{};
    ka.in = a.in;
    ka.out = a.out;
    ka.n_outer = a.n_outer;
    ka.n_inner = a.n_inner;
    ka.in_ostride = a.in_ostride;
    ka.out_ostride = a.out_ostride;
    ka.n_in = a.n_in;
    ka.n_out = a.n_out;
    ka.L = a.L;
    ka.in_map = a.in_map;
    ka.out_map = a.out_map;
    ka.out_off = a.out_off;
    ka.sign = a.sign;
    ka.sign2 = a.sign2;
    ka.pre = a.pre;
    ka.linefac = a.linefac;
    ka.post = a.post;
    ka.scale = a.scale;
    ka.mid = a.mid;
    ka.mid_ra = a.mid_ra;
    ka.mid_fold = a.mid_fold ? 1 : 0;
    ka.logC = logC;
    if (a.n_inner == 1) {
        blocks = (a.n_outer + C - 1) / C;
        ka.blocks_per_outer = 1;
    } else {
        ka.blocks_per_outer = (a.n_inner + C - 1) / C;
        blocks = a.n_outer * ka.blocks_per_outer;
    }
    LC_REQUIRE(blocks < (1L << 31), "axis FFT: grid too large");
    return ka;
}

// one launch of the transform with C = 1 << logC lines per CTA
void run_axis(Context &ctx, const AxisFFT &a, const FFTPlan &pl, int logC, int threads) {
    const size_t esz = a.fp64 ? sizeof(double2) : sizeof(float2);
    long blocks = 0;
    const KArgs ka = make_kargs(a, logC, blocks);
    const size_t smem = 2 * ((size_t)a.L << logC) * esz;
    if (a.fp64) dispatch<double>(ctx, a, ka, pl, threads, smem, blocks);
    else dispatch<float>(ctx, a, ka, pl, threads, smem, blocks);
}

// log2 of the lines per CTA (a power of two) and the CTA size: rows are
// grouped so that a CTA moves >= 2048 elements, column groups take 16 adjacent
// lines (128 contiguous bytes of float2) when the inner extent allows; both
// ping-pong buffers must fit in shared memory.
int choose_lines(const AxisFFT &a, size_t esz, size_t max_smem, int &threads) {
    LC_REQUIRE(!a.mid || a.n_inner > 1, "axis FFT: a spectral multiply needs column lines");
    const size_t smem_cap = std::min<size_t>(max_smem, 200 * 1024);
    int logC = 0;
    if (a.lines_per_cta > 0) {
        while ((2 << logC) <= a.lines_per_cta) ++logC;
    } else if (a.n_inner == 1) {
        while ((a.L << (logC + 1)) <= 2048 && (1L << (logC + 1)) <= a.n_outer) ++logC;
    } else {
        logC = 4;
        while (logC > 0 && (1L << logC) > a.n_inner * 2) --logC;
    }
    while (logC > 0 && 2 * ((size_t)a.L << logC) * esz > smem_cap) --logC;
    LC_REQUIRE(2 * (size_t)a.L * esz <= max_smem, "axis FFT: line does not fit shared memory");
    const long work = ((long)a.L << logC) / 2;
    threads = work >= 4096 ? 512 : (work >= 1024 ? 256 : 128);
    return logC;
}

// ---- launch autotuner -------------------------------------------------------
// The lines per CTA and the CTA size of an FP32 transform are chosen per
// transform shape by timing the candidates once (CUDA events on the launching
// stream) and kept per device for the life of the process.  Column candidates
// keep groups of >= 4 lines (whole 32-byte sectors of float2).  A trial of a
// transform whose output overwrites its input writes to a scratch buffer.
// Tuning is skipped while the stream is being captured into a graph (the
// heuristic of choose_lines is used), and LC_FFT_AUTOTUNE=0 turns it off.
struct TuneKey {
    int dev, L, n_in, n_out, in_map, out_map, in_t, out_t, mid, pre, post, linefac;
    long n_outer, n_inner, in_ostride, out_ostride;
    auto tie() const {
        return std::tie(dev, L, n_in, n_out, in_map, out_map, in_t, out_t, mid, pre, post, linefac,
                        n_outer, n_inner, in_ostride, out_ostride);
    }
    bool operator<(const TuneKey &o) const { return tie() < o.tie(); }
};

struct TuneVal {
    int logC, threads;
    float ms;
};

std::mutex g_tune_mu;
std::map<TuneKey, TuneVal> g_tune;

bool autotune_enabled() {
    static const bool on = [] {
        const char *e = std::getenv("LC_FFT_AUTOTUNE");
        return !(e && e[0] == '0');
    }();
    return on;
}

TuneKey tune_key(int dev, const AxisFFT &a) {
    return TuneKey{dev, a.L, a.n_in, a.n_out, (int)a.in_map, (int)a.out_map, (int)a.in_t,
                   (int)a.out_t, a.mid != nullptr, a.pre != nullptr, a.post != nullptr,
                   a.linefac != nullptr, a.n_outer, a.n_inner, a.in_ostride, a.out_ostride};
}

// elements spanned by the output lines
long out_extent(const AxisFFT &a) {
    if (a.n_inner == 1) return (a.n_outer - 1) * a.out_ostride + a.n_out;
    return (a.n_outer - 1) * a.out_ostride + (long)(a.n_out - 1) * a.n_inner + a.n_inner;
}

TuneVal autotune(Context &ctx, const AxisFFT &a0, const FFTPlan &pl) {
    cudaStream_t st = ctx.stream();
    const size_t esz = sizeof(float2);
    const size_t cap = std::min<size_t>(ctx.max_smem(), 200 * 1024);
    int base_threads = 0;
    const int base_logC = choose_lines(a0, esz, ctx.max_smem(), base_threads);
    std::vector<std::pair<int, int>> cands{{base_logC, base_threads}};
    const bool rows = a0.n_inner == 1;
    for (int logC = rows ? 0 : 2; logC <= (rows ? 6 : 5); ++logC) {
        if (rows && (((long)a0.L << logC) > 8192 || (1L << logC) > std::max<long>(1, a0.n_outer)))
            break;
        if (!rows && (1L << logC) > 2 * a0.n_inner) break;
        if (2 * ((size_t)a0.L << logC) * esz > cap) break;
        for (int th : {128, 256, 512}) {
            if (((long)a0.L << logC) < th) continue;
            if (logC == base_logC && th == base_threads) continue;
            cands.emplace_back(logC, th);
        }
    }
    AxisFFT a = a0;
    DevBuf<char> scratch;
    if (a0.out == a0.in) {
        const size_t oesz = (a0.out_t == E_F32) ? sizeof(float) : sizeof(float2);
        scratch.alloc(out_extent(a0) * oesz, st);
        a.out = scratch.get();
    }
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    TuneVal best{base_logC, base_threads, 1e30f};
    try {
        LC_CUDA(cudaEventCreate(&e0));
        LC_CUDA(cudaEventCreate(&e1));
        for (auto [logC, th] : cands) {
            run_axis(ctx, a, pl, logC, th);  // warm
            float tbest = 1e30f;
            for (int rep = 0; rep < 2; ++rep) {
                LC_CUDA(cudaEventRecord(e0, st));
                run_axis(ctx, a, pl, logC, th);
                LC_CUDA(cudaEventRecord(e1, st));
                LC_CUDA(cudaEventSynchronize(e1));
                float ms = 0.f;
                LC_CUDA(cudaEventElapsedTime(&ms, e0, e1));
                tbest = std::min(tbest, ms);
            }
            if (tbest < best.ms) best = TuneVal{logC, th, tbest};
        }
        LC_CUDA(cudaStreamSynchronize(st));  // the scratch buffer is released on return
    } catch (...) {
        if (e0) cudaEventDestroy(e0);
        if (e1) cudaEventDestroy(e1);
        throw;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    return best;
}

}  // namespace

// ---- batched launches ------------------------------------------------------
// A CTA of a batched launch holds at most this many elements per buffer
// (lines x length), except that column transforms keep at least two lines.
#ifndef LC_BATCH_ELEMS
#define LC_BATCH_ELEMS 4096
#endif
#ifndef LC_BATCH_THREADS
#define LC_BATCH_THREADS 256
#endif
constexpr int kBatchElems = LC_BATCH_ELEMS;
constexpr int kBatchThreads = LC_BATCH_THREADS;
// Items are launched in shared-memory classes (<= 32 KB, <= 64 KB, more per
// CTA), so that small transforms keep several CTAs per SM beside large ones.
constexpr size_t kBatchClassSmem[2] = {32 * 1024, 64 * 1024};

struct AxisFFTBatch::Impl {
    struct Group {
        std::vector<FFTBatchItem> items;
        DevBuf<FFTBatchItem> dev;
        size_t smem = 0;
        long blocks = 0;
    };
    Group g[3];
    int in_real = -1, out_real = -1;
};

AxisFFTBatch::AxisFFTBatch() : impl_(new Impl) {}
AxisFFTBatch::~AxisFFTBatch() = default;
bool AxisFFTBatch::empty() const {
    return impl_->g[0].items.empty() && impl_->g[1].items.empty() && impl_->g[2].items.empty();
}
long AxisFFTBatch::blocks() const { return impl_->g[0].blocks + impl_->g[1].blocks + impl_->g[2].blocks; }

void AxisFFTBatch::add(Context &ctx, const AxisFFT &a, const int *skip) {
    LC_REQUIRE(!a.fp64 && !a.cg && a.lines_per_cta == 0, "batched axis FFT: FP32 transforms without CG fusion");
    LC_REQUIRE((a.in_t == E_F32 || a.in_t == E_C64) && (a.out_t == E_F32 || a.out_t == E_C64),
               "batched axis FFT: float or float2 elements only");
    const int ir = a.in_t == E_F32, orl = a.out_t == E_F32;
    LC_REQUIRE(impl_->in_real < 0 || (impl_->in_real == ir && impl_->out_real == orl),
               "batched axis FFT: all transforms of a batch share their element types");
    LC_REQUIRE(is_smooth23(a.L), "batched axis FFT: lengths must be 2^p 3^q");
    if (a.in_map == IN_HERM) LC_REQUIRE(a.n_in == a.L / 2 + 1, "IN_HERM needs n_in = L/2+1");
    else if (a.in_map == IN_C2R_PACK) LC_REQUIRE(a.n_in == a.L + 1, "IN_C2R_PACK needs n_in = L+1");
    else LC_REQUIRE(a.n_in <= (a.in_map == IN_REAL_PACKED ? 2 * a.L : a.L), "axis FFT: n_in > L");
    if (a.out_map == OUT_WINDOW) LC_REQUIRE(a.out_off >= 0 && a.out_off + a.n_out <= a.L, "window");
    else if (a.out_map == OUT_R2C_UNPACK) LC_REQUIRE(a.n_out <= a.L + 1, "axis FFT: n_out > L+1");
    else if (a.out_map == OUT_REAL_UNPACK) LC_REQUIRE(a.n_out <= 2 * a.L, "axis FFT: n_out > 2L");
    else LC_REQUIRE(a.n_out <= a.L, "axis FFT: n_out > L");
    LC_REQUIRE(!a.mid || a.n_inner > 1, "axis FFT: a spectral multiply needs column lines");
    if (a.n_outer <= 0 || a.n_inner <= 0 || a.n_out == 0) return;
    impl_->in_real = ir;
    impl_->out_real = orl;
    int logC = 0;
    const size_t cap = std::min<size_t>(ctx.max_smem(), 160 * 1024);
    auto fits = [&](int lc) { return 2 * ((size_t)a.L << lc) * sizeof(float2) <= cap; };
    if (a.n_inner == 1) {
        while ((a.L << (logC + 1)) <= kBatchElems && (1L << (logC + 1)) <= a.n_outer) ++logC;
    } else {
        while (logC < 4 && (1L << (logC + 1)) <= 2 * a.n_inner &&
               ((a.L << (logC + 1)) <= kBatchElems || (logC == 0 && fits(1))))
            ++logC;
    }
    const size_t need = 2 * ((size_t)a.L << logC) * sizeof(float2);
    LC_REQUIRE(need <= ctx.max_smem(), "batched axis FFT: line does not fit shared memory");
    Impl::Group &grp = impl_->g[need <= kBatchClassSmem[0] ? 0 : (need <= kBatchClassSmem[1] ? 1 : 2)];
    FFTBatchItem it{};
    long nb = 0;
    it.a = make_kargs(a, logC, nb);
    it.pl = ctx.plans().get(a.L, false, ctx.stream());
    it.first_block = grp.blocks;
    it.skip = skip;
    grp.items.push_back(it);
    grp.blocks += nb;
    grp.smem = std::max(grp.smem, need);
    LC_REQUIRE(grp.blocks < (1L << 31), "batched axis FFT: grid too large");
}

template <typename TI, typename TO>
static void batch_launch_t(cudaStream_t st, const FFTBatchItem *items, int n, long blocks, size_t smem) {
    axis_fft_batch_kernel<TI, TO><<<(unsigned)blocks, kBatchThreads, smem, st>>>(items, n);
    LC_CHECK_LAUNCH();
}

void AxisFFTBatch::finalize(Context &ctx) {
    for (Impl::Group &grp : impl_->g)
        if (!grp.items.empty()) grp.dev.upload(grp.items.data(), grp.items.size(), ctx.stream());
    if (empty()) return;
    // the shared-memory limit is set here, outside any stream capture
    if (impl_->in_real && impl_->out_real) allow_max_dynamic_smem(ctx, axis_fft_batch_kernel<float, float>);
    else if (impl_->in_real) allow_max_dynamic_smem(ctx, axis_fft_batch_kernel<float, float2>);
    else if (impl_->out_real) allow_max_dynamic_smem(ctx, axis_fft_batch_kernel<float2, float>);
    else allow_max_dynamic_smem(ctx, axis_fft_batch_kernel<float2, float2>);
}

struct RegLineBatch::Impl {
    RegBatchKey key;
    std::vector<unsigned char> items;
    DevBuf<unsigned char> dev;
    int n = 0;
    long blocks = 0;
};

RegLineBatch::RegLineBatch() : impl_(new Impl) {}
RegLineBatch::~RegLineBatch() = default;
bool RegLineBatch::empty() const { return impl_->n == 0; }

bool RegLineBatch::add(const AxisFFT &a, const int *skip) {
    if (!line_kernels_enabled()) return false;
    if (a.n_outer <= 0 || a.n_inner <= 0 || a.n_out == 0) return false;
    RegBatchKey k;
    std::vector<unsigned char> item;
    long nb = 0;
    const bool ok = a.n_inner == 1 ? row_batch_item(a, skip, impl_->blocks, k, item, nb)
                                   : col_batch_item(a, skip, impl_->blocks, k, item, nb);
    if (!ok) return false;
    if (impl_->n > 0 && (k.kind != impl_->key.kind || k.M != impl_->key.M || k.mode != impl_->key.mode))
        return false;
    impl_->key = k;
    impl_->items.insert(impl_->items.end(), item.begin(), item.end());
    impl_->blocks += nb;
    impl_->n += 1;
    LC_REQUIRE(impl_->blocks < (1L << 31), "batched line FFT: grid too large");
    return true;
}

void RegLineBatch::finalize(Context &ctx) {
    if (impl_->n == 0) return;
    impl_->dev.upload(impl_->items.data(), impl_->items.size(), ctx.stream());
    impl_->key.configure();  // outside any stream capture
}

void RegLineBatch::launch(cudaStream_t st) const {
    if (impl_->n == 0) return;
    LC_REQUIRE(impl_->dev.size() == impl_->items.size(), "batched line FFT: finalize() before launch()");
    impl_->key.launch(st, impl_->dev.get(), impl_->n, impl_->blocks);
}

void AxisFFTBatch::launch(cudaStream_t st) const {
    for (const Impl::Group &grp : impl_->g) {
        if (grp.items.empty()) continue;
        LC_REQUIRE(grp.dev.size() == grp.items.size(), "batched axis FFT: finalize() before launch()");
        const FFTBatchItem *d = grp.dev.get();
        const int n = (int)grp.items.size();
        if (impl_->in_real && impl_->out_real) batch_launch_t<float, float>(st, d, n, grp.blocks, grp.smem);
        else if (impl_->in_real) batch_launch_t<float, float2>(st, d, n, grp.blocks, grp.smem);
        else if (impl_->out_real) batch_launch_t<float2, float>(st, d, n, grp.blocks, grp.smem);
        else batch_launch_t<float2, float2>(st, d, n, grp.blocks, grp.smem);
    }
}


// LC_LINE_KERNELS=0 routes every transform through the generic kernel (for
// A/B timing of the register-plan line kernels).
bool line_kernels_enabled() {
    static const bool on = [] {
        const char *e = std::getenv("LC_LINE_KERNELS");
        return !(e && e[0] == '0');
    }();
    return on;
}

void launch_axis_fft(Context &ctx, const AxisFFT &a) {
    LC_REQUIRE(is_smooth23(a.L), "axis FFT length must be 2^p*3^q");
    LC_REQUIRE(a.n_in >= 0 && a.n_out >= 0, "axis FFT: bad lengths");
    const bool packed_in = a.in_map == IN_REAL_PACKED || a.in_map == IN_C2R_PACK;
    const bool packed_out = a.out_map == OUT_R2C_UNPACK || a.out_map == OUT_REAL_UNPACK;
    LC_REQUIRE(!(packed_in || packed_out) || a.n_inner == 1, "axis FFT: packed real maps need rows");
    if (a.in_map == IN_HERM) LC_REQUIRE(a.n_in == a.L / 2 + 1, "IN_HERM needs n_in = L/2+1");
    else if (a.in_map == IN_REAL_PACKED) LC_REQUIRE(a.n_in <= 2 * a.L, "axis FFT: n_in > 2L");
    else if (a.in_map == IN_C2R_PACK) LC_REQUIRE(a.n_in == a.L + 1, "IN_C2R_PACK needs n_in = L+1");
    else LC_REQUIRE(a.n_in <= a.L, "axis FFT: n_in > L");
    if (a.out_map == OUT_WINDOW) LC_REQUIRE(a.out_off >= 0 && a.out_off + a.n_out <= a.L, "window");
    else if (a.out_map == OUT_R2C_UNPACK) LC_REQUIRE(a.n_out <= a.L + 1, "axis FFT: n_out > L+1");
    else if (a.out_map == OUT_REAL_UNPACK) LC_REQUIRE(a.n_out <= 2 * a.L, "axis FFT: n_out > 2L");
    else LC_REQUIRE(a.n_out <= a.L, "axis FFT: n_out > L");
    if (a.n_outer <= 0 || a.n_inner <= 0 || a.n_out == 0) return;
    if (line_kernels_enabled() && (launch_col_fft(ctx.stream(), a) || launch_row_fft(ctx.stream(), a))) return;
    LC_REQUIRE(a.cg_parts == 0, "axis FFT: fused CG work needs a register-plan row kernel");

    const FFTPlan &pl = ctx.plans().get(a.L, a.fp64, ctx.stream());
    const size_t esz = a.fp64 ? sizeof(double2) : sizeof(float2);
    int threads = 0;
    int logC = choose_lines(a, esz, ctx.max_smem(), threads);
    if (!a.fp64 && a.lines_per_cta == 0 && autotune_enabled()) {
        const TuneKey key = tune_key(ctx.device(), a);
        bool found = false;
        {
            std::lock_guard<std::mutex> lk(g_tune_mu);
            auto it = g_tune.find(key);
            if (it != g_tune.end()) {
                logC = it->second.logC;
                threads = it->second.threads;
                found = true;
            }
        }
        cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
        LC_CUDA(cudaStreamIsCapturing(ctx.stream(), &cs));
        if (!found && cs == cudaStreamCaptureStatusNone) {
            const TuneVal v = autotune(ctx, a, pl);
            std::lock_guard<std::mutex> lk(g_tune_mu);
            g_tune.emplace(key, v);
            logC = v.logC;
            threads = v.threads;
        }
    }
    run_axis(ctx, a, pl, logC, threads);
}

void launch_axis_fft_f32_with_plan(cudaStream_t stream, size_t max_smem, const AxisFFT &a,
                                   const FFTPlan &pl) {
    LC_REQUIRE(!a.fp64, "explicit-plan axis FFT is FP32 only");
    LC_REQUIRE(pl.L == a.L, "explicit-plan axis FFT: plan length mismatch");
    if (a.in_map == IN_HERM) LC_REQUIRE(a.n_in == a.L / 2 + 1, "IN_HERM needs n_in = L/2+1");
    else LC_REQUIRE(a.n_in <= a.L, "axis FFT: n_in > L");
    if (a.out_map == OUT_WINDOW) LC_REQUIRE(a.out_off >= 0 && a.out_off + a.n_out <= a.L, "window");
    else LC_REQUIRE(a.n_out <= a.L, "axis FFT: n_out > L");
    if (a.n_outer <= 0 || a.n_inner <= 0 || a.n_out == 0) return;
    const size_t esz = sizeof(float2);
    int threads = 0;
    const int logC = choose_lines(a, esz, max_smem, threads);
    const int C = 1 << logC;
    KArgs ka{};
    ka.in = a.in;
    ka.out = a.out;
    ka.n_outer = a.n_outer;
    ka.n_inner = a.n_inner;
    ka.in_ostride = a.in_ostride;
    ka.out_ostride = a.out_ostride;
    ka.n_in = a.n_in;
    ka.n_out = a.n_out;
    ka.L = a.L;
    ka.in_map = a.in_map;
    ka.out_map = a.out_map;
    ka.out_off = a.out_off;
    ka.sign = a.sign;
    ka.sign2 = a.sign2;
    ka.pre = a.pre;
    ka.linefac = a.linefac;
    ka.post = a.post;
    ka.scale = a.scale;
    ka.mid = a.mid;
    ka.mid_ra = a.mid_ra;
    ka.mid_fold = a.mid_fold ? 1 : 0;
    ka.logC = logC;
    long blocks;
    if (a.n_inner == 1) {
        blocks = (a.n_outer + C - 1) / C;
        ka.blocks_per_outer = 1;
    } else {
        ka.blocks_per_outer = (a.n_inner + C - 1) / C;
        blocks = a.n_outer * ka.blocks_per_outer;
    }
    LC_REQUIRE(blocks < (1L << 31), "axis FFT: grid too large");
    size_t smem = 2 * (size_t)a.L * C * esz;
    bool in_real = a.in_t == E_F32, out_real = a.out_t == E_F32;
    LC_REQUIRE((a.in_t == E_F32 || a.in_t == E_C64) && (a.out_t == E_F32 || a.out_t == E_C64),
               "explicit-plan axis FFT: float or float2 elements only");
    if (in_real && out_real) {
        auto k = axis_fft_kernel<float, float, float>;
        LC_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)max_smem));
        k<<<(unsigned)blocks, threads, smem, stream>>>(ka, pl);
    } else if (in_real) {
        auto k = axis_fft_kernel<float, float, float2>;
        LC_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)max_smem));
        k<<<(unsigned)blocks, threads, smem, stream>>>(ka, pl);
    } else if (out_real) {
        auto k = axis_fft_kernel<float, float2, float>;
        LC_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)max_smem));
        k<<<(unsigned)blocks, threads, smem, stream>>>(ka, pl);
    } else {
        auto k = axis_fft_kernel<float, float2, float2>;
        LC_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)max_smem));
        k<<<(unsigned)blocks, threads, smem, stream>>>(ka, pl);
    }
    LC_CHECK_LAUNCH();
}

// ---------------------------------------------------------------------------
// direct DFT of arbitrary length (float)
// ---------------------------------------------------------------------------
namespace {

struct DArgs {
    const void *in;
    void *out;
    long n_outer, n_inner, in_ostride, out_ostride;
    int n, d_pre, d_post, sign, C;
    float scale;
    long blocks_per_outer;
    const float2 *tw;
};

template <typename TI, typename TO>
__global__ void axis_dft_kernel(DArgs a) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int n = a.n, C = a.C;
    float2 *tw = reinterpret_cast<float2 *>(smem_raw);
    float2 *buf = tw + n;  // [n][C]
    const TI *in = reinterpret_cast<const TI *>(a.in);
    TO *out = reinterpret_cast<TO *>(a.out);
    const bool rows = (a.n_inner == 1);
    long o_base, c_base;
    if (rows) {
        o_base = (long)blockIdx.x * C;
        c_base = 0;
    } else {
        o_base = (long)blockIdx.x / a.blocks_per_outer;
        c_base = ((long)blockIdx.x % a.blocks_per_outer) * C;
    }
    const int tid = threadIdx.x, nt = blockDim.x;
    for (int m = tid; m < n; m += nt) {
        float2 w = a.tw[m];
        if (a.sign > 0) w.y = -w.y;
        tw[m] = w;
    }
    for (int idx = tid; idx < n * C; idx += nt) {
        int m, cl;
        if (rows) {
            m = idx % n;
            cl = idx / n;
        } else {
            cl = idx % C;
            m = idx / C;
        }
        long o = rows ? o_base + cl : o_base;
        long c = rows ? 0 : c_base + cl;
        float2 v = make_float2(0.f, 0.f);
        if (o < a.n_outer && c < a.n_inner) {
            // v[m'] = in[(m' + d_pre) % n]  <=>  in[m] lands at m' = (m - d_pre) mod n
            int mp = m - a.d_pre;
            if (mp < 0) mp += n;
            cx<float> t = ld_elem<float, TI>(in + o * a.in_ostride + (long)m * a.n_inner + c);
            v = t;
            buf[mp * C + cl] = v;
        } else {
            buf[m * C + cl] = v;
        }
    }
    __syncthreads();
    for (int idx = tid; idx < n * C; idx += nt) {
        int k, cl;
        if (rows) {
            k = idx % n;
            cl = idx / n;
        } else {
            cl = idx % C;
            k = idx / C;
        }
        long o = rows ? o_base + cl : o_base;
        long c = rows ? 0 : c_base + cl;
        if (!(o < a.n_outer && c < a.n_inner)) continue;
        int kk = k + a.d_post;
        if (kk >= n) kk -= n;
        float sr = 0.f, si = 0.f;
        int ti = 0;
        for (int m = 0; m < n; ++m) {
            float2 x = buf[m * C + cl];
            float2 w = tw[ti];
            sr = fmaf(x.x, w.x, fmaf(-x.y, w.y, sr));
            si = fmaf(x.x, w.y, fmaf(x.y, w.x, si));
            ti += kk;
            if (ti >= n) ti -= n;
        }
        st_elem<float, TO>(out + o * a.out_ostride + (long)k * a.n_inner + c,
                           make_float2(sr * a.scale, si * a.scale));
    }
}

template <typename TI, typename TO>
void dft_launch(Context &ctx, const DArgs &d, long blocks, int threads, size_t smem) {
    auto kern = axis_dft_kernel<TI, TO>;
    static thread_local int configured_dev = -1;
    if (configured_dev != ctx.device()) {
        LC_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)ctx.max_smem()));
        configured_dev = ctx.device();
    }
    kern<<<(unsigned)blocks, threads, smem, ctx.stream()>>>(d);
    LC_CHECK_LAUNCH();
}

}  // namespace

// ---------------------------------------------------------------------------
// Bluestein (chirp-z) DFT of arbitrary length on the Stockham core:
//   X[k] = sum_m x[m] e^{s 2 pi i m k / n} = a[k] sum_m (x[m] a[m]) conj(a[k-m]),
//   a[j] = e^{s i pi j^2 / n},
// a cyclic convolution of length L = next 2^p 3^q >= 2n - 1 done as
// FFT -> multiply by V = FFT(conj a, wrapped) / L -> inverse FFT.
// ---------------------------------------------------------------------------
struct BArgs {
    const void *in;
    void *out;
    long n_outer, n_inner, in_ostride, out_ostride;
    int n, L, d_pre, d_post, logC;
    float scale;
    long blocks_per_outer;
    const float2 *chirp, *V;
};

template <typename TI, typename TO>
__global__ void bluestein_kernel(BArgs a, FFTPlan pl) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const long bid = (long)blockIdx.x;
    const int logC = a.logC, C = 1 << logC, L = a.L, n = a.n;
    float2 *buf = reinterpret_cast<float2 *>(smem_raw);
    float2 *alt = buf + ((long)L << logC);
    const TI *in = reinterpret_cast<const TI *>(a.in);
    TO *out = reinterpret_cast<TO *>(a.out);
    const int tid = threadIdx.x, nt = blockDim.x;
    const bool rows = (a.n_inner == 1);
    long o_base, c_base;
    if (rows) {
        o_base = bid << logC;
        c_base = 0;
    } else {
        o_base = bid / a.blocks_per_outer;
        c_base = (bid % a.blocks_per_outer) << logC;
    }
    const int nlines = rows ? (int)min((long)C, a.n_outer - o_base) : (int)min((long)C, a.n_inner - c_base);
    for (int idx = tid; idx < ((L - n) << logC); idx += nt)
        buf[((n + (idx >> logC)) << logC) + (idx & (C - 1))] = make_float2(0.f, 0.f);
    // load with the pre-roll: line value m is in[(m + d_pre) % n], times chirp[m]
    if (rows) {
        for (int cl = 0; cl < nlines; ++cl) {
            const TI *src = in + (o_base + cl) * a.in_ostride;
            for (int m = tid; m < n; m += nt) {
                int s = m + a.d_pre;
                if (s >= n) s -= n;
                buf[(m << logC) + cl] = cmul(ld_elem<float, TI>(src + s), a.chirp[m]);
            }
        }
    } else {
        const TI *src = in + o_base * a.in_ostride + c_base;
        for (int idx = tid; idx < (n << logC); idx += nt) {
            const int cl = idx & (C - 1), m = idx >> logC;
            if (cl >= nlines) continue;
            int s = m + a.d_pre;
            if (s >= n) s -= n;
            buf[idx] = cmul(ld_elem<float, TI>(src + (long)s * a.n_inner + cl), a.chirp[m]);
        }
    }
    __syncthreads();
    float2 *res = smem_fft<float>(buf, alt, logC, pl, -1);
    float2 *oth = (res == buf) ? alt : buf;
    for (int idx = tid; idx < (L << logC); idx += nt) res[idx] = cmul(res[idx], a.V[idx >> logC]);
    __syncthreads();
    res = smem_fft<float>(res, oth, logC, pl, +1);
    // store with the post-roll: out[k] = X[(k + d_post) % n], X[q] = a[q] * conv[q]
    if (rows) {
        for (int cl = 0; cl < nlines; ++cl) {
            TO *dst = out + (o_base + cl) * a.out_ostride;
            for (int k = tid; k < n; k += nt) {
                int q = k + a.d_post;
                if (q >= n) q -= n;
                st_elem<float, TO>(dst + k, cscale(cmul(res[(q << logC) + cl], a.chirp[q]), a.scale));
            }
        }
    } else {
        TO *dst = out + o_base * a.out_ostride + c_base;
        for (int idx = tid; idx < (n << logC); idx += nt) {
            const int cl = idx & (C - 1), k = idx >> logC;
            if (cl >= nlines) continue;
            int q = k + a.d_post;
            if (q >= n) q -= n;
            st_elem<float, TO>(dst + (long)k * a.n_inner + cl,
                               cscale(cmul(res[(q << logC) + cl], a.chirp[q]), a.scale));
        }
    }
}

__global__ void c128_to_c64_kernel(const double2 *in, float2 *out, int n, double scale) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        out[i] = make_float2((float)(in[i].x * scale), (float)(in[i].y * scale));
}

const BluesteinEntry &bluestein_tables(Context &ctx, int n, int sign) {
    if (BluesteinEntry *e = ctx.plans().find_bluestein(n, sign)) return *e;
    cudaStream_t st = ctx.stream();
    auto e = std::make_unique<BluesteinEntry>();
    e->n = n;
    e->sign = sign;
    e->L = (int)next_smooth23(2L * n - 1);
    const int L = e->L;
    const double pi = 3.14159265358979323846;
    std::vector<double2> a(n), v(L, make_double2(0.0, 0.0));
    for (int j = 0; j < n; ++j) {
        long t = ((long)j * j) % (2L * n);  // exact j^2 mod 2n
        double ang = sign * pi * (double)t / (double)n;
        a[j] = make_double2(std::cos(ang), std::sin(ang));
    }
    for (int j = 0; j < n; ++j) {
        double2 c = make_double2(a[j].x, -a[j].y);
        v[j] = c;
        if (j > 0) v[L - j] = c;
    }
    std::vector<float2> af(n);
    for (int j = 0; j < n; ++j) af[j] = make_float2((float)a[j].x, (float)a[j].y);
    e->chirp.upload(af.data(), n, st);
    DevBuf<double2> dv, dV;
    dv.upload(v.data(), L, st);
    dV.alloc(L, st);
    AxisFFT f;
    f.in = dv.get();
    f.in_t = E_C128;
    f.out = dV.get();
    f.out_t = E_C128;
    f.fp64 = true;
    f.n_outer = 1;
    f.n_inner = 1;
    f.in_ostride = L;
    f.out_ostride = L;
    f.n_in = L;
    f.L = L;
    f.n_out = L;
    f.sign = -1;
    launch_axis_fft(ctx, f);
    e->V.alloc(L, st);
    c128_to_c64_kernel<<<(L + 255) / 256, 256, 0, st>>>(dV.get(), e->V.get(), L, 1.0 / (double)L);
    LC_CHECK_LAUNCH();
    LC_CUDA(cudaStreamSynchronize(st));  // host vectors and dv/dV die on return
    return *ctx.plans().store_bluestein(std::move(e));
}

template <typename TI, typename TO>
void bluestein_launch(Context &ctx, const BArgs &b, const FFTPlan &pl, long blocks, int threads,
                      size_t smem) {
    auto kern = bluestein_kernel<TI, TO>;
    LC_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)ctx.max_smem()));
    kern<<<(unsigned)blocks, threads, smem, ctx.stream()>>>(b, pl);
    LC_CHECK_LAUNCH();
}

void launch_bluestein(Context &ctx, const AxisDFT &a) {
    const BluesteinEntry &e = bluestein_tables(ctx, a.n, a.sign);
    if (line_kernels_enabled() && launch_bluestein_lines(ctx.stream(), a, e)) return;
    const FFTPlan &pl = ctx.plans().get(e.L, false, ctx.stream());
    AxisFFT shape;  // only to pick the line grouping
    shape.L = e.L;
    shape.n_inner = a.n_inner;
    shape.n_outer = a.n_outer;
    int threads = 0;
    const int logC = choose_lines(shape, sizeof(float2), ctx.max_smem(), threads);
    const int C = 1 << logC;
    BArgs b{};
    b.in = a.in;
    b.out = a.out;
    b.n_outer = a.n_outer;
    b.n_inner = a.n_inner;
    b.in_ostride = a.in_ostride;
    b.out_ostride = a.out_ostride;
    b.n = a.n;
    b.L = e.L;
    b.d_pre = ((a.d_pre % a.n) + a.n) % a.n;
    b.d_post = ((a.d_post % a.n) + a.n) % a.n;
    b.logC = logC;
    b.scale = a.scale;
    b.chirp = e.chirp.get();
    b.V = e.V.get();
    long blocks;
    if (a.n_inner == 1) {
        blocks = (a.n_outer + C - 1) / C;
        b.blocks_per_outer = 1;
    } else {
        b.blocks_per_outer = (a.n_inner + C - 1) / C;
        blocks = a.n_outer * b.blocks_per_outer;
    }
    LC_REQUIRE(blocks < (1L << 31), "DFT: grid too large");
    size_t smem = 2 * ((size_t)e.L << logC) * sizeof(float2);
    bool in_real = a.in_t == E_F32, out_real = a.out_t == E_F32;
    if (in_real && out_real) bluestein_launch<float, float>(ctx, b, pl, blocks, threads, smem);
    else if (in_real) bluestein_launch<float, float2>(ctx, b, pl, blocks, threads, smem);
    else if (out_real) bluestein_launch<float2, float>(ctx, b, pl, blocks, threads, smem);
    else bluestein_launch<float2, float2>(ctx, b, pl, blocks, threads, smem);
}

void launch_axis_dft(Context &ctx, const AxisDFT &a) {
    LC_REQUIRE(a.n > 0, "DFT length must be positive");
    const double lines = (double)a.n_outer * a.n_inner;
    ProfScope ps(ctx, PS_DFT,
                 lines * a.n * ((a.in_t == E_F32 ? 4.0 : 8.0) + (a.out_t == E_F32 ? 4.0 : 8.0)));
    LC_REQUIRE(a.in_t == E_F32 || a.in_t == E_C64, "DFT input must be float or float2");
    LC_REQUIRE(a.out_t == E_F32 || a.out_t == E_C64, "DFT output must be float or float2");
    if (a.n_outer <= 0 || a.n_inner <= 0) return;
    if (a.n >= 16 && next_smooth23(2L * a.n - 1) <= 8192) {
        launch_bluestein(ctx, a);
        return;
    }
    DArgs d{};
    d.in = a.in;
    d.out = a.out;
    d.n_outer = a.n_outer;
    d.n_inner = a.n_inner;
    d.in_ostride = a.in_ostride;
    d.out_ostride = a.out_ostride;
    d.n = a.n;
    d.d_pre = ((a.d_pre % a.n) + a.n) % a.n;
    d.d_post = ((a.d_post % a.n) + a.n) % a.n;
    d.sign = a.sign;
    d.scale = a.scale;
    d.tw = ctx.plans().dft_twiddles(a.n, ctx.stream());
    int C = a.n_inner == 1 ? 1 : (int)std::min<long>(8, a.n_inner);
    while (C > 1 && (size_t)(a.n * (C + 1)) * sizeof(float2) > 160 * 1024) --C;
    d.C = C;
    size_t smem = (size_t)a.n * (C + 1) * sizeof(float2);
    LC_REQUIRE(smem <= ctx.max_smem(), "DFT line too long");
    long blocks;
    if (a.n_inner == 1) {
        blocks = (a.n_outer + C - 1) / C;
        d.blocks_per_outer = 1;
    } else {
        d.blocks_per_outer = (a.n_inner + C - 1) / C;
        blocks = a.n_outer * d.blocks_per_outer;
    }
    int threads = std::min(1024, std::max(64, ((a.n * C + 31) / 32) * 32));
    threads = std::min(threads, 512);
    bool in_real = a.in_t == E_F32, out_real = a.out_t == E_F32;
    if (in_real && out_real) dft_launch<float, float>(ctx, d, blocks, threads, smem);
    else if (in_real) dft_launch<float, float2>(ctx, d, blocks, threads, smem);
    else if (out_real) dft_launch<float2, float>(ctx, d, blocks, threads, smem);
    else dft_launch<float2, float2>(ctx, d, blocks, threads, smem);
}

}  // namespace lc
