// Axis FFT / DFT kernels.  One CTA transforms C lines held in shared memory;
// global loads and stores are arranged so that consecutive threads touch
// consecutive addresses (along i for contiguous lines, along c otherwise).
#include <algorithm>

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
    int C;
    long blocks_per_outer;
};

template <typename T, typename TI, typename TO>
__global__ void axis_fft_kernel(KArgs a, FFTPlan pl) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    using V = cx<T>;
    const int C = a.C;
    const int L = a.L;
    V *buf = reinterpret_cast<V *>(smem_raw);
    V *alt = buf + (long)L * C;
    const TI *in = reinterpret_cast<const TI *>(a.in);
    TO *out = reinterpret_cast<TO *>(a.out);
    const T *pre = reinterpret_cast<const T *>(a.pre);
    const T *linefac = reinterpret_cast<const T *>(a.linefac);
    const T *post = reinterpret_cast<const T *>(a.post);

    // lines handled by this CTA
    long o_base, c_base;
    const bool rows = (a.n_inner == 1);
    if (rows) {
        o_base = (long)blockIdx.x * C;
        c_base = 0;
    } else {
        o_base = (long)blockIdx.x / a.blocks_per_outer;
        c_base = ((long)blockIdx.x % a.blocks_per_outer) * C;
    }
    auto line_ok = [&](int cl, long &o, long &c) -> bool {
        if (rows) {
            o = o_base + cl;
            c = 0;
        } else {
            o = o_base;
            c = c_base + cl;
        }
        return o < a.n_outer && c < a.n_inner;
    };

    const int tid = threadIdx.x, nt = blockDim.x;
    for (int idx = tid; idx < L * C; idx += nt) buf[idx] = mk<T>(T(0), T(0));
    __syncthreads();

    // ---- load ----
    if (a.in_map == IN_HERM) {
        const int nh = L / 2 + 1;
        for (int idx = tid; idx < L * C; idx += nt) {
            int f, cl;
            if (rows) {
                f = idx % L;
                cl = idx / L;
            } else {
                cl = idx % C;
                f = idx / C;
            }
            long o, c;
            if (!line_ok(cl, o, c)) continue;
            int j = f < nh ? f : L - f;
            V v = ld_elem<T, TI>(in + o * a.in_ostride + (long)j * a.n_inner + c);
            if (f >= nh) v.y = -v.y;
            buf[f * C + cl] = v;
        }
    } else {
        for (int idx = tid; idx < a.n_in * C; idx += nt) {
            int j, cl;
            if (rows) {
                j = idx % a.n_in;
                cl = idx / a.n_in;
            } else {
                cl = idx % C;
                j = idx / C;
            }
            long o, c;
            if (!line_ok(cl, o, c)) continue;
            V v = ld_elem<T, TI>(in + o * a.in_ostride + (long)j * a.n_inner + c);
            T s = T(1);
            if (pre) s *= pre[j];
            if (linefac) s *= linefac[c];
            if (pre || linefac) v = cscale(v, s);
            int f;
            if (a.in_map == IN_MODES) {
                f = j - a.n_in / 2;
                if (f < 0) f += L;
            } else {
                f = j;
            }
            buf[f * C + cl] = v;
        }
    }
    __syncthreads();

    buf = smem_fft<T>(buf, alt, C, pl, a.sign);
    alt = (buf == reinterpret_cast<V *>(smem_raw)) ? buf + (long)L * C : reinterpret_cast<V *>(smem_raw);

    if (a.mid) {
        for (int idx = tid; idx < L * C; idx += nt) {
            int cl = idx % C;
            int f = idx / C;
            long o, c;
            if (!line_ok(cl, o, c)) continue;
            buf[idx] = cscale(buf[idx], (T)__ldg(a.mid + (long)f * a.mid_ra + c));
        }
        __syncthreads();
        buf = smem_fft<T>(buf, alt, C, pl, a.sign2);
    }

    // ---- store ----
    for (int idx = tid; idx < a.n_out * C; idx += nt) {
        int j, cl;
        if (rows) {
            j = idx % a.n_out;
            cl = idx / a.n_out;
        } else {
            cl = idx % C;
            j = idx / C;
        }
        long o, c;
        if (!line_ok(cl, o, c)) continue;
        int f;
        if (a.out_map == OUT_MODES) {
            f = j - a.n_out / 2;
            if (f < 0) f += L;
        } else if (a.out_map == OUT_WINDOW) {
            f = j + a.out_off;
        } else {
            f = j;
        }
        V v = buf[f * C + cl];
        T s = (T)a.scale;
        if (post) s *= post[j];
        v = cscale(v, s);
        st_elem<T, TO>(out + o * a.out_ostride + (long)j * a.n_inner + c, v);
    }
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

}  // namespace

void launch_axis_fft(Context &ctx, const AxisFFT &a) {
    LC_REQUIRE(is_smooth23(a.L), "axis FFT length must be 2^p*3^q");
    LC_REQUIRE(a.n_in >= 0 && a.n_out >= 0, "axis FFT: bad lengths");
    if (a.in_map == IN_HERM) LC_REQUIRE(a.n_in == a.L / 2 + 1, "IN_HERM needs n_in = L/2+1");
    else LC_REQUIRE(a.n_in <= a.L, "axis FFT: n_in > L");
    if (a.out_map == OUT_WINDOW) LC_REQUIRE(a.out_off >= 0 && a.out_off + a.n_out <= a.L, "window");
    else LC_REQUIRE(a.n_out <= a.L, "axis FFT: n_out > L");
    if (a.n_outer <= 0 || a.n_inner <= 0 || a.n_out == 0) return;

    const FFTPlan &pl = ctx.plans().get(a.L, a.fp64, ctx.stream());
    const size_t esz = a.fp64 ? sizeof(double2) : sizeof(float2);
    const size_t smem_cap = std::min<size_t>(ctx.max_smem(), 200 * 1024);

    int C = a.lines_per_cta;
    if (C <= 0) {
        if (a.n_inner == 1) {
            C = std::max(1, 2048 / a.L);
        } else {
            C = 16;
            while (C > 1 && (long)C > a.n_inner * 2) C /= 2;
        }
    }
    // two ping-pong buffers of L*C elements must fit in shared memory
    while (C > 1 && 2 * (size_t)a.L * C * esz > smem_cap) --C;
    LC_REQUIRE(2 * (size_t)a.L * C * esz <= ctx.max_smem(), "axis FFT: line does not fit shared memory");
    long work = (long)a.L * C / 2;
    int threads = work >= 4096 ? 512 : (work >= 1024 ? 256 : 128);

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
    ka.C = C;
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
    if (a.fp64) dispatch<double>(ctx, a, ka, pl, threads, smem, blocks);
    else dispatch<float>(ctx, a, ka, pl, threads, smem, blocks);
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

void launch_axis_dft(Context &ctx, const AxisDFT &a) {
    LC_REQUIRE(a.n > 0, "DFT length must be positive");
    const double lines = (double)a.n_outer * a.n_inner;
    ProfScope ps(ctx, PS_DFT,
                 lines * a.n * ((a.in_t == E_F32 ? 4.0 : 8.0) + (a.out_t == E_F32 ? 4.0 : 8.0)));
    LC_REQUIRE(a.in_t == E_F32 || a.in_t == E_C64, "DFT input must be float or float2");
    LC_REQUIRE(a.out_t == E_F32 || a.out_t == E_C64, "DFT output must be float or float2");
    if (a.n_outer <= 0 || a.n_inner <= 0) return;
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
