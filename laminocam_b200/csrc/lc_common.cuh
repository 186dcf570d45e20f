// Shared device/host helpers for the laminocam_b200 kernels (sm_100a).
//
//  * complex helpers over float2 / double2
//  * the exponential-of-semicircle (ES) spreading kernel
//  * a shared-memory Stockham FFT core (radices 2, 3, 4, 8) used by every
//    line-FFT kernel in this library
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <cmath>
#include <stdexcept>
#include <string>

namespace lc {

// ---------------------------------------------------------------------------
// errors
// ---------------------------------------------------------------------------
struct Error : std::runtime_error {
    int code;
    Error(int c, const std::string &m) : std::runtime_error(m), code(c) {}
};

// file name without its directories, for error messages
constexpr const char *lc_basename(const char *p) {
    const char *b = p;
    for (const char *q = p; *q; ++q)
        if (*q == '/') b = q + 1;
    return b;
}

#define LC_CUDA(call)                                                                          \
    do {                                                                                       \
        cudaError_t e_ = (call);                                                               \
        if (e_ != cudaSuccess)                                                                 \
            throw ::lc::Error(3, std::string(#call) + " (" + ::lc::lc_basename(__FILE__) + ":" + \
                                     std::to_string(__LINE__) + "): " + cudaGetErrorString(e_)); \
    } while (0)

// Kernel launches issued by this library (every launch site is followed by
// LC_CHECK_LAUNCH(), which also counts it).
long kernel_launch_count();
void note_kernel_launch();

#define LC_CHECK_LAUNCH()              \
    do {                               \
        ::lc::note_kernel_launch();    \
        LC_CUDA(cudaGetLastError());   \
    } while (0)

#define LC_REQUIRE(cond, msg)                                                           \
    do {                                                                                \
        if (!(cond)) throw ::lc::Error(1, std::string(msg));                           \
    } while (0)

// ---------------------------------------------------------------------------
// complex arithmetic
// ---------------------------------------------------------------------------
template <typename T> struct C2;
template <> struct C2<float> { using type = float2; };
template <> struct C2<double> { using type = double2; };
template <typename T> using cx = typename C2<T>::type;

template <typename T> __host__ __device__ __forceinline__ cx<T> mk(T r, T i) {
    cx<T> z;
    z.x = r;
    z.y = i;
    return z;
}
template <typename V> __host__ __device__ __forceinline__ V cadd(V a, V b) {
    a.x += b.x;
    a.y += b.y;
    return a;
}
template <typename V> __host__ __device__ __forceinline__ V csub(V a, V b) {
    a.x -= b.x;
    a.y -= b.y;
    return a;
}
template <typename V> __host__ __device__ __forceinline__ V cmul(V a, V b) {
    V z;
    z.x = a.x * b.x - a.y * b.y;
    z.y = a.x * b.y + a.y * b.x;
    return z;
}
template <typename V> __host__ __device__ __forceinline__ V cconj(V a) {
    a.y = -a.y;
    return a;
}
template <typename V, typename S> __host__ __device__ __forceinline__ V cscale(V a, S s) {
    a.x *= s;
    a.y *= s;
    return a;
}
// multiply by sign*i
template <typename V> __device__ __forceinline__ V cmul_i(V a, int sign) {
    V z;
    if (sign > 0) {
        z.x = -a.y;
        z.y = a.x;
    } else {
        z.x = a.y;
        z.y = -a.x;
    }
    return z;
}

// ---------------------------------------------------------------------------
// line-FFT plans
// ---------------------------------------------------------------------------
constexpr int kMaxStages = 16;

// Device-side description of one FFT length: radix sequence, the multiplier
// that divides by Ns (the product of the earlier radices) at each stage, and
// the twiddle table tw[m] = exp(-2*pi*i*m/L), m in [0, L), in the plan's
// precision.
struct FFTPlan {
    int L;
    int nst;
    int radix[kMaxStages];
    unsigned long long ns_magic[kMaxStages];  // ceil(2^40 / Ns)
    const void *tw;
};

// floor(n / d) for n, d < 2^20 from magic = ceil(2^40 / d): the error term
// n * (magic * d - 2^40) < n * d < 2^40 keeps the quotient exact.
__host__ __device__ __forceinline__ unsigned fast_div(unsigned n, unsigned long long magic) {
    return (unsigned)(((unsigned long long)n * magic) >> 40);
}
__host__ __device__ __forceinline__ unsigned long long fast_div_magic(unsigned d) {
    return ((1ULL << 40) + d - 1) / d;
}

// Fills radices (8, 9, 4, 2, 3 preferred in that order) and division
// multipliers; returns false unless L = 2^p 3^q fits in kMaxStages stages.
inline bool fft_factorise(int L, FFTPlan &pl) {
    pl.L = L;
    pl.nst = 0;
    int r = L;
    auto push = [&](int R) {
        if (pl.nst >= kMaxStages) return false;
        pl.radix[pl.nst++] = R;
        r /= R;
        return true;
    };
    while (r % 8 == 0)
        if (!push(8)) return false;
    while (r % 9 == 0)
        if (!push(9)) return false;
    if (r % 4 == 0 && !push(4)) return false;
    if (r % 2 == 0 && !push(2)) return false;
    while (r % 3 == 0)
        if (!push(3)) return false;
    if (r != 1) return false;
    unsigned ns = 1;
    for (int s = 0; s < pl.nst; ++s) {
        pl.ns_magic[s] = fast_div_magic(ns);
        ns *= (unsigned)pl.radix[s];
    }
    return true;
}

template <typename V, int R>
__device__ __forceinline__ void dft_small(V *v, int sign) {
    using T = decltype(v[0].x);
    if constexpr (R == 2) {
        V a = v[0], b = v[1];
        v[0] = cadd(a, b);
        v[1] = csub(a, b);
    } else if constexpr (R == 3) {
        const T c1 = T(-0.5);
        const T s1 = T(0.86602540378443864676) * T(sign);
        V a = v[0], b = v[1], c = v[2];
        V t1 = cadd(b, c);
        V t2 = csub(b, c);
        v[0] = cadd(a, t1);
        V m = mk<T>(a.x + c1 * t1.x, a.y + c1 * t1.y);
        // (b - c) * i * s1
        V r = mk<T>(-s1 * t2.y, s1 * t2.x);
        v[1] = cadd(m, r);
        v[2] = csub(m, r);
    } else if constexpr (R == 4) {
        V a = v[0], b = v[1], c = v[2], d = v[3];
        V t0 = cadd(a, c), t1 = csub(a, c), t2 = cadd(b, d), t3 = cmul_i(csub(b, d), sign);
        v[0] = cadd(t0, t2);
        v[2] = csub(t0, t2);
        v[1] = cadd(t1, t3);
        v[3] = csub(t1, t3);
    } else if constexpr (R == 9) {
        // 3 x 3: DFT3 over n1 for each n2, twiddle W9^(n2 k1), DFT3 over n2
        const T c1 = T(0.76604444311897803520), s1 = T(0.64278760968653932632) * T(sign);
        const T c2 = T(0.17364817766693034885), s2 = T(0.98480775301220805936) * T(sign);
        const T c4 = T(-0.93969262078590838405), s4 = T(0.34202014332566873304) * T(sign);
        V y[3][3];
#pragma unroll
        for (int n2 = 0; n2 < 3; ++n2) {
            V t[3] = {v[n2], v[n2 + 3], v[n2 + 6]};
            dft_small<V, 3>(t, sign);
            y[n2][0] = t[0];
            y[n2][1] = t[1];
            y[n2][2] = t[2];
        }
        y[1][1] = cmul(y[1][1], mk<T>(c1, s1));  // W9^1
        y[1][2] = cmul(y[1][2], mk<T>(c2, s2));  // W9^2
        y[2][1] = cmul(y[2][1], mk<T>(c2, s2));  // W9^2
        y[2][2] = cmul(y[2][2], mk<T>(c4, s4));  // W9^4
#pragma unroll
        for (int k1 = 0; k1 < 3; ++k1) {
            V t[3] = {y[0][k1], y[1][k1], y[2][k1]};
            dft_small<V, 3>(t, sign);
            v[k1] = t[0];
            v[k1 + 3] = t[1];
            v[k1 + 6] = t[2];
        }
    } else if constexpr (R == 8) {
        const T h = T(0.70710678118654752440);
        // radix-2 over even/odd, then radix-4 each
        V e[4] = {v[0], v[2], v[4], v[6]};
        V o[4] = {v[1], v[3], v[5], v[7]};
        dft_small<V, 4>(e, sign);
        dft_small<V, 4>(o, sign);
        // twiddles w8^k for k=0..3 with sign: exp(sign*i*2*pi*k/8)
        V o1 = mk<T>(h * (o[1].x - T(sign) * o[1].y), h * (o[1].y + T(sign) * o[1].x));
        V o2 = cmul_i(o[2], sign);
        V o3 = mk<T>(h * (-o[3].x - T(sign) * o[3].y), h * (-o[3].y + T(sign) * o[3].x));
        v[0] = cadd(e[0], o[0]);
        v[4] = csub(e[0], o[0]);
        v[1] = cadd(e[1], o1);
        v[5] = csub(e[1], o1);
        v[2] = cadd(e[2], o2);
        v[6] = csub(e[2], o2);
        v[3] = cadd(e[3], o3);
        v[7] = csub(e[3], o3);
    }
}

// One Stockham stage of radix R over C lines of length L, out of place:
// element (i, c) of line c lives at src[i*C + c] / dst[i*C + c].  C is a power
// of two (1 << logC); the division by Ns uses the plan's multiplier.
template <typename T, int R>
__device__ __forceinline__ void stockham_stage(const cx<T> *__restrict__ src, cx<T> *__restrict__ dst,
                                               int L, int logC, int Ns, unsigned long long ns_magic,
                                               const cx<T> *__restrict__ tw, int sign) {
    using V = cx<T>;
    const int C = 1 << logC;
    const int nb = L / R;
    const int items = nb << logC;
    const int tstride = L / (Ns * R);
    for (int it = threadIdx.x; it < items; it += blockDim.x) {
        const int c = it & (C - 1);
        const int j = it >> logC;
        const int g = (int)fast_div((unsigned)j, ns_magic);
        const int k = j - g * Ns;
        V v[R];
        const V *s0 = src + (j << logC) + c;
        const int sstep = nb << logC;
#pragma unroll
        for (int r = 0; r < R; ++r) v[r] = s0[r * sstep];
        if (Ns > 1) {
            // twiddles w^r from w = tw[k * tstride], with w^2 also taken from
            // the table for radices above 4 (halves the recurrence depth)
            V w1 = tw[k * tstride];
            if (sign > 0) w1.y = -w1.y;
            v[1] = cmul(v[1], w1);
            if (R > 2) {
                V w2;
                if (R > 4) {
                    w2 = tw[2 * k * tstride];
                    if (sign > 0) w2.y = -w2.y;
                } else {
                    w2 = cmul(w1, w1);
                }
                v[2] = cmul(v[2], w2);
                V wo = w1, we = w2;
#pragma unroll
                for (int r = 3; r < R; ++r) {
                    if (r & 1) {
                        wo = cmul(wo, w2);
                        v[r] = cmul(v[r], wo);
                    } else {
                        we = cmul(we, w2);
                        v[r] = cmul(v[r], we);
                    }
                }
            }
        }
        dft_small<V, R>(v, sign);
        const int base = g * Ns * R + k;
        V *d0 = dst + (base << logC) + c;
        const int dstep = Ns << logC;
#pragma unroll
        for (int r = 0; r < R; ++r) d0[r * dstep] = v[r];
    }
}

// Unnormalised DFT of C = 1 << logC lines held in shared memory ([L][C]
// layout), natural order in and out, ping-ponging between a and b.  Returns
// the buffer that holds the result.  sign = -1: forward (e^{-i}); +1: backward.
// The data must be complete in `a` (__syncthreads() before the call); the
// result is complete when the call returns.
template <typename T>
__device__ cx<T> *smem_fft(cx<T> *a, cx<T> *b, int logC, const FFTPlan &pl, int sign) {
    const cx<T> *tw = reinterpret_cast<const cx<T> *>(pl.tw);
    cx<T> *src = a, *dst = b;
    int Ns = 1;
    for (int s = 0; s < pl.nst; ++s) {
        const int R = pl.radix[s];
        const unsigned long long mg = pl.ns_magic[s];
        switch (R) {
            case 2: stockham_stage<T, 2>(src, dst, pl.L, logC, Ns, mg, tw, sign); break;
            case 3: stockham_stage<T, 3>(src, dst, pl.L, logC, Ns, mg, tw, sign); break;
            case 4: stockham_stage<T, 4>(src, dst, pl.L, logC, Ns, mg, tw, sign); break;
            case 9: stockham_stage<T, 9>(src, dst, pl.L, logC, Ns, mg, tw, sign); break;
            default: stockham_stage<T, 8>(src, dst, pl.L, logC, Ns, mg, tw, sign); break;
        }
        __syncthreads();
        cx<T> *t = src;
        src = dst;
        dst = t;
        Ns *= R;
    }
    return src;
}

// ---------------------------------------------------------------------------
// exponential-of-semicircle kernel  phi(z) = exp(beta*(sqrt(1-z^2)-1)), |z|<=1
// (Barnett, Magland & af Klinteberg, SIAM J. Sci. Comput. 41(5), 2019)
// ---------------------------------------------------------------------------
struct ESParams {
    int w;        // kernel width in fine-grid cells
    float beta;   // shape parameter
    float half_w; // w/2
};

template <typename T>
__device__ __forceinline__ T es_eval(T z, T beta) {
    T s = T(1) - z * z;
    return s > T(0) ? exp(beta * (sqrt(s) - T(1))) : T(0);
}

__device__ __forceinline__ float es_evalf(float z, float beta) {
    float s = 1.0f - z * z;
    return s > 0.0f ? expf(beta * (sqrtf(s) - 1.0f)) : 0.0f;
}

// The same kernel as 2^x with x = beta_l2e (sqrt(1 - z^2) - 1), beta_l2e =
// beta log2(e) rounded to float: exp2f and a correctly rounded square root.
// Rounding beta_l2e and the product moves x by at most 2^-23 |x|, so a weight
// 2^x changes by at most 2^-23 ln(2) |x| 2^x <= 4.4e-8 of the peak weight 1,
// besides exp2f's own error of 2 ulp.
__device__ __forceinline__ float es_eval2f(float z, float beta_l2e) {
    const float s = fmaf(-z, z, 1.0f);
    return s > 0.0f ? exp2f(beta_l2e * (__fsqrt_rn(s) - 1.0f)) : 0.0f;
}

// Fine-grid placement of a coordinate x (radians, any real value, taken
// 2*pi-periodic) on a grid of nf cells of width 2*pi/nf.  Computes the first
// covered cell l0 (not yet wrapped) and the offset of x from l0 in cells, in
// double precision so that the float kernel evaluation sees an exact offset.
__device__ __forceinline__ void es_place(double x, int nf, int w, int &l0, float &off) {
    double u = x * (double)nf * 0.15915494309189533577;  // x / h, h = 2*pi/nf
    double lo = ceil(u - 0.5 * (double)w);
    l0 = (int)lo;
    off = (float)(u - lo);  // in (w/2 - 1, w/2]; cell l0+m sits at z = (m - off)/(w/2)
}

__device__ __forceinline__ int wrap(int l, int n) {
    l %= n;
    return l < 0 ? l + n : l;
}

}  // namespace lc
