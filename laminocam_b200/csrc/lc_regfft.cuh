// Register-resident small DFTs and Stockham stages with compile-time radices,
// shared by the Toeplitz z-stage kernel and the column / row line kernels.
//
// Stockham stage of radix R over a line of M points, after stages whose
// radices multiply to NS (NS = 1 for the first stage): butterfly j in
// [0, M/R) reads the elements j + r (M/R), r < R, multiplies element r by
// w_M^(r k M/(NS R)) with k = j mod NS, does a DFT of length R and writes
// element r of the result to (j div NS) NS R + k + r NS.  After the last
// stage the line is in natural order; the last stage writes j + r (M/R).
#pragma once

#include "lc_common.cuh"

namespace lc {

// exp(sign * 2 pi i m / N) for the composite radices 6, 12, 16 and 18
template <int N>
__device__ __forceinline__ float2 unit_root(int m, int sign) {
    const float h = 0.70710678118654752440f, c30 = 0.86602540378443864676f;
    const float c22 = 0.92387953251128675613f, s22 = 0.38268343236508977173f;
    float c = 1.f, s = 0.f;
    if constexpr (N == 6) {
        const float cs[6] = {1.f, 0.5f, -0.5f, -1.f, -0.5f, 0.5f};
        const float sn[6] = {0.f, c30, c30, 0.f, -c30, -c30};
        c = cs[m];
        s = sn[m];
    } else if constexpr (N == 12) {
        const float cs[12] = {1.f, c30, 0.5f, 0.f, -0.5f, -c30, -1.f, -c30, -0.5f, 0.f, 0.5f, c30};
        const float sn[12] = {0.f, 0.5f, c30, 1.f, c30, 0.5f, 0.f, -0.5f, -c30, -1.f, -c30, -0.5f};
        c = cs[m];
        s = sn[m];
    } else if constexpr (N == 16) {
        const float cs[16] = {1.f, c22, h, s22, 0.f, -s22, -h, -c22, -1.f, -c22, -h, -s22, 0.f, s22, h, c22};
        const float sn[16] = {0.f, s22, h, c22, 1.f, c22, h, s22, 0.f, -s22, -h, -c22, -1.f, -c22, -h, -s22};
        c = cs[m];
        s = sn[m];
    } else if constexpr (N == 18) {
        // cos and sin of 20 m degrees
        const float a = 0.93969262078590838405f, b = 0.34202014332566873304f;  // 20
        const float d = 0.76604444311897803520f, e = 0.64278760968653932632f;  // 40
        const float f = 0.17364817766693034885f, g = 0.98480775301220805936f;  // 80
        const float cs[18] = {1.f, a, d, 0.5f, f, -f, -0.5f, -d, -a, -1.f, -a, -d, -0.5f, -f, f, 0.5f, d, a};
        const float sn[18] = {0.f, b, e, c30, g, g, c30, e, b, 0.f, -b, -e, -c30, -g, -g, -c30, -e, -b};
        c = cs[m];
        s = sn[m];
    }
    return make_float2(c, sign * s);
}

// N = R1 * R2 from two small DFTs: n = b + R2 a, k = k1 + R1 k2
template <int R1, int R2>
__device__ __forceinline__ void dft_composite(float2 *v, int sign) {
    constexpr int N = R1 * R2;
    float2 y[R2][R1];
#pragma unroll
    for (int b = 0; b < R2; ++b) {
        float2 t[R1];
#pragma unroll
        for (int a = 0; a < R1; ++a) t[a] = v[b + R2 * a];
        dft_small<float2, R1>(t, sign);
#pragma unroll
        for (int k1 = 0; k1 < R1; ++k1) y[b][k1] = (b * k1 == 0) ? t[k1] : cmul(t[k1], unit_root<N>(b * k1, sign));
    }
#pragma unroll
    for (int k1 = 0; k1 < R1; ++k1) {
        float2 t[R2];
#pragma unroll
        for (int b = 0; b < R2; ++b) t[b] = y[b][k1];
        dft_small<float2, R2>(t, sign);
#pragma unroll
        for (int k2 = 0; k2 < R2; ++k2) v[k1 + R1 * k2] = t[k2];
    }
}

// unnormalised DFT of length N in registers (sign -1 forward, +1 backward)
template <int N>
__device__ __forceinline__ void dft_reg(float2 *v, int sign) {
    if constexpr (N == 1) return;
    else if constexpr (N == 6) dft_composite<3, 2>(v, sign);
    else if constexpr (N == 12) dft_composite<3, 4>(v, sign);
    else if constexpr (N == 16) dft_composite<4, 4>(v, sign);
    else if constexpr (N == 18) dft_composite<9, 2>(v, sign);
    else dft_small<float2, N>(v, sign);
}

// Stage twiddles of NV lines at once: element r of butterfly j of every line
// times w_M^(r k TS), k = j mod NS, TS = M / (NS R); tw[m] = exp(-2 pi i m / M).
// w and w^2 come from the table, the higher powers from products of them.
template <int M, int R, int NS, int NV, int RM>
__device__ __forceinline__ void stage_twiddle(float2 (&v)[NV][RM], int j, const float2 *tw, int sign) {
    if constexpr (NS > 1 && R > 1) {
        constexpr int TS = M / (NS * R);
        const int k = j % NS;
        float2 w1 = tw[k * TS];
        if (sign > 0) w1.y = -w1.y;
#pragma unroll
        for (int q = 0; q < NV; ++q) v[q][1] = cmul(v[q][1], w1);
        if constexpr (R > 2) {
            float2 w2;
            if constexpr (R > 4) {
                w2 = tw[2 * k * TS];
                if (sign > 0) w2.y = -w2.y;
            } else {
                w2 = cmul(w1, w1);
            }
#pragma unroll
            for (int q = 0; q < NV; ++q) v[q][2] = cmul(v[q][2], w2);
            float2 wo = w1, we = w2;
#pragma unroll
            for (int r = 3; r < R; ++r) {
                float2 w;
                if (r & 1) {
                    wo = cmul(wo, w2);
                    w = wo;
                } else {
                    we = cmul(we, w2);
                    w = we;
                }
#pragma unroll
                for (int q = 0; q < NV; ++q) v[q][r] = cmul(v[q][r], w);
            }
        }
    }
}

// ---- compile-time twiddle tables -------------------------------------------
// sin and cos of 2 pi num / den: the angle is reduced exactly (in integers) to
// within 1/16 turn of a multiple of 1/8 turn, the remainder x (|x| <= pi/8)
// goes through the Taylor series of sin and cos (12 terms: the truncation
// error is far below double rounding), and the result is rotated by the
// octant.  Used only to build constant tables at compile time.
constexpr void ct_sincos(long num, long den, double &s, double &c) {
    num %= den;
    if (num < 0) num += den;
    const long o8 = 8 * num;
    const long oct = (o8 + den / 2) / den;
    const double x = 2.0 * 3.14159265358979323846 * (double)(o8 - oct * den) / (8.0 * (double)den);
    const double x2 = x * x;
    double ts = x, ss = x, tc = 1.0, cc = 1.0;
    for (int k = 1; k < 12; ++k) {
        ts *= -x2 / ((2.0 * k) * (2.0 * k + 1.0));
        ss += ts;
        tc *= -x2 / ((2.0 * k - 1.0) * (2.0 * k));
        cc += tc;
    }
    const double h = 0.70710678118654752440;
    const double co[8] = {1, h, 0, -h, -1, -h, 0, h};
    const double so[8] = {0, h, 1, h, 0, -h, -1, -h};
    const int q = (int)(oct % 8);
    s = ss * co[q] + cc * so[q];
    c = cc * co[q] - ss * so[q];
}

// v[m] = exp(-2 pi i m / M) and v[M + m] = exp(-pi i m / M), m < M
template <int M>
struct LineTwiddles {
    alignas(16) float2 v[2 * M];
    constexpr LineTwiddles() : v() {
        for (int m = 0; m < M; ++m) {
            double s = 0.0, c = 0.0;
            ct_sincos(m, M, s, c);
            v[m] = float2{(float)c, (float)-s};
            ct_sincos(m, 2 * M, s, c);
            v[M + m] = float2{(float)c, (float)-s};
        }
    }
};

template <int M>
__device__ const LineTwiddles<M> g_line_twiddles = LineTwiddles<M>();

// copy the 2M table entries into shared memory (all threads of the CTA)
template <int M>
__device__ __forceinline__ void load_line_twiddles(float2 *dst) {
    const float4 *src = reinterpret_cast<const float4 *>(g_line_twiddles<M>.v);
    float4 *d4 = reinterpret_cast<float4 *>(dst);
    for (int i = threadIdx.x; i < M; i += blockDim.x) d4[i] = __ldg(src + i);
}

constexpr int cmax(int a, int b) { return a > b ? a : b; }
constexpr int cmin(int a, int b) { return a < b ? a : b; }

// A line of M = R0 R1 R2 points on NT threads (one butterfly each per stage)
template <int R0, int R1, int R2>
struct RegPlan {
    static constexpr int M = R0 * R1 * R2;
    static constexpr int NT = M / cmin(R0, cmin(R1, R2));  // threads per line
    static constexpr int RM = cmax(R0, cmax(R1, R2));      // registers per line
};

// Line lengths M with a register plan: X(M, R0, R1, R2), radices in stage
// order.  Every 2^p 3^q length from 64 to 1296 whose three radices are at most
// 16 with M / min(R) <= 144 threads per line.  An odd first radix keeps the
// first stage's strided shared-memory writes free of bank conflicts.
#define LC_LINE_PLANS(X) \
    X(64, 4, 4, 4)       \
    X(72, 3, 4, 6)       \
    X(81, 9, 3, 3)       \
    X(96, 3, 8, 4)       \
    X(108, 3, 6, 6)      \
    X(128, 8, 4, 4)      \
    X(144, 9, 4, 4)      \
    X(162, 9, 6, 3)      \
    X(192, 3, 8, 8)      \
    X(216, 9, 6, 4)      \
    X(243, 9, 9, 3)      \
    X(256, 8, 8, 4)      \
    X(288, 9, 8, 4)      \
    X(324, 9, 6, 6)      \
    X(384, 6, 8, 8)      \
    X(432, 9, 6, 8)      \
    X(486, 9, 9, 6)      \
    X(512, 8, 8, 8)      \
    X(576, 9, 8, 8)      \
    X(648, 9, 9, 8)      \
    X(729, 9, 9, 9)      \
    X(768, 12, 8, 8)     \
    X(864, 9, 12, 8)     \
    X(972, 9, 9, 12)     \
    X(1024, 16, 8, 8)    \
    X(1152, 9, 16, 8)    \
    X(1296, 9, 12, 12)

inline bool line_plan_exists(int M) {
    switch (M) {
#define LC_LINE_HAS(m, r0, r1, r2) case m:
        LC_LINE_PLANS(LC_LINE_HAS)
#undef LC_LINE_HAS
        return true;
        default: return false;
    }
}

// Three Stockham stages (radices RA, RB, RC) of NV lines of M points.  The
// thread (index t within its line group) holds the elements t + r M/RA,
// r < RA, of line q in v[q]; on return it holds the elements t + r M/RC of
// the transforms.  at(q, i) is the shared-memory slot of element i of line
// q; the lines cross shared memory twice, in place.  tw[m] = exp(-2 pi i m/M).
// Every thread of the CTA must call it (it synchronises the CTA).
template <int M, int RA, int RB, int RC, int NV, int RM, class At>
__device__ __forceinline__ void xform3(float2 (&v)[NV][RM], const At &at, int t, const float2 *tw, int sign) {
    constexpr int NA = M / RA, NB = M / RB, NC = M / RC;
    if (t < NA) {
#pragma unroll
        for (int q = 0; q < NV; ++q) dft_reg<RA>(v[q], sign);
    }
    __syncthreads();  // earlier readers of the slots are done
    if (t < NA) {
#pragma unroll
        for (int q = 0; q < NV; ++q)
#pragma unroll
            for (int r = 0; r < RA; ++r) at(q, t * RA + r) = v[q][r];
    }
    __syncthreads();
    if (t < NB) {
#pragma unroll
        for (int q = 0; q < NV; ++q) {
#pragma unroll
            for (int r = 0; r < RB; ++r) v[q][r] = at(q, t + r * NB);
        }
        stage_twiddle<M, RB, RA>(v, t, tw, sign);
#pragma unroll
        for (int q = 0; q < NV; ++q) dft_reg<RB>(v[q], sign);
    }
    __syncthreads();
    if (t < NB) {
        const int o = (t / RA) * RA * RB + t % RA;
#pragma unroll
        for (int q = 0; q < NV; ++q)
#pragma unroll
            for (int r = 0; r < RB; ++r) at(q, o + r * RA) = v[q][r];
    }
    __syncthreads();
    if (t < NC) {
#pragma unroll
        for (int q = 0; q < NV; ++q) {
#pragma unroll
            for (int r = 0; r < RC; ++r) v[q][r] = at(q, t + r * NC);
        }
        stage_twiddle<M, RC, RA * RB>(v, t, tw, sign);
#pragma unroll
        for (int q = 0; q < NV; ++q) dft_reg<RC>(v[q], sign);
    }
}

}  // namespace lc
