// The z stage of the 3D Toeplitz apply as one register-resident kernel.
//
// For every column (ky, kx) of the half spectrum, the stage takes the n1
// values along z, zero-pads them to L = P1, transforms, multiplies by the real
// spectrum column, transforms back and keeps the first n1 values (the cropped
// circular convolution of include/toeplitz.h:95-129 along z).  L is small for
// laminography volumes (P1 <= 128), so a line is split as L = A * B over
// max(A, B) threads: each thread keeps A (then B) elements in registers and
// does its radix-A (radix-B) DFTs there, and the line crosses shared memory
// once per transform.  The generic shared-memory Stockham kernel instead
// passes through shared memory and a barrier at every radix stage, and spends
// about 280 instructions per element at L = 48.
//
// Decomposition (n = b + B a, k = k1 + A k2, w = exp(-2 pi i / L)):
//   Y_b[k1]        = sum_a x[b + B a] w^(B a k1)            (DFT_A in thread b)
//   X[k1 + A k2]   = sum_b (Y_b[k1] w^(b k1)) w^(A b k2)    (DFT_B in thread k1)
// and the inverse runs the same steps backwards with conjugate roots.
//
// HALF (n_in, n_out <= L/2, always so for a Toeplitz line, L >= 2 n - 1 with
// L even): the inputs x[b + B a] with a >= A/2 vanish and the outputs with
// a >= A/2 are not kept, so the outer radix-A steps run as two DFTs of A/2
// (the even/odd split of the column kernels): forward
// Y[2m] = DFT_{A/2}(x)[m], Y[2m+1] = DFT_{A/2}(x h)[m] with
// h(a) = exp(-2 pi i a / A) = w^(B a); inverse
// x[a] = DFT+_{A/2}(Y_even)[a] + conj h(a) DFT+_{A/2}(Y_odd)[a].
//
// Direct form.  When the kernel is even in z (the angle set is closed under
// the mirror that negates kz), the stage for one column is a real symmetric
// Toeplitz matrix times the column: with b(dz) = the kernel's z-profile of
// the column (the kernel after the x and y transforms), the FFT form computes
// L sum_{z'} b(z - z') x[z'] and b(-dz) = b(dz) is real.  At n = 29 rows
// that is 2 n^2 = 1682 FMAs per column against about 4100 instructions for
// the 64-point FFT route, and the column never leaves registers, so the
// stage runs at the rate its bytes allow.  The taps L b(dz), dz < n, are
// stored per column (n planes instead of the L/2 + 1 spectrum planes).
#include <cstdlib>

#include "lc_fft.hpp"
#include "lc_regfft.cuh"

#ifndef LC_Z64_COLS
#define LC_Z64_COLS 32  // columns per CTA of the 64-point z convolution
#endif

namespace lc {
namespace {

template <int A, int B, int C, bool HALF>
__global__ void __launch_bounds__(C *(A > B ? A : B))
    zconv_kernel(float2 *data, long n_inner, int n_in, int n_out, const float *__restrict__ spec, int fold) {
    constexpr int L = A * B;
    constexpr int TPL = A > B ? A : B;
    __shared__ float2 sm[L * C];
    __shared__ float2 tw[L];  // exp(-2 pi i m / L)
    for (int m = threadIdx.x; m < L; m += blockDim.x) {
        float s, c;
        sincospif(2.0f * (float)m / (float)L, &s, &c);
        tw[m] = make_float2(c, -s);
    }
    const int cl = threadIdx.x % C, j = threadIdx.x / C;
    const long col = (long)blockIdx.x * C + cl;
    const bool valid = col < n_inner;
    float2 v[TPL];
    // forward, radix A in thread b = j: x[b + B a] -> Y_b[k1] w^(b k1)
    constexpr int AH = HALF ? A / 2 : A;  // radix-A inputs (outputs) that can be nonzero (kept)
    if (j < B) {
#pragma unroll
        for (int a = 0; a < AH; ++a) {
            const int n = j + B * a;
            v[a] = (valid && n < n_in) ? data[(long)n * n_inner + col] : make_float2(0.f, 0.f);
        }
    }
    __syncthreads();  // twiddle table ready
    if (j < B) {
        if constexpr (HALF) {
            float2 e[AH], o[AH];
#pragma unroll
            for (int a = 0; a < AH; ++a) {
                e[a] = v[a];
                o[a] = a ? cmul(v[a], tw[a * B]) : v[a];
            }
            dft_reg<AH>(e, -1);
            dft_reg<AH>(o, -1);
#pragma unroll
            for (int m = 0; m < AH; ++m) {
                v[2 * m] = e[m];
                v[2 * m + 1] = o[m];
            }
        } else {
            dft_reg<A>(v, -1);
        }
#pragma unroll
        for (int k1 = 1; k1 < A; ++k1) v[k1] = cmul(v[k1], tw[(j * k1) % L]);
#pragma unroll
        for (int k1 = 0; k1 < A; ++k1) sm[(k1 * B + j) * C + cl] = v[k1];
    }
    __syncthreads();
    // radix B in thread k1 = j, spectral multiply, inverse radix B
    if (j < A) {
#pragma unroll
        for (int b = 0; b < B; ++b) v[b] = sm[(j * B + b) * C + cl];
        dft_reg<B>(v, -1);
#pragma unroll
        for (int k2 = 0; k2 < B; ++k2) {
            int f = j + A * k2;
            if (fold && f > L / 2) f = L - f;
            const float r = valid ? __ldg(spec + (long)f * n_inner + col) : 0.f;
            v[k2] = make_float2(v[k2].x * r, v[k2].y * r);
        }
        dft_reg<B>(v, +1);
#pragma unroll
        for (int b = 1; b < B; ++b) {
            const float2 w = tw[(j * b) % L];
            v[b] = cmul(v[b], make_float2(w.x, -w.y));
        }
#pragma unroll
        for (int b = 0; b < B; ++b) sm[(j * B + b) * C + cl] = v[b];
    }
    __syncthreads();
    // inverse radix A in thread b = j, keep the first n_out rows
    if (j < B) {
#pragma unroll
        for (int k1 = 0; k1 < A; ++k1) v[k1] = sm[(k1 * B + j) * C + cl];
        if constexpr (HALF) {
            float2 e[AH], o[AH];
#pragma unroll
            for (int m = 0; m < AH; ++m) {
                e[m] = v[2 * m];
                o[m] = v[2 * m + 1];
            }
            dft_reg<AH>(e, +1);
            dft_reg<AH>(o, +1);
#pragma unroll
            for (int a = 0; a < AH; ++a) {
                const float2 h = tw[a * B];
                v[a] = a ? cadd(e[a], cmul(make_float2(h.x, -h.y), o[a])) : cadd(e[a], o[a]);
            }
        } else {
            dft_reg<A>(v, +1);
        }
#pragma unroll
        for (int a = 0; a < AH; ++a) {
            const int n = j + B * a;
            if (valid && n < n_out) data[(long)n * n_inner + col] = v[a];
        }
    }
}

// Direct z stage, one column per thread.  N is the compile-time row count
// (n rounded up; rows n..N-1 are zero and not stored).  The column's n
// values and n taps stay in registers; every output is one fixed-order sum
// of N products, so the result does not depend on the launch shape.
template <int N>
__global__ void __launch_bounds__(128, (N <= 32 ? 4 : 2))
    zdirect_kernel(float2 *data, long n_inner, int n, const float *__restrict__ taps) {
    const long col = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (col >= n_inner) return;
    float2 x[N];
    float k[N];
#pragma unroll
    for (int z = 0; z < N; ++z) {
        x[z] = z < n ? data[(long)z * n_inner + col] : make_float2(0.f, 0.f);
        k[z] = z < n ? __ldg(taps + (long)z * n_inner + col) : 0.f;
    }
#pragma unroll
    for (int z = 0; z < N; ++z) {
        if (z >= n) break;
        float ax = 0.f, ay = 0.f;
#pragma unroll
        for (int q = 0; q < N; ++q) {
            const float t = k[z > q ? z - q : q - z];
            ax = fmaf(t, x[q].x, ax);
            ay = fmaf(t, x[q].y, ay);
        }
        data[(long)z * n_inner + col] = make_float2(ax, ay);
    }
}

template <int N>
void launch_zd(cudaStream_t st, float2 *data, long n_inner, int n, const float *taps) {
    const long blocks = (n_inner + 127) / 128;
    LC_REQUIRE(blocks < (1L << 31), "direct z stage: grid too large");
    zdirect_kernel<N><<<(unsigned)blocks, 128, 0, st>>>(data, n_inner, n, taps);
    LC_CHECK_LAUNCH();
}

template <int A, int B, int C>
void launch_z(cudaStream_t st, float2 *data, long n_inner, int n_in, int n_out, const float *spec, int fold) {
    constexpr int TPL = A > B ? A : B;
    const long blocks = (n_inner + C - 1) / C;
    LC_REQUIRE(blocks < (1L << 31), "z convolution: grid too large");
    if (A % 2 == 0 && 2 * n_in <= A * B && 2 * n_out <= A * B)
        zconv_kernel<A, B, C, (A % 2 == 0)><<<(unsigned)blocks, C * TPL, 0, st>>>(data, n_inner, n_in, n_out,
                                                                                  spec, fold);
    else
        zconv_kernel<A, B, C, false><<<(unsigned)blocks, C * TPL, 0, st>>>(data, n_inner, n_in, n_out, spec,
                                                                          fold);
    LC_CHECK_LAUNCH();
}

}  // namespace

int zdirect_max_rows() { return 48; }

bool zdirect_enabled() {
    static const bool on = [] {
        const char *e = std::getenv("LC_ZDIRECT");
        return !(e && e[0] == '0');
    }();
    return on;
}

bool launch_zdirect(cudaStream_t st, float2 *data, long n_inner, int n, const float *taps) {
    LC_REQUIRE(n >= 0, "direct z stage: bad row count");
    if (n > zdirect_max_rows()) return false;
    if (n_inner <= 0 || n == 0) return true;
    if (n <= 4) launch_zd<4>(st, data, n_inner, n, taps);
    else if (n <= 8) launch_zd<8>(st, data, n_inner, n, taps);
    else if (n <= 12) launch_zd<12>(st, data, n_inner, n, taps);
    else if (n <= 16) launch_zd<16>(st, data, n_inner, n, taps);
    else if (n <= 20) launch_zd<20>(st, data, n_inner, n, taps);
    else if (n <= 24) launch_zd<24>(st, data, n_inner, n, taps);
    else if (n <= 28) launch_zd<28>(st, data, n_inner, n, taps);
    else if (n <= 32) launch_zd<32>(st, data, n_inner, n, taps);
    else if (n <= 40) launch_zd<40>(st, data, n_inner, n, taps);
    else launch_zd<48>(st, data, n_inner, n, taps);
    return true;
}

bool launch_zconv(cudaStream_t st, float2 *data, long n_inner, int L, int n_in, int n_out,
                  const float *spec, bool fold) {
    LC_REQUIRE(n_in >= 0 && n_in <= L && n_out >= 0 && n_out <= L, "z convolution: bad lengths");
    if (n_inner <= 0 || n_out == 0) return true;
    switch (L) {
        case 16: launch_z<4, 4, 32>(st, data, n_inner, n_in, n_out, spec, fold ? 1 : 0); return true;
        case 24: launch_z<8, 3, 32>(st, data, n_inner, n_in, n_out, spec, fold ? 1 : 0); return true;
        case 32: launch_z<8, 4, 32>(st, data, n_inner, n_in, n_out, spec, fold ? 1 : 0); return true;
        case 36: launch_z<6, 6, 32>(st, data, n_inner, n_in, n_out, spec, fold ? 1 : 0); return true;
        case 48: launch_z<8, 6, 32>(st, data, n_inner, n_in, n_out, spec, fold ? 1 : 0); return true;
        case 64: launch_z<8, 8, LC_Z64_COLS>(st, data, n_inner, n_in, n_out, spec, fold ? 1 : 0); return true;
        case 72: launch_z<8, 9, 16>(st, data, n_inner, n_in, n_out, spec, fold ? 1 : 0); return true;
        case 96: launch_z<8, 12, 16>(st, data, n_inner, n_in, n_out, spec, fold ? 1 : 0); return true;
        case 128: launch_z<8, 16, 16>(st, data, n_inner, n_in, n_out, spec, fold ? 1 : 0); return true;
        default: return false;
    }
}

}  // namespace lc
