// Detector-domain DFTs of odd length n by Bluestein's chirp-z convolution on
// the register-plan line kernels.
//
//   X[k] = chirp[k] * sum_j (x[j] chirp[j]) conj(chirp[k - j])
// is a convolution of length L = next 2^p 3^q >= 2n - 1, done as FFT, a
// multiply by the precomputed spectrum V of the chirp kernel, and an inverse
// FFT.  L is even here, and both the padded input and the kept output fit in
// the first M = L/2 points (n <= M), so each of the two transforms runs as
// two transforms of length M in one thread (the even/odd split of the column
// kernels):
//   forward  X[2k] = DFT_M(a)[k],  X[2k+1] = DFT_M(h a)[k],   h(j) = exp(-i pi j / M)
//   inverse  c[j] = DFT+_M(Y_even)[j] + conj h(j) DFT+_M(Y_odd)[j]
// The fftshift/ifftshift rolls are index maps at the load and the store
// (value j of the line is in[(j + d_pre) mod n]; out[k] = X[(k + d_post) mod n]).
// A CTA takes 4 lines: adjacent rows (contiguous lines) or 4 adjacent columns
// (32-byte row segments).  Real rows go two to a line: rows a and b are
// transformed as the complex line a + i b, whose DFT Z gives
//   A[k] = (Z[k] + conj Z[n-k]) / 2,   B[k] = (Z[k] - conj Z[n-k]) / (2i)
// (the DFT of a real sequence is Hermitian), paired through shared memory.
#include <atomic>
#include <type_traits>

#include "lc_fft.hpp"
#include "lc_regfft.cuh"

namespace lc {
namespace {

constexpr int kBlueLines = 4;

struct BlueArgs {
    const void *in;
    float2 *out;
    long n_outer, n_inner, in_ostride, out_ostride, bpo;
    int n, d_pre, d_post;
    float scale;
    const float2 *chirp, *V;
};

template <int R0, int R1, int R2>
constexpr size_t blue_smem() {
    constexpr int M = RegPlan<R0, R1, R2>::M;
    return (2 * (size_t)M * kBlueLines + 2 * (size_t)M) * sizeof(float2);
}

template <typename TI>
__device__ __forceinline__ float2 load_c(const TI *p) {
    if constexpr (std::is_same_v<TI, float>) return make_float2(*p, 0.f);
    else return *p;
}

template <int R0, int R1, int R2, bool ROWS, typename TI>
__global__ void __launch_bounds__(RegPlan<R0, R1, R2>::NT *kBlueLines) blue_kernel(BlueArgs a) {
    using P = RegPlan<R0, R1, R2>;
    constexpr int M = P::M, RM = P::RM, NT = P::NT, C = kBlueLines;
    extern __shared__ __align__(16) float2 blue_sm[];
    float2 *tw = blue_sm + 2 * M * C;  // exp(-2 pi i m / M)
    float2 *th = tw + M;               // exp(-pi i m / M)
    load_line_twiddles<M>(tw);
    // ROWS: thread (c, t) with t fastest (contiguous samples); columns: (t, c)
    // with c fastest (adjacent columns)
    const int t = ROWS ? (int)threadIdx.x % NT : (int)threadIdx.x / C;
    const int c = ROWS ? (int)threadIdx.x / NT : (int)threadIdx.x % C;
    // real rows, two to a line (rows 2 line and 2 line + 1)
    constexpr bool PACK = ROWS && std::is_same_v<TI, float>;
    long base_in, base_out, step;
    bool valid, valid_b = false;
    if constexpr (PACK) {
        const long line = (long)blockIdx.x * C + c;
        valid = 2 * line < a.n_outer;
        valid_b = 2 * line + 1 < a.n_outer;
        base_in = (valid ? 2 * line : 0) * a.in_ostride;
        base_out = (valid ? 2 * line : 0) * a.out_ostride;
        step = 1;
    } else if constexpr (ROWS) {
        const long line = (long)blockIdx.x * C + c;
        valid = line < a.n_outer;
        base_in = (valid ? line : 0) * a.in_ostride;
        base_out = (valid ? line : 0) * a.out_ostride;
        step = 1;
    } else {
        const long o = (long)blockIdx.x / a.bpo;
        const long col = ((long)blockIdx.x - o * a.bpo) * C + c;
        valid = col < a.n_inner;
        base_in = o * a.in_ostride + (valid ? col : 0);
        base_out = o * a.out_ostride + (valid ? col : 0);
        step = a.n_inner;
    }
    const TI *in = static_cast<const TI *>(a.in) + base_in;
    const auto at = [&](int q, int i) -> float2 & {
        return ROWS ? blue_sm[q * M * C + c * M + i] : blue_sm[q * M * C + i * C + c];
    };
    float2 v[2][RM];
    constexpr int NA = M / R0;
    if (t < NA) {
#pragma unroll
        for (int r = 0; r < R0; ++r) {
            const int j = t + r * NA;
            float2 x = make_float2(0.f, 0.f);
            if (valid && j < a.n) {
                int s = j + a.d_pre;
                if (s >= a.n) s -= a.n;
                if constexpr (PACK) {
                    const float xa = static_cast<const float *>(a.in)[base_in + s];
                    const float xb = valid_b ? static_cast<const float *>(a.in)[base_in + a.in_ostride + s] : 0.f;
                    x = cmul(make_float2(xa, xb), __ldg(a.chirp + j));
                } else {
                    x = cmul(load_c<TI>(in + (long)s * step), __ldg(a.chirp + j));
                }
            }
            v[0][r] = x;
        }
    }
    __syncthreads();  // twiddle tables ready
    if (t < NA) {
#pragma unroll
        for (int r = 0; r < R0; ++r) v[1][r] = cmul(v[0][r], th[t + r * NA]);
    }
    xform3<M, R0, R1, R2>(v, at, t, tw, -1);
    constexpr int NC = M / R2;
    if (t < NC) {
#pragma unroll
        for (int r = 0; r < R2; ++r) {
            const int k = t + r * NC;
            v[0][r] = cmul(v[0][r], __ldg(a.V + 2 * k));
            v[1][r] = cmul(v[1][r], __ldg(a.V + 2 * k + 1));
        }
    }
    xform3<M, R2, R1, R0>(v, at, t, tw, +1);
    constexpr int NF = M / R0;
    if constexpr (PACK) {
        // Z[q] of the line into its shared-memory row, then the two rows'
        // values from the pairs (q, n - q)
        __syncthreads();  // the transform's last shared-memory reads are done
        if (t < NF) {
#pragma unroll
            for (int r = 0; r < R0; ++r) {
                const int q = t + r * NF;
                if (q < a.n) {
                    const float2 h = th[q];
                    const float2 y = cadd(v[0][r], cmul(make_float2(h.x, -h.y), v[1][r]));
                    at(0, q) = cscale(cmul(y, __ldg(a.chirp + q)), 0.5f * a.scale);
                }
            }
        }
        __syncthreads();
        if (t < NF && valid) {
#pragma unroll
            for (int r = 0; r < R0; ++r) {
                const int q = t + r * NF;
                if (q < a.n) {
                    const float2 zq = at(0, q), zm = at(0, q == 0 ? 0 : a.n - q);
                    int k = q - a.d_post;
                    if (k < 0) k += a.n;
                    a.out[base_out + k] = make_float2(zq.x + zm.x, zq.y - zm.y);
                    if (valid_b) a.out[base_out + a.out_ostride + k] = make_float2(zq.y + zm.y, zm.x - zq.x);
                }
            }
        }
        return;
    }
    if (t < NF && valid) {
#pragma unroll
        for (int r = 0; r < R0; ++r) {
            const int q = t + r * NF;
            if (q < a.n) {
                const float2 h = th[q];
                const float2 y = cadd(v[0][r], cmul(make_float2(h.x, -h.y), v[1][r]));
                int k = q - a.d_post;
                if (k < 0) k += a.n;
                a.out[base_out + (long)k * step] = cscale(cmul(y, __ldg(a.chirp + q)), a.scale);
            }
        }
    }
}

template <int R0, int R1, int R2, bool ROWS, typename TI>
void launch_blue_t(cudaStream_t st, const BlueArgs &a, long blocks) {
    constexpr size_t smem = blue_smem<R0, R1, R2>();
    auto kern = blue_kernel<R0, R1, R2, ROWS, TI>;
    static std::atomic<unsigned long long> configured{0};
    int dev = 0;
    LC_CUDA(cudaGetDevice(&dev));
    const unsigned long long bit = 1ull << (dev & 63);
    if (!(configured.load() & bit)) {
        LC_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        configured.fetch_or(bit);
    }
    kern<<<(unsigned)blocks, RegPlan<R0, R1, R2>::NT * kBlueLines, smem, st>>>(a);
    LC_CHECK_LAUNCH();
}

template <int R0, int R1, int R2>
void launch_blue_plan(cudaStream_t st, bool rows, bool in_real, const BlueArgs &a, long blocks) {
    if (rows && in_real) launch_blue_t<R0, R1, R2, true, float>(st, a, blocks);
    else if (rows) launch_blue_t<R0, R1, R2, true, float2>(st, a, blocks);
    else if (in_real) launch_blue_t<R0, R1, R2, false, float>(st, a, blocks);
    else launch_blue_t<R0, R1, R2, false, float2>(st, a, blocks);
}

}  // namespace

bool launch_bluestein_lines(cudaStream_t st, const AxisDFT &a, const BluesteinEntry &e) {
    if (a.out_t != E_C64 || e.L % 2 != 0 || a.n > e.L / 2) return false;
    const int M = e.L / 2;
    if (!line_plan_exists(M)) return false;
    if (a.n_outer <= 0 || a.n_inner <= 0) return true;
    BlueArgs b{};
    b.in = a.in;
    b.out = static_cast<float2 *>(a.out);
    b.n_outer = a.n_outer;
    b.n_inner = a.n_inner;
    b.in_ostride = a.in_ostride;
    b.out_ostride = a.out_ostride;
    b.n = a.n;
    b.d_pre = ((a.d_pre % a.n) + a.n) % a.n;
    b.d_post = ((a.d_post % a.n) + a.n) % a.n;
    b.scale = a.scale;
    b.chirp = e.chirp.get();
    b.V = e.V.get();
    const bool rows = a.n_inner == 1;
    long blocks;
    if (rows) {
        // real rows go two to a line
        const long lines = a.in_t == E_F32 ? (a.n_outer + 1) / 2 : a.n_outer;
        blocks = (lines + kBlueLines - 1) / kBlueLines;
        b.bpo = 1;
    } else {
        b.bpo = (a.n_inner + kBlueLines - 1) / kBlueLines;
        blocks = a.n_outer * b.bpo;
    }
    LC_REQUIRE(blocks < (1L << 31), "DFT: grid too large");
    const bool in_real = a.in_t == E_F32;
    switch (M) {
#define LC_BLUE_CASE(m, r0, r1, r2) \
    case m: launch_blue_plan<r0, r1, r2>(st, rows, in_real, b, blocks); return true;
        LC_LINE_PLANS(LC_BLUE_CASE)
#undef LC_BLUE_CASE
        default: return false;
    }
}

}  // namespace lc
