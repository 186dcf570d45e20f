// Column passes of the axis FFT (lines at stride n_inner, no index maps or
// per-index factors) as register-resident Stockham FFTs with compile-time
// radix plans.  These are the y passes of the 3D Toeplitz apply and the y
// pass (FFT, spectral multiply, inverse FFT) of the 2D one.
//
// A CTA transforms kCols adjacent columns.  A line of M = R0 R1 R2 points is
// handled by M / min(R) threads: in every stage a thread keeps its
// butterfly's R elements in registers, and the line crosses shared memory
// twice per transform, in one buffer (no ping-pong).  The global load feeds
// the first stage straight from registers; the last stage feeds the store,
// or the spectral multiply and the inverse transform, whose first stage
// reads exactly the elements the forward transform left in the thread.
//
// Even lengths L = 2M whose input, or output, occupies at most M elements
// run as two transforms of length M (h(n) = exp(sign i pi n / M)):
//   input x[n] = 0 for n >= M:  X[2k] = DFT_M(x)[k],  X[2k+1] = DFT_M(h x)[k]
//   output kept for n < M:       x[n] = DFT_M(X_even)[n] + h(n) DFT_M(X_odd)[n]
// This is the Toeplitz case: the padded length is P >= 2n - 1, the line holds
// n <= P/2 values and the cropped result keeps n.  Both halves go through the
// same thread as two independent instruction streams.
#include <atomic>
#include <cstring>
#include <vector>

#include "lc_fft.hpp"
#include "lc_regfft.cuh"

namespace lc {
namespace {

#ifndef LC_COL_LINES
#define LC_COL_LINES 4
#endif
constexpr int kCols = LC_COL_LINES;  // columns per CTA: 32-byte row segments
static_assert(kCols % 2 == 0, "the twiddle tables after the line buffers need 16-byte alignment");

enum ColMode { CM_PLAIN = 0, CM_PLAIN_MID = 1, CM_SPLIT_IN = 2, CM_SPLIT_OUT = 3, CM_SPLIT_MID = 4 };

struct ColArgs {
    const float2 *in;
    float2 *out;
    long n_inner, in_ostride, out_ostride, bpo;
    int n_in, n_out, sign, sign2;
    const float *spec;
    long spec_ra;
};

template <int MODE>
constexpr int col_nv() { return MODE >= CM_SPLIT_IN ? 2 : 1; }

template <int R0, int R1, int R2, int MODE>
constexpr size_t col_smem() {
    constexpr int M = RegPlan<R0, R1, R2>::M;
    return ((size_t)col_nv<MODE>() * M * kCols + 2 * (size_t)M) * sizeof(float2);
}

// CTAs per SM the register budget is sized for: three for the small CTAs,
// fewer for the long lines (whose threads hold up to 2 x 16 elements)
#ifndef LC_COL_MIN_BLOCKS_SMALL
#define LC_COL_MIN_BLOCKS_SMALL 3  // CTAs per SM for CTAs of up to 352 threads
#endif
template <int R0, int R1, int R2>
constexpr int col_min_blocks() {
    constexpr int t = RegPlan<R0, R1, R2>::NT * kCols;
    return t <= 352 ? LC_COL_MIN_BLOCKS_SMALL : (t <= 448 ? 2 : 1);
}

template <int R0, int R1, int R2, int MODE>
__device__ __forceinline__ void col_fft_body(const ColArgs &a, long bid) {
    using P = RegPlan<R0, R1, R2>;
    constexpr int M = P::M, RM = P::RM, C = kCols;
    constexpr bool SPLIT = MODE >= CM_SPLIT_IN;
    constexpr int NV = col_nv<MODE>();
    extern __shared__ __align__(16) float2 col_sm[];
    float2 *tw = col_sm + NV * M * C;  // exp(-2 pi i m / M)
    float2 *th = tw + M;               // exp(-pi i m / M)
    load_line_twiddles<M>(tw);
    const int c = threadIdx.x % C, t = threadIdx.x / C;
    const long o = bid / a.bpo;
    const long col = (bid - o * a.bpo) * C + c;
    const bool valid = col < a.n_inner;
    const long ni = a.n_inner;
    const float2 *in = a.in + o * a.in_ostride + col;
    float2 *out = a.out + o * a.out_ostride + col;
    const float2 zero = make_float2(0.f, 0.f);

    float2 v[NV][RM];
    constexpr int NA = M / R0;
    if (t < NA) {
#pragma unroll
        for (int r = 0; r < R0; ++r) {
            const int i = t + r * NA;
            if constexpr (MODE == CM_SPLIT_OUT) {
                v[0][r] = (valid && 2 * i < a.n_in) ? in[(long)(2 * i) * ni] : zero;
                v[1][r] = (valid && 2 * i + 1 < a.n_in) ? in[(long)(2 * i + 1) * ni] : zero;
            } else {
                v[0][r] = (valid && i < a.n_in) ? in[(long)i * ni] : zero;
            }
        }
    }
    __syncthreads();  // twiddle tables ready
    if constexpr (MODE == CM_SPLIT_IN || MODE == CM_SPLIT_MID) {
        if (t < NA) {
#pragma unroll
            for (int r = 0; r < R0; ++r) {
                float2 h = th[t + r * NA];
                if (a.sign > 0) h.y = -h.y;
                v[1][r] = cmul(v[0][r], h);
            }
        }
    }
    const auto at = [&](int q, int i) -> float2 & { return col_sm[q * M * C + i * C + c]; };
    xform3<M, R0, R1, R2>(v, at, t, tw, a.sign);
    constexpr int NC = M / R2;
    if constexpr (MODE == CM_PLAIN) {
        if (t < NC && valid) {
#pragma unroll
            for (int r = 0; r < R2; ++r) {
                const int k = t + r * NC;
                if (k < a.n_out) out[(long)k * ni] = v[0][r];
            }
        }
    } else if constexpr (MODE == CM_SPLIT_IN) {
        if (t < NC && valid) {
#pragma unroll
            for (int r = 0; r < R2; ++r) {
                const int k = t + r * NC;
                if (2 * k < a.n_out) out[(long)(2 * k) * ni] = v[0][r];
                if (2 * k + 1 < a.n_out) out[(long)(2 * k + 1) * ni] = v[1][r];
            }
        }
    } else if constexpr (MODE == CM_SPLIT_OUT) {
        if (t < NC && valid) {
#pragma unroll
            for (int r = 0; r < R2; ++r) {
                const int n = t + r * NC;
                if (n < a.n_out) {
                    float2 h = th[n];
                    if (a.sign > 0) h.y = -h.y;
                    out[(long)n * ni] = cadd(v[0][r], cmul(h, v[1][r]));
                }
            }
        }
    } else {
        // spectral multiply (row f of the spectrum scales FFT index f), then
        // the inverse transform with the radices reversed
        if (t < NC) {
            const float *sp = a.spec + (valid ? col : 0);
#pragma unroll
            for (int r = 0; r < R2; ++r) {
                const int k = t + r * NC;
                if constexpr (SPLIT) {
                    const float s0 = valid ? __ldg(sp + (long)(2 * k) * a.spec_ra) : 0.f;
                    const float s1 = valid ? __ldg(sp + (long)(2 * k + 1) * a.spec_ra) : 0.f;
                    v[0][r] = cscale(v[0][r], s0);
                    v[1][r] = cscale(v[1][r], s1);
                } else {
                    const float s0 = valid ? __ldg(sp + (long)k * a.spec_ra) : 0.f;
                    v[0][r] = cscale(v[0][r], s0);
                }
            }
        }
        xform3<M, R2, R1, R0>(v, at, t, tw, a.sign2);
        constexpr int NF = M / R0;
        if (t < NF && valid) {
#pragma unroll
            for (int r = 0; r < R0; ++r) {
                const int n = t + r * NF;
                if (n < a.n_out) {
                    float2 x = v[0][r];
                    if constexpr (SPLIT) {
                        float2 h = th[n];
                        if (a.sign2 > 0) h.y = -h.y;
                        x = cadd(x, cmul(h, v[1][r]));
                    }
                    out[(long)n * ni] = x;
                }
            }
        }
    }
}

template <int R0, int R1, int R2, int MODE>
__global__ void __launch_bounds__(RegPlan<R0, R1, R2>::NT *kCols, (col_min_blocks<R0, R1, R2>()))
    col_fft_kernel(ColArgs a) {
    col_fft_body<R0, R1, R2, MODE>(a, (long)blockIdx.x);
}

// one launch over several column transforms of one plan and mode: CTA b runs
// block b - first_block of the item whose range holds b
struct ColBatchItem {
    ColArgs a;
    long first_block;
    const int *skip;
};

template <int R0, int R1, int R2, int MODE>
__global__ void __launch_bounds__(RegPlan<R0, R1, R2>::NT *kCols, (col_min_blocks<R0, R1, R2>()))
    col_fft_batch_kernel(const ColBatchItem *__restrict__ items, int nitems) {
    const long b = (long)blockIdx.x;
    int lo = 0, hi = nitems - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (items[mid].first_block <= b) lo = mid;
        else hi = mid - 1;
    }
    if (items[lo].skip && *items[lo].skip) return;
    col_fft_body<R0, R1, R2, MODE>(items[lo].a, b - items[lo].first_block);
}

template <int R0, int R1, int R2, int MODE>
void col_batch_configure() {
    LC_CUDA(cudaFuncSetAttribute(col_fft_batch_kernel<R0, R1, R2, MODE>,
                                 cudaFuncAttributeMaxDynamicSharedMemorySize, (int)col_smem<R0, R1, R2, MODE>()));
}

template <int R0, int R1, int R2, int MODE>
void col_batch_launch(cudaStream_t st, const void *items, int n, long blocks) {
    col_fft_batch_kernel<R0, R1, R2, MODE><<<(unsigned)blocks, RegPlan<R0, R1, R2>::NT * kCols,
                                             col_smem<R0, R1, R2, MODE>(), st>>>(
        static_cast<const ColBatchItem *>(items), n);
    LC_CHECK_LAUNCH();
}

template <int R0, int R1, int R2>
void col_batch_fns(int mode, RegBatchKey &k) {
    switch (mode) {
        case CM_PLAIN: k.launch = col_batch_launch<R0, R1, R2, CM_PLAIN>; k.configure = col_batch_configure<R0, R1, R2, CM_PLAIN>; break;
        case CM_PLAIN_MID: k.launch = col_batch_launch<R0, R1, R2, CM_PLAIN_MID>; k.configure = col_batch_configure<R0, R1, R2, CM_PLAIN_MID>; break;
        case CM_SPLIT_IN: k.launch = col_batch_launch<R0, R1, R2, CM_SPLIT_IN>; k.configure = col_batch_configure<R0, R1, R2, CM_SPLIT_IN>; break;
        case CM_SPLIT_OUT: k.launch = col_batch_launch<R0, R1, R2, CM_SPLIT_OUT>; k.configure = col_batch_configure<R0, R1, R2, CM_SPLIT_OUT>; break;
        default: k.launch = col_batch_launch<R0, R1, R2, CM_SPLIT_MID>; k.configure = col_batch_configure<R0, R1, R2, CM_SPLIT_MID>; break;
    }
}

template <int R0, int R1, int R2, int MODE>
void launch_mode(cudaStream_t st, const ColArgs &a, long blocks) {
    constexpr size_t smem = col_smem<R0, R1, R2, MODE>();
    auto kern = col_fft_kernel<R0, R1, R2, MODE>;
    static std::atomic<unsigned long long> configured{0};
    int dev = 0;
    LC_CUDA(cudaGetDevice(&dev));
    const unsigned long long bit = 1ull << (dev & 63);
    if (!(configured.load() & bit)) {
        LC_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        configured.fetch_or(bit);
    }
    kern<<<(unsigned)blocks, RegPlan<R0, R1, R2>::NT * kCols, smem, st>>>(a);
    LC_CHECK_LAUNCH();
}

template <int R0, int R1, int R2>
void launch_plan(cudaStream_t st, int mode, const ColArgs &a, long blocks) {
    switch (mode) {
        case CM_PLAIN: launch_mode<R0, R1, R2, CM_PLAIN>(st, a, blocks); break;
        case CM_PLAIN_MID: launch_mode<R0, R1, R2, CM_PLAIN_MID>(st, a, blocks); break;
        case CM_SPLIT_IN: launch_mode<R0, R1, R2, CM_SPLIT_IN>(st, a, blocks); break;
        case CM_SPLIT_OUT: launch_mode<R0, R1, R2, CM_SPLIT_OUT>(st, a, blocks); break;
        default: launch_mode<R0, R1, R2, CM_SPLIT_MID>(st, a, blocks); break;
    }
}

bool launch_plan_for(cudaStream_t st, int M, int mode, const ColArgs &a, long blocks) {
    switch (M) {
#define LC_COL_CASE(m, r0, r1, r2) \
    case m: launch_plan<r0, r1, r2>(st, mode, a, blocks); return true;
        LC_LINE_PLANS(LC_COL_CASE)
#undef LC_COL_CASE
        default: return false;
    }
}

}  // namespace

// The column plan of a transform: M and the mode, and its arguments; false
// when no register plan covers it.
static bool col_plan_args(const AxisFFT &a, int &M, int &mode, ColArgs &ca) {
    if (a.fp64 || a.in_t != E_C64 || a.out_t != E_C64 || a.n_inner <= 1) return false;
    if (a.in_map != IN_DIRECT) return false;
    if (!(a.out_map == OUT_DIRECT || (a.out_map == OUT_WINDOW && a.out_off == 0))) return false;
    if (a.pre || a.linefac || a.post || a.scale != 1.0 || a.lines_per_cta > 0 || a.mid_fold) return false;
    const int L = a.L;
    if (a.n_in < 0 || a.n_in > L || a.n_out < 0 || a.n_out > L) return false;
    const bool mid = a.mid != nullptr;
    M = L;
    mode = mid ? CM_PLAIN_MID : CM_PLAIN;
    if (L % 2 == 0 && line_plan_exists(L / 2)) {
        const int h = L / 2;
        if (mid && a.n_in <= h && a.n_out <= h) {
            M = h;
            mode = CM_SPLIT_MID;
        } else if (!mid && a.n_in <= h) {
            M = h;
            mode = CM_SPLIT_IN;
        } else if (!mid && a.n_out <= h) {
            M = h;
            mode = CM_SPLIT_OUT;
        }
    }
    if (!line_plan_exists(M)) return false;
    ca.in = static_cast<const float2 *>(a.in);
    ca.out = static_cast<float2 *>(a.out);
    ca.n_inner = a.n_inner;
    ca.in_ostride = a.in_ostride;
    ca.out_ostride = a.out_ostride;
    ca.bpo = (a.n_inner + kCols - 1) / kCols;
    ca.n_in = a.n_in;
    ca.n_out = a.n_out;
    ca.sign = a.sign;
    ca.sign2 = a.sign2;
    ca.spec = a.mid;
    ca.spec_ra = a.mid_ra;
    return true;
}

bool launch_col_fft(cudaStream_t st, const AxisFFT &a) {
    int M = 0, mode = 0;
    ColArgs ca;
    if (!col_plan_args(a, M, mode, ca)) return false;
    if (a.n_outer <= 0 || a.n_out == 0) return true;
    const long blocks = a.n_outer * ca.bpo;
    LC_REQUIRE(blocks < (1L << 31), "column FFT: grid too large");
    return launch_plan_for(st, M, mode, ca, blocks);
}

bool col_batch_item(const AxisFFT &a, const int *skip, long first_block, RegBatchKey &key,
                    std::vector<unsigned char> &item, long &blocks) {
    int M = 0, mode = 0;
    ColArgs ca;
    if (!col_plan_args(a, M, mode, ca)) return false;
    key.kind = 1;
    key.M = M;
    key.mode = mode;
    key.item_size = sizeof(ColBatchItem);
    switch (M) {
#define LC_COL_BATCH_CASE(m, r0, r1, r2) \
    case m: col_batch_fns<r0, r1, r2>(mode, key); break;
        LC_LINE_PLANS(LC_COL_BATCH_CASE)
#undef LC_COL_BATCH_CASE
        default: return false;
    }
    blocks = a.n_outer * ca.bpo;
    ColBatchItem it{ca, first_block, skip};
    item.resize(sizeof it);
    std::memcpy(item.data(), &it, sizeof it);
    return true;
}

}  // namespace lc
