// Real row passes of the axis FFT (the x passes of the Toeplitz apply) as
// register-resident Stockham FFTs with compile-time radix plans.
//
// A real line of N = 2M samples is transformed as one complex line of M
// points (the even/odd packing that the generic kernel implements with
// IN_REAL_PACKED / OUT_R2C_UNPACK and IN_C2R_PACK / OUT_REAL_UNPACK):
//   forward  z[e] = x[2e] + i x[2e+1];  Z = DFT_M(z);
//            X[k] = (Z[k] + conj Z[M-k]) / 2 - (i/2) h(k) (Z[k] - conj Z[M-k]),
//            k = 0..M, h(k) = exp(-i pi k / M)
//   inverse  Z[k] = (X[k] + conj X[M-k]) + i conj h(k) (X[k] - conj X[M-k]),
//            z = DFT_M^+(Z);  x[2e] = Re z[e], x[2e+1] = Im z[e]
// A CTA transforms kRowLines lines of M points on M / min(R) threads each;
// consecutive threads walk consecutive samples of a line, so the loads and
// stores are contiguous.  The line crosses shared memory twice in the
// transform, and once more in the forward unpack (which pairs k with M - k).
#include <atomic>
#include <cstring>
#include <vector>

#include "lc_fft.hpp"
#include "lc_reduce.cuh"
#include "lc_regfft.cuh"

namespace lc {
namespace {

constexpr int kRowLines = 4;

enum RowMode { RM_R2C = 0, RM_C2R = 1 };

struct RowArgs {
    const void *in;
    void *out;
    long n_lines, in_stride, out_stride;
    int n_in, n_out;
    float scale;
    // fused CG work (R2C: direction update of the input; C2R: p . output)
    CGFusion cg;
    int cg_upd, cg_dot;
};

template <int R0, int R1, int R2>
constexpr size_t row_smem() {
    constexpr int M = RegPlan<R0, R1, R2>::M;
    return ((size_t)M * kRowLines + 2 * (size_t)M) * sizeof(float2);
}

// HOOK: the fused CG work of RowArgs (compiled out when unused)
template <int R0, int R1, int R2, int MODE, bool HOOK>
__device__ __forceinline__ void row_fft_body(const RowArgs &a, long bid) {
    using P = RegPlan<R0, R1, R2>;
    constexpr int M = P::M, RM = P::RM, NT = P::NT;
    extern __shared__ __align__(16) float2 row_sm[];
    float2 *tw = row_sm + M * kRowLines;  // exp(-2 pi i m / M)
    float2 *th = tw + M;                  // h(m) = exp(-pi i m / M)
    load_line_twiddles<M>(tw);
    const int t = threadIdx.x % NT, c = threadIdx.x / NT;
    const long line = bid * kRowLines + c;
    const bool valid = line < a.n_lines;
    float2 *buf = row_sm + c * M;
    const auto at = [&](int, int i) -> float2 & { return buf[i]; };
    constexpr int NA = M / R0;
    float2 v[1][RM];
    if constexpr (MODE == RM_R2C) {
        const long lo = (valid ? line : 0) * a.in_stride;
        const float *in = static_cast<const float *>(a.in) + lo;
        // fused direction update p = r + beta p (the input is p)
        const bool upd = HOOK && a.cg_upd && !a.cg.st->done;
        const float beta = upd ? (float)a.cg.st->beta : 0.f;
        if (t < NA) {
#pragma unroll
            for (int r = 0; r < R0; ++r) {
                const int e = t + r * NA;
                float re = (valid && 2 * e < a.n_in) ? in[2 * e] : 0.f;
                float im = (valid && 2 * e + 1 < a.n_in) ? in[2 * e + 1] : 0.f;
                if (upd && valid) {
                    if (2 * e < a.n_in) {
                        re = fmaf(beta, re, a.cg.r[lo + 2 * e]);
                        a.cg.p[lo + 2 * e] = re;
                    }
                    if (2 * e + 1 < a.n_in) {
                        im = fmaf(beta, im, a.cg.r[lo + 2 * e + 1]);
                        a.cg.p[lo + 2 * e + 1] = im;
                    }
                }
                v[0][r] = make_float2(re, im);
            }
        }
        __syncthreads();  // twiddle tables ready
        xform3<M, R0, R1, R2>(v, at, t, tw, -1);
        constexpr int NC = M / R2;
        __syncthreads();  // the last stage's reads are done
        if (t < NC) {
#pragma unroll
            for (int r = 0; r < R2; ++r) buf[t + r * NC] = v[0][r];
        }
        __syncthreads();
        if (valid) {
            float2 *out = static_cast<float2 *>(a.out) + line * a.out_stride;
            for (int k = t; k < a.n_out; k += NT) {
                const float2 za = buf[k == M ? 0 : k];
                const float2 zb = buf[k == 0 ? 0 : M - k];
                const float2 sm = make_float2(0.5f * (za.x + zb.x), 0.5f * (za.y - zb.y));
                const float2 df = make_float2(0.5f * (za.x - zb.x), 0.5f * (za.y + zb.y));
                const float2 wd = cmul(k == M ? make_float2(-1.f, 0.f) : th[k], df);
                out[k] = make_float2(a.scale * (sm.x + wd.y), a.scale * (sm.y - wd.x));
            }
        }
    } else {
        const float2 *in = static_cast<const float2 *>(a.in) + (valid ? line : 0) * a.in_stride;
        float2 xb[RM];
        if (t < NA) {
#pragma unroll
            for (int r = 0; r < R0; ++r) {
                const int k = t + r * NA;
                v[0][r] = valid ? in[k] : make_float2(0.f, 0.f);
                xb[r] = valid ? in[M - k] : make_float2(0.f, 0.f);
            }
        }
        __syncthreads();  // twiddle tables ready
        if (t < NA) {
#pragma unroll
            for (int r = 0; r < R0; ++r) {
                const int k = t + r * NA;
                const float2 xa = v[0][r];
                const float2 sm = make_float2(xa.x + xb[r].x, xa.y - xb[r].y);
                const float2 df = make_float2(xa.x - xb[r].x, xa.y + xb[r].y);
                const float2 h = th[k];
                const float2 wd = cmul(make_float2(h.x, -h.y), df);
                v[0][r] = make_float2(sm.x - wd.y, sm.y + wd.x);
            }
        }
        xform3<M, R0, R1, R2>(v, at, t, tw, +1);
        constexpr int NC = M / R2;
        const bool dot = HOOK && a.cg_dot && !a.cg.st->done;  // uniform over the grid
        float accf = 0.f;
        double accd = 0.0;
        if (t < NC && valid) {
            const long lo = line * a.out_stride;
            float *out = static_cast<float *>(a.out) + lo;
#pragma unroll
            for (int r = 0; r < R2; ++r) {
                const int e = t + r * NC;
                const float y0 = a.scale * v[0][r].x, y1 = a.scale * v[0][r].y;
                if (2 * e < a.n_out) {
                    out[2 * e] = y0;
                    if constexpr (HOOK) if (dot) {
                        const float pv = a.cg.p[lo + 2 * e];
                        accf += pv * y0;
                        accd += (double)pv * (double)y0;
                    }
                }
                if (2 * e + 1 < a.n_out) {
                    out[2 * e + 1] = y1;
                    if constexpr (HOOK) if (dot) {
                        const float pv = a.cg.p[lo + 2 * e + 1];
                        accf += pv * y1;
                        accd += (double)pv * (double)y1;
                    }
                }
            }
        }
        if constexpr (HOOK) if (dot) {
            // p.Ap over the transform's blocks (all of the grid in a plain
            // launch, the item's blocks in a batched one), then alpha and the
            // |p.Ap| stop (as the CG dot kernel)
            const long nblk = (a.n_lines + kRowLines - 1) / kRowLines;
            double pap = 0.0;
            bool last;
            if (a.cg.fp32) {
                float vv[1] = {accf};
                last = red_block_partials_at<float, 1>(vv, a.cg.part, a.cg.counter, bid, nblk);
                if (last) pap = red_total<float>(a.cg.part, 0, (int)nblk);
            } else {
                double vv[1] = {accd};
                last = red_block_partials_at<double, 1>(vv, a.cg.part, a.cg.counter, bid, nblk);
                if (last) pap = red_total<double>(a.cg.part, 0, (int)nblk);
            }
            if (last && threadIdx.x == 0) {
                CGState *st = a.cg.st;
                st->pAp = pap;
                if (fabs(pap) < 1e-10) {
                    st->done = 1;
                    st->reason = 3;
                } else {
                    st->alpha = a.cg.fp32 ? (double)((float)st->rs_old / (float)pap) : st->rs_old / pap;
                }
                *a.cg.counter = 0;
            }
        }
    }
}

template <int R0, int R1, int R2, int MODE, bool HOOK>
__global__ void __launch_bounds__(RegPlan<R0, R1, R2>::NT *kRowLines) row_fft_kernel(RowArgs a) {
    row_fft_body<R0, R1, R2, MODE, HOOK>(a, (long)blockIdx.x);
}

// one launch over several row transforms of one plan and mode: CTA b runs
// block b - first_block of the item whose range holds b, with the item's
// fused CG work (its partials and ticket are the item's own)
struct RowBatchItem {
    RowArgs a;
    long first_block;
    const int *skip;
};

template <int R0, int R1, int R2, int MODE>
__global__ void __launch_bounds__(RegPlan<R0, R1, R2>::NT *kRowLines)
    row_fft_batch_kernel(const RowBatchItem *__restrict__ items, int nitems) {
    const long b = (long)blockIdx.x;
    int lo = 0, hi = nitems - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (items[mid].first_block <= b) lo = mid;
        else hi = mid - 1;
    }
    if (items[lo].skip && *items[lo].skip) return;
    row_fft_body<R0, R1, R2, MODE, true>(items[lo].a, b - items[lo].first_block);
}

template <int R0, int R1, int R2, int MODE>
void row_batch_configure() {
    LC_CUDA(cudaFuncSetAttribute(row_fft_batch_kernel<R0, R1, R2, MODE>,
                                 cudaFuncAttributeMaxDynamicSharedMemorySize, (int)row_smem<R0, R1, R2>()));
}

template <int R0, int R1, int R2, int MODE>
void row_batch_launch(cudaStream_t st, const void *items, int n, long blocks) {
    row_fft_batch_kernel<R0, R1, R2, MODE><<<(unsigned)blocks, RegPlan<R0, R1, R2>::NT * kRowLines,
                                             row_smem<R0, R1, R2>(), st>>>(
        static_cast<const RowBatchItem *>(items), n);
    LC_CHECK_LAUNCH();
}

template <int R0, int R1, int R2, int MODE, bool HOOK>
void launch_row_mode(cudaStream_t st, const RowArgs &a, long blocks) {
    constexpr size_t smem = row_smem<R0, R1, R2>();
    auto kern = row_fft_kernel<R0, R1, R2, MODE, HOOK>;
    static std::atomic<unsigned long long> configured{0};
    int dev = 0;
    LC_CUDA(cudaGetDevice(&dev));
    const unsigned long long bit = 1ull << (dev & 63);
    if (!(configured.load() & bit)) {
        LC_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        configured.fetch_or(bit);
    }
    kern<<<(unsigned)blocks, RegPlan<R0, R1, R2>::NT * kRowLines, smem, st>>>(a);
    LC_CHECK_LAUNCH();
}

bool launch_row_plan(cudaStream_t st, int M, int mode, const RowArgs &a, long blocks) {
    switch (M) {
#define LC_ROW_CASE(m, r0, r1, r2)                                                      \
    case m:                                                                             \
        if (mode == RM_R2C) {                                                           \
            if (a.cg_upd) launch_row_mode<r0, r1, r2, RM_R2C, true>(st, a, blocks);     \
            else launch_row_mode<r0, r1, r2, RM_R2C, false>(st, a, blocks);             \
        } else {                                                                        \
            if (a.cg_dot) launch_row_mode<r0, r1, r2, RM_C2R, true>(st, a, blocks);     \
            else launch_row_mode<r0, r1, r2, RM_C2R, false>(st, a, blocks);             \
        }                                                                               \
        return true;
        LC_LINE_PLANS(LC_ROW_CASE)
#undef LC_ROW_CASE
        default: return false;
    }
}

}  // namespace

long row_fft_ctas(long n_lines) { return (n_lines + kRowLines - 1) / kRowLines; }

// The row plan of a transform (M, mode) and its arguments; false when no
// register plan covers it.
static bool row_plan_args(const AxisFFT &a, int &M, int &mode, RowArgs &ra) {
    if (a.fp64 || a.n_inner != 1 || a.lines_per_cta > 0) return false;
    if (a.pre || a.linefac || a.post) return false;
    M = a.L;
    if (a.in_map == IN_REAL_PACKED && a.out_map == OUT_R2C_UNPACK && a.in_t == E_F32 && a.out_t == E_C64 &&
        a.sign < 0 && a.n_in <= 2 * M && a.n_out <= M + 1) {
        mode = RM_R2C;
    } else if (a.in_map == IN_C2R_PACK && a.out_map == OUT_REAL_UNPACK && a.in_t == E_C64 &&
               a.out_t == E_F32 && a.sign > 0 && a.n_in == M + 1 && a.n_out <= 2 * M) {
        mode = RM_C2R;
    } else {
        return false;
    }
    if (!line_plan_exists(M)) return false;
    ra.in = a.in;
    ra.out = a.out;
    ra.n_lines = a.n_outer;
    ra.in_stride = a.in_ostride;
    ra.out_stride = a.out_ostride;
    ra.n_in = a.n_in;
    ra.n_out = a.n_out;
    ra.scale = (float)a.scale;
    ra.cg_upd = ra.cg_dot = 0;
    return true;
}

bool launch_row_fft(cudaStream_t st, const AxisFFT &a) {
    int M = 0, mode = 0;
    RowArgs ra;
    if (!row_plan_args(a, M, mode, ra)) return false;
    if (a.n_outer <= 0 || a.n_out == 0) return true;
    if (a.cg_parts) {
        LC_REQUIRE(a.cg != nullptr, "row FFT: fused CG work without its state");
        ra.cg = *a.cg;
        ra.cg_upd = (mode == RM_R2C && (a.cg_parts & kFusedUpdate)) ? 1 : 0;
        ra.cg_dot = (mode == RM_C2R && (a.cg_parts & kFusedDot)) ? 1 : 0;
    }
    const long blocks = (a.n_outer + kRowLines - 1) / kRowLines;
    LC_REQUIRE(blocks < (1L << 31), "row FFT: grid too large");
    return launch_row_plan(st, M, mode, ra, blocks);
}

bool row_batch_item(const AxisFFT &a, const int *skip, long first_block, RegBatchKey &key,
                    std::vector<unsigned char> &item, long &blocks) {
    int M = 0, mode = 0;
    RowArgs ra;
    if (!row_plan_args(a, M, mode, ra)) return false;
    if (a.cg_parts) {
        LC_REQUIRE(a.cg != nullptr, "row FFT: fused CG work without its state");
        ra.cg = *a.cg;
        ra.cg_upd = (mode == RM_R2C && (a.cg_parts & kFusedUpdate)) ? 1 : 0;
        ra.cg_dot = (mode == RM_C2R && (a.cg_parts & kFusedDot)) ? 1 : 0;
    }
    key.kind = 2;
    key.M = M;
    key.mode = mode;
    key.item_size = sizeof(RowBatchItem);
    switch (M) {
#define LC_ROW_BATCH_CASE(m, r0, r1, r2)                                   \
    case m:                                                                \
        if (mode == RM_R2C) {                                              \
            key.launch = row_batch_launch<r0, r1, r2, RM_R2C>;             \
            key.configure = row_batch_configure<r0, r1, r2, RM_R2C>;       \
        } else {                                                           \
            key.launch = row_batch_launch<r0, r1, r2, RM_C2R>;             \
            key.configure = row_batch_configure<r0, r1, r2, RM_C2R>;       \
        }                                                                  \
        break;
        LC_LINE_PLANS(LC_ROW_BATCH_CASE)
#undef LC_ROW_BATCH_CASE
        default: return false;
    }
    blocks = (a.n_outer + kRowLines - 1) / kRowLines;
    RowBatchItem it{ra, first_block, skip};
    item.resize(sizeof it);
    std::memcpy(item.data(), &it, sizeof it);
    return true;
}

}  // namespace lc
