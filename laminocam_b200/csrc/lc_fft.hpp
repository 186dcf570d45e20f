// Line transforms along one axis of a strided 3D array:
//  * launch_axis_fft: 2^p*3^q shared-memory Stockham FFT with fused zero
//    padding, mode (CMCL) placement/extraction, Hermitian expansion, per-index
//    scale factors (NUFFT deapodisation), an optional spectral multiply between
//    a forward and an inverse transform (Toeplitz), and real or complex output.
//  * launch_axis_dft: direct DFT of arbitrary length with fused circular
//    shifts (fftshift / ifftshift index maps), used for detector-domain
//    transforms whose lengths are odd.
#pragma once

#include <memory>
#include <vector>

#include "lc_cgstate.hpp"
#include "lc_runtime.hpp"

namespace lc {

enum Elem { E_F32 = 0, E_C64 = 1, E_F64 = 2, E_C128 = 3 };  // float, float2, double, double2
enum InMap { IN_DIRECT = 0, IN_MODES = 1, IN_HERM = 2, IN_REAL_PACKED = 3, IN_C2R_PACK = 4 };
enum OutMap { OUT_DIRECT = 0, OUT_MODES = 1, OUT_WINDOW = 2, OUT_R2C_UNPACK = 3, OUT_REAL_UNPACK = 4 };

// Lines are indexed by (o, c), o in [0, n_outer), c in [0, n_inner); element i
// of line (o, c) is at  o*ostride + i*n_inner + c  (input and output alike).
//
// Input maps (element j of the input line -> FFT index f):
//   IN_DIRECT  f = j (j < n_in, zero padded to L)
//   IN_MODES   f = (j - n_in/2) mod L        (mode k = j - floor(n_in/2))
//   IN_HERM    f in [0, L): in[f] for f <= L/2, conj(in[L-f]) otherwise
//              (n_in = L/2 + 1, half spectrum of a real line)
// Output maps (output element j <- FFT index f):
//   OUT_DIRECT f = j; OUT_MODES f = (j - n_out/2) mod L; OUT_WINDOW f = j + out_off
//
// Real lines of even length N = 2L as complex transforms of length L (rows
// only; the usual even/odd packing):
//   IN_REAL_PACKED  z[e] = x[2e] + i x[2e+1] (real input of n_in <= 2L samples)
//   OUT_R2C_UNPACK  X[k] = E[k] + exp(-i pi k / L) O[k], k < n_out <= L+1, with
//                   E = (Z[k] + conj Z[L-k]) / 2 and O = (Z[k] - conj Z[L-k]) / 2i:
//                   the half spectrum of the length-N real DFT
//   IN_C2R_PACK     Z[k] = (X[k] + conj X[L-k]) + i exp(+i pi k / L) (X[k] - conj X[L-k])
//                   from a half spectrum of n_in = L+1 values
//   OUT_REAL_UNPACK out[j] = Re z[j/2] (j even) or Im z[j/2] (j odd), j < n_out <= 2L:
//                   with sign +1 the unnormalised length-N inverse real DFT
struct AxisFFT {
    const void *in = nullptr;
    Elem in_t = E_C64;
    void *out = nullptr;
    Elem out_t = E_C64;
    long n_outer = 1, n_inner = 1;
    long in_ostride = 0, out_ostride = 0;
    int n_in = 0, n_out = 0, L = 0;
    InMap in_map = IN_DIRECT;
    OutMap out_map = OUT_DIRECT;
    int out_off = 0;
    int sign = -1;
    const void *pre = nullptr;      // real factor per input index j
    const void *linefac = nullptr;  // real factor per line inner index c
    const void *post = nullptr;     // real factor per output index j
    double scale = 1.0;
    // spectral multiply between a transform of `sign` and one of `sign2`:
    // the value at FFT index f of line (o, c) is multiplied by mid[f*mid_ra + c]
    const float *mid = nullptr;
    long mid_ra = 0;
    bool mid_fold = false;  // mid holds only f <= L/2; index f > L/2 reads L - f
    int sign2 = +1;
    bool fp64 = false;  // compute precision
    int lines_per_cta = 0;  // 0 = choose automatically
    // CG work fused into a real row pass (row kernels only; see CGFusion):
    // kFusedUpdate on IN_REAL_PACKED rows, whose input is then the direction p;
    // kFusedDot on OUT_REAL_UNPACK rows, whose output is then A p
    const CGFusion *cg = nullptr;
    unsigned cg_parts = 0;
};

// Many FP32 transforms with one element-type pairing (float or float2 in and
// out) as one launch of the generic kernel per shared-memory class (at most
// three: up to 32 KB, 64 KB and more per CTA): each keeps its own length
// (2^p 3^q), plan, index maps, strides, spectral multiply and lines per CTA;
// those of a class share the CTA size and the largest's shared memory.  An
// optional per-transform flag (device int, nonzero = skip) lets finished jobs
// drop out without rebuilding the batch.  add() the transforms, finalize()
// once (uploads the table on the context stream), then launch() as often as
// needed: launch() only launches, so it can be captured into a graph.
class AxisFFTBatch {
  public:
    AxisFFTBatch();
    ~AxisFFTBatch();
    AxisFFTBatch(const AxisFFTBatch &) = delete;
    AxisFFTBatch &operator=(const AxisFFTBatch &) = delete;
    void add(Context &ctx, const AxisFFT &a, const int *skip = nullptr);
    void finalize(Context &ctx);
    void launch(cudaStream_t st) const;
    bool empty() const;
    long blocks() const;

  private:
    struct Impl;
    std::unique_ptr<Impl> impl_;
};

// Which batched register-plan launch a transform takes: kernel kind (1
// column, 2 row), plan length M and mode, and the functions that configure
// and launch that kernel on a device table of items.
struct RegBatchKey {
    int kind = 0, M = 0, mode = 0;
    size_t item_size = 0;
    void (*configure)() = nullptr;
    void (*launch)(cudaStream_t, const void *, int, long) = nullptr;
};
// The batch item of a transform for the register column (row) kernels; false
// when no register plan covers it.  blocks = the CTAs it needs.
bool col_batch_item(const AxisFFT &a, const int *skip, long first_block, RegBatchKey &key,
                    std::vector<unsigned char> &item, long &blocks);
bool row_batch_item(const AxisFFT &a, const int *skip, long first_block, RegBatchKey &key,
                    std::vector<unsigned char> &item, long &blocks);

// Register-plan line transforms (the row and column kernels) of several
// transforms as one launch.  Every transform added must take the same kernel,
// plan and mode: add() returns false, and adds nothing, when no register plan
// covers the transform or it differs from those already added.  No fused CG
// work.  finalize() once, then launch() as often as needed (capturable).
class RegLineBatch {
  public:
    RegLineBatch();
    ~RegLineBatch();
    RegLineBatch(const RegLineBatch &) = delete;
    RegLineBatch &operator=(const RegLineBatch &) = delete;
    bool add(const AxisFFT &a, const int *skip = nullptr);
    void finalize(Context &ctx);
    void launch(cudaStream_t st) const;
    bool empty() const;

  private:
    struct Impl;
    std::unique_ptr<Impl> impl_;
};

// CTAs of a real row pass over n_lines lines (the partials a fused dot needs)
long row_fft_ctas(long n_lines);

void launch_axis_fft(Context &ctx, const AxisFFT &a);

// The Toeplitz z stage in place on `data` (n_inner columns, rows of n_inner
// complex values): zero-pad n_in rows to L, FFT, multiply row f by the real
// spec[f * n_inner + column] (with fold: rows f <= L/2 only, row L - f for
// f > L/2), inverse FFT, keep n_out rows.  Register-resident
// kernels for L in {16, 24, 32, 36, 48, 64, 72, 96, 128}; returns false for
// other lengths (the caller then uses launch_axis_fft).
bool launch_zconv(cudaStream_t st, float2 *data, long n_inner, int L, int n_in, int n_out,
                  const float *spec, bool fold = false);

// The z stage of a Toeplitz kernel that is even in z, as the direct product
// with a real symmetric Toeplitz matrix per column, in place:
//     data[z][c] <- sum_{z' < n} taps[|z - z'|][c] data[z'][c],   z < n,
// taps = the first n planes of the kernel's z-profile per (ky, kx) column
// (times L).  Returns false for n above zdirect_max_rows() (the caller then
// runs the FFT form, launch_zconv).
bool launch_zdirect(cudaStream_t st, float2 *data, long n_inner, int n, const float *taps);
int zdirect_max_rows();
// false when the environment sets LC_ZDIRECT=0 (the FFT form everywhere)
bool zdirect_enabled();

// Column transforms (n_inner > 1) without index maps, per-index factors or
// scale, in FP32 complex, as register-resident kernels with compile-time
// radix plans; even lengths whose input or output fits in half the line run
// as two half-length transforms.  Returns false for shapes without a plan
// (the caller then uses the generic kernel).  launch_axis_fft tries it first.
bool launch_col_fft(cudaStream_t st, const AxisFFT &a);

// Real row passes (n_inner == 1) in the packed forms IN_REAL_PACKED ->
// OUT_R2C_UNPACK (sign -1) and IN_C2R_PACK -> OUT_REAL_UNPACK (sign +1),
// optionally scaled, as register-resident kernels for lengths with a plan.
// Returns false otherwise.  launch_axis_fft tries it first.
bool launch_row_fft(cudaStream_t st, const AxisFFT &a);

// false when LC_LINE_KERNELS=0: every transform then takes the generic
// shared-memory kernel (A/B timing of the register-plan kernels)
bool line_kernels_enabled();

// Same transform with a caller-supplied FP32 plan (radices and twiddle table)
// on an explicit stream; touches no context, plan cache or allocator.
void launch_axis_fft_f32_with_plan(cudaStream_t stream, size_t max_smem, const AxisFFT &a,
                                   const FFTPlan &pl);

struct AxisDFT {
    const void *in = nullptr;
    Elem in_t = E_C64;
    void *out = nullptr;
    Elem out_t = E_C64;
    long n_outer = 1, n_inner = 1;
    long in_ostride = 0, out_ostride = 0;
    int n = 0;
    int d_pre = 0;   // loaded line:  v[m] = in[(m + d_pre) % n]
    int d_post = 0;  // stored line:  out[k] = DFT(v)[(k + d_post) % n]
    int sign = -1;
    float scale = 1.0f;
};

void launch_axis_dft(Context &ctx, const AxisDFT &a);

// Bluestein transforms with complex output whose convolution length is even
// with a register plan for half of it, on the line kernels; false otherwise
// (the generic Bluestein kernel then runs).
bool launch_bluestein_lines(cudaStream_t st, const AxisDFT &a, const BluesteinEntry &e);

}  // namespace lc
