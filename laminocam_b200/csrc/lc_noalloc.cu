// Allocation-free variant of the 2D Toeplitz apply (A^T A of a stack of slices).
//
// Some callers cannot allocate device memory once they are running: an online
// reconstruction embedded in a detector's acquisition loop that reserves the
// whole device for frame buffers up front, or a host framework that forbids
// allocation after start-up because cudaMalloc / cudaFree can synchronise the
// device and stall the data stream.  lc_sysmat2d_toeplitz_noalloc serves them:
// the caller passes the inputs (slices and PSF spectrum) and the output, and
// the intermediate half spectrum lives in a fixed array compiled into this
// library, so the call allocates nothing.
//
// The scratch array (16 MiB) and the twiddle table (32 KiB) below are
// file-scope __device__ arrays: every GPU that loads the library holds them
// until the process exits.  In host code their names are host-side stand-ins,
// not device addresses, so every call looks up their device addresses with
// cudaGetSymbolAddress for the current device and passes those to the
// kernels.  Looking them up per call (a table lookup once the module is
// loaded) keeps the addresses right after a cudaDeviceReset, which unloads
// the module; a per-device cache would keep stale ones.
//
// CUDA loads a library's device code lazily, on its first use on a device,
// and that load is what places the two arrays in device memory.  A caller
// that reserves the whole device must therefore make one call first: the
// set-up call (all pointers NULL, all sizes 0) only loads the module and
// resolves the addresses, and later calls allocate nothing.
#include "../../include/laminocam.h"
#include "lc_fft.hpp"

namespace lc {
namespace {

constexpr long kScratchElems = 2L * 1024 * 1024;  // float2 elements: 16 MiB
constexpr int kMaxP = 4096;                        // longest transform (twiddle table size)

static __device__ __align__(256) float2 g_noalloc_scratch[kScratchElems];
static __device__ __align__(256) float2 g_noalloc_twiddles[kMaxP];

// tw[m] = exp(-2 pi i m / L), evaluated with sincospi in double precision
__global__ void noalloc_twiddle_kernel(float2 *tw, int L) {
    for (int m = blockIdx.x * blockDim.x + threadIdx.x; m < L; m += gridDim.x * blockDim.x) {
        double s, c;
        sincospi(2.0 * (double)m / (double)L, &s, &c);
        tw[m] = make_float2((float)c, (float)-s);
    }
}

bool plan_radices(int L, FFTPlan &pl) { return fft_factorise(L, pl); }

// Device addresses of the static arrays on the current device and its
// shared-memory limit, looked up on every call.
bool resolve_current_device(float2 *&scratch, float2 *&tw, size_t &max_smem) {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return false;
    void *p = nullptr, *q = nullptr;
    if (cudaGetSymbolAddress(&p, g_noalloc_scratch) != cudaSuccess) return false;
    if (cudaGetSymbolAddress(&q, g_noalloc_twiddles) != cudaSuccess) return false;
    int smem = 0;
    if (cudaDeviceGetAttribute(&smem, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev) != cudaSuccess) return false;
    scratch = static_cast<float2 *>(p);
    tw = static_cast<float2 *>(q);
    max_smem = (size_t)smem;
    return true;
}

}  // namespace
}  // namespace lc

using namespace lc;

extern "C" int lc_sysmat2d_toeplitz_noalloc(void *stream, const float *spectrum, int P, const float *x,
                                            float *y, int nslices, int n) {
    float2 *scratch = nullptr, *tw = nullptr;
    size_t max_smem = 0;
    if (!spectrum && !x && !y && nslices == 0 && n == 0 && P == 0)  // set-up call
        return resolve_current_device(scratch, tw, max_smem) ? LC_OK : LC_ERR_CUDA;
    if (!spectrum || !x || !y || nslices <= 0 || n <= 0 || P <= 0) return LC_ERR_INVALID;
    if (P != (int)next_smooth23(2L * n - 1)) return LC_ERR_INVALID;
    const long P3h = P / 2 + 1;
    if (P > kMaxP || (long)nslices * n * P3h > kScratchElems) return LC_ERR_TOO_LARGE;
    FFTPlan pl{};
    if (!plan_radices(P, pl)) return LC_ERR_INVALID;
    if (!resolve_current_device(scratch, tw, max_smem)) return LC_ERR_CUDA;
    cudaStream_t s = (cudaStream_t)stream;
    try {
        noalloc_twiddle_kernel<<<(P + 255) / 256, 256, 0, s>>>(tw, P);
        LC_CHECK_LAUNCH();
        pl.tw = tw;
        // rows: real slices -> half spectrum in the scratch array
        AxisFFT a;
        a.in = x;
        a.in_t = E_F32;
        a.out = scratch;
        a.out_t = E_C64;
        a.n_outer = (long)nslices * n;
        a.n_inner = 1;
        a.in_ostride = n;
        a.out_ostride = P3h;
        a.n_in = n;
        a.L = P;
        a.n_out = (int)P3h;
        a.sign = -1;
        launch_axis_fft_f32_with_plan(s, max_smem, a, pl);
        // columns: forward, multiply by the real spectrum, inverse, keep n rows (in place)
        AxisFFT b;
        b.in = scratch;
        b.in_t = E_C64;
        b.out = scratch;
        b.out_t = E_C64;
        b.n_outer = nslices;
        b.n_inner = P3h;
        b.in_ostride = (long)n * P3h;
        b.out_ostride = (long)n * P3h;
        b.n_in = n;
        b.L = P;
        b.n_out = n;
        b.out_map = OUT_WINDOW;
        b.out_off = 0;
        b.sign = -1;
        b.mid = spectrum;
        b.mid_ra = P3h;
        b.sign2 = +1;
        launch_axis_fft_f32_with_plan(s, max_smem, b, pl);
        // rows: half spectrum -> real, first n samples, scaled as the reference's norm
        AxisFFT c;
        c.in = scratch;
        c.in_t = E_C64;
        c.out = y;
        c.out_t = E_F32;
        c.n_outer = (long)nslices * n;
        c.n_inner = 1;
        c.in_ostride = P3h;
        c.out_ostride = n;
        c.n_in = (int)P3h;
        c.in_map = IN_HERM;
        c.L = P;
        c.n_out = n;
        c.out_map = OUT_WINDOW;
        c.out_off = 0;
        c.sign = +1;
        c.scale = 1.0 / ((double)P * (double)P * (double)n);
        launch_axis_fft_f32_with_plan(s, max_smem, c, pl);
    } catch (const Error &e) {
        return e.code == 1 ? LC_ERR_INVALID : LC_ERR_CUDA;
    }
    return LC_OK;
}
