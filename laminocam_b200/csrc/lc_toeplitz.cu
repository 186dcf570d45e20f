// PSF generation (closed form, FP64) and the fused-FFT Toeplitz apply.
#include <algorithm>

#include "lc_toeplitz.hpp"

namespace lc {

namespace {

constexpr double kPiD = 3.14159265358979323846;

// sum_{m=0}^{n-1} exp(i u (2 pi/n)(m - (n-1)/2)) = sin(pi u) / sin(pi u / n)
__device__ __forceinline__ double dirichlet(double u, int n) {
    double v = u / (double)n;
    double sv = sinpi(v);
    if (fabs(sv) < 1e-13) {
        // u/n is (numerically) an integer: limit n cos(pi u) / cos(pi u / n)
        return (double)n * cospi(u) / cospi(v);
    }
    return sinpi(u) / sv;
}

// K[ky][kx] over modes k = j - P/2, 2D polar grid: sum_theta D_nr(kx c + ky s)
__global__ void psf2d_kernel(const double2 *__restrict__ cs, int ntheta, int nr, int P2, int P3,
                             double *__restrict__ K) {
    long total = (long)P2 * P3;
    for (long idx = (long)blockIdx.x * blockDim.x + threadIdx.x; idx < total;
         idx += (long)gridDim.x * blockDim.x) {
        int jy = (int)(idx / P3), jx = (int)(idx - (long)jy * P3);
        double kx = (double)(jx - P3 / 2), ky = (double)(jy - P2 / 2);
        double s = 0.0;
        for (int i = 0; i < ntheta; ++i) {
            double2 t = cs[i];
            s += dirichlet(kx * t.x + ky * t.y, nr);
        }
        K[idx] = s;
    }
}

// K[kz][ky][kx], 3D rotated detector lattice:
// sum_theta D_ncols(uX) D_nrows(uY), uX = R00 kx + R10 ky + R20 kz, uY = R01 kx + R11 ky + R21 kz
__global__ void psf3d_kernel(const double *__restrict__ rot, int ntheta, int nrows, int ncols,
                             int P1, int P2, int P3, double *__restrict__ K) {
    extern __shared__ double srot[];
    for (int i = threadIdx.x; i < 6 * ntheta; i += blockDim.x) srot[i] = rot[i];
    __syncthreads();
    long total = (long)P1 * P2 * P3;
    for (long idx = (long)blockIdx.x * blockDim.x + threadIdx.x; idx < total;
         idx += (long)gridDim.x * blockDim.x) {
        int jz = (int)(idx / ((long)P2 * P3));
        long r = idx - (long)jz * P2 * P3;
        int jy = (int)(r / P3), jx = (int)(r - (long)jy * P3);
        double kx = (double)(jx - P3 / 2), ky = (double)(jy - P2 / 2), kz = (double)(jz - P1 / 2);
        double s = 0.0;
        for (int i = 0; i < ntheta; ++i) {
            const double *R = srot + 6 * i;
            double uX = R[0] * kx + R[2] * ky + R[4] * kz;
            double uY = R[1] * kx + R[3] * ky + R[5] * kz;
            s += dirichlet(uX, ncols) * dirichlet(uY, nrows);
        }
        K[idx] = s;
    }
}

// Zero the planes of mode -P/2 (index 0 in mode order) along every axis of even
// length.  Their values are never reached by the cropped convolution
// (|i - j| <= n - 1 < P/2), and without them the zero-centred kernel is
// exactly point-symmetric, so its spectrum is real.
__global__ void zero_unpaired_kernel(double *__restrict__ K, int P1, int P2, int P3) {
    long total = (long)P1 * P2 * P3;
    for (long idx = (long)blockIdx.x * blockDim.x + threadIdx.x; idx < total;
         idx += (long)gridDim.x * blockDim.x) {
        int jz = (int)(idx / ((long)P2 * P3));
        long r = idx - (long)jz * P2 * P3;
        int jy = (int)(r / P3), jx = (int)(r - (long)jy * P3);
        if ((P1 % 2 == 0 && jz == 0) || (P2 % 2 == 0 && jy == 0) || (P3 % 2 == 0 && jx == 0))
            K[idx] = 0.0;
    }
}

__global__ void d2f_kernel(const double *__restrict__ in, float *__restrict__ out, long n) {
    for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x)
        out[i] = (float)in[i];
}

// y += mu * (-laplacian(x)) with the zero-padded central-difference gradient and
// divergence of the reference GPU build (src/gpu/finitediff.cu:28-222):
// per axis  lap_a(x)[i] = 0.5*(g[i+1] - g[i-1]),  g[k] = 0.5*(x[k+1] - x[k-1]),
// g = 0 outside the volume and x = 0 outside the volume.
__global__ void neg_lap_axpy_kernel(const float *__restrict__ x, float *__restrict__ y, long n1,
                                    long n2, long n3, float mu) {
    long total = n1 * n2 * n3;
    for (long idx = (long)blockIdx.x * blockDim.x + threadIdx.x; idx < total;
         idx += (long)gridDim.x * blockDim.x) {
        long i = idx / (n2 * n3);
        long r = idx - i * n2 * n3;
        long j = r / n3, k = r - j * n3;
        float c = x[idx];
        float lap = 0.f;
        // axis k (n3), stride 1
        {
            float p2 = (k + 2 < n3) ? x[idx + 2] : 0.f;
            float m2 = (k - 2 >= 0) ? x[idx - 2] : 0.f;
            float gp = (k + 1 < n3) ? 0.5f * (p2 - c) : 0.f;
            float gm = (k - 1 >= 0) ? 0.5f * (c - m2) : 0.f;
            lap += 0.5f * (gp - gm);
        }
        {
            long s = n3;
            float p2 = (j + 2 < n2) ? x[idx + 2 * s] : 0.f;
            float m2 = (j - 2 >= 0) ? x[idx - 2 * s] : 0.f;
            float gp = (j + 1 < n2) ? 0.5f * (p2 - c) : 0.f;
            float gm = (j - 1 >= 0) ? 0.5f * (c - m2) : 0.f;
            lap += 0.5f * (gp - gm);
        }
        {
            long s = n2 * n3;
            float p2 = (i + 2 < n1) ? x[idx + 2 * s] : 0.f;
            float m2 = (i - 2 >= 0) ? x[idx - 2 * s] : 0.f;
            float gp = (i + 1 < n1) ? 0.5f * (p2 - c) : 0.f;
            float gm = (i - 1 >= 0) ? 0.5f * (c - m2) : 0.f;
            lap += 0.5f * (gp - gm);
        }
        y[idx] = fmaf(-mu, lap, y[idx]);
    }
}

inline unsigned grid_for(long n, int threads, int sms) {
    long b = (n + threads - 1) / threads;
    return (unsigned)std::max<long>(1, std::min<long>(b, (long)sms * 32));
}

}  // namespace

void launch_neg_laplacian_axpy(Context &ctx, const float *x, float *y, const long dims[3], float mu) {
    long n = dims[0] * dims[1] * dims[2];
    ProfScope ps(ctx, PS_NEG_LAP, 12.0 * n);
    neg_lap_axpy_kernel<<<grid_for(n, 256, ctx.num_sms()), 256, 0, ctx.stream()>>>(
        x, y, dims[0], dims[1], dims[2], mu);
    LC_CHECK_LAUNCH();
}

static int next_fast_dim(long n) { return (int)next_smooth23(n); }

Toeplitz::Toeplitz(Context &ctx, const PolarGeometry &g, const long dims[3], bool three_d)
    : three_d_(three_d), g_(&g) {
    for (int d = 0; d < 3; ++d) n_[d] = dims[d];
    LC_REQUIRE(n_[0] > 0 && n_[1] > 0 && n_[2] > 0, "Toeplitz: dims must be positive");
    if (three_d) {
        LC_REQUIRE(g.pts.dim == 3, "Toeplitz3D needs a 3D geometry");
        for (int d = 0; d < 3; ++d) P_[d] = next_fast_dim(2 * n_[d] - 1);
        for (int d = 0; d < 3; ++d) Ph_[d] = P_[d] / 2 + 1;
        scale_ = 1.0 / ((double)P_[0] * P_[1] * P_[2] * (double)n_[1] * (double)n_[2]);
    } else {
        LC_REQUIRE(g.pts.dim == 2, "Toeplitz2D needs a 2D geometry");
        P_[0] = 1;
        P_[1] = P_[2] = next_fast_dim(2 * n_[2] - 1);
        Ph_[0] = 1;
        Ph_[1] = Ph_[2] = P_[2] / 2 + 1;
        scale_ = 1.0 / ((double)P_[1] * P_[2] * (double)n_[2]);
    }
    cudaStream_t st = ctx.stream();
    DevBuf<double> K;
    build_kernel(ctx, K);
    {
        long total = (long)P_[0] * P_[1] * P_[2];
        zero_unpaired_kernel<<<grid_for(total, 256, ctx.num_sms()), 256, 0, st>>>(K.get(), P_[0], P_[1],
                                                                                  P_[2]);
        LC_CHECK_LAUNCH();
    }
    // Spectrum of the zero-centred kernel: FFT with the mode placement k -> k mod P.
    // It is real and point-symmetric; keep x in [0, P3/2] (the R2C half) and all
    // of y and z, i.e. a real {P1, P2, P3/2+1} array.
    ProfScope ps(ctx, PS_PSF_FFT, 0.0);
    DevBuf<double2> a, b;
    DevBuf<double> Rd(spectrum_elems(), st);
    const int P1 = P_[0], P2 = P_[1], P3 = P_[2], P3h = Ph_[2];
    a.alloc((long)P1 * P2 * P3h, st);
    {
        AxisFFT x;
        x.in = K.get();
        x.in_t = E_F64;
        x.out = a.get();
        x.out_t = E_C128;
        x.fp64 = true;
        x.n_outer = (long)P1 * P2;
        x.n_inner = 1;
        x.in_ostride = P3;
        x.out_ostride = P3h;
        x.n_in = P3;
        x.in_map = IN_MODES;
        x.L = P3;
        x.n_out = P3h;
        x.sign = -1;
        launch_axis_fft(ctx, x);
    }
    K.release();
    {
        AxisFFT y;
        y.in = a.get();
        y.in_t = E_C128;
        y.fp64 = true;
        y.n_outer = P1;
        y.n_inner = P3h;
        y.in_ostride = (long)P2 * P3h;
        y.out_ostride = (long)P2 * P3h;
        y.n_in = P2;
        y.in_map = IN_MODES;
        y.L = P2;
        y.n_out = P2;
        y.sign = -1;
        if (three_d) {
            b.alloc((long)P1 * P2 * P3h, st);
            y.out = b.get();
            y.out_t = E_C128;
        } else {
            y.out = Rd.get();
            y.out_t = E_F64;
        }
        launch_axis_fft(ctx, y);
    }
    a.release();
    if (three_d) {
        AxisFFT z;
        z.in = b.get();
        z.in_t = E_C128;
        z.out = Rd.get();
        z.out_t = E_F64;
        z.fp64 = true;
        z.n_outer = 1;
        z.n_inner = (long)P2 * P3h;
        z.in_ostride = 0;
        z.out_ostride = 0;
        z.n_in = P1;
        z.in_map = IN_MODES;
        z.L = P1;
        z.n_out = P1;
        z.sign = -1;
        launch_axis_fft(ctx, z);
    }
    long nR = spectrum_elems();
    R_.alloc(nR, st);
    d2f_kernel<<<grid_for(nR, 256, ctx.num_sms()), 256, 0, st>>>(Rd.get(), R_.get(), nR);
    LC_CHECK_LAUNCH();
    LC_CUDA(cudaStreamSynchronize(st));
    // work buffers
    if (three_d) {
        t1_.alloc(n_[0] * n_[1] * Ph_[2], st);
        t2_.alloc(n_[0] * (long)P_[1] * Ph_[2], st);
    } else {
        t1_.alloc(n_[0] * n_[1] * Ph_[2], st);
    }
}

void Toeplitz::build_kernel(Context &ctx, DevBuf<double> &K) {
    cudaStream_t st = ctx.stream();
    ProfScope ps(ctx, PS_PSF_GEN, 0.0);
    if (!three_d_) {
        const int P = P_[2];
        K.alloc((long)P * P, st);
        long total = (long)P * P;
        psf2d_kernel<<<grid_for(total, 128, ctx.num_sms()), 128, 0, st>>>(
            g_->pts.cs, g_->pts.ntheta, g_->pts.nr, P, P, K.get());
    } else {
        long total = (long)P_[0] * P_[1] * P_[2];
        K.alloc(total, st);
        size_t smem = 6 * sizeof(double) * g_->pts.ntheta;
        LC_REQUIRE(smem <= 200 * 1024, "Toeplitz3D: too many angles for one PSF launch");
        auto kern = psf3d_kernel;
        LC_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        kern<<<grid_for(total, 128, ctx.num_sms()), 128, smem, st>>>(
            g_->pts.rot, g_->pts.ntheta, g_->pts.nrows, g_->pts.ncols, P_[0], P_[1], P_[2], K.get());
    }
    LC_CHECK_LAUNCH();
}

void Toeplitz::kernel_fp64(Context &ctx, double *host_out) {
    DevBuf<double> K;
    build_kernel(ctx, K);
    long total = three_d_ ? (long)P_[0] * P_[1] * P_[2] : (long)P_[2] * P_[2];
    LC_CUDA(cudaMemcpyAsync(host_out, K.get(), total * sizeof(double), cudaMemcpyDeviceToHost,
                            ctx.stream()));
    LC_CUDA(cudaStreamSynchronize(ctx.stream()));
}

double Toeplitz::algorithmic_bytes() const {
    // read x, write y, read the real spectrum octant once
    return 8.0 * (double)nvox() + 4.0 * (double)spectrum_elems();
}

void Toeplitz::apply(Context &ctx, const float *x, float *y) {
    const long n1 = n_[0], n2 = n_[1], n3 = n_[2];
    const int P1 = P_[0], P2 = P_[1], P3 = P_[2];
    const int P3h = Ph_[2];
    const double N = (double)n1 * n2 * n3;
    const double T1 = (double)n1 * n2 * P3h * 8.0;      // half-spectrum rows, complex
    const double T2 = (double)n1 * P2 * P3h * 8.0;      // after the y transform
    const double Rb = 4.0 * (double)spectrum_elems();
    // x rows: real -> half spectrum
    {
        ProfScope ps(ctx, PS_TOEP_X_FWD, 4.0 * N + T1);
        AxisFFT a;
        a.in = x;
        a.in_t = E_F32;
        a.out = t1_.get();
        a.out_t = E_C64;
        a.n_outer = n1 * n2;
        a.n_inner = 1;
        a.in_ostride = n3;
        a.out_ostride = P3h;
        a.n_in = (int)n3;
        a.L = P3;
        a.n_out = P3h;
        a.sign = -1;
        launch_axis_fft(ctx, a);
    }
    if (!three_d_) {
        ProfScope ps(ctx, PS_TOEP_Y_MID, 2.0 * T1 + Rb);
        AxisFFT a;
        a.in = t1_.get();
        a.in_t = E_C64;
        a.out = t1_.get();
        a.out_t = E_C64;
        a.n_outer = n1;
        a.n_inner = P3h;
        a.in_ostride = n2 * P3h;
        a.out_ostride = n2 * P3h;
        a.n_in = (int)n2;
        a.L = P2;
        a.n_out = (int)n2;
        a.out_map = OUT_WINDOW;
        a.out_off = 0;
        a.sign = -1;
        a.mid = R_.get();
        a.mid_ra = P3h;
        a.sign2 = +1;
        launch_axis_fft(ctx, a);
    } else {
        {
            ProfScope ps(ctx, PS_TOEP_Y_FWD, T1 + T2);
            AxisFFT a;
            a.in = t1_.get();
            a.in_t = E_C64;
            a.out = t2_.get();
            a.out_t = E_C64;
            a.n_outer = n1;
            a.n_inner = P3h;
            a.in_ostride = n2 * P3h;
            a.out_ostride = (long)P2 * P3h;
            a.n_in = (int)n2;
            a.L = P2;
            a.n_out = P2;
            a.sign = -1;
            launch_axis_fft(ctx, a);
        }
        {
            ProfScope ps(ctx, PS_TOEP_Z_MID, 2.0 * T2 + Rb);
            AxisFFT a;
            a.in = t2_.get();
            a.in_t = E_C64;
            a.out = t2_.get();
            a.out_t = E_C64;
            a.n_outer = 1;
            a.n_inner = (long)P2 * P3h;
            a.in_ostride = 0;
            a.out_ostride = 0;
            a.n_in = (int)n1;
            a.L = P1;
            a.n_out = (int)n1;
            a.out_map = OUT_WINDOW;
            a.out_off = 0;
            a.sign = -1;
            a.mid = R_.get();
            a.mid_ra = (long)P2 * P3h;
            a.sign2 = +1;
            launch_axis_fft(ctx, a);
        }
        {
            ProfScope ps(ctx, PS_TOEP_Y_INV, T1 + T2);
            AxisFFT a;
            a.in = t2_.get();
            a.in_t = E_C64;
            a.out = t1_.get();
            a.out_t = E_C64;
            a.n_outer = n1;
            a.n_inner = P3h;
            a.in_ostride = (long)P2 * P3h;
            a.out_ostride = n2 * P3h;
            a.n_in = P2;
            a.L = P2;
            a.n_out = (int)n2;
            a.out_map = OUT_WINDOW;
            a.out_off = 0;
            a.sign = +1;
            launch_axis_fft(ctx, a);
        }
    }
    {
        ProfScope ps(ctx, PS_TOEP_X_INV, T1 + 4.0 * N);
        AxisFFT a;
        a.in = t1_.get();
        a.in_t = E_C64;
        a.out = y;
        a.out_t = E_F32;
        a.n_outer = n1 * n2;
        a.n_inner = 1;
        a.in_ostride = P3h;
        a.out_ostride = n3;
        a.n_in = P3h;
        a.in_map = IN_HERM;
        a.L = P3;
        a.n_out = (int)n3;
        a.out_map = OUT_WINDOW;
        a.out_off = 0;
        a.sign = +1;
        a.scale = scale_;
        launch_axis_fft(ctx, a);
    }
}

void Toeplitz::apply_reg(Context &ctx, const float *x, float *y, float mu) {
    apply(ctx, x, y);
    if (mu != 0.0f) launch_neg_laplacian_axpy(ctx, x, y, n_, mu);
}

}  // namespace lc
