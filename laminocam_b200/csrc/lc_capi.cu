// extern "C" boundary of laminocam_b200 (declared in include/laminocam.h).
#include <algorithm>
#include <chrono>
#include <cfloat>
#include <cmath>
#include <cstdio>
#include <map>
#include <memory>
#include <tuple>

#include "lc_internal.hpp"

using namespace lc;

namespace lc {
long odd_pad(long n, float factor) {
    long v = (long)((float)n * factor);
    return v % 2 == 0 ? v - 1 : v;
}
}  // namespace lc

namespace {

int fail(lc_context c, int code, const char *msg) {
    if (c) c->err = msg;
    return code;
}

double eff_tol(double tol) { return tol > 0 ? tol : 1e-6; }

NufftPlan &plan_for(lc_geometry g, int n3, int n2, int n1, double tol) {
    Context &ctx = *g->owner->ctx;
    int tq = (int)std::lround(-std::log10(tol) * 100.0);
    auto key = std::make_tuple(n3, n2, n1, tq);
    auto it = g->plans.find(key);
    if (it != g->plans.end()) return *it->second;
    int modes[3] = {n3, n2, n1};
    auto p = std::make_unique<NufftPlan>(ctx, g->g, modes, tol);
    auto &ref = *p;
    g->plans[key] = std::move(p);
    return ref;
}

// ---- small kernels used by the drivers ---------------------------------
__global__ void max_kernel(const float *__restrict__ a, long n, unsigned *out_bits) {
    float m = -FLT_MAX;
    for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x)
        m = fmaxf(m, a[i]);
    for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_down_sync(0xffffffffu, m, o));
    if ((threadIdx.x & 31) == 0) {
        // order-preserving float -> unsigned map
        unsigned b = __float_as_uint(m);
        b = (b & 0x80000000u) ? ~b : (b | 0x80000000u);
        atomicMax(out_bits, b);
    }
}

// out {nt, N2, N3} = in {nt, n2, n3} / scale placed at (d2, d3), zero elsewhere
__global__ void norm_pad_kernel(const float *__restrict__ in, long nt, long n2, long n3,
                                float *__restrict__ out, long N2, long N3, long d2, long d3,
                                const unsigned *max_bits) {
    unsigned b = *max_bits;
    b = (b & 0x80000000u) ? (b & 0x7fffffffu) : ~b;
    float mx = __uint_as_float(b);
    bool scale = mx > 0.f;
    long total = nt * N2 * N3;
    for (long idx = (long)blockIdx.x * blockDim.x + threadIdx.x; idx < total;
         idx += (long)gridDim.x * blockDim.x) {
        long t = idx / (N2 * N3);
        long r = idx - t * N2 * N3;
        long j = r / N3 - d2, k = r % N3 - d3;
        float v = 0.f;
        if (j >= 0 && j < n2 && k >= 0 && k < n3) {
            v = in[(t * n2 + j) * n3 + k];
            if (scale) v = v / mx;
        }
        out[idx] = v;
    }
}

__global__ void crop_kernel(const float *__restrict__ in, long N1, long N2, long N3,
                            float *__restrict__ out, long n1, long n2, long n3, long d1, long d2,
                            long d3) {
    long total = n1 * n2 * n3;
    for (long idx = (long)blockIdx.x * blockDim.x + threadIdx.x; idx < total;
         idx += (long)gridDim.x * blockDim.x) {
        long i = idx / (n2 * n3);
        long r = idx - i * n2 * n3;
        long j = r / n3, k = r % n3;
        out[idx] = in[((i + d1) * N2 + (j + d2)) * N3 + (k + d3)];
    }
}

unsigned grid_for(long n, int threads, int sms) {
    long b = (n + threads - 1) / threads;
    return (unsigned)std::max<long>(1, std::min<long>(b, (long)sms * 32));
}

// --- operator implementations shared by the API and the drivers ----------
void do_backproj2d(lc_geometry g, const float *sino, int ns, int n2, int n3, float *vol, double tol) {
    Context &ctx = *g->owner->ctx;
    LC_REQUIRE(g->g.pts.dim == 2, "backproj2d needs a 2D geometry");
    const int nth = g->g.pts.ntheta, nr = g->g.pts.nr;
    const long M = g->g.pts.M;
    g->work.ensure((long)ns * M, ctx.stream());
    AxisDFT d;
    d.in = sino;
    d.in_t = E_F32;
    d.out = g->work.get();
    d.out_t = E_C64;
    d.n_outer = (long)ns * nth;
    d.n_inner = 1;
    d.in_ostride = nr;
    d.out_ostride = nr;
    d.n = nr;
    d.d_pre = nr / 2;         // fftshift1
    d.d_post = (nr + 1) / 2;  // ifftshift1
    d.sign = -1;
    launch_axis_dft(ctx, d);
    plan_for(g, n3, n2, 1, tol).type1_real(ctx, g->work.get(), ns, vol, 1.0f / (float)nr, PT_PLAIN);
}

void do_forward2d(lc_geometry g, const float *vol, int ns, int n2, int n3, float *sino, double tol) {
    Context &ctx = *g->owner->ctx;
    LC_REQUIRE(g->g.pts.dim == 2, "forward2d needs a 2D geometry");
    const int nth = g->g.pts.ntheta, nr = g->g.pts.nr;
    const long M = g->g.pts.M;
    g->work.ensure((long)ns * M, ctx.stream());
    plan_for(g, n3, n2, 1, tol).type2_real(ctx, vol, ns, g->work.get(), PT_PLAIN);
    AxisDFT d;
    d.in = g->work.get();
    d.in_t = E_C64;
    d.out = sino;
    d.out_t = E_F32;
    d.n_outer = (long)ns * nth;
    d.n_inner = 1;
    d.in_ostride = nr;
    d.out_ostride = nr;
    d.n = nr;
    d.d_pre = (nr + 1) / 2;  // ifftshift1
    d.d_post = nr / 2;       // fftshift1
    d.sign = +1;
    d.scale = 1.0f / (float)nr;
    launch_axis_dft(ctx, d);
}

void do_backproj3d(lc_geometry g, const float *proj, int n1, int n2, int n3, bool shifts,
                   float *vol, double tol) {
    Context &ctx = *g->owner->ctx;
    LC_REQUIRE(g->g.pts.dim == 3, "backproj3d needs a 3D geometry");
    const int nth = g->g.pts.ntheta, nrows = g->g.pts.nrows, ncols = g->g.pts.ncols;
    const long M = g->g.pts.M;
    g->work.ensure(M, ctx.stream());
    {
        AxisDFT d;  // along ncols: fftshift -> FFT -> ifftshift
        d.in = proj;
        d.in_t = E_F32;
        d.out = g->work.get();
        d.out_t = E_C64;
        d.n_outer = (long)nth * nrows;
        d.n_inner = 1;
        d.in_ostride = ncols;
        d.out_ostride = ncols;
        d.n = ncols;
        d.d_pre = ncols / 2;
        d.d_post = (ncols + 1) / 2;
        d.sign = -1;
        launch_axis_dft(ctx, d);
    }
    {
        AxisDFT d;  // along nrows, in place
        d.in = g->work.get();
        d.in_t = E_C64;
        d.out = g->work.get();
        d.out_t = E_C64;
        d.n_outer = nth;
        d.n_inner = ncols;
        d.in_ostride = (long)nrows * ncols;
        d.out_ostride = (long)nrows * ncols;
        d.n = nrows;
        d.d_pre = nrows / 2;
        d.d_post = (nrows + 1) / 2;
        d.sign = -1;
        launch_axis_dft(ctx, d);
    }
    plan_for(g, n3, n2, n1, tol).type1_real(ctx, g->work.get(), 1, vol,
                                            1.0f / ((float)nrows * (float)ncols),
                                            shifts ? PT_SHIFT : PT_MASK);
}

void do_forward3d(lc_geometry g, const float *vol, int n1, int n2, int n3, float *proj, double tol) {
    Context &ctx = *g->owner->ctx;
    LC_REQUIRE(g->g.pts.dim == 3, "forward3d needs a 3D geometry");
    const int nth = g->g.pts.ntheta, nrows = g->g.pts.nrows, ncols = g->g.pts.ncols;
    const long M = g->g.pts.M;
    g->work.ensure(M, ctx.stream());
    plan_for(g, n3, n2, n1, tol).type2_real(ctx, vol, 1, g->work.get(), PT_MASK);
    {
        AxisDFT d;  // along ncols: fftshift -> IFFT -> ifftshift, in place
        d.in = g->work.get();
        d.in_t = E_C64;
        d.out = g->work.get();
        d.out_t = E_C64;
        d.n_outer = (long)nth * nrows;
        d.n_inner = 1;
        d.in_ostride = ncols;
        d.out_ostride = ncols;
        d.n = ncols;
        d.d_pre = ncols / 2;
        d.d_post = (ncols + 1) / 2;
        d.sign = +1;
        launch_axis_dft(ctx, d);
    }
    {
        AxisDFT d;  // along nrows, real part / (nrows*ncols)
        d.in = g->work.get();
        d.in_t = E_C64;
        d.out = proj;
        d.out_t = E_F32;
        d.n_outer = nth;
        d.n_inner = ncols;
        d.in_ostride = (long)nrows * ncols;
        d.out_ostride = (long)nrows * ncols;
        d.n = nrows;
        d.d_pre = nrows / 2;
        d.d_post = (nrows + 1) / 2;
        d.sign = +1;
        d.scale = 1.0f / ((float)nrows * (float)ncols);
        launch_axis_dft(ctx, d);
    }
}

void check_solver_params(const lc_solver_params *p) {
    LC_REQUIRE(p != nullptr, "solver params must not be NULL");
    LC_REQUIRE(p->max_iters >= 0 && p->inner_iters >= 0, "iteration counts must be >= 0");
    LC_REQUIRE(std::isfinite(p->tol) && std::isfinite(p->xtol), "tolerances must be finite");
    LC_REQUIRE(std::isfinite(p->lambda) && std::isfinite(p->mu), "lambda and mu must be finite");
}

SolverParams to_sp(const lc_solver_params *p) {
    SolverParams s;
    s.max_iters = p->max_iters;
    s.inner_iters = p->inner_iters;
    s.tol = p->tol;
    s.xtol = p->xtol;
    s.lambda = p->lambda;
    s.mu = p->mu;
    s.fp32_scalars = p->fp32_scalars;
    s.poll_every = p->poll_every;
    s.use_graph = p->use_graph;
    s.residual_refresh = p->residual_refresh;
    return s;
}

void run_solver(lc_psf psf, int method, const float *rhs, float *x, const lc_solver_params *p,
                lc_solver_stats *stats) {
    Context &ctx = *psf->owner->ctx;
    check_solver_params(p);
    if (method == 1) LC_REQUIRE(p->mu != 0.0f, "split_bregman: mu must be non-zero");
    Toeplitz *T = psf->T.get();
    // Split-Bregman runs on rows padded to a multiple of 4 values (zeros past
    // the row), so that its stencil kernels take four voxels per thread
    const long *d = T->dims();
    const long pitch = (d[2] + 3) / 4 * 4;
    const bool padded = method == 1 && pitch != d[2];
    const long need = padded ? d[0] * d[1] * pitch : T->nvox();
    if (!psf->solver || psf->solver->size() != need) psf->solver = std::make_unique<Solver>(ctx, need);
    Operator A = [&ctx, T](const float *in, float *out) { T->apply(ctx, in, out); };
    // CG iterations fuse the direction update and p.Ap into the x passes
    FusedOperator F;
    F.caps = T->cg_caps();
    F.partials = T->cg_partials();
    const unsigned caps = F.caps;
    F.apply = [&ctx, T, caps](const float *in, float *out, const CGFusion &f) {
        T->apply(ctx, in, out, &f, caps);
    };
    cudaEvent_t e0, e1;
    LC_CUDA(cudaEventCreate(&e0));
    LC_CUDA(cudaEventCreate(&e1));
    LC_CUDA(cudaEventRecord(e0, ctx.stream()));
    SolverStats st;
    SolverParams sp = to_sp(p);
    if (method == 0) {
        psf->solver->cg(ctx, A, rhs, x, sp, &st, &F);
    } else if (!padded) {
        psf->solver->split_bregman(ctx, A, d, rhs, x, sp, &st);
    } else {
        cudaStream_t s = ctx.stream();
        const long rows = d[0] * d[1], np = need;
        DevBuf<float> yp(np, s), xp(np, s);
        yp.zero(s);
        xp.zero(s);
        const size_t w = (size_t)d[2] * sizeof(float), wp = (size_t)pitch * sizeof(float);
        LC_CUDA(cudaMemcpy2DAsync(yp.get(), wp, rhs, w, w, rows, cudaMemcpyDeviceToDevice, s));
        LC_CUDA(cudaMemcpy2DAsync(xp.get(), wp, x, w, w, rows, cudaMemcpyDeviceToDevice, s));
        Operator Ap = [&ctx, T, pitch](const float *in, float *out) { T->apply(ctx, in, out, nullptr, 0, pitch); };
        psf->solver->split_bregman(ctx, Ap, d, yp.get(), xp.get(), sp, &st, pitch);
        LC_CUDA(cudaMemcpy2DAsync(x, w, xp.get(), wp, w, rows, cudaMemcpyDeviceToDevice, s));
    }
    LC_CUDA(cudaEventRecord(e1, ctx.stream()));
    LC_CUDA(cudaEventSynchronize(e1));
    float ms = 0;
    const cudaError_t te = cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    LC_CUDA(te);
    if (stats) {
        stats->iters = st.iters;
        stats->cg_iters_total = st.cg_iters_total;
        stats->residual = st.residual;
        stats->dx = st.dx;
        stats->stop_reason = st.stop_reason;
        stats->elapsed_ms = ms;
    }
}

}  // namespace

// Destroys a geometry or PSF without touching its owner handle, which may
// already be gone; the shared lc::Context keeps the streams alive meanwhile.
template <typename H>
static int destroy_child(H *h) {
    if (!h) return LC_ERR_INVALID;
    const std::shared_ptr<Context> keep = h->keep;
    int rc = LC_OK;
    try {
        DeviceGuard dg(keep->device());
        if (cudaStreamSynchronize(keep->stream()) != cudaSuccess) rc = LC_ERR_CUDA;
        delete h;
    } catch (...) {
        rc = LC_ERR_CUDA;
    }
    return rc;
}

extern "C" {

int lc_version(void) { return 100; }

long lc_kernel_launches(void) { return kernel_launch_count(); }

void lc_solver_params_default(lc_solver_params *p) {
    if (!p) return;
    p->max_iters = 50;
    p->inner_iters = 1;
    p->tol = 1e-5f;
    p->xtol = 1e-5f;
    p->lambda = 0.1f;
    p->mu = 10.0f;
    p->fp32_scalars = 0;
    p->poll_every = 8;
    p->use_graph = 0;
    p->residual_refresh = 1;
}

void lc_recon_params_default(lc_recon_params *p) {
    if (!p) return;
    p->method = 0;
    lc_solver_params_default(&p->solver);
    p->nufft_tol = 1e-6;
    p->pad_factor = 1.4142f;
    p->psf_fp32 = 0;
}

int lc_context_create(int device, void *stream, lc_context *out) {
    if (!out) return LC_ERR_INVALID;
    *out = nullptr;
    try {
        int n = 0;
        if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) return LC_ERR_CUDA;
        if (device < 0 || device >= n) return LC_ERR_INVALID;
        auto c = new lc_context_s;
        c->ctx = std::make_unique<Context>(device, (cudaStream_t)stream);
        *out = c;
        return LC_OK;
    } catch (...) {
        return LC_ERR_CUDA;
    }
}

int lc_context_destroy(lc_context c) {
    if (!c) return LC_ERR_INVALID;
    {
        DeviceGuard dg(c->ctx->device());
        cudaStreamSynchronize(c->ctx->stream());
        c->ctx.reset();
    }
    delete c;
    return LC_OK;
}

int lc_context_set_stream(lc_context c, void *stream) {
    return guarded(c, [&] { c->ctx->set_stream((cudaStream_t)stream); });
}

int lc_context_synchronize(lc_context c) {
    return guarded(c, [&] { LC_CUDA(cudaStreamSynchronize(c->ctx->stream())); });
}

const char *lc_last_error(lc_context c) { return c ? c->err.c_str() : "null context"; }

int lc_geometry2d_create(lc_context c, const double *theta, int ntheta, int nradial,
                         lc_geometry *out) {
    if (!out) return fail(c, LC_ERR_INVALID, "out is NULL");
    *out = nullptr;
    return guarded(c, [&] {
        LC_REQUIRE(theta != nullptr, "theta is NULL");
        for (int i = 0; i < ntheta; ++i) LC_REQUIRE(std::isfinite(theta[i]), "theta must be finite");
        auto g = std::make_unique<lc_geometry_s>();
        g->keep = c->ctx;
        g->owner = c;
        geometry_init_2d(*c->ctx, g->g, theta, ntheta, nradial);
        *out = g.release();
    });
}

int lc_geometry3d_create(lc_context c, const double *theta, const double *gamma,
                         const double *beta, const float *shifts, int ntheta, int nrows,
                         int ncols, lc_geometry *out) {
    if (!out) return fail(c, LC_ERR_INVALID, "out is NULL");
    *out = nullptr;
    return guarded(c, [&] {
        LC_REQUIRE(theta && gamma && beta, "theta, gamma and beta must not be NULL");
        for (int i = 0; i < ntheta; ++i)
            LC_REQUIRE(std::isfinite(theta[i]) && std::isfinite(gamma[i]) && std::isfinite(beta[i]),
                       "angles must be finite");
        auto g = std::make_unique<lc_geometry_s>();
        g->keep = c->ctx;
        g->owner = c;
        geometry_init_3d(*c->ctx, g->g, theta, gamma, beta, shifts, ntheta, nrows, ncols);
        *out = g.release();
    });
}

int lc_geometry_destroy(lc_geometry g) { return destroy_child(g); }

int lc_forward2d(lc_context c, lc_geometry g, const float *volume, int ns, int n2, int n3,
                 float *sino, double tol) {
    return guarded(c, [&] {
        LC_REQUIRE(g && volume && sino, "NULL argument");
        LC_REQUIRE(ns > 0 && n2 > 0 && n3 > 0, "sizes must be positive");
        do_forward2d(g, volume, ns, n2, n3, sino, eff_tol(tol));
    });
}

int lc_backproj2d(lc_context c, lc_geometry g, const float *sino, int ns, int n2, int n3,
                  float *volume, double tol) {
    return guarded(c, [&] {
        LC_REQUIRE(g && volume && sino, "NULL argument");
        LC_REQUIRE(ns > 0 && n2 > 0 && n3 > 0, "sizes must be positive");
        do_backproj2d(g, sino, ns, n2, n3, volume, eff_tol(tol));
    });
}

int lc_sysmat2d_nufft(lc_context c, lc_geometry g, const float *x, int ns, int n2, int n3, float *y,
                      double tol) {
    return guarded(c, [&] {
        LC_REQUIRE(g && x && y, "NULL argument");
        LC_REQUIRE(ns > 0 && n2 > 0 && n3 > 0, "sizes must be positive");
        LC_REQUIRE(g->g.pts.dim == 2, "sysmat2d needs a 2D geometry");
        Context &ctx = *c->ctx;
        NufftPlan &pl = plan_for(g, n3, n2, 1, eff_tol(tol));
        g->work.ensure((long)ns * g->g.pts.M, ctx.stream());
        pl.type2_real(ctx, x, ns, g->work.get(), PT_PLAIN);
        pl.type1_real(ctx, g->work.get(), ns, y, 1.0f / (float)g->g.pts.nr, PT_PLAIN);
    });
}

int lc_forward3d(lc_context c, lc_geometry g, const float *volume, int n1, int n2, int n3,
                 float *proj, double tol) {
    return guarded(c, [&] {
        LC_REQUIRE(g && volume && proj, "NULL argument");
        LC_REQUIRE(n1 > 0 && n2 > 0 && n3 > 0, "sizes must be positive");
        do_forward3d(g, volume, n1, n2, n3, proj, eff_tol(tol));
    });
}

int lc_backproj3d(lc_context c, lc_geometry g, const float *proj, int n1, int n2, int n3,
                  int apply_shifts, float *volume, double tol) {
    return guarded(c, [&] {
        LC_REQUIRE(g && volume && proj, "NULL argument");
        LC_REQUIRE(n1 > 0 && n2 > 0 && n3 > 0, "sizes must be positive");
        do_backproj3d(g, proj, n1, n2, n3, apply_shifts != 0, volume, eff_tol(tol));
    });
}

int lc_sysmat3d_nufft(lc_context c, lc_geometry g, const float *x, int n1, int n2, int n3, float *y,
                      double tol) {
    return guarded(c, [&] {
        LC_REQUIRE(g && x && y, "NULL argument");
        LC_REQUIRE(n1 > 0 && n2 > 0 && n3 > 0, "sizes must be positive");
        LC_REQUIRE(g->g.pts.dim == 3, "sysmat3d needs a 3D geometry");
        Context &ctx = *c->ctx;
        NufftPlan &pl = plan_for(g, n3, n2, n1, eff_tol(tol));
        g->work.ensure(g->g.pts.M, ctx.stream());
        pl.type2_real(ctx, x, 1, g->work.get(), PT_PLAIN);
        pl.type1_real(ctx, g->work.get(), 1, y,
                      1.0f / ((float)g->g.pts.nrows * (float)g->g.pts.ncols), PT_PLAIN);
    });
}

int lc_psf_create(lc_context c, lc_geometry g, int n1, int n2, int n3, lc_psf *out) {
    return lc_psf_create_ex(c, g, n1, n2, n3, 0, out);
}

int lc_psf_create_ex(lc_context c, lc_geometry g, int n1, int n2, int n3, int flags, lc_psf *out) {
    if (!out) return fail(c, LC_ERR_INVALID, "out is NULL");
    *out = nullptr;
    return guarded(c, [&] {
        LC_REQUIRE(g != nullptr, "geometry is NULL");
        LC_REQUIRE(n1 > 0 && n2 > 0 && n3 > 0, "sizes must be positive");
        LC_REQUIRE((flags & ~LC_PSF_FP32_NUFFT) == 0, "unknown PSF flags");
        bool three = g->g.pts.dim == 3;
        if (!three) LC_REQUIRE(n2 == n3, "2D PSF needs square slices (n2 == n3)");
        long dims[3] = {n1, n2, n3};
        auto p = std::make_unique<lc_psf_s>();
        p->keep = c->ctx;
        p->owner = c;
        p->geom = g;
        p->T = std::make_unique<Toeplitz>(*c->ctx, g->g, dims, three, (flags & LC_PSF_FP32_NUFFT) != 0);
        // complete on return: the caller may use it on another stream
        LC_CUDA(cudaStreamSynchronize(c->ctx->stream()));
        *out = p.release();
    });
}

int lc_psf_destroy(lc_psf p) { return destroy_child(p); }

int lc_psf_info(lc_psf p, int *P, long *spectrum_elems) {
    if (!p) return LC_ERR_INVALID;
    if (P)
        for (int d = 0; d < 3; ++d) P[d] = p->T->P()[d];
    if (spectrum_elems) *spectrum_elems = p->T->spectrum_elems();
    return LC_OK;
}

int lc_psf_kernel(lc_context c, lc_psf p, double *host_out) {
    return guarded(c, [&] {
        LC_REQUIRE(p && host_out, "NULL argument");
        p->T->kernel_fp64(*c->ctx, host_out);
    });
}

int lc_psf_spectrum(lc_context c, lc_psf p, float *host_out) {
    return guarded(c, [&] {
        LC_REQUIRE(p && host_out, "NULL argument");
        Toeplitz &T = *p->T;
        T.ensure_spectrum(*c->ctx);
        LC_CUDA(cudaMemcpyAsync(host_out, T.spectrum(), T.stored_spectrum_elems() * sizeof(float),
                                cudaMemcpyDeviceToHost, c->ctx->stream()));
        LC_CUDA(cudaStreamSynchronize(c->ctx->stream()));
        if (T.spectrum_zfold()) {
            // the device keeps planes f1 <= P1/2; plane f1 > P1/2 equals plane P1 - f1
            const int P1 = T.P()[0];
            const long plane = T.spectrum_elems() / P1;
            for (int f = P1 / 2 + 1; f < P1; ++f)
                std::copy(host_out + (long)(P1 - f) * plane, host_out + (long)(P1 - f + 1) * plane,
                          host_out + (long)f * plane);
        }
    });
}

int lc_sysmat_toeplitz(lc_context c, lc_psf p, const float *x, float *y) {
    return guarded(c, [&] {
        LC_REQUIRE(p && x && y, "NULL argument");
        p->T->apply(*c->ctx, x, y);
    });
}

int lc_cgsolver(lc_context c, lc_psf p, const float *rhs, float *x, const lc_solver_params *prm,
                lc_solver_stats *stats) {
    return guarded(c, [&] {
        LC_REQUIRE(p && rhs && x, "NULL argument");
        run_solver(p, 0, rhs, x, prm, stats);
    });
}

int lc_split_bregman(lc_context c, lc_psf p, const float *rhs, float *x,
                     const lc_solver_params *prm, lc_solver_stats *stats) {
    return guarded(c, [&] {
        LC_REQUIRE(p && rhs && x, "NULL argument");
        run_solver(p, 1, rhs, x, prm, stats);
    });
}

// The solvers over an operator given as a callback (opt::Function<T>,
// include/optimize.h:30-31): each application calls op(user, in, out, n,
// stream) with device vectors of n floats; a nonzero return stops the solve
// with LC_ERR_INVALID and the callback's code in the message.
static void run_solver_op(lc_context c, int method, lc_operator_fn op, void *user, const long dims[3],
                          const float *rhs, float *x, const lc_solver_params *prm, lc_solver_stats *stats) {
    LC_REQUIRE(op && rhs && x, "NULL argument");
    check_solver_params(prm);
    if (method == 1) LC_REQUIRE(prm->mu != 0.0f, "split_bregman: mu must be non-zero");
    Context &ctx = *c->ctx;
    const long n = dims[0] * dims[1] * dims[2];
    LC_REQUIRE(n > 0, "operator size must be positive");
    Solver solver(ctx, n);
    Operator A = [&ctx, op, user, n](const float *in, float *out) {
        const int rc = op(user, in, out, n, (void *)ctx.stream());
        if (rc) throw Error(1, "operator callback returned " + std::to_string(rc));
    };
    SolverStats st;
    const auto t0 = std::chrono::steady_clock::now();
    if (method == 0) solver.cg(ctx, A, rhs, x, to_sp(prm), &st, nullptr);
    else solver.split_bregman(ctx, A, dims, rhs, x, to_sp(prm), &st);
    LC_CUDA(cudaStreamSynchronize(ctx.stream()));
    if (stats) {
        stats->iters = st.iters;
        stats->cg_iters_total = st.cg_iters_total;
        stats->residual = st.residual;
        stats->dx = st.dx;
        stats->stop_reason = st.stop_reason;
        stats->elapsed_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    }
}

int lc_cgsolver_op(lc_context c, lc_operator_fn op, void *user, long n, const float *rhs, float *x,
                   const lc_solver_params *prm, lc_solver_stats *stats) {
    return guarded(c, [&] {
        const long dims[3] = {1, 1, n};
        run_solver_op(c, 0, op, user, dims, rhs, x, prm, stats);
    });
}

int lc_split_bregman_op(lc_context c, lc_operator_fn op, void *user, const int *dims, const float *rhs,
                        float *x, const lc_solver_params *prm, lc_solver_stats *stats) {
    return guarded(c, [&] {
        LC_REQUIRE(dims && dims[0] > 0 && dims[1] > 0 && dims[2] > 0, "dims must be positive");
        const long d[3] = {dims[0], dims[1], dims[2]};
        run_solver_op(c, 1, op, user, d, rhs, x, prm, stats);
    });
}

}  // extern "C"

namespace lc {

static std::shared_ptr<Toeplitz> make_psf(Context &ctx, const PolarGeometry &g, const long dims[3],
                                          bool three_d, const PsfProvider *psf, bool *hit, bool fp32 = false) {
    if (hit) *hit = false;
    if (fp32) return std::make_shared<Toeplitz>(ctx, g, dims, three_d, true);
    if (psf && *psf) return (*psf)(ctx, g, dims, three_d, hit);
    return std::make_shared<Toeplitz>(ctx, g, dims, three_d);
}

void mbir2d_core(lc_context c, const float *dsino, int ns, int ntheta, int nradial,
                 const double *theta, const int *recon_dims, const lc_recon_params *p,
                 float *drecon, lc_solver_stats *stats, const PsfProvider *psfp, bool *psf_hit) {
    LC_REQUIRE(dsino && theta && recon_dims && p && drecon, "NULL argument");
    LC_REQUIRE(ns > 0 && ntheta > 0 && nradial > 0, "sizes must be positive");
    LC_REQUIRE(recon_dims[0] == ns, "recon_dims[0] must equal the number of sinogram slices");
    LC_REQUIRE(recon_dims[1] == recon_dims[2] && recon_dims[1] > 0, "recon_dims must be square in-plane");
    LC_REQUIRE(p->method == 0 || p->method == 1, "method must be 0 (CG) or 1 (Split-Bregman)");
    check_solver_params(&p->solver);
    Context &ctx = *c->ctx;
    cudaStream_t s = ctx.stream();
    const int n = recon_dims[1];
    const long nv = (long)ns * n * n;
    lc_geometry g = nullptr;
    int rc = lc_geometry2d_create(c, theta, ntheta, nradial, &g);
    if (rc) throw Error(rc == LC_ERR_INVALID ? 1 : 3, c->err);
    std::unique_ptr<lc_geometry_s> gown(g);
    DevBuf<float> rhs(nv, s);
    do_backproj2d(g, dsino, ns, n, n, rhs.get(), eff_tol(p->nufft_tol));
    g->work.release();
    g->plans.clear();
    lc_psf_s psf;
    psf.owner = c;
    psf.geom = g;
    long dims[3] = {ns, n, n};
    psf.T = make_psf(ctx, g->g, dims, false, psfp, psf_hit, p->psf_fp32 != 0);
    LC_CUDA(cudaMemsetAsync(drecon, 0, nv * sizeof(float), s));
    run_solver(&psf, p->method, rhs.get(), drecon, &p->solver, stats);
}

}  // namespace lc

extern "C" {

int lc_mbir2d(lc_context c, const float *sino, int ns, int ntheta, int nradial,
              const double *theta, const int *recon_dims, const lc_recon_params *p, float *recon,
              lc_solver_stats *stats) {
    return guarded(c, [&] {
        LC_REQUIRE(sino && theta && recon_dims && p && recon, "NULL argument");
        LC_REQUIRE(ns > 0 && ntheta > 0 && nradial > 0, "sizes must be positive");
        Context &ctx = *c->ctx;
        cudaStream_t s = ctx.stream();
        const long nsino = (long)ns * ntheta * nradial;
        const long nv = (long)ns * recon_dims[1] * recon_dims[2];
        LC_REQUIRE(nv > 0, "recon_dims must be positive");
        DevBuf<float> dsino, x(nv, s);
        dsino.upload(sino, nsino, s);
        mbir2d_core(c, dsino.get(), ns, ntheta, nradial, theta, recon_dims, p, x.get(), stats, nullptr,
                    nullptr);
        LC_CUDA(cudaMemcpyAsync(recon, x.get(), nv * sizeof(float), cudaMemcpyDeviceToHost, s));
        LC_CUDA(cudaStreamSynchronize(s));
    });
}

}  // extern "C"

namespace lc {

void with_overlapped_upload(Context &ctx, float *dst, const float *src, long n,
                            const std::function<void(const std::function<void()> &)> &body) {
    cudaStream_t s = ctx.stream(), cs = ctx.copy_stream();
    cudaEvent_t allocated = nullptr, arrived = nullptr;
    LC_CUDA(cudaEventCreateWithFlags(&allocated, cudaEventDisableTiming));
    const cudaError_t e2 = cudaEventCreateWithFlags(&arrived, cudaEventDisableTiming);
    if (e2 != cudaSuccess) {
        cudaEventDestroy(allocated);
        LC_CUDA(e2);
    }
    auto done = [&] {
        cudaEventDestroy(allocated);
        cudaEventDestroy(arrived);
    };
    try {
        // recorded before the body queues its work, so the copy waits only for
        // the allocation of dst (stream-ordered on s)
        LC_CUDA(cudaEventRecord(allocated, s));
        bool started = false;
        auto load = [&] {
            LC_REQUIRE(!started, "upload started twice");
            started = true;
            LC_CUDA(cudaStreamWaitEvent(cs, allocated, 0));
            LC_CUDA(cudaMemcpyAsync(dst, src, n * sizeof(float), cudaMemcpyHostToDevice, cs));
            LC_CUDA(cudaEventRecord(arrived, cs));
            LC_CUDA(cudaStreamWaitEvent(s, arrived, 0));
        };
        body(load);
    } catch (...) {
        // the copy may still be running into dst: let it finish first
        cudaStreamSynchronize(cs);
        done();
        throw;
    }
    done();
}

void mbir3d_core(lc_context c, const float *dprojs_in, int ntheta, int nrows, int ncols,
                 const double *theta, const double *gamma, const double *beta, const float *shifts,
                 const int *recon_dims, const lc_recon_params *p, float *dout,
                 lc_solver_stats *stats, const PsfProvider *psfp, bool *psf_hit,
                 const std::function<void()> &load_input) {
    LC_REQUIRE(theta && gamma && beta && recon_dims && p, "NULL argument");
    LC_REQUIRE(ntheta > 0 && nrows > 0 && ncols > 0, "sizes must be positive");
    LC_REQUIRE(recon_dims[0] > 0 && recon_dims[1] > 0 && recon_dims[2] > 0,
               "recon_dims must be positive");
    LC_REQUIRE(p->method == 0 || p->method == 1, "method must be 0 (CG) or 1 (Split-Bregman)");
    LC_REQUIRE(p->pad_factor >= 1.0f && p->pad_factor < 4.0f, "pad_factor must be in [1, 4)");
    check_solver_params(&p->solver);
    Context &ctx = *c->ctx;
    cudaStream_t s = ctx.stream();
    const float pf = p->pad_factor;
    // padded reconstruction box (src/gpu/mbir.cu:46-60)
    long N[3];
    for (int d = 0; d < 3; ++d) {
        N[d] = odd_pad(recon_dims[d], pf);
        LC_REQUIRE(N[d] >= recon_dims[d], "recon_dims must be odd when pad_factor is 1");
    }
    // padded projections (symmetric, odd), normalised by the global maximum
    long PR = odd_pad(nrows, pf), PC = odd_pad(ncols, pf);
    if (pf - 1.0f < 1e-6f) {
        PR = nrows;
        PC = ncols;
    }
    const long np = (long)ntheta * nrows * ncols;
    lc_geometry g = nullptr;
    int rc = lc_geometry3d_create(c, theta, gamma, beta, shifts, ntheta, (int)PR, (int)PC, &g);
    if (rc) throw Error(rc == LC_ERR_INVALID ? 1 : 3, c->err);
    std::unique_ptr<lc_geometry_s> gown(g);
    // the PSF depends on the angles only: it is built while the projections
    // may still be arriving
    lc_psf_s psf;
    psf.owner = c;
    psf.geom = g;
    psf.T = make_psf(ctx, g->g, N, true, psfp, psf_hit, p->psf_fp32 != 0);
    if (load_input) load_input();
    DevBuf<unsigned> mx(1, s);
    mx.zero(s);
    max_kernel<<<grid_for(np, 256, ctx.num_sms()), 256, 0, s>>>(dprojs_in, np, mx.get());
    LC_CHECK_LAUNCH();
    DevBuf<float> dproj((long)ntheta * PR * PC, s);
    norm_pad_kernel<<<grid_for((long)ntheta * PR * PC, 256, ctx.num_sms()), 256, 0, s>>>(
        dprojs_in, ntheta, nrows, ncols, dproj.get(), PR, PC, (PR - nrows) / 2, (PC - ncols) / 2,
        mx.get());
    LC_CHECK_LAUNCH();
    const long nvp = N[0] * N[1] * N[2];
    DevBuf<float> yT(nvp, s), x(nvp, s);
    do_backproj3d(g, dproj.get(), (int)N[0], (int)N[1], (int)N[2], shifts != nullptr, yT.get(),
                  eff_tol(p->nufft_tol));
    dproj.release();
    g->work.release();
    g->plans.clear();
    x.zero(s);
    run_solver(&psf, p->method, yT.get(), x.get(), &p->solver, stats);
    const long nv = (long)recon_dims[0] * recon_dims[1] * recon_dims[2];
    crop_kernel<<<grid_for(nv, 256, ctx.num_sms()), 256, 0, s>>>(
        x.get(), N[0], N[1], N[2], dout, recon_dims[0], recon_dims[1], recon_dims[2],
        (N[0] - recon_dims[0]) / 2, (N[1] - recon_dims[1]) / 2, (N[2] - recon_dims[2]) / 2);
    LC_CHECK_LAUNCH();
}

}  // namespace lc

extern "C" {

int lc_mbir3d(lc_context c, const float *projs, int ntheta, int nrows, int ncols,
              const double *theta, const double *gamma, const double *beta, const float *shifts,
              const int *recon_dims, const lc_recon_params *p, float *recon,
              lc_solver_stats *stats) {
    return guarded(c, [&] {
        LC_REQUIRE(projs && recon && recon_dims, "NULL argument");
        LC_REQUIRE(ntheta > 0 && nrows > 0 && ncols > 0, "sizes must be positive");
        Context &ctx = *c->ctx;
        cudaStream_t s = ctx.stream();
        const long np = (long)ntheta * nrows * ncols;
        const long nv = (long)recon_dims[0] * recon_dims[1] * recon_dims[2];
        LC_REQUIRE(nv > 0, "recon_dims must be positive");
        // the projections travel on the copy stream while the geometry and
        // the PSF are built
        DevBuf<float> draw(np, s);
        DevBuf<float> out(nv, s);
        with_overlapped_upload(ctx, draw.get(), projs, np, [&](const std::function<void()> &load) {
            mbir3d_core(c, draw.get(), ntheta, nrows, ncols, theta, gamma, beta, shifts, recon_dims, p,
                        out.get(), stats, nullptr, nullptr, load);
            LC_CUDA(cudaMemcpyAsync(recon, out.get(), nv * sizeof(float), cudaMemcpyDeviceToHost, s));
            LC_CUDA(cudaStreamSynchronize(s));
        });
    });
}

int lc_mbir3d_device(lc_context c, const float *projs, int ntheta, int nrows, int ncols,
                     const double *theta, const double *gamma, const double *beta,
                     const float *shifts, const int *recon_dims, const lc_recon_params *p,
                     float *recon, lc_solver_stats *stats) {
    return guarded(c, [&] {
        LC_REQUIRE(projs && recon, "NULL argument");
        mbir3d_core(c, projs, ntheta, nrows, ncols, theta, gamma, beta, shifts, recon_dims, p,
                    recon, stats, nullptr, nullptr);
        // the reconstruction is complete on return, as with lc_mbir3d
        LC_CUDA(cudaStreamSynchronize(c->ctx->stream()));
    });
}

int lc_profile_enable(lc_context c, int on) {
    return guarded(c, [&] {
        c->ctx->prof.reset();
        c->ctx->prof.on = on != 0;
    });
}

int lc_profile_read(lc_context c, lc_profile_entry *out, int max_entries, int *n_entries) {
    return guarded(c, [&] {
        LC_REQUIRE(out && n_entries, "NULL argument");
        c->ctx->prof.collect();
        int n = 0;
        for (int sct = 0; sct < PS_COUNT && n < max_entries; ++sct) {
            if (c->ctx->prof.count[sct] == 0) continue;
            lc_profile_entry &e = out[n++];
            std::snprintf(e.name, sizeof(e.name), "%s", prof_name(sct));
            e.count = c->ctx->prof.count[sct];
            e.total_ms = c->ctx->prof.ms[sct];
            e.bytes = c->ctx->prof.bytes[sct];
        }
        *n_entries = n;
    });
}

}  // extern "C"
