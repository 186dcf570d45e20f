// Definitions shared by the C ABI (lc_capi.cu) and the job server
// (lc_server.cu): the handle structs and the reconstruction drivers on
// device buffers.
#pragma once

#include <functional>
#include <map>
#include <memory>
#include <vector>
#include <string>
#include <tuple>

#include "../../include/laminocam.h"
#include "lc_nufft.hpp"
#include "lc_solver.hpp"
#include "lc_toeplitz.hpp"

// A context handle shares its lc::Context with the geometries and PSFs made
// from it, so that those can still be destroyed (their device memory freed on
// the context's streams) after the context handle itself was destroyed.
struct lc_context_s {
    std::shared_ptr<lc::Context> ctx;
    std::string err;
    // worker contexts of lc_mbir2d_batch's setup, created on first use and
    // kept (with their streams) until this context is destroyed
    std::vector<std::unique_ptr<lc_context_s>> batch_workers;
};

struct lc_geometry_s {
    std::shared_ptr<lc::Context> keep;  // first member: released after the rest
    lc_context owner = nullptr;
    lc::PolarGeometry g;
    std::map<std::tuple<int, int, int, int>, std::unique_ptr<lc::NufftPlan>> plans;
    lc::DevBuf<float2> work;
};

struct lc_psf_s {
    std::shared_ptr<lc::Context> keep;  // first member: released after the rest
    lc_context owner = nullptr;
    lc_geometry geom = nullptr;
    std::shared_ptr<lc::Toeplitz> T;
    std::unique_ptr<lc::Solver> solver;
};

namespace lc {

// Supplies the Toeplitz operator of a reconstruction: either a new one or one
// that shares a cached spectrum.  `hit` is set when the spectrum was reused.
using PsfProvider = std::function<std::shared_ptr<Toeplitz>(Context &ctx, const PolarGeometry &g,
                                                            const long dims[3], bool three_d,
                                                            bool *hit)>;

// gpu::MBIR2D on a device sinogram {ns, ntheta, nradial}; drecon {ns, n, n}
void mbir2d_core(lc_context c, const float *dsino, int ns, int ntheta, int nradial,
                 const double *theta, const int *recon_dims, const lc_recon_params *p,
                 float *drecon, lc_solver_stats *stats, const PsfProvider *psf, bool *psf_hit);

// gpu::MBIR on device projections {ntheta, nrows, ncols}; drecon = recon_dims.
// load_input (optional) runs once the geometry and the PSF, which need only
// the angles, are queued: it starts filling dprojs and makes the context
// stream wait for it, so the upload overlaps the PSF construction.
void mbir3d_core(lc_context c, const float *dprojs, int ntheta, int nrows, int ncols,
                 const double *theta, const double *gamma, const double *beta, const float *shifts,
                 const int *recon_dims, const lc_recon_params *p, float *drecon,
                 lc_solver_stats *stats, const PsfProvider *psf, bool *psf_hit,
                 const std::function<void()> &load_input = {});

// body(load): load() copies n floats from host src into dst (allocated in the
// order of ctx.stream()) on the context's copy stream and makes ctx.stream()
// wait for them, so work the body queued before calling it overlaps the copy.
// On an exception the copy is finished before dst can be released.
void with_overlapped_upload(Context &ctx, float *dst, const float *src, long n,
                            const std::function<void(const std::function<void()> &)> &body);

// padded size of the reference: int(n * factor) in float, forced odd
long odd_pad(long n, float factor);

// Runs f and maps an exception to its C status code; the message goes to err.
template <typename F>
int run_guarded(std::string &err, F &&f) {
    try {
        f();
        return LC_OK;
    } catch (const Error &e) {
        err = e.what();
        if (err.find("out of memory") != std::string::npos) return LC_ERR_NOMEM;
        if (e.code == LC_ERR_TOO_LARGE) return LC_ERR_TOO_LARGE;
        return e.code == 1 ? LC_ERR_INVALID : (e.code == 3 ? LC_ERR_CUDA : LC_ERR_INTERNAL);
    } catch (const std::bad_alloc &) {
        err = "host allocation failed";
        return LC_ERR_NOMEM;
    } catch (const std::exception &e) {
        err = e.what();
        return LC_ERR_INTERNAL;
    }
}

// run_guarded on the context's device, recording the message in the context
template <typename F>
int guarded(lc_context c, F &&f) {
    if (!c) return LC_ERR_INVALID;
    return run_guarded(c->err, [&] {
        DeviceGuard dg(c->ctx->device());
        f();
    });
}

}  // namespace lc
