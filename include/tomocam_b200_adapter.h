/* C++ adapter: the reference's reconstruction API over the laminocam_b200 C ABI.
 *
 * A LaminoCam maintainer includes this header, after the reference's array.h
 * and recon_params.h, in place of the CUDA sources of the tomocam library and
 * links liblaminocam_b200.so and the CUDA runtime.  It provides:
 *
 *   tomocam::gpu::MBIR2D<float>, tomocam::gpu::MBIR<float>
 *       definitions of the templates declared in include/gpu/tomocam.h:60-93
 *       (gpu::MBIR2D, src/gpu/mbir2d.cu:36-85; gpu::MBIR, src/gpu/mbir.cu:41-167),
 *       so that src/mbir2d.cpp and src/recon.cpp build unchanged;
 *   tomocam::b200::{forward2d, backproj2d, sysmat2d, forward, backproj, sysmat}
 *       the operators of include/projection.h:38-68 on host Array<float>s,
 *       with the geometry and PSF types below in place of cpu::PolarGrid{,2D}
 *       and cpu::PointSpreadFunction{,2D} (include/toeplitz.h:54-129,
 *       include/toeplitz2d.h:71-125);
 *   tomocam::b200::opt::{cgsolver, split_bregman}
 *       opt::cgsolver / opt::split_bregman (include/optimize.h:74-91) over a
 *       B200 PSF (the whole solve on the device) or over any
 *       tomocam::opt::Function<float> (applied on the host each iteration).
 *
 * Status codes become std::runtime_error with the library's message, as the
 * reference's SAFE_CALL does (include/gpu/utils.h:31-39).  The path is
 * float32 (the reference GPU path's precision); the templates accept T = float
 * only.  One process-wide context on the current device serves every call; it
 * is not thread-safe, like the reference's plan caches
 * (include/gpu/multigpu.h:123-126). */
#ifndef TOMOCAM_B200_ADAPTER_H
#define TOMOCAM_B200_ADAPTER_H

#include <cuda_runtime.h>

#include <array>
#include <functional>
#include <stdexcept>
#include <string>
#include <type_traits>
#include <vector>

#include "array.h"
#include "laminocam.h"
#include "recon_params.h"

namespace tomocam::b200 {

    inline lc_context context() {
        static lc_context ctx = [] {
            int dev = 0;
            cudaGetDevice(&dev);
            lc_context c = nullptr;
            if (lc_context_create(dev, nullptr, &c) != LC_OK)
                throw std::runtime_error("laminocam_b200: no CUDA device");
            return c;
        }();
        return ctx;
    }

    inline void check(int rc) {
        if (rc != LC_OK) throw std::runtime_error(std::string("laminocam_b200: ") + lc_last_error(context()));
    }

    inline void check_cuda(cudaError_t e) {
        if (e != cudaSuccess) throw std::runtime_error(std::string("laminocam_b200: ") + cudaGetErrorString(e));
    }

    inline lc_recon_params params(const ReconParams &p) {
        lc_recon_params r;
        lc_recon_params_default(&r);
        r.method = p.regularizer == Regularizer::SPLIT_BREGMAN ? 1 : 0;
        r.solver.max_iters = (int)p.maxIters;
        r.solver.inner_iters = (int)p.innerIters;
        r.solver.tol = p.tol;
        r.solver.xtol = p.xtol;
        r.solver.lambda = p.lambda;
        r.solver.mu = p.mu;
        r.pad_factor = p.PAD_FACTOR;
        return r;
    }

    // device copy of a host array (owned, freed on destruction)
    class DeviceBuffer {
      public:
        explicit DeviceBuffer(size_t n) : n_(n) {
            if (n) check_cuda(cudaMalloc(&p_, n * sizeof(float)));
        }
        DeviceBuffer(const float *host, size_t n) : DeviceBuffer(n) {
            if (n) check_cuda(cudaMemcpy(p_, host, n * sizeof(float), cudaMemcpyHostToDevice));
        }
        ~DeviceBuffer() {
            if (p_) cudaFree(p_);
        }
        DeviceBuffer(const DeviceBuffer &) = delete;
        DeviceBuffer &operator=(const DeviceBuffer &) = delete;
        float *get() const { return p_; }
        void to_host(float *host) const {
            // the library's work is ordered on the context's stream
            check(lc_context_synchronize(context()));
            check_cuda(cudaMemcpy(host, p_, n_ * sizeof(float), cudaMemcpyDeviceToHost));
        }

      private:
        float *p_ = nullptr;
        size_t n_ = 0;
    };

    template <typename T>
    void require_float() {
        static_assert(std::is_same_v<T, float>, "the laminocam_b200 path is float32");
    }

    // cpu::PolarGrid2D (include/polar_grid2d.h:35-66): angles in radians, ncols radial samples
    class PolarGrid2D {
      public:
        PolarGrid2D(const std::vector<float> &theta, size_t ncols) : ntheta_(theta.size()), ncols_(ncols) {
            std::vector<double> th(theta.begin(), theta.end());
            check(lc_geometry2d_create(context(), th.data(), (int)th.size(), (int)ncols, &g_));
        }
        ~PolarGrid2D() {
            if (g_) lc_geometry_destroy(g_);
        }
        PolarGrid2D(const PolarGrid2D &) = delete;
        PolarGrid2D &operator=(const PolarGrid2D &) = delete;
        lc_geometry handle() const { return g_; }
        size_t ntheta() const { return ntheta_; }
        size_t ncols() const { return ncols_; }

      private:
        lc_geometry g_ = nullptr;
        size_t ntheta_, ncols_;
    };

    // cpu::PolarGrid (include/polar_grid.h:34-95) plus per-projection shifts
    class PolarGrid {
      public:
        PolarGrid(const std::vector<float> &theta, const std::vector<float> &gamma, const std::vector<float> &beta,
                  size_t nrows, size_t ncols, const std::vector<std::array<float, 2>> &shifts = {})
            : ntheta_(theta.size()), nrows_(nrows), ncols_(ncols) {
            std::vector<double> th(theta.begin(), theta.end()), ga(gamma.begin(), gamma.end()),
                be(beta.begin(), beta.end());
            std::vector<float> sh;
            for (const auto &s : shifts) {
                sh.push_back(s[0]);
                sh.push_back(s[1]);
            }
            check(lc_geometry3d_create(context(), th.data(), ga.data(), be.data(), sh.empty() ? nullptr : sh.data(),
                                       (int)th.size(), (int)nrows, (int)ncols, &g_));
        }
        ~PolarGrid() {
            if (g_) lc_geometry_destroy(g_);
        }
        PolarGrid(const PolarGrid &) = delete;
        PolarGrid &operator=(const PolarGrid &) = delete;
        lc_geometry handle() const { return g_; }
        size_t ntheta() const { return ntheta_; }
        size_t nrows() const { return nrows_; }
        size_t ncols() const { return ncols_; }

      private:
        lc_geometry g_ = nullptr;
        size_t ntheta_, nrows_, ncols_;
    };

    // cpu::PointSpreadFunction{,2D}: the Toeplitz operator A^T A of a geometry
    class PointSpreadFunction {
      public:
        PointSpreadFunction(const PolarGrid2D &g, size_t image_size, size_t nslices = 1)
            : dims_(nslices, image_size, image_size) {
            check(lc_psf_create(context(), g.handle(), (int)nslices, (int)image_size, (int)image_size, &p_));
        }
        PointSpreadFunction(const PolarGrid &g, dims_t recon_dims) : dims_(recon_dims) {
            check(lc_psf_create(context(), g.handle(), (int)recon_dims.n1, (int)recon_dims.n2, (int)recon_dims.n3,
                                &p_));
        }
        ~PointSpreadFunction() {
            if (p_) lc_psf_destroy(p_);
        }
        PointSpreadFunction(const PointSpreadFunction &) = delete;
        PointSpreadFunction &operator=(const PointSpreadFunction &) = delete;
        lc_psf handle() const { return p_; }
        dims_t dims() const { return dims_; }

        // PointSpreadFunction::convolve (include/toeplitz.h:95-129)
        Array<float> convolve(const Array<float> &x) const {
            if (!(x.dims() == dims_)) throw std::invalid_argument("convolve: input dims differ from the PSF's");
            DeviceBuffer in(x.data(), x.size()), out(x.size());
            check(lc_sysmat_toeplitz(context(), p_, in.get(), out.get()));
            Array<float> y(dims_);
            out.to_host(y.data());
            return y;
        }

      private:
        lc_psf p_ = nullptr;
        dims_t dims_;
    };

    // forward2d / backproj2d / sysmat2d (include/projection.h:57-68)
    inline Array<float> forward2d(const Array<float> &vol, const PolarGrid2D &g, double tol = 0.0) {
        DeviceBuffer in(vol.data(), vol.size()), out(vol.nslices() * g.ntheta() * g.ncols());
        check(lc_forward2d(context(), g.handle(), in.get(), (int)vol.nslices(), (int)vol.nrows(), (int)vol.ncols(),
                           out.get(), tol));
        Array<float> s(dims_t{vol.nslices(), g.ntheta(), g.ncols()});
        out.to_host(s.data());
        return s;
    }

    inline Array<float> backproj2d(const Array<float> &sino, const PolarGrid2D &g, const dims_t &recon_dims,
                                   double tol = 0.0) {
        DeviceBuffer in(sino.data(), sino.size()), out(recon_dims.n1 * recon_dims.n2 * recon_dims.n3);
        check(lc_backproj2d(context(), g.handle(), in.get(), (int)recon_dims.n1, (int)recon_dims.n2,
                            (int)recon_dims.n3, out.get(), tol));
        Array<float> v(recon_dims);
        out.to_host(v.data());
        return v;
    }

    inline Array<float> sysmat2d(const Array<float> &x, const PolarGrid2D &g, double tol = 0.0) {
        DeviceBuffer in(x.data(), x.size()), out(x.size());
        check(lc_sysmat2d_nufft(context(), g.handle(), in.get(), (int)x.nslices(), (int)x.nrows(), (int)x.ncols(),
                                out.get(), tol));
        Array<float> y(x.dims());
        out.to_host(y.data());
        return y;
    }

    inline Array<float> sysmat2d(const Array<float> &x, const PointSpreadFunction &psf) { return psf.convolve(x); }

    // forward / backproj (+ shifts) / sysmat (include/projection.h:38-55)
    inline Array<float> forward(const Array<float> &vol, const PolarGrid &g, double tol = 0.0) {
        DeviceBuffer in(vol.data(), vol.size()), out(g.ntheta() * g.nrows() * g.ncols());
        check(lc_forward3d(context(), g.handle(), in.get(), (int)vol.nslices(), (int)vol.nrows(), (int)vol.ncols(),
                           out.get(), tol));
        Array<float> p(dims_t{g.ntheta(), g.nrows(), g.ncols()});
        out.to_host(p.data());
        return p;
    }

    inline Array<float> backproj(const Array<float> &proj, const PolarGrid &g, const dims_t &dims,
                                 bool apply_shifts = false, double tol = 0.0) {
        DeviceBuffer in(proj.data(), proj.size()), out(dims.n1 * dims.n2 * dims.n3);
        check(lc_backproj3d(context(), g.handle(), in.get(), (int)dims.n1, (int)dims.n2, (int)dims.n3,
                            apply_shifts ? 1 : 0, out.get(), tol));
        Array<float> v(dims);
        out.to_host(v.data());
        return v;
    }

    inline Array<float> sysmat(const Array<float> &x, const PolarGrid &g, double tol = 0.0) {
        DeviceBuffer in(x.data(), x.size()), out(x.size());
        check(lc_sysmat3d_nufft(context(), g.handle(), in.get(), (int)x.nslices(), (int)x.nrows(), (int)x.ncols(),
                                out.get(), tol));
        Array<float> y(x.dims());
        out.to_host(y.data());
        return y;
    }

    inline Array<float> sysmat(const Array<float> &x, const PointSpreadFunction &psf) { return psf.convolve(x); }

    namespace opt {

        inline lc_solver_params solver_params(size_t iters, size_t inner, float tol, float xtol, float lam, float mu) {
            lc_solver_params p;
            lc_solver_params_default(&p);
            p.max_iters = (int)iters;
            p.inner_iters = (int)inner;
            p.tol = tol;
            p.xtol = xtol;
            p.lambda = lam;
            p.mu = mu;
            return p;
        }

        // opt::cgsolver over a B200 PSF: every iteration stays on the device
        inline Array<float> cgsolver(const PointSpreadFunction &A, const Array<float> &y, const Array<float> &x0,
                                     size_t max_iter, float tol, float xtol) {
            DeviceBuffer dy(y.data(), y.size()), dx(x0.data(), x0.size());
            lc_solver_params p = solver_params(max_iter, 1, tol, xtol, 0.0f, 1.0f);
            check(lc_cgsolver(context(), A.handle(), dy.get(), dx.get(), &p, nullptr));
            Array<float> x(x0.dims());
            dx.to_host(x.data());
            return x;
        }

        inline Array<float> split_bregman(const PointSpreadFunction &A, const Array<float> &yT, const Array<float> &x0,
                                          float lambda, float mu, size_t outer_max, size_t inner_max, float tol,
                                          float xtol) {
            DeviceBuffer dy(yT.data(), yT.size()), dx(x0.data(), x0.size());
            lc_solver_params p = solver_params(outer_max, inner_max, tol, xtol, lambda, mu);
            check(lc_split_bregman(context(), A.handle(), dy.get(), dx.get(), &p, nullptr));
            Array<float> x(x0.dims());
            dx.to_host(x.data());
            return x;
        }

        // An opt::Function<float> applied on the host: each call copies the
        // device vector out, applies the function and copies the result in.
        struct HostOperator {
            const std::function<Array<float>(const Array<float> &)> *f;
            dims_t dims;
            std::string error;
        };

        inline int host_operator(void *user, const float *in, float *out, long n, void *stream) {
            auto *h = static_cast<HostOperator *>(user);
            try {
                Array<float> x(h->dims);
                cudaStream_t s = static_cast<cudaStream_t>(stream);
                check_cuda(cudaMemcpyAsync(x.data(), in, n * sizeof(float), cudaMemcpyDeviceToHost, s));
                check_cuda(cudaStreamSynchronize(s));
                Array<float> y = (*h->f)(x);
                if (y.size() != (size_t)n) throw std::invalid_argument("operator changed the vector size");
                check_cuda(cudaMemcpyAsync(out, y.data(), n * sizeof(float), cudaMemcpyHostToDevice, s));
                check_cuda(cudaStreamSynchronize(s));
                return 0;
            } catch (const std::exception &e) {
                h->error = e.what();
                return 1;
            }
        }

        inline Array<float> cgsolver(const std::function<Array<float>(const Array<float> &)> &A,
                                     const Array<float> &y, const Array<float> &x0, size_t max_iter, float tol,
                                     float xtol) {
            DeviceBuffer dy(y.data(), y.size()), dx(x0.data(), x0.size());
            lc_solver_params p = solver_params(max_iter, 1, tol, xtol, 0.0f, 1.0f);
            HostOperator h{&A, y.dims(), {}};
            const int rc = lc_cgsolver_op(context(), host_operator, &h, (long)y.size(), dy.get(), dx.get(), &p, nullptr);
            if (!h.error.empty()) throw std::runtime_error(h.error);
            check(rc);
            Array<float> x(x0.dims());
            dx.to_host(x.data());
            return x;
        }

        inline Array<float> split_bregman(const std::function<Array<float>(const Array<float> &)> &A,
                                          const Array<float> &yT, const Array<float> &x0, float lambda, float mu,
                                          size_t outer_max, size_t inner_max, float tol, float xtol) {
            DeviceBuffer dy(yT.data(), yT.size()), dx(x0.data(), x0.size());
            lc_solver_params p = solver_params(outer_max, inner_max, tol, xtol, lambda, mu);
            HostOperator h{&A, yT.dims(), {}};
            const int dims[3] = {(int)yT.nslices(), (int)yT.nrows(), (int)yT.ncols()};
            const int rc = lc_split_bregman_op(context(), host_operator, &h, dims, dy.get(), dx.get(), &p, nullptr);
            if (!h.error.empty()) throw std::runtime_error(h.error);
            check(rc);
            Array<float> x(x0.dims());
            dx.to_host(x.data());
            return x;
        }

    } // namespace opt

} // namespace tomocam::b200

namespace tomocam::gpu {

    // gpu::MBIR2D (include/gpu/tomocam.h:72-74, src/gpu/mbir2d.cu:36-85) on a
    // prepared sinogram {n_slices, n_angles, n_cols}
    template <typename T>
    Array<T> MBIR2D(const Array<T> &sinogram, const std::vector<T> &theta, const ReconParams &params) {
        b200::require_float<T>();
        std::vector<double> th(theta.begin(), theta.end());
        int rd[3] = {(int)params.recon_dims[0], (int)params.recon_dims[1], (int)params.recon_dims[2]};
        Array<T> out(dims_t{params.recon_dims[0], params.recon_dims[1], params.recon_dims[2]});
        lc_recon_params r = b200::params(params);
        b200::check(lc_mbir2d(b200::context(), sinogram.data(), (int)sinogram.nslices(), (int)sinogram.nrows(),
                              (int)sinogram.ncols(), th.data(), rd, &r, out.data(), nullptr));
        return out;
    }

    // gpu::MBIR (include/gpu/tomocam.h:60-62, src/gpu/mbir.cu:41-167): the
    // datasets are stacked along the angle axis as the reference does
    template <typename T>
    Array<T> MBIR(const std::vector<Dataset_t<T>> &datasets, const ReconParams &params) {
        b200::require_float<T>();
        if (datasets.empty()) throw std::invalid_argument("MBIR: no datasets");
        std::vector<float> projs;
        std::vector<double> th, ga, be;
        std::vector<float> sh;
        const size_t nrows = datasets[0].projs.nrows(), ncols = datasets[0].projs.ncols();
        bool shifts = false;
        for (const auto &d : datasets) {
            if (d.projs.nrows() != nrows || d.projs.ncols() != ncols)
                throw std::invalid_argument("MBIR: datasets differ in detector size");
            projs.insert(projs.end(), d.projs.data(), d.projs.data() + d.projs.size());
            for (size_t i = 0; i < d.angles.size(); ++i) {
                th.push_back(d.angles[i]);
                ga.push_back(d.gamma);
                be.push_back(d.beta);
                const float dx = i < d.shifts.size() ? d.shifts[i][0] : 0.0f;
                const float dy = i < d.shifts.size() ? d.shifts[i][1] : 0.0f;
                shifts = shifts || dx != 0.0f || dy != 0.0f;
                sh.push_back(dx);
                sh.push_back(dy);
            }
        }
        int rd[3] = {(int)params.recon_dims[0], (int)params.recon_dims[1], (int)params.recon_dims[2]};
        Array<T> out(dims_t{params.recon_dims[0], params.recon_dims[1], params.recon_dims[2]});
        lc_recon_params r = b200::params(params);
        b200::check(lc_mbir3d(b200::context(), projs.data(), (int)th.size(), (int)nrows, (int)ncols, th.data(),
                              ga.data(), be.data(), shifts ? sh.data() : nullptr, rd, &r, out.data(), nullptr));
        return out;
    }

} // namespace tomocam::gpu

#endif
