// Command-line driver around the reference's own C++ hot-path sources, compiled
// unmodified against the shim headers in ./shim.  TEST INFRASTRUCTURE ONLY: its
// outputs pin the numpy oracle (oracle/oracle.py) to the reference's code.
//
// Usage:  ref_driver <op> <in.f64> <out.f64>
// Input and output are flat little-endian float64 streams; integers are stored
// as float64 too.  Ops and their layouts are listed in run() below.
#include <array>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <iostream>
#include <stdexcept>
#include <string>
#include <vector>

#include "array.h"
#include "bregman.h"
#include "optimize.h"
#include "polar_grid.h"
#include "polar_grid2d.h"
#include "projection.h"
#include "recon_params.h"
#include "toeplitz.h"
#include "toeplitz2d.h"
#include "tomocam.h"

using namespace tomocam;

#ifdef LC_GPU_STENCIL
#include "gpu_stencil.h"
#endif

struct Reader {
    std::vector<double> v;
    size_t pos = 0;
    explicit Reader(const char *path) {
        std::ifstream f(path, std::ios::binary | std::ios::ate);
        if (!f) throw std::runtime_error("cannot open input");
        size_t n = (size_t)f.tellg() / sizeof(double);
        f.seekg(0);
        v.resize(n);
        f.read((char *)v.data(), n * sizeof(double));
    }
    double d() { return v.at(pos++); }
    size_t i() { return (size_t)v.at(pos++); }
    std::vector<double> vec(size_t n) {
        std::vector<double> out(v.begin() + pos, v.begin() + pos + n);
        pos += n;
        return out;
    }
    Array<double> arr(dims_t dims) {
        Array<double> a(dims);
        for (size_t k = 0; k < dims.size(); ++k) a[k] = v.at(pos++);
        return a;
    }
};

struct Writer {
    std::vector<double> v;
    void put(double x) { v.push_back(x); }
    void put(const Array<double> &a) {
        for (size_t k = 0; k < a.size(); ++k) v.push_back(a[k]);
    }
    void put(const Array<std::complex<double>> &a) {
        for (size_t k = 0; k < a.size(); ++k) {
            v.push_back(a[k].real());
            v.push_back(a[k].imag());
        }
    }
    void save(const char *path) {
        std::ofstream f(path, std::ios::binary);
        f.write((const char *)v.data(), v.size() * sizeof(double));
    }
};

static void run(const std::string &op, Reader &r, Writer &w) {
    if (op == "forward2d") {  // ns n2 n3 nth nr theta[nth] vol
        size_t ns = r.i(), n2 = r.i(), n3 = r.i(), nth = r.i(), nr = r.i();
        auto th = r.vec(nth);
        auto vol = r.arr({ns, n2, n3});
        cpu::PolarGrid2D<double> pg(th, nr);
        w.put(forward2d(vol, pg));
    } else if (op == "backproj2d") {  // ns nth nr n2 n3 theta sino
        size_t ns = r.i(), nth = r.i(), nr = r.i(), n2 = r.i(), n3 = r.i();
        auto th = r.vec(nth);
        auto sino = r.arr({ns, nth, nr});
        cpu::PolarGrid2D<double> pg(th, nr);
        w.put(backproj2d(sino, pg, dims_t{ns, n2, n3}));
    } else if (op == "psf2d") {  // nth nr n theta x(ns n n) -> P, khat, conv(x)
        size_t nth = r.i(), nr = r.i(), n = r.i(), ns = r.i();
        auto th = r.vec(nth);
        auto x = r.arr({ns, n, n});
        cpu::PolarGrid2D<double> pg(th, nr);
        cpu::PointSpreadFunction2D<double> psf(pg, n);
        w.put((double)psf.psf_size());
        w.put(psf.kernel_hat());
        w.put(sysmat2d(x, psf));
        w.put(sysmat2d(x, pg));
    } else if (op == "mbir2d") {  // ns nth nr n method iters tol xtol lam mu inner theta sino
        size_t ns = r.i(), nth = r.i(), nr = r.i(), n = r.i(), method = r.i(), iters = r.i();
        double tol = r.d(), xtol = r.d(), lam = r.d(), mu = r.d();
        size_t inner = r.i();
        auto th = r.vec(nth);
        auto sino = r.arr({ns, nth, nr});
        dims_t rd{ns, n, n};
        cpu::PolarGrid2D<double> pg(th, nr);
        cpu::PointSpreadFunction2D<double> psf(pg, n);
        opt::Function<double> A = [&psf](const Array<double> &x) { return sysmat2d(x, psf); };
        auto rhs = backproj2d(sino, pg, rd);
        auto x0 = Array<double>::zeros(rd);
        if (method == 0)
            w.put(opt::cgsolver<double>(A, rhs, x0, iters, tol, xtol));
        else
            w.put(opt::split_bregman<double>(A, rhs, x0, lam, mu, iters, inner, tol, xtol));
    } else if (op == "grad") {  // n1 n2 n3 u -> grad[3], divergence(grad)
        size_t n1 = r.i(), n2 = r.i(), n3 = r.i();
        auto u = r.arr({n1, n2, n3});
        auto g = opt::grad_u(u);
        for (int a = 0; a < 3; ++a) w.put(g[a]);
        w.put(opt::divergence(g));
    } else if (op == "proj3d") {  // nth nrows ncols n1 n2 n3 theta gamma beta shifts(2*nth) vol proj
        size_t nth = r.i(), nrows = r.i(), ncols = r.i(), n1 = r.i(), n2 = r.i(), n3 = r.i();
        auto th = r.vec(nth), ga = r.vec(nth), be = r.vec(nth), sh = r.vec(2 * nth);
        auto vol = r.arr({n1, n2, n3});
        auto proj = r.arr({nth, nrows, ncols});
        std::vector<std::array<double, 2>> shifts(nth);
        for (size_t k = 0; k < nth; ++k) shifts[k] = {sh[2 * k], sh[2 * k + 1]};
        cpu::PolarGrid<double> pg(th, ga, be, nrows, ncols);
        w.put(forward(vol, pg));
        w.put(backproj(proj, pg, dims_t{n1, n2, n3}));
        w.put(backproj(proj, pg, dims_t{n1, n2, n3}, shifts));
        w.put(sysmat(vol, pg));
        cpu::PointSpreadFunction<double> psf(pg, dims_t{n1, n2, n3});
        w.put((double)psf.dims().n1);
        w.put((double)psf.dims().n2);
        w.put((double)psf.dims().n3);
        w.put(psf.kernel_hat());
        w.put(sysmat(vol, psf));
    } else if (op == "mbir3d") {  // nth nrows ncols r1 r2 r3 method iters tol xtol lam mu inner gamma beta theta projs
        size_t nth = r.i(), nrows = r.i(), ncols = r.i(), r1 = r.i(), r2 = r.i(), r3 = r.i();
        size_t method = r.i(), iters = r.i();
        double tol = r.d(), xtol = r.d(), lam = r.d(), mu = r.d();
        size_t inner = r.i();
        double gamma = r.d(), beta = r.d();
        auto th = r.vec(nth);
        auto projs = r.arr({nth, nrows, ncols});
        Dataset_t<double> ds{std::move(projs), th, gamma, beta,
                             std::vector<std::array<double, 2>>(nth, {0.0, 0.0})};
        ReconParams p;
        p.regularizer = method == 0 ? Regularizer::UNCONSTRAINED : Regularizer::SPLIT_BREGMAN;
        p.recon_dims = {r1, r2, r3};
        p.maxIters = iters;
        p.innerIters = inner;
        p.lambda = (float)lam;
        p.mu = (float)mu;
        p.tol = (float)tol;
        p.xtol = (float)xtol;
        std::vector<Dataset_t<double>> dss;
        dss.push_back(std::move(ds));
        w.put(MBIR<double>(dss, p));
    } else {
        throw std::runtime_error("unknown op " + op);
    }
}

int main(int argc, char **argv) {
    if (argc != 4) {
        std::fprintf(stderr, "usage: %s <op> <in> <out>\n", argv[0]);
        return 2;
    }
    try {
        std::cout.setstate(std::ios::failbit);  // silence per-iteration logging
        Reader r(argv[2]);
        Writer w;
        run(argv[1], r, w);
        w.save(argv[3]);
    } catch (const std::exception &e) {
        std::fprintf(stderr, "ref_driver: %s\n", e.what());
        return 1;
    }
    return 0;
}
