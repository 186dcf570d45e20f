// Timing driver around the reference's own C++ hot-path sources (src/projection.cpp,
// src/gradient.cpp, src/conjgrad.cpp, src/bregman.cpp, src/finitediff.cpp,
// src/mbir.cpp, include/toeplitz.h), compiled unmodified against the fast shim
// headers in ./shim_fast (multithreaded FFT and ES-kernel NUFFT standing in for
// FFTW and FINUFFT).  TEST INFRASTRUCTURE ONLY: it gives bench.py's CPU
// baseline (the reference arm) and checks its own shims.
//
//   ref_bench check_fft   <in.f64> <out.f64>   FFTW-shim transform (tests)
//   ref_bench check_nufft <in.f64> <out.f64>   FINUFFT-shim transform (tests)
//   ref_bench lamino <phantom.f32> <n1> <n2> <n3> <nangles> <gamma_deg> <warmup> <steps> [full]
//   ref_prec  forward2d[_f32]  <in.f64> <out.f64>    forward2d in double (FINUFFT
//                                                    tol 1e-12) or float (5e-4)
//   ref_prec  precision2d[_f32] <in.f64> <out.f64>   backproj2d, sysmat2d(x, PSF), CG and
//                                                    Split-Bregman in double or float,
//                                                    for the precision study
// (ref_prec is this file built with -DLC_GPU_STENCIL: the zero-padded finite
// differences of the reference's GPU build, gpu_stencil.h, in place of
// src/finitediff.cpp, whose interior-only stencil vanishes on single slices.)
//
// lamino: the laminography Split-Bregman workload in float, the reference's
// CPU precision.  Projections are the reference's own forward() of the given
// phantom plus 1% Gaussian noise (not timed).  Then, timed and printed as one
// JSON line each:
//   setup  the steps of tomocam::MBIR before its solver (src/mbir.cpp:103-131):
//          max normalisation, sqrt(2) padding, polar grid, backprojection and
//          the PSF (NUFFT of ones + R2C FFT), with the reference's own calls;
//   outer  one Split-Bregman outer iteration (opt::split_bregman with
//          outer_max = 1, inner 1, lambda 0.1, mu 10): warmup untimed, then
//          `steps` timed;
//   full   (optional) one complete tomocam::MBIR with 100 outer iterations.
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <iostream>
#include <random>
#include <stdexcept>
#include <string>
#include <vector>

#include "array.h"
#include "array_ops.h"
#include "fftw3.h"
#include "finufft.h"
#include "optimize.h"
#include "padding.h"
#include "polar_grid.h"
#include "projection.h"
#include "recon_params.h"
#include "toeplitz.h"
#include "tomocam.h"
#include "toeplitz2d.h"
#ifdef LC_GPU_STENCIL
#include "gpu_stencil.h"
#endif

using namespace tomocam;

static std::vector<double> read_f64(const char *path) {
    std::ifstream f(path, std::ios::binary | std::ios::ate);
    if (!f) throw std::runtime_error("cannot open input");
    size_t n = (size_t)f.tellg() / sizeof(double);
    f.seekg(0);
    std::vector<double> v(n);
    f.read((char *)v.data(), n * sizeof(double));
    return v;
}

static void write_f64(const char *path, const std::vector<double> &v) {
    std::ofstream f(path, std::ios::binary);
    f.write((const char *)v.data(), v.size() * sizeof(double));
}

static double now_s() {
    return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

// kind precision rank dims... sign data -> out (complex as re, im pairs)
template <typename R>
static std::vector<double> check_fft_t(const std::vector<double> &v, size_t pos, int kind, int rank,
                                       const int *n, int sign) {
    long sz = 1;
    for (int d = 0; d < rank; ++d) sz *= n[d];
    const long nh = (long)n[rank - 1] / 2 + 1, hsz = sz / n[rank - 1] * nh;
    std::vector<double> out;
    if (kind == 0) {
        std::vector<std::complex<R>> a(sz);
        for (long i = 0; i < sz; ++i) a[i] = {(R)v[pos + 2 * i], (R)v[pos + 2 * i + 1]};
        lc_shim::Plan *p = lc_shim::make(rank, n, 1, (int)sz, (int)sz, sign, lc_shim::C2C);
        lc_shim::run_c2c<R>(*p, a.data(), a.data());
        delete p;
        for (auto c : a) { out.push_back(c.real()); out.push_back(c.imag()); }
    } else if (kind == 1) {
        std::vector<R> a(sz);
        for (long i = 0; i < sz; ++i) a[i] = (R)v[pos + i];
        std::vector<std::complex<R>> b(hsz);
        lc_shim::Plan *p = lc_shim::make(rank, n, 1, (int)sz, (int)hsz, -1, lc_shim::R2C);
        lc_shim::run_r2c<R>(*p, a.data(), b.data());
        delete p;
        for (auto c : b) { out.push_back(c.real()); out.push_back(c.imag()); }
    } else {
        std::vector<std::complex<R>> a(hsz);
        for (long i = 0; i < hsz; ++i) a[i] = {(R)v[pos + 2 * i], (R)v[pos + 2 * i + 1]};
        std::vector<R> b(sz);
        lc_shim::Plan *p = lc_shim::make(rank, n, 1, (int)hsz, (int)sz, +1, lc_shim::C2R);
        lc_shim::run_c2r<R>(*p, a.data(), b.data());
        delete p;
        for (auto c : b) out.push_back(c);
    }
    return out;
}

// type dim n1 n2 n3 iflag tol precision M x[M] y[M] z[M] data -> out
template <typename R>
static std::vector<double> check_nufft_t(const std::vector<double> &v, size_t pos, int type, int dim,
                                         int64_t *nm, int iflag, double tol, int64_t M) {
    std::vector<R> x(M), y(M), z(M);
    for (int64_t j = 0; j < M; ++j) x[j] = (R)v[pos + j];
    for (int64_t j = 0; j < M; ++j) y[j] = (R)v[pos + M + j];
    for (int64_t j = 0; j < M; ++j) z[j] = (R)v[pos + 2 * M + j];
    pos += 3 * M;
    const int64_t nmod = nm[0] * (dim > 1 ? nm[1] : 1) * (dim > 2 ? nm[2] : 1);
    std::vector<std::complex<R>> c(M), f(nmod);
    lc_shim::NuPlan p;
    lc_shim::init_plan(&p, type, dim, nm, iflag, tol);
    p.M = M;
    p.x = x.data();
    p.y = y.data();
    p.z = z.data();
    if (type == 1) {
        for (int64_t j = 0; j < M; ++j) c[j] = {(R)v[pos + 2 * j], (R)v[pos + 2 * j + 1]};
        lc_shim::make_schedule<R>(p);
    } else {
        for (int64_t k = 0; k < nmod; ++k) f[k] = {(R)v[pos + 2 * k], (R)v[pos + 2 * k + 1]};
    }
    lc_shim::nu_execute<R>(&p, c.data(), f.data());
    std::vector<double> out;
    for (auto a : (type == 1 ? f : c)) { out.push_back(a.real()); out.push_back(a.imag()); }
    return out;
}

// n nth nr theta[nth] vol[n n] -> sino[nth nr], in precision T (the FINUFFT
// tolerance of the reference for T: 1e-12 double, 5e-4 float)
template <typename T>
static std::vector<double> forward2d_op(const std::vector<double> &v, size_t pos) {
    const size_t n = (size_t)v[pos++], nth = (size_t)v[pos++], nr = (size_t)v[pos++];
    std::vector<T> th(nth);
    for (size_t i = 0; i < nth; ++i) th[i] = (T)v[pos + i];
    pos += nth;
    Array<T> vol(dims_t{1, n, n});
    for (size_t i = 0; i < n * n; ++i) vol[i] = (T)v[pos + i];
    cpu::PolarGrid2D<T> pg(th, nr);
    Array<T> s = forward2d(vol, pg);
    return std::vector<double>(s.begin(), s.end());
}

// n nth nr cg_iters sb_outer sb_inner lam mu theta[nth] sino[nth nr] xprobe[n n]
//   -> backproj2d rhs, sysmat2d(xprobe, PSF), CG recon, Split-Bregman recon
template <typename T>
static std::vector<double> precision2d_op(const std::vector<double> &v, size_t pos) {
    const size_t n = (size_t)v[pos++], nth = (size_t)v[pos++], nr = (size_t)v[pos++];
    const size_t cg_iters = (size_t)v[pos++], sb_outer = (size_t)v[pos++], sb_inner = (size_t)v[pos++];
    const T lam = (T)v[pos++], mu = (T)v[pos++];
    std::vector<T> th(nth);
    for (size_t i = 0; i < nth; ++i) th[i] = (T)v[pos + i];
    pos += nth;
    Array<T> sino(dims_t{1, nth, nr}), xp(dims_t{1, n, n});
    for (size_t i = 0; i < nth * nr; ++i) sino[i] = (T)v[pos + i];
    pos += nth * nr;
    for (size_t i = 0; i < n * n; ++i) xp[i] = (T)v[pos + i];
    cpu::PolarGrid2D<T> pg(th, nr);
    const dims_t rd{1, n, n};
    Array<T> rhs = backproj2d(sino, pg, rd);
    cpu::PointSpreadFunction2D<T> psf(pg, n);
    opt::Function<T> A = [&psf](const Array<T> &x) { return sysmat2d(x, psf); };
    Array<T> ax = A(xp);
    auto x0 = Array<T>::zeros(rd);
    Array<T> cg = opt::cgsolver<T>(A, rhs, x0, cg_iters, T(0), T(0));
    Array<T> sb = opt::split_bregman<T>(A, rhs, x0, lam, mu, sb_outer, sb_inner, T(0), T(0));
    std::vector<double> out;
    for (const Array<T> *a : {&rhs, &ax, &cg, &sb}) out.insert(out.end(), a->begin(), a->end());
    return out;
}

static int lamino(int argc, char **argv) {
    if (argc < 10) throw std::runtime_error("lamino: arguments missing");
    const char *phantom = argv[2];
    const size_t n1 = std::stoul(argv[3]), n2 = std::stoul(argv[4]), n3 = std::stoul(argv[5]);
    const size_t nang = std::stoul(argv[6]);
    const float gamma_deg = std::stof(argv[7]);
    const int warmup = std::stoi(argv[8]), steps = std::stoi(argv[9]);
    const bool full = argc > 10 && std::string(argv[10]) == "full";
    const float lam = 0.1f, mu = 10.0f, tol = 1e-5f, xtol = 0.0f;
    const size_t outer = 100, inner = 1;

    // phantom (float32, n1 x n2 x n3) -> projections by the reference's forward()
    Array<float> vol(dims_t{n1, n2, n3});
    {
        std::ifstream f(phantom, std::ios::binary);
        if (!f) throw std::runtime_error("cannot open phantom");
        f.read((char *)vol.begin(), vol.size() * sizeof(float));
    }
    std::vector<float> theta(nang), gamma(nang, -gamma_deg * (float)M_PI / 180.0f), beta(nang, 0.0f);
    for (size_t i = 0; i < nang; ++i) theta[i] = (float)(2.0 * M_PI * (double)i / (double)nang);
    double t0 = now_s();
    Array<float> projs;
    {
        cpu::PolarGrid<float> pg0(theta, gamma, beta, n2, n3);
        projs = forward(vol, pg0);
    }
    {
        std::mt19937_64 rng(2000);
        std::normal_distribution<float> nd(0.0f, 1.0f);
        const float sigma = 0.01f * array::max(projs);
        for (size_t i = 0; i < projs.size(); ++i) projs[i] += sigma * nd(rng);
    }
    std::printf("{\"phase\": \"data\", \"seconds\": %.3f}\n", now_s() - t0);
    std::fflush(stdout);

    ReconParams prm;
    prm.regularizer = Regularizer::SPLIT_BREGMAN;
    prm.recon_dims = {n1, n2, n3};
    prm.maxIters = outer;
    prm.innerIters = inner;
    prm.lambda = lam;
    prm.mu = mu;
    prm.tol = tol;
    prm.xtol = xtol;
    const float padfac = (float)prm.PAD_FACTOR;
    auto pad = [padfac](size_t n) {
        size_t p = (size_t)(n * padfac);
        return p % 2 == 0 ? p - 1 : p;
    };
    dims_t out_dims{pad(n1), pad(n2), pad(n3)};

    // setup: the calls of tomocam::MBIR before its solver (src/mbir.cpp:103-131)
    t0 = now_s();
    Array<float> work = projs.clone();
    float mx = array::max(work);
    if (mx > 0) work /= mx;
    work = pad2d(work, padfac, PadType::SYMMETRIC);
    cpu::PolarGrid<float> pg(theta, gamma, beta, work.nrows(), work.ncols());
    std::vector<std::array<float, 2>> shifts(nang, {0.0f, 0.0f});
    double tb = now_s();
    Array<float> yT = backproj(work, pg, out_dims, shifts);
    double tp = now_s();
    cpu::PointSpreadFunction<float> psf(pg, out_dims);
    double t1 = now_s();
    std::printf("{\"phase\": \"setup\", \"seconds\": %.3f, \"backproj_s\": %.3f, \"psf_s\": %.3f}\n", t1 - t0,
                tp - tb, t1 - tp);
    std::fflush(stdout);

    opt::Function<float> A = [&psf](const Array<float> &x) { return sysmat(x, psf); };
    Array<float> x = Array<float>::zeros(out_dims);
    for (int s = 0; s < warmup + steps; ++s) {
        double a = now_s();
        x = opt::split_bregman<float>(A, yT, x, lam, mu, 1, inner, tol, xtol);
        double b = now_s();
        std::printf("{\"phase\": \"%s\", \"seconds\": %.4f}\n", s < warmup ? "warmup" : "outer", b - a);
        std::fflush(stdout);
    }
    if (full) {
        std::vector<Dataset_t<float>> dss;
        dss.push_back(Dataset_t<float>{projs.clone(), theta, gamma[0], 0.0f,
                                       std::vector<std::array<float, 2>>(nang, {0.0f, 0.0f})});
        double a = now_s();
        Array<float> rec = MBIR<float>(dss, prm);
        double b = now_s();
        std::printf("{\"phase\": \"full\", \"seconds\": %.3f, \"outer_iters\": %zu}\n", b - a, outer);
        std::fflush(stdout);
    }
    return 0;
}

int main(int argc, char **argv) {
    if (argc < 2) {
        std::fprintf(stderr, "usage: %s check_fft|check_nufft|lamino ...\n", argv[0]);
        return 2;
    }
    try {
        const std::string op = argv[1];
        if (op != "check_fft" && op != "check_nufft") {
            // the reference prints per-iteration progress; keep stdout for the JSON lines
            std::cout.setstate(std::ios::failbit);
        }
        if (op == "lamino") {
            return lamino(argc, argv);
        }
        if (argc != 4) throw std::runtime_error("expected <in> <out>");
        auto v = read_f64(argv[2]);
        size_t pos = 0;
        std::vector<double> out;
        if (op == "check_fft") {
            int kind = (int)v[pos++], prec = (int)v[pos++], rank = (int)v[pos++];
            std::vector<int> n(rank);
            for (int d = 0; d < rank; ++d) n[d] = (int)v[pos++];
            int sign = (int)v[pos++];
            out = prec ? check_fft_t<double>(v, pos, kind, rank, n.data(), sign)
                       : check_fft_t<float>(v, pos, kind, rank, n.data(), sign);
        } else if (op == "forward2d" || op == "forward2d_f32") {
            out = op == "forward2d" ? forward2d_op<double>(v, pos) : forward2d_op<float>(v, pos);
        } else if (op == "precision2d" || op == "precision2d_f32") {
            out = op == "precision2d" ? precision2d_op<double>(v, pos) : precision2d_op<float>(v, pos);
        } else if (op == "check_nufft") {
            int type = (int)v[pos++], dim = (int)v[pos++];
            int64_t nm[3] = {(int64_t)v[pos], (int64_t)v[pos + 1], (int64_t)v[pos + 2]};
            pos += 3;
            int iflag = (int)v[pos++];
            double tol = v[pos++];
            int prec = (int)v[pos++];
            int64_t M = (int64_t)v[pos++];
            out = prec ? check_nufft_t<double>(v, pos, type, dim, nm, iflag, tol, M)
                       : check_nufft_t<float>(v, pos, type, dim, nm, iflag, tol, M);
        } else {
            throw std::runtime_error("unknown op " + op);
        }
        write_f64(argv[3], out);
    } catch (const std::exception &e) {
        std::fprintf(stderr, "ref_bench: %s\n", e.what());
        return 1;
    }
    return 0;
}
