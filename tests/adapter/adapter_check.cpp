// Check program for include/tomocam_b200_adapter.h, compiled against the
// reference's own headers (array.h, recon_params.h, optimize.h): it runs the
// reference-shaped API over the B200 library and writes the results for
// tests/test_adapter.py to compare.
//
//   adapter_check <in.f64> <out.f64>
// in:  n nth theta[nth] sino[nth n] vol[n n]   (one slice)
// out: forward2d(vol), backproj2d(sino), PSF convolve(vol),
//      gpu::MBIR2D CG(5), opt::cgsolver(Function, 5) on the NUFFT normal operator
#include <fstream>
#include <iostream>
#include <vector>

#include "array.h"
#include "optimize.h"
#include "recon_params.h"
#include "tomocam_b200_adapter.h"

using namespace tomocam;

int main(int argc, char **argv) {
    if (argc != 3) {
        std::cerr << "usage: adapter_check <in.f64> <out.f64>\n";
        return 2;
    }
    try {
        std::ifstream f(argv[1], std::ios::binary | std::ios::ate);
        std::vector<double> v((size_t)f.tellg() / sizeof(double));
        f.seekg(0);
        f.read((char *)v.data(), v.size() * sizeof(double));
        size_t pos = 0;
        const size_t n = (size_t)v[pos++], nth = (size_t)v[pos++];
        std::vector<float> theta(nth);
        for (auto &t : theta) t = (float)v[pos++];
        Array<float> sino(dims_t{1, nth, n}), vol(dims_t{1, n, n});
        for (size_t i = 0; i < sino.size(); ++i) sino[i] = (float)v[pos++];
        for (size_t i = 0; i < vol.size(); ++i) vol[i] = (float)v[pos++];

        b200::PolarGrid2D pg(theta, n);
        Array<float> fw = b200::forward2d(vol, pg);
        Array<float> bp = b200::backproj2d(sino, pg, dims_t{1, n, n});
        b200::PointSpreadFunction psf(pg, n);
        Array<float> ax = psf.convolve(vol);
        ReconParams p;
        p.regularizer = Regularizer::UNCONSTRAINED;
        p.recon_dims = {1, n, n};
        p.maxIters = 5;
        p.tol = 0.0f;
        p.xtol = 0.0f;
        Array<float> rec = gpu::MBIR2D<float>(sino, theta, p);
        opt::Function<float> A = [&pg](const Array<float> &x) { return b200::sysmat2d(x, pg); };
        Array<float> cg = b200::opt::cgsolver(A, bp, Array<float>::zeros(dims_t{1, n, n}), 5, 0.0f, 0.0f);

        std::vector<double> out;
        for (const Array<float> *a : {&fw, &bp, &ax, &rec, &cg})
            for (size_t i = 0; i < a->size(); ++i) out.push_back((*a)[i]);
        std::ofstream o(argv[2], std::ios::binary);
        o.write((const char *)out.data(), out.size() * sizeof(double));
    } catch (const std::exception &e) {
        std::cerr << "adapter_check: " << e.what() << "\n";
        return 1;
    }
    return 0;
}
