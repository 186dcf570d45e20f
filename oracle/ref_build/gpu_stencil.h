// Zero-padded central differences of the reference's GPU build
// (src/gpu/finitediff.cu:28-133), restated in plain C++ so that the unmodified
// src/bregman.cpp runs with the production (GPU) boundary semantics on the
// CPU.  TEST INFRASTRUCTURE ONLY; included by the reference drivers built with
// -DLC_GPU_STENCIL in place of src/finitediff.cpp.
#pragma once

#include <array>

#include "array.h"
#include "bregman.h"

// grad = [d/dn3, d/dn2, d/dn1], divergence = the matching sum.
namespace tomocam::opt {
    template <typename T>
    static T at(const Array<T> &u, long i, long j, long k) {
        if (i < 0 || j < 0 || k < 0 || i >= (long)u.nslices() || j >= (long)u.nrows() ||
            k >= (long)u.ncols())
            return T(0);
        return u[{(size_t)i, (size_t)j, (size_t)k}];
    }
    template <typename T>
    std::array<Array<T>, 3> grad_u(const Array<T> &u) {
        std::array<Array<T>, 3> g;
        for (int a = 0; a < 3; ++a) g[a] = Array<T>::zeros(u.dims());
        for (long i = 0; i < (long)u.nslices(); ++i)
            for (long j = 0; j < (long)u.nrows(); ++j)
                for (long k = 0; k < (long)u.ncols(); ++k) {
                    dims_t id{(size_t)i, (size_t)j, (size_t)k};
                    g[0][id] = T(0.5) * (at(u, i, j, k + 1) - at(u, i, j, k - 1));
                    g[1][id] = T(0.5) * (at(u, i, j + 1, k) - at(u, i, j - 1, k));
                    g[2][id] = T(0.5) * (at(u, i + 1, j, k) - at(u, i - 1, j, k));
                }
        return g;
    }
    template <typename T>
    Array<T> divergence(const std::array<Array<T>, 3> &du) {
        Array<T> d = Array<T>::zeros(du[0].dims());
        for (long i = 0; i < (long)d.nslices(); ++i)
            for (long j = 0; j < (long)d.nrows(); ++j)
                for (long k = 0; k < (long)d.ncols(); ++k) {
                    dims_t id{(size_t)i, (size_t)j, (size_t)k};
                    d[id] = T(0.5) * (at(du[0], i, j, k + 1) - at(du[0], i, j, k - 1)) +
                            T(0.5) * (at(du[1], i, j + 1, k) - at(du[1], i, j - 1, k)) +
                            T(0.5) * (at(du[2], i + 1, j, k) - at(du[2], i - 1, j, k));
                }
        return d;
    }
    template std::array<Array<double>, 3> grad_u(const Array<double> &);
    template Array<double> divergence(const std::array<Array<double>, 3> &);
    template std::array<Array<float>, 3> grad_u(const Array<float> &);
    template Array<float> divergence(const std::array<Array<float>, 3> &);
} // namespace tomocam::opt
