/* Self-written stand-in for the subset of the FFTW3 API that the LaminoCam
 * reference calls (include/fftw_plan.h:43-197), backed by the multithreaded
 * transforms of lc_fastfft.h: the timing build (oracle/ref_build, target
 * ref_bench) runs the reference's own sources on it to give bench.py's CPU
 * baseline.  TEST INFRASTRUCTURE ONLY.  FFTW's conventions: unnormalised,
 * FFTW_FORWARD = e^{-i}, row-major with the last dimension fastest, batches
 * contiguous (stride 1, distance idist / odist); R2C keeps n/2 + 1 values of
 * the last dimension; C2R assumes Hermitian symmetry and, like FFTW's
 * default for multi-dimensional C2R, may overwrite its input. */
#ifndef LC_SHIM_FAST_FFTW3_H
#define LC_SHIM_FAST_FFTW3_H

#include <complex>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "lc_fastfft.h"

#define FFTW_FORWARD (-1)
#define FFTW_BACKWARD (+1)
#define FFTW_MEASURE (0U)
#define FFTW_ESTIMATE (1U << 6)

typedef double fftw_complex[2];
typedef float fftwf_complex[2];

namespace lc_shim {

enum Kind { C2C, R2C, C2R };

struct Plan {
    std::vector<long> n;
    int howmany;
    int sign;
    Kind kind;
    long idist, odist;
};

inline Plan *make(int rank, const int *n, int howmany, int idist, int odist, int sign, Kind k) {
    Plan *p = new Plan;
    p->n.assign(n, n + rank);
    p->howmany = howmany;
    p->idist = idist;
    p->odist = odist;
    p->sign = sign;
    p->kind = k;
    return p;
}

// transforms along every axis but the last of a row-major array whose last
// extent is `last`
template <typename R>
void c2c_leading(std::complex<R> *a, const std::vector<long> &n, long last, int sign) {
    const int rank = (int)n.size();
    long total = last;
    for (int d = 0; d + 1 < rank; ++d) total *= n[d];
    for (int d = rank - 2; d >= 0; --d) {
        long inner = last;
        for (int e = d + 1; e + 1 < rank; ++e) inner *= n[e];
        if (n[d] > 1) lc_fast::c2c_axis(a, total / (inner * n[d]), n[d], inner, sign);
    }
}

template <typename R>
void run_c2c(const Plan &p, const std::complex<R> *in, std::complex<R> *out) {
    long sz = 1;
    for (long v : p.n) sz *= v;
    for (int b = 0; b < p.howmany; ++b) {
        std::complex<R> *o = out + b * p.odist;
        if ((const void *)(in + b * p.idist) != (const void *)o) std::memcpy(o, in + b * p.idist, sz * sizeof(*o));
        lc_fast::c2c_nd(o, p.n, p.sign);
    }
}

template <typename R>
void run_r2c(const Plan &p, const R *in, std::complex<R> *out) {
    const long N = p.n.back(), nh = N / 2 + 1;
    long rows = 1;
    for (size_t d = 0; d + 1 < p.n.size(); ++d) rows *= p.n[d];
    for (int b = 0; b < p.howmany; ++b) {
        const R *x = in + b * p.idist;
        std::complex<R> *y = out + b * p.odist;
        if (N % 2 == 0) {
            lc_fast::r2c_rows(x, y, rows, N);
        } else {  // odd rows: complex transforms of the real rows, first halves kept
            std::vector<std::complex<R>> t((size_t)(rows * N));
#pragma omp parallel for schedule(static)
            for (long i = 0; i < rows * N; ++i) t[i] = std::complex<R>(x[i], 0);
            lc_fast::c2c_rows(t.data(), rows, N, -1);
#pragma omp parallel for schedule(static)
            for (long r = 0; r < rows; ++r)
                for (long k = 0; k < nh; ++k) y[r * nh + k] = t[r * N + k];
        }
        c2c_leading(y, p.n, nh, -1);
    }
}

template <typename R>
void run_c2r(const Plan &p, std::complex<R> *in, R *out) {
    const long N = p.n.back(), nh = N / 2 + 1;
    long rows = 1;
    for (size_t d = 0; d + 1 < p.n.size(); ++d) rows *= p.n[d];
    for (int b = 0; b < p.howmany; ++b) {
        std::complex<R> *x = in + b * p.idist;
        R *y = out + b * p.odist;
        c2c_leading(x, p.n, nh, +1);
        if (N % 2 == 0) {
            lc_fast::c2r_rows(x, y, rows, N);
        } else {
            std::vector<std::complex<R>> t((size_t)(rows * N));
#pragma omp parallel for schedule(static)
            for (long r = 0; r < rows; ++r)
                for (long k = 0; k < N; ++k)
                    t[r * N + k] = k < nh ? x[r * nh + k] : std::conj(x[r * nh + (N - k)]);
            lc_fast::c2c_rows(t.data(), rows, N, +1);
#pragma omp parallel for schedule(static)
            for (long i = 0; i < rows * N; ++i) y[i] = t[i].real();
        }
    }
}

}  // namespace lc_shim

typedef lc_shim::Plan *fftw_plan;
typedef lc_shim::Plan *fftwf_plan;

inline void *fftw_malloc(size_t n) { return std::malloc(n); }
inline void fftw_free(void *p) { std::free(p); }
inline void *fftwf_malloc(size_t n) { return std::malloc(n); }
inline void fftwf_free(void *p) { std::free(p); }
inline void fftw_destroy_plan(fftw_plan p) { delete p; }
inline void fftwf_destroy_plan(fftwf_plan p) { delete p; }

#define LC_SHIM_FFTW_API(PFX, R, CPLX)                                                        \
    inline lc_shim::Plan *PFX##_plan_many_dft(int rank, const int *n, int howmany, CPLX *,    \
                                              const int *, int, int idist, CPLX *,            \
                                              const int *, int, int odist, int sign,          \
                                              unsigned) {                                     \
        return lc_shim::make(rank, n, howmany, idist, odist, sign, lc_shim::C2C);             \
    }                                                                                         \
    inline lc_shim::Plan *PFX##_plan_many_dft_r2c(int rank, const int *n, int howmany, R *,   \
                                                  const int *, int, int idist, CPLX *,        \
                                                  const int *, int, int odist, unsigned) {    \
        return lc_shim::make(rank, n, howmany, idist, odist, FFTW_FORWARD, lc_shim::R2C);     \
    }                                                                                         \
    inline lc_shim::Plan *PFX##_plan_many_dft_c2r(int rank, const int *n, int howmany,        \
                                                  CPLX *, const int *, int, int idist, R *,   \
                                                  const int *, int, int odist, unsigned) {    \
        return lc_shim::make(rank, n, howmany, idist, odist, FFTW_BACKWARD, lc_shim::C2R);    \
    }                                                                                         \
    inline void PFX##_execute_dft(lc_shim::Plan *p, CPLX *in, CPLX *out) {                    \
        lc_shim::run_c2c<R>(*p, (const std::complex<R> *)in, (std::complex<R> *)out);         \
    }                                                                                         \
    inline void PFX##_execute_dft_r2c(lc_shim::Plan *p, R *in, CPLX *out) {                   \
        lc_shim::run_r2c<R>(*p, in, (std::complex<R> *)out);                                  \
    }                                                                                         \
    inline void PFX##_execute_dft_c2r(lc_shim::Plan *p, CPLX *in, R *out) {                   \
        lc_shim::run_c2r<R>(*p, (std::complex<R> *)in, out);                                  \
    }

LC_SHIM_FFTW_API(fftw, double, fftw_complex)
LC_SHIM_FFTW_API(fftwf, float, fftwf_complex)

#endif
