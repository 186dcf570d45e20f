/* Self-written stand-in for the subset of the FFTW3 API that the LaminoCam
 * reference calls (include/fftw_plan.h:43-197).  TEST INFRASTRUCTURE ONLY: it
 * lets the reference's own sources compile unmodified so that their outputs can
 * pin the numpy oracle.  Transforms are evaluated as direct separable DFTs in
 * long double (exact to rounding), with FFTW's conventions: unnormalised,
 * FFTW_FORWARD = e^{-i}, row-major, last dimension fastest; R2C keeps n/2+1
 * entries of the last dimension; C2R assumes Hermitian symmetry. */
#ifndef LC_SHIM_FFTW3_H
#define LC_SHIM_FFTW3_H

#include <cmath>
#include <complex>
#include <cstdlib>
#include <cstring>
#include <vector>

#define FFTW_FORWARD (-1)
#define FFTW_BACKWARD (+1)
#define FFTW_MEASURE (0U)
#define FFTW_ESTIMATE (1U << 6)

typedef double fftw_complex[2];
typedef float fftwf_complex[2];

namespace lc_shim {

enum Kind { C2C, R2C, C2R };

struct Plan {
    int rank;
    std::vector<int> n;
    int howmany;
    int sign;
    Kind kind;
    long idist, odist;
};

typedef std::complex<long double> cld;

/* in-place separable DFT of a row-major array with dims n[0..rank) */
inline void dft_nd(std::vector<cld> &a, const std::vector<int> &n, int sign) {
    int rank = (int)n.size();
    size_t total = 1;
    for (int d = 0; d < rank; ++d) total *= (size_t)n[d];
    for (int d = 0; d < rank; ++d) {
        size_t L = (size_t)n[d];
        size_t inner = 1;
        for (int e = d + 1; e < rank; ++e) inner *= (size_t)n[e];
        size_t outer = total / (L * inner);
        std::vector<cld> tw(L);
        for (size_t k = 0; k < L; ++k) {
            long double ang = (long double)sign * 2.0L * 3.14159265358979323846264338327950288L *
                              (long double)k / (long double)L;
            tw[k] = cld(cosl(ang), sinl(ang));
        }
        std::vector<cld> tmp(L);
#pragma omp parallel for collapse(2) firstprivate(tmp)
        for (size_t o = 0; o < outer; ++o) {
            for (size_t i = 0; i < inner; ++i) {
                cld *base = a.data() + o * L * inner + i;
                for (size_t k = 0; k < L; ++k) {
                    cld s = 0;
                    for (size_t j = 0; j < L; ++j) s += base[j * inner] * tw[(j * k) % L];
                    tmp[k] = s;
                }
                for (size_t k = 0; k < L; ++k) base[k * inner] = tmp[k];
            }
        }
    }
}

template <typename R>
void run_c2c(const Plan &p, const R *in, R *out) {
    size_t sz = 1;
    for (int v : p.n) sz *= (size_t)v;
    for (int b = 0; b < p.howmany; ++b) {
        std::vector<cld> a(sz);
        for (size_t i = 0; i < sz; ++i)
            a[i] = cld(in[2 * (b * p.idist + i)], in[2 * (b * p.idist + i) + 1]);
        dft_nd(a, p.n, p.sign);
        for (size_t i = 0; i < sz; ++i) {
            out[2 * (b * p.odist + i)] = (R)a[i].real();
            out[2 * (b * p.odist + i) + 1] = (R)a[i].imag();
        }
    }
}

template <typename R>
void run_r2c(const Plan &p, const R *in, R *out) {
    size_t sz = 1;
    for (int v : p.n) sz *= (size_t)v;
    int nl = p.n.back();
    int nh = nl / 2 + 1;
    size_t rows = sz / nl;
    for (int b = 0; b < p.howmany; ++b) {
        std::vector<cld> a(sz);
        for (size_t i = 0; i < sz; ++i) a[i] = cld(in[b * p.idist + i], 0);
        dft_nd(a, p.n, FFTW_FORWARD);
        for (size_t r = 0; r < rows; ++r)
            for (int k = 0; k < nh; ++k) {
                cld v = a[r * nl + k];
                out[2 * (b * p.odist + r * nh + k)] = (R)v.real();
                out[2 * (b * p.odist + r * nh + k) + 1] = (R)v.imag();
            }
    }
}

template <typename R>
void run_c2r(const Plan &p, const R *in, R *out) {
    size_t sz = 1;
    for (int v : p.n) sz *= (size_t)v;
    int rank = (int)p.n.size();
    int nl = p.n.back();
    int nh = nl / 2 + 1;
    size_t rows = sz / nl;
    for (int b = 0; b < p.howmany; ++b) {
        std::vector<cld> a(sz);
        for (size_t r = 0; r < rows; ++r) {
            /* mirror index of row r: negate every leading coordinate */
            size_t rem = r, mr = 0, mul = 1;
            std::vector<size_t> idx(rank - 1);
            for (int d = rank - 2; d >= 0; --d) {
                idx[d] = rem % p.n[d];
                rem /= p.n[d];
            }
            for (int d = rank - 2; d >= 0; --d) {
                mr += ((p.n[d] - idx[d]) % p.n[d]) * mul;
                mul *= p.n[d];
            }
            for (int k = 0; k < nl; ++k) {
                if (k < nh) {
                    size_t o = b * p.idist + r * nh + k;
                    a[r * nl + k] = cld(in[2 * o], in[2 * o + 1]);
                } else {
                    size_t o = b * p.idist + mr * nh + (nl - k);
                    a[r * nl + k] = std::conj(cld(in[2 * o], in[2 * o + 1]));
                }
            }
        }
        dft_nd(a, p.n, FFTW_BACKWARD);
        for (size_t i = 0; i < sz; ++i) out[b * p.odist + i] = (R)a[i].real();
    }
}

inline Plan *make(int rank, const int *n, int howmany, int idist, int odist, int sign, Kind k) {
    Plan *p = new Plan;
    p->rank = rank;
    p->n.assign(n, n + rank);
    p->howmany = howmany;
    p->idist = idist;
    p->odist = odist;
    p->sign = sign;
    p->kind = k;
    return p;
}

} // namespace lc_shim

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
        lc_shim::run_c2c<R>(*p, (const R *)in, (R *)out);                                     \
    }                                                                                         \
    inline void PFX##_execute_dft_r2c(lc_shim::Plan *p, R *in, CPLX *out) {                   \
        lc_shim::run_r2c<R>(*p, in, (R *)out);                                                \
    }                                                                                         \
    inline void PFX##_execute_dft_c2r(lc_shim::Plan *p, CPLX *in, R *out) {                   \
        lc_shim::run_c2r<R>(*p, (const R *)in, out);                                          \
    }

LC_SHIM_FFTW_API(fftw, double, fftw_complex)
LC_SHIM_FFTW_API(fftwf, float, fftwf_complex)

#endif
