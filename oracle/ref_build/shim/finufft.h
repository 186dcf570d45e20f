/* Self-written stand-in for the subset of the FINUFFT API that the LaminoCam
 * reference calls (include/finufft_plan.h:39-83).  TEST INFRASTRUCTURE ONLY.
 * The transforms are the exact non-uniform DFTs that FINUFFT approximates
 * (FINUFFT semantics: type 1 f_k = sum_j c_j e^{+-i k.x_j}, type 2
 * c_j = sum_k f_k e^{+-i k.x_j}; modes k in [-floor(N/2), floor((N-1)/2)]
 * increasing; dimension 1 fastest), evaluated in long double with separable
 * exponentials.  The requested tolerance is ignored: the result is exact to
 * rounding. */
#ifndef LC_SHIM_FINUFFT_H
#define LC_SHIM_FINUFFT_H

#include <cmath>
#include <complex>
#include <cstdint>
#include <vector>

typedef struct finufft_opts {
    int modeord;
    int debug;
} finufft_opts;

namespace lc_shim {

struct NuPlan {
    int type, dim, iflag;
    int64_t n[3];
    int64_t M;
    const void *x, *y, *z;
};

typedef std::complex<long double> cld;

template <typename R>
int nu_execute(NuPlan *p, std::complex<R> *c, std::complex<R> *f) {
    int64_t n1 = p->n[0], n2 = p->dim > 1 ? p->n[1] : 1, n3 = p->dim > 2 ? p->n[2] : 1;
    const R *xs = (const R *)p->x, *ys = (const R *)p->y, *zs = (const R *)p->z;
    int64_t nm = n1 * n2 * n3;
    long double s = (long double)p->iflag;
    if (p->type == 1) {
        std::vector<cld> acc(nm, cld(0, 0));
#pragma omp parallel
        {
            std::vector<cld> loc(nm, cld(0, 0));
            std::vector<cld> e1(n1), e2(n2), e3(n3);
#pragma omp for
            for (int64_t j = 0; j < p->M; ++j) {
                for (int64_t a = 0; a < n1; ++a) {
                    long double k = (long double)(a - n1 / 2);
                    e1[a] = std::polar(1.0L, s * k * (long double)xs[j]);
                }
                for (int64_t a = 0; a < n2; ++a) {
                    long double k = (long double)(a - n2 / 2);
                    e2[a] = p->dim > 1 ? std::polar(1.0L, s * k * (long double)ys[j]) : cld(1, 0);
                }
                for (int64_t a = 0; a < n3; ++a) {
                    long double k = (long double)(a - n3 / 2);
                    e3[a] = p->dim > 2 ? std::polar(1.0L, s * k * (long double)zs[j]) : cld(1, 0);
                }
                cld cj((long double)c[j].real(), (long double)c[j].imag());
                for (int64_t c3 = 0; c3 < n3; ++c3)
                    for (int64_t c2 = 0; c2 < n2; ++c2) {
                        cld w = cj * e3[c3] * e2[c2];
                        cld *row = loc.data() + (c3 * n2 + c2) * n1;
                        for (int64_t c1 = 0; c1 < n1; ++c1) row[c1] += w * e1[c1];
                    }
            }
#pragma omp critical
            for (int64_t i = 0; i < nm; ++i) acc[i] += loc[i];
        }
        for (int64_t i = 0; i < nm; ++i) f[i] = std::complex<R>((R)acc[i].real(), (R)acc[i].imag());
    } else {
#pragma omp parallel
        {
            std::vector<cld> e1(n1), e2(n2), e3(n3);
#pragma omp for
            for (int64_t j = 0; j < p->M; ++j) {
                for (int64_t a = 0; a < n1; ++a)
                    e1[a] = std::polar(1.0L, s * (long double)(a - n1 / 2) * (long double)xs[j]);
                for (int64_t a = 0; a < n2; ++a)
                    e2[a] = p->dim > 1 ? std::polar(1.0L, s * (long double)(a - n2 / 2) * (long double)ys[j])
                                       : cld(1, 0);
                for (int64_t a = 0; a < n3; ++a)
                    e3[a] = p->dim > 2 ? std::polar(1.0L, s * (long double)(a - n3 / 2) * (long double)zs[j])
                                       : cld(1, 0);
                cld sum(0, 0);
                for (int64_t c3 = 0; c3 < n3; ++c3)
                    for (int64_t c2 = 0; c2 < n2; ++c2) {
                        cld w = e3[c3] * e2[c2];
                        const std::complex<R> *row = f + (c3 * n2 + c2) * n1;
                        cld rs(0, 0);
                        for (int64_t c1 = 0; c1 < n1; ++c1)
                            rs += cld((long double)row[c1].real(), (long double)row[c1].imag()) * e1[c1];
                        sum += w * rs;
                    }
                c[j] = std::complex<R>((R)sum.real(), (R)sum.imag());
            }
        }
    }
    return 0;
}

} // namespace lc_shim

typedef lc_shim::NuPlan *finufft_plan;
typedef lc_shim::NuPlan *finufftf_plan;

inline void finufft_default_opts(finufft_opts *o) { o->modeord = 0; o->debug = 0; }
inline void finufftf_default_opts(finufft_opts *o) { o->modeord = 0; o->debug = 0; }

#define LC_SHIM_NUFFT_API(PFX, R)                                                              \
    inline int PFX##_makeplan(int type, int dim, int64_t *n_modes, int iflag, int, R,          \
                              lc_shim::NuPlan **plan, finufft_opts *) {                        \
        lc_shim::NuPlan *p = new lc_shim::NuPlan;                                              \
        p->type = type; p->dim = dim; p->iflag = iflag > 0 ? 1 : -1;                           \
        for (int d = 0; d < 3; ++d) p->n[d] = n_modes[d];                                      \
        p->M = 0; p->x = p->y = p->z = nullptr;                                                \
        *plan = p;                                                                             \
        return 0;                                                                              \
    }                                                                                          \
    inline int PFX##_setpts(lc_shim::NuPlan *p, int64_t M, R *x, R *y, R *z, int64_t, R *,     \
                            R *, R *) {                                                        \
        p->M = M; p->x = x; p->y = y; p->z = z;                                                \
        return 0;                                                                              \
    }                                                                                          \
    inline int PFX##_execute(lc_shim::NuPlan *p, std::complex<R> *c, std::complex<R> *f) {     \
        return lc_shim::nu_execute<R>(p, c, f);                                                \
    }                                                                                          \
    inline int PFX##_destroy(lc_shim::NuPlan *p) { delete p; return 0; }

LC_SHIM_NUFFT_API(finufft, double)
LC_SHIM_NUFFT_API(finufftf, float)

#endif
