/* Self-written stand-in for the subset of the FINUFFT API that the LaminoCam
 * reference calls (include/finufft_plan.h:39-83), built for speed: the timing
 * build (oracle/ref_build, target ref_bench) runs the reference's own sources
 * on it to give bench.py's CPU baseline.  TEST INFRASTRUCTURE ONLY.
 *
 * It implements the published "exponential of semicircle" NUFFT (A. Barnett,
 * J. Magland, L. af Klinteberg, "A parallel nonuniform fast Fourier transform
 * library based on an exponential of semicircle kernel", SIAM J. Sci. Comput.
 * 41(5), 2019), with FINUFFT's semantics:
 *   type 1: f_k = sum_j c_j e^{iflag i k.x_j};  type 2: c_j = sum_k f_k e^{iflag i k.x_j};
 *   modes k in [-floor(N/2), floor((N-1)/2)] increasing, dimension 1 fastest;
 *   points taken 2 pi periodic.
 * Kernel: phi(z) = exp(beta (sqrt(1 - z^2) - 1)) on |z| <= 1, width
 * w = ceil(log10(1/tol)) + 1 cells (at least 2), beta = 2.30 w, upsampling 2
 * (fine grid next 2^p 3^q >= max(2N, 2w)); deconvolution by the kernel's
 * Fourier transform, by Gauss-Legendre quadrature.  The tolerance is the one
 * the caller passes: 5e-4 for the reference's float path, as in FINUFFT.
 *
 * Type 1 spreads without atomics: setpts sorts the points by the block of
 * their footprint's first cell (blocks of at least w cells along y and z),
 * and spreading runs in colour phases in which blocks two apart (or three,
 * across the periodic wrap of an odd block count) never write the same cell;
 * OpenMP threads take the blocks of a phase. */
#ifndef LC_SHIM_FAST_FINUFFT_H
#define LC_SHIM_FAST_FINUFFT_H

#include <algorithm>
#include <cmath>
#include <complex>
#include <cstdint>
#include <vector>

#include "lc_fastfft.h"

typedef struct finufft_opts {
    int modeord;
    int debug;
} finufft_opts;

namespace lc_shim {

inline void gauss_legendre(int n, std::vector<double> &x, std::vector<double> &wt) {
    x.assign(n, 0.0);
    wt.assign(n, 0.0);
    const double pi = 3.14159265358979323846;
    for (int i = 0; i < (n + 1) / 2; ++i) {
        double z = std::cos(pi * (i + 0.75) / (n + 0.5)), z1, pp;
        do {
            double p1 = 1.0, p2 = 0.0;
            for (int j = 1; j <= n; ++j) {
                double p3 = p2;
                p2 = p1;
                p1 = ((2.0 * j - 1.0) * z * p2 - (j - 1.0) * p3) / j;
            }
            pp = n * (z * p1 - p2) / (z * z - 1.0);
            z1 = z;
            z = z1 - p1 / pp;
        } while (std::fabs(z - z1) > 1e-15);
        x[i] = -z;
        x[n - 1 - i] = z;
        wt[i] = wt[n - 1 - i] = 2.0 / ((1.0 - z * z) * pp * pp);
    }
}

struct NuPlan {
    int type = 1, dim = 1, iflag = 1, w = 7;
    double beta = 16.1;
    int64_t n[3] = {1, 1, 1};   // modes per dimension (dimension 1 fastest)
    int64_t nf[3] = {1, 1, 1};  // fine grid
    std::vector<double> corr[3];
    int64_t M = 0;
    const void *x = nullptr, *y = nullptr, *z = nullptr;
    bool is_float = true;
    // spreading schedule
    int64_t nb[3] = {1, 1, 1};  // blocks per dimension
    std::vector<int64_t> start;  // per block, its first index into perm (plus one end)
    std::vector<int32_t> perm;
};

// fine-grid coordinate in [0, nf) of the 2 pi periodic point x
inline double fine_coord(double x, int64_t nf) {
    double u = x * (double)nf / (2.0 * 3.14159265358979323846);
    u -= (double)nf * std::floor(u / (double)nf);
    if (u >= (double)nf) u -= (double)nf;
    if (u < 0) u = 0;
    return u;
}

template <typename R>
inline double coord_of(const NuPlan &p, int d, int64_t j) {
    const R *a = (const R *)(d == 0 ? p.x : (d == 1 ? p.y : p.z));
    return (double)a[j];
}

inline int64_t first_cell(double u, int w) { return (int64_t)std::ceil(u - 0.5 * w); }

inline int64_t wrapi(int64_t v, int64_t n) {
    v %= n;
    return v < 0 ? v + n : v;
}

inline int block_colour(int64_t b, int64_t nb) {
    if (nb == 1) return 0;
    if (nb % 2 == 1 && b == nb - 1) return 2;
    return (int)(b % 2);
}

// block of cell l (of nf) when nf is cut into nb blocks [b nf / nb, (b + 1) nf / nb)
inline int64_t block_of(int64_t l, int64_t nf, int64_t nb) {
    int64_t b = (l * nb) / nf;
    while (b + 1 < nb && ((b + 1) * nf) / nb <= l) ++b;
    while (b > 0 && (b * nf) / nb > l) --b;
    return b;
}

template <typename R>
void make_schedule(NuPlan &p) {
    // y (2D) or y and z (3D) cut into blocks of at least max(w, 16) cells, so
    // a footprint reaches its own block and the next one (wrapped) only; x is
    // not cut
    int64_t nblocks = 1;
    for (int d = 0; d < 3; ++d) {
        p.nb[d] = (d == 0 || d >= p.dim) ? 1 : std::max<int64_t>(1, p.nf[d] / std::max<int64_t>(p.w, 16));
        nblocks *= p.nb[d];
    }
    std::vector<int64_t> cnt(nblocks + 1, 0);
    std::vector<int32_t> key(p.M);
#pragma omp parallel for schedule(static)
    for (int64_t j = 0; j < p.M; ++j) {
        int64_t b = 0, mul = 1;
        for (int d = 1; d < p.dim; ++d) {
            int64_t l0 = wrapi(first_cell(fine_coord(coord_of<R>(p, d, j), p.nf[d]), p.w), p.nf[d]);
            b += block_of(l0, p.nf[d], p.nb[d]) * mul;
            mul *= p.nb[d];
        }
        key[j] = (int32_t)b;
    }
    for (int64_t j = 0; j < p.M; ++j) ++cnt[key[j] + 1];
    for (int64_t b = 0; b < nblocks; ++b) cnt[b + 1] += cnt[b];
    p.start = cnt;
    p.perm.resize(p.M);
    for (int64_t j = 0; j < p.M; ++j) p.perm[cnt[key[j]]++] = (int32_t)j;
}

// kernel weights in the transform's precision R
template <typename R>
inline void es_weights(double u, int w, double beta, int64_t &l0, R *wt) {
    l0 = first_cell(u, w);
    const double hw = 0.5 * w;
    for (int m = 0; m < w; ++m) {
        const double z = ((double)(l0 + m) - u) / hw;
        const double t = 1.0 - z * z;
        wt[m] = t > 0 ? (R)std::exp(beta * (std::sqrt(t) - 1.0)) : R(0);
    }
}

// spread point j (value v) into the fine grid g (complex, x fastest)
template <typename R>
inline void spread_one(const NuPlan &p, int64_t j, std::complex<R> v, std::complex<R> *g) {
    const int w = p.w;
    R wx[16], wy[16], wz[16];
    int64_t l0[3] = {0, 0, 0};
    es_weights(fine_coord(coord_of<R>(p, 0, j), p.nf[0]), w, p.beta, l0[0], wx);
    if (p.dim > 1) es_weights(fine_coord(coord_of<R>(p, 1, j), p.nf[1]), w, p.beta, l0[1], wy);
    else wy[0] = R(1);
    if (p.dim > 2) es_weights(fine_coord(coord_of<R>(p, 2, j), p.nf[2]), w, p.beta, l0[2], wz);
    else wz[0] = R(1);
    const int wyn = p.dim > 1 ? w : 1, wzn = p.dim > 2 ? w : 1;
    const int64_t nx = p.nf[0], ny = p.nf[1], nz = p.nf[2];
    const bool xin = l0[0] >= 0 && l0[0] + w <= nx;
    for (int dz = 0; dz < wzn; ++dz) {
        const int64_t iz = p.dim > 2 ? wrapi(l0[2] + dz, nz) : 0;
        for (int dy = 0; dy < wyn; ++dy) {
            const int64_t iy = p.dim > 1 ? wrapi(l0[1] + dy, ny) : 0;
            const R f = wz[dz] * wy[dy];
            const R vr = v.real() * f, vi = v.imag() * f;
            std::complex<R> *row = g + (iz * ny + iy) * nx;
            if (xin) {
                R *r = reinterpret_cast<R *>(row + l0[0]);
#pragma omp simd
                for (int dx = 0; dx < w; ++dx) {
                    r[2 * dx] += vr * wx[dx];
                    r[2 * dx + 1] += vi * wx[dx];
                }
            } else {
                for (int dx = 0; dx < w; ++dx) row[wrapi(l0[0] + dx, nx)] += std::complex<R>(vr * wx[dx], vi * wx[dx]);
            }
        }
    }
}

template <typename R>
inline std::complex<R> interp_one(const NuPlan &p, int64_t j, const std::complex<R> *g) {
    const int w = p.w;
    R wx[16], wy[16], wz[16];
    int64_t l0[3] = {0, 0, 0};
    es_weights(fine_coord(coord_of<R>(p, 0, j), p.nf[0]), w, p.beta, l0[0], wx);
    if (p.dim > 1) es_weights(fine_coord(coord_of<R>(p, 1, j), p.nf[1]), w, p.beta, l0[1], wy);
    else wy[0] = R(1);
    if (p.dim > 2) es_weights(fine_coord(coord_of<R>(p, 2, j), p.nf[2]), w, p.beta, l0[2], wz);
    else wz[0] = R(1);
    const int wyn = p.dim > 1 ? w : 1, wzn = p.dim > 2 ? w : 1;
    const int64_t nx = p.nf[0], ny = p.nf[1], nz = p.nf[2];
    R ar = 0, ai = 0;
    for (int dz = 0; dz < wzn; ++dz) {
        const int64_t iz = p.dim > 2 ? wrapi(l0[2] + dz, nz) : 0;
        for (int dy = 0; dy < wyn; ++dy) {
            const int64_t iy = p.dim > 1 ? wrapi(l0[1] + dy, ny) : 0;
            const std::complex<R> *row = g + (iz * ny + iy) * nx;
            R rr = 0, ri = 0;
            for (int dx = 0; dx < w; ++dx) {
                const std::complex<R> c = row[wrapi(l0[0] + dx, nx)];
                rr += c.real() * wx[dx];
                ri += c.imag() * wx[dx];
            }
            const R f = wz[dz] * wy[dy];
            ar += rr * f;
            ai += ri * f;
        }
    }
    return {ar, ai};
}

template <typename R>
int nu_execute(NuPlan *p, std::complex<R> *c, std::complex<R> *f) {
    const int64_t nx = p->nf[0], ny = p->nf[1], nz = p->nf[2];
    const int64_t gsize = nx * ny * nz;
    std::vector<std::complex<R>> g(gsize);
    std::vector<long> dims;  // row-major: slowest first
    for (int d = p->dim - 1; d >= 0; --d) dims.push_back((long)p->nf[d]);
    const int64_t n0 = p->n[0], n1 = p->dim > 1 ? p->n[1] : 1, n2 = p->dim > 2 ? p->n[2] : 1;
    if (p->type == 1) {
        const int64_t nby = p->nb[1], nbz = p->nb[2];
        const int ncy = nby == 1 ? 1 : (nby % 2 ? 3 : 2), ncz = nbz == 1 ? 1 : (nbz % 2 ? 3 : 2);
        for (int cz = 0; cz < ncz; ++cz)
            for (int cy = 0; cy < ncy; ++cy) {
                std::vector<int64_t> blocks;
                for (int64_t bz = 0; bz < nbz; ++bz)
                    for (int64_t by = 0; by < nby; ++by)
                        if (block_colour(bz, nbz) == cz && block_colour(by, nby) == cy)
                            blocks.push_back(bz * nby + by);
#pragma omp parallel for schedule(dynamic, 1)
                for (size_t t = 0; t < blocks.size(); ++t) {
                    const int64_t b = blocks[t];
                    for (int64_t q = p->start[b]; q < p->start[b + 1]; ++q) {
                        const int64_t j = p->perm[q];
                        spread_one<R>(*p, j, c[j], g.data());
                    }
                }
            }
        lc_fast::c2c_nd<R>(g.data(), dims, p->iflag > 0 ? +1 : -1);
        // modes k at fine index k mod nf, deconvolved
#pragma omp parallel for collapse(2) schedule(static)
        for (int64_t a2 = 0; a2 < n2; ++a2)
            for (int64_t a1 = 0; a1 < n1; ++a1) {
                const int64_t k2 = a2 - n2 / 2, k1 = a1 - n1 / 2;
                const int64_t i2 = wrapi(k2, nz), i1 = wrapi(k1, ny);
                const double c21 = p->corr[2].empty() ? 1.0 : p->corr[2][a2];
                const double c1 = c21 * (p->corr[1].empty() ? 1.0 : p->corr[1][a1]);
                const std::complex<R> *row = g.data() + (i2 * ny + i1) * nx;
                std::complex<R> *out = f + (a2 * n1 + a1) * n0;
                for (int64_t a0 = 0; a0 < n0; ++a0) {
                    const int64_t i0 = wrapi(a0 - n0 / 2, nx);
                    out[a0] = row[i0] * (R)(c1 * p->corr[0][a0]);
                }
            }
    } else {
#pragma omp parallel for collapse(2) schedule(static)
        for (int64_t a2 = 0; a2 < n2; ++a2)
            for (int64_t a1 = 0; a1 < n1; ++a1) {
                const int64_t i2 = wrapi(a2 - n2 / 2, nz), i1 = wrapi(a1 - n1 / 2, ny);
                const double c21 = p->corr[2].empty() ? 1.0 : p->corr[2][a2];
                const double c1 = c21 * (p->corr[1].empty() ? 1.0 : p->corr[1][a1]);
                std::complex<R> *row = g.data() + (i2 * ny + i1) * nx;
                const std::complex<R> *in = f + (a2 * n1 + a1) * n0;
                for (int64_t a0 = 0; a0 < n0; ++a0) row[wrapi(a0 - n0 / 2, nx)] = in[a0] * (R)(c1 * p->corr[0][a0]);
            }
        lc_fast::c2c_nd<R>(g.data(), dims, p->iflag > 0 ? +1 : -1);
#pragma omp parallel for schedule(static)
        for (int64_t j = 0; j < p->M; ++j) c[j] = interp_one<R>(*p, j, g.data());
    }
    return 0;
}

inline void init_plan(NuPlan *p, int type, int dim, const int64_t *n_modes, int iflag, double tol) {
    p->type = type;
    p->dim = dim;
    p->iflag = iflag > 0 ? 1 : -1;
    p->w = std::max(2, std::min(16, (int)std::ceil(std::log10(1.0 / tol)) + 1));
    p->beta = 2.30 * p->w;
    std::vector<double> gx, gw;
    gauss_legendre(4 * p->w + 60, gx, gw);
    for (int d = 0; d < 3; ++d) {
        p->n[d] = d < dim ? n_modes[d] : 1;
        p->nf[d] = d < dim ? lc_fast::next_smooth23(std::max<int64_t>(2 * p->n[d], 2 * p->w)) : 1;
        p->corr[d].clear();
        if (d >= dim) continue;
        // 2 / (w phihat(k w pi / nf)), phihat(xi) = int_{-1}^{1} phi(t) cos(xi t) dt
        p->corr[d].resize(p->n[d]);
        for (int64_t a = 0; a < p->n[d]; ++a) {
            const double xi = (double)(a - p->n[d] / 2) * p->w * 3.14159265358979323846 / (double)p->nf[d];
            double s = 0;
            for (size_t q = 0; q < gx.size(); ++q)
                s += gw[q] * std::exp(p->beta * (std::sqrt(1.0 - gx[q] * gx[q]) - 1.0)) * std::cos(xi * gx[q]);
            p->corr[d][a] = 2.0 / (p->w * s);
        }
    }
}

}  // namespace lc_shim

typedef lc_shim::NuPlan *finufft_plan;
typedef lc_shim::NuPlan *finufftf_plan;

inline void finufft_default_opts(finufft_opts *o) { o->modeord = 0; o->debug = 0; }
inline void finufftf_default_opts(finufft_opts *o) { o->modeord = 0; o->debug = 0; }

#define LC_SHIM_NUFFT_API(PFX, R)                                                              \
    inline int PFX##_makeplan(int type, int dim, int64_t *n_modes, int iflag, int, R tol,      \
                              lc_shim::NuPlan **plan, finufft_opts *) {                        \
        lc_shim::NuPlan *p = new lc_shim::NuPlan;                                              \
        lc_shim::init_plan(p, type, dim, n_modes, iflag, (double)tol);                         \
        *plan = p;                                                                             \
        return 0;                                                                              \
    }                                                                                          \
    inline int PFX##_setpts(lc_shim::NuPlan *p, int64_t M, R *x, R *y, R *z, int64_t, R *,     \
                            R *, R *) {                                                        \
        p->M = M; p->x = x; p->y = y; p->z = z;                                                \
        if (p->type == 1) lc_shim::make_schedule<R>(*p);                                       \
        return 0;                                                                              \
    }                                                                                          \
    inline int PFX##_execute(lc_shim::NuPlan *p, std::complex<R> *c, std::complex<R> *f) {     \
        return lc_shim::nu_execute<R>(p, c, f);                                                \
    }                                                                                          \
    inline int PFX##_destroy(lc_shim::NuPlan *p) { delete p; return 0; }

LC_SHIM_NUFFT_API(finufft, double)
LC_SHIM_NUFFT_API(finufftf, float)

#endif
