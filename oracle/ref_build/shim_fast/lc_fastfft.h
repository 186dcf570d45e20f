/* Multithreaded FFTs for the timing build of the reference's sources
 * (oracle/ref_build, target ref_bench).  TEST INFRASTRUCTURE ONLY: the CPU
 * baseline that bench.py reports runs the reference's own code on these
 * transforms in place of FFTW and FINUFFT, which are not available here.
 *
 * Conventions are FFTW's: unnormalised, sign -1 = e^{-i}, row-major arrays
 * with the last dimension fastest.
 *
 *  * Lengths 2^p 3^q: Stockham autosort passes of radix 4, 2 and 3
 *    (decimation in frequency; a published formulation, e.g. C. Van Loan,
 *    "Computational Frameworks for the Fast Fourier Transform", SIAM 1992,
 *    section 1.7).
 *  * Other lengths: Bluestein's chirp-z algorithm (L. Bluestein, 1970) over a
 *    2^p 3^q transform of length >= 2n - 1.
 *  * Lines are transformed B at a time in a split real / imaginary scratch
 *    laid out [element][line], so the inner loops run over B * stride
 *    contiguous values and vectorise; OpenMP threads take groups of lines.
 *  * Real transforms pack a real row of even length N as a complex row of
 *    N / 2 points and unpack the half spectrum. */
#ifndef LC_FASTFFT_H
#define LC_FASTFFT_H

#include <algorithm>
#include <cmath>
#include <complex>
#include <cstdint>
#include <map>
#include <memory>
#include <mutex>
#include <vector>

namespace lc_fast {

constexpr int kLines = 16;  // lines per group

inline long next_smooth23(long n) {
    long best = 1;
    while (best < n) best <<= 1;
    for (long p3 = 1; p3 < best; p3 *= 3)
        for (long v = p3; v < best; v <<= 1)
            if (v >= n) { best = std::min(best, v); break; }
    return best;
}

inline bool smooth23(long n) {
    while (n % 2 == 0) n /= 2;
    while (n % 3 == 0) n /= 3;
    return n == 1;
}

/* One length, one sign, one precision: a Stockham plan, or Bluestein over one. */
template <typename R>
struct Line {
    int n = 0, sign = -1;
    // Stockham: per stage the radix and the twiddles w^(j u), u = 1..p-1,
    // j < m, with w = e^{sign 2 pi i / len} (len = the stage's sub-length)
    std::vector<int> radix;
    std::vector<std::vector<R>> twr, twi;
    // Bluestein
    bool blue = false;
    int L = 0;
    std::vector<R> chr, chi;    // e^{sign i pi j^2 / n}, j < n
    std::vector<R> vr, vi;      // FFT_L of the wrapped conjugate chirp, / L
    std::unique_ptr<Line<R>> fwd, inv;

    void init(int n_, int sign_) {
        n = n_;
        sign = sign_;
        if (smooth23(n)) {
            int len = n;
            while (len > 1) {
                int p = (len % 4 == 0) ? 4 : (len % 2 == 0 ? 2 : 3);
                int m = len / p;
                radix.push_back(p);
                std::vector<R> tr((size_t)m * (p - 1)), ti((size_t)m * (p - 1));
                for (int j = 0; j < m; ++j)
                    for (int u = 1; u < p; ++u) {
                        long double a = (long double)sign * 2.0L * 3.14159265358979323846264338327950288L *
                                        (long double)((long)j * u) / (long double)len;
                        tr[(size_t)j * (p - 1) + u - 1] = (R)cosl(a);
                        ti[(size_t)j * (p - 1) + u - 1] = (R)sinl(a);
                    }
                twr.push_back(std::move(tr));
                twi.push_back(std::move(ti));
                len = m;
            }
        } else {
            blue = true;
            L = (int)next_smooth23(2L * n - 1);
            fwd.reset(new Line<R>());
            fwd->init(L, -1);
            inv.reset(new Line<R>());
            inv->init(L, +1);
            chr.resize(n);
            chi.resize(n);
            for (long j = 0; j < n; ++j) {
                long q = (j * j) % (2L * n);
                long double a = (long double)sign * 3.14159265358979323846264338327950288L * (long double)q /
                                (long double)n;
                chr[j] = (R)cosl(a);
                chi[j] = (R)sinl(a);
            }
            // b_m = conj(chirp_|m|), wrapped into [0, L)
            std::vector<R> br((size_t)L * kLines, 0), bi((size_t)L * kLines, 0);
            for (long j = 0; j < n; ++j) {
                br[(size_t)j * kLines] = chr[j];
                bi[(size_t)j * kLines] = -chi[j];
                if (j > 0) {
                    br[(size_t)(L - j) * kLines] = chr[j];
                    bi[(size_t)(L - j) * kLines] = -chi[j];
                }
            }
            std::vector<R> sr((size_t)L * kLines), si((size_t)L * kLines);
            fwd->run(br.data(), bi.data(), sr.data(), si.data(), 1);
            vr.resize(L);
            vi.resize(L);
            for (int k = 0; k < L; ++k) {
                vr[k] = br[(size_t)k * kLines] / (R)L;
                vi[k] = bi[(size_t)k * kLines] / (R)L;
            }
        }
    }

    /* In place on x (split, [element][kLines]) for the first nb lines, with
     * scratch y of the same size.  Lines nb..kLines-1 are left as garbage. */
    void run(R *xr, R *xi, R *yr, R *yi, int nb) const {
        if (blue) return run_blue(xr, xi, yr, yi, nb);
        R *ar = xr, *ai = xi, *br = yr, *bi = yi;
        long s = 1;  // stride in lines-groups of kLines
        int len = n;
        for (size_t st = 0; st < radix.size(); ++st) {
            const int p = radix[st];
            const int m = len / p;
            const R *tr = twr[st].data(), *ti = twi[st].data();
            const long S = s * kLines;  // contiguous values per (j, t)
            for (int j = 0; j < m; ++j) {
                const R *a0r = ar + (size_t)j * S, *a0i = ai + (size_t)j * S;
                R *b0r = br + (size_t)p * j * S, *b0i = bi + (size_t)p * j * S;
                const size_t sm = (size_t)m * S;
                if (p == 2) {
                    const R w1r = tr[j], w1i = ti[j];
#pragma omp simd
                    for (long q = 0; q < S; ++q) {
                        R xr0 = a0r[q], xi0 = a0i[q], xr1 = a0r[q + sm], xi1 = a0i[q + sm];
                        b0r[q] = xr0 + xr1;
                        b0i[q] = xi0 + xi1;
                        R dr = xr0 - xr1, di = xi0 - xi1;
                        b0r[q + S] = dr * w1r - di * w1i;
                        b0i[q + S] = dr * w1i + di * w1r;
                    }
                } else if (p == 4) {
                    const R w1r = tr[3 * j], w1i = ti[3 * j], w2r = tr[3 * j + 1], w2i = ti[3 * j + 1],
                            w3r = tr[3 * j + 2], w3i = ti[3 * j + 2];
                    const R sg = (R)sign;  // multiply by sign * i
#pragma omp simd
                    for (long q = 0; q < S; ++q) {
                        R x0r = a0r[q], x0i = a0i[q], x1r = a0r[q + sm], x1i = a0i[q + sm];
                        R x2r = a0r[q + 2 * sm], x2i = a0i[q + 2 * sm], x3r = a0r[q + 3 * sm],
                          x3i = a0i[q + 3 * sm];
                        R s02r = x0r + x2r, s02i = x0i + x2i, d02r = x0r - x2r, d02i = x0i - x2i;
                        R s13r = x1r + x3r, s13i = x1i + x3i, d13r = x1r - x3r, d13i = x1i - x3i;
                        // (sign i) * d13
                        R jr = -sg * d13i, ji = sg * d13r;
                        R y0r = s02r + s13r, y0i = s02i + s13i;
                        R y2r = s02r - s13r, y2i = s02i - s13i;
                        R y1r = d02r + jr, y1i = d02i + ji;
                        R y3r = d02r - jr, y3i = d02i - ji;
                        b0r[q] = y0r;
                        b0i[q] = y0i;
                        b0r[q + S] = y1r * w1r - y1i * w1i;
                        b0i[q + S] = y1r * w1i + y1i * w1r;
                        b0r[q + 2 * S] = y2r * w2r - y2i * w2i;
                        b0i[q + 2 * S] = y2r * w2i + y2i * w2r;
                        b0r[q + 3 * S] = y3r * w3r - y3i * w3i;
                        b0i[q + 3 * S] = y3r * w3i + y3i * w3r;
                    }
                } else {  // 3
                    const R w1r = tr[2 * j], w1i = ti[2 * j], w2r = tr[2 * j + 1], w2i = ti[2 * j + 1];
                    const R c = (R)-0.5, sn = (R)(sign * 0.86602540378443864676);
#pragma omp simd
                    for (long q = 0; q < S; ++q) {
                        R x0r = a0r[q], x0i = a0i[q], x1r = a0r[q + sm], x1i = a0i[q + sm];
                        R x2r = a0r[q + 2 * sm], x2i = a0i[q + 2 * sm];
                        R sr = x1r + x2r, si = x1i + x2i, dr = x1r - x2r, di = x1i - x2i;
                        R y0r = x0r + sr, y0i = x0i + si;
                        R tr_ = x0r + c * sr, ti_ = x0i + c * si;
                        // sin term: sign * sin(2pi/3) * i * d
                        R ur = -sn * di, ui = sn * dr;
                        R y1r = tr_ + ur, y1i = ti_ + ui, y2r = tr_ - ur, y2i = ti_ - ui;
                        b0r[q] = y0r;
                        b0i[q] = y0i;
                        b0r[q + S] = y1r * w1r - y1i * w1i;
                        b0i[q + S] = y1r * w1i + y1i * w1r;
                        b0r[q + 2 * S] = y2r * w2r - y2i * w2i;
                        b0i[q + 2 * S] = y2r * w2i + y2i * w2r;
                    }
                }
            }
            std::swap(ar, br);
            std::swap(ai, bi);
            s *= p;
            len = m;
        }
        if (ar != xr) {
            std::copy(ar, ar + (size_t)n * kLines, xr);
            std::copy(ai, ai + (size_t)n * kLines, xi);
        }
    }

    void run_blue(R *xr, R *xi, R *, R *, int nb) const {
        // a = x * chirp, zero-padded to L; A = FFT_L(a); A *= V; c = IFFT_L(A); X = c * chirp
        std::vector<R> ar((size_t)L * kLines, 0), ai((size_t)L * kLines, 0);
        std::vector<R> tr((size_t)L * kLines), ti((size_t)L * kLines);
        for (int j = 0; j < n; ++j) {
            const R cr = chr[j], ci = chi[j];
            for (int b = 0; b < kLines; ++b) {
                R vr_ = xr[(size_t)j * kLines + b], vi_ = xi[(size_t)j * kLines + b];
                ar[(size_t)j * kLines + b] = vr_ * cr - vi_ * ci;
                ai[(size_t)j * kLines + b] = vr_ * ci + vi_ * cr;
            }
        }
        fwd->run(ar.data(), ai.data(), tr.data(), ti.data(), nb);
        for (int k = 0; k < L; ++k) {
            const R v_r = vr[k], v_i = vi[k];
#pragma omp simd
            for (int b = 0; b < kLines; ++b) {
                R a = ar[(size_t)k * kLines + b], c = ai[(size_t)k * kLines + b];
                ar[(size_t)k * kLines + b] = a * v_r - c * v_i;
                ai[(size_t)k * kLines + b] = a * v_i + c * v_r;
            }
        }
        inv->run(ar.data(), ai.data(), tr.data(), ti.data(), nb);
        for (int j = 0; j < n; ++j) {
            const R cr = chr[j], ci = chi[j];
            for (int b = 0; b < kLines; ++b) {
                R a = ar[(size_t)j * kLines + b], c = ai[(size_t)j * kLines + b];
                xr[(size_t)j * kLines + b] = a * cr - c * ci;
                xi[(size_t)j * kLines + b] = a * ci + c * cr;
            }
        }
    }
};

template <typename R>
const Line<R> &line_plan(int n, int sign) {
    static std::mutex mu;
    static std::map<std::pair<int, int>, std::unique_ptr<Line<R>>> cache;
    std::lock_guard<std::mutex> lk(mu);
    auto &slot = cache[{n, sign}];
    if (!slot) {
        slot.reset(new Line<R>());
        slot->init(n, sign);
    }
    return *slot;
}

/* Transform of every line along one axis of a row-major array of complex
 * values: L = the axis length, inner = product of the later extents, outer =
 * product of the earlier extents.  In place. */
template <typename R>
void c2c_axis(std::complex<R> *a, long outer, long L, long inner, int sign) {
    const Line<R> &pl = line_plan<R>((int)L, sign);
    const long groups_per_outer = (inner + kLines - 1) / kLines;
    const long ngroups = outer * groups_per_outer;
#pragma omp parallel
    {
        std::vector<R> xr((size_t)L * kLines), xi((size_t)L * kLines), yr((size_t)L * kLines),
            yi((size_t)L * kLines);
#pragma omp for schedule(dynamic, 4)
        for (long g = 0; g < ngroups; ++g) {
            const long o = g / groups_per_outer, i0 = (g % groups_per_outer) * kLines;
            const int nb = (int)std::min<long>(kLines, inner - i0);
            std::complex<R> *base = a + o * L * inner + i0;
            if (inner == 1) {
                // the lines are contiguous rows (nb == 1 here: inner == 1 gives one line per outer)
                for (long j = 0; j < L; ++j) {
                    xr[(size_t)j * kLines] = base[j].real();
                    xi[(size_t)j * kLines] = base[j].imag();
                }
            } else {
                for (long j = 0; j < L; ++j) {
                    const std::complex<R> *src = base + j * inner;
                    for (int b = 0; b < nb; ++b) {
                        xr[(size_t)j * kLines + b] = src[b].real();
                        xi[(size_t)j * kLines + b] = src[b].imag();
                    }
                }
            }
            pl.run(xr.data(), xi.data(), yr.data(), yi.data(), nb);
            for (long j = 0; j < L; ++j) {
                std::complex<R> *dst = base + j * inner;
                for (int b = 0; b < nb; ++b)
                    dst[b] = std::complex<R>(xr[(size_t)j * kLines + b], xi[(size_t)j * kLines + b]);
            }
        }
    }
}

/* Contiguous rows (inner == 1) in groups of kLines rows per scratch. */
template <typename R>
void c2c_rows(std::complex<R> *a, long rows, long L, int sign) {
    const Line<R> &pl = line_plan<R>((int)L, sign);
    const long ngroups = (rows + kLines - 1) / kLines;
#pragma omp parallel
    {
        std::vector<R> xr((size_t)L * kLines), xi((size_t)L * kLines), yr((size_t)L * kLines),
            yi((size_t)L * kLines);
#pragma omp for schedule(dynamic, 4)
        for (long g = 0; g < ngroups; ++g) {
            const long r0 = g * kLines;
            const int nb = (int)std::min<long>(kLines, rows - r0);
            for (int b = 0; b < nb; ++b) {
                const std::complex<R> *src = a + (r0 + b) * L;
                for (long j = 0; j < L; ++j) {
                    xr[(size_t)j * kLines + b] = src[j].real();
                    xi[(size_t)j * kLines + b] = src[j].imag();
                }
            }
            pl.run(xr.data(), xi.data(), yr.data(), yi.data(), nb);
            for (int b = 0; b < nb; ++b) {
                std::complex<R> *dst = a + (r0 + b) * L;
                for (long j = 0; j < L; ++j)
                    dst[j] = std::complex<R>(xr[(size_t)j * kLines + b], xi[(size_t)j * kLines + b]);
            }
        }
    }
}

/* n-dimensional c2c in place (row-major dims n[0..rank)). */
template <typename R>
void c2c_nd(std::complex<R> *a, const std::vector<long> &n, int sign) {
    const int rank = (int)n.size();
    long total = 1;
    for (long v : n) total *= v;
    for (int d = rank - 1; d >= 0; --d) {
        long inner = 1;
        for (int e = d + 1; e < rank; ++e) inner *= n[e];
        const long outer = total / (inner * n[d]);
        if (n[d] == 1) continue;
        if (inner == 1) c2c_rows(a, outer, n[d], sign);
        else c2c_axis(a, outer, n[d], inner, sign);
    }
}

/* Real rows of even length N -> half spectra of N/2 + 1 values (sign -1), by
 * a complex transform of N/2 points of the packed row. */
template <typename R>
void r2c_rows(const R *in, std::complex<R> *out, long rows, long N) {
    const long M = N / 2, nh = M + 1;
    const Line<R> &pl = line_plan<R>((int)M, -1);
    std::vector<R> wr(M + 1), wi(M + 1);
    for (long k = 0; k <= M; ++k) {
        long double a = -2.0L * 3.14159265358979323846264338327950288L * (long double)k / (long double)N;
        wr[k] = (R)cosl(a);
        wi[k] = (R)sinl(a);
    }
    const long ngroups = (rows + kLines - 1) / kLines;
#pragma omp parallel
    {
        std::vector<R> xr((size_t)M * kLines), xi((size_t)M * kLines), yr((size_t)M * kLines),
            yi((size_t)M * kLines);
#pragma omp for schedule(dynamic, 4)
        for (long g = 0; g < ngroups; ++g) {
            const long r0 = g * kLines;
            const int nb = (int)std::min<long>(kLines, rows - r0);
            for (int b = 0; b < nb; ++b) {
                const R *src = in + (r0 + b) * N;
                for (long e = 0; e < M; ++e) {
                    xr[(size_t)e * kLines + b] = src[2 * e];
                    xi[(size_t)e * kLines + b] = src[2 * e + 1];
                }
            }
            pl.run(xr.data(), xi.data(), yr.data(), yi.data(), nb);
            for (int b = 0; b < nb; ++b) {
                std::complex<R> *dst = out + (r0 + b) * nh;
                for (long k = 0; k <= M; ++k) {
                    const long k1 = k % M, k2 = (M - k) % M;
                    const R zr = xr[(size_t)k1 * kLines + b], zi = xi[(size_t)k1 * kLines + b];
                    const R cr = xr[(size_t)k2 * kLines + b], ci = -xi[(size_t)k2 * kLines + b];
                    const R er = (zr + cr) * (R)0.5, ei = (zi + ci) * (R)0.5;      // E = (Z + conj Z')/2
                    const R odr = (zi - ci) * (R)0.5, odi = -(zr - cr) * (R)0.5;  // O = (Z - conj Z')/2i
                    dst[k] = std::complex<R>(er + wr[k] * odr - wi[k] * odi, ei + wr[k] * odi + wi[k] * odr);
                }
            }
        }
    }
}

/* Half spectra of N/2 + 1 values -> real rows of even length N (sign +1,
 * unnormalised), by packing into a complex row of N/2 points. */
template <typename R>
void c2r_rows(const std::complex<R> *in, R *out, long rows, long N) {
    const long M = N / 2, nh = M + 1;
    const Line<R> &pl = line_plan<R>((int)M, +1);
    std::vector<R> wr(M), wi(M);
    for (long k = 0; k < M; ++k) {
        long double a = 2.0L * 3.14159265358979323846264338327950288L * (long double)k / (long double)N;
        wr[k] = (R)cosl(a);
        wi[k] = (R)sinl(a);
    }
    const long ngroups = (rows + kLines - 1) / kLines;
#pragma omp parallel
    {
        std::vector<R> xr((size_t)M * kLines), xi((size_t)M * kLines), yr((size_t)M * kLines),
            yi((size_t)M * kLines);
#pragma omp for schedule(dynamic, 4)
        for (long g = 0; g < ngroups; ++g) {
            const long r0 = g * kLines;
            const int nb = (int)std::min<long>(kLines, rows - r0);
            for (int b = 0; b < nb; ++b) {
                const std::complex<R> *src = in + (r0 + b) * nh;
                for (long k = 0; k < M; ++k) {
                    const std::complex<R> X = src[k], Y = std::conj(src[M - k]);
                    const std::complex<R> s = X + Y, d = X - Y;
                    // Z = s + i w d
                    const R tdr = wr[k] * d.real() - wi[k] * d.imag(), tdi = wr[k] * d.imag() + wi[k] * d.real();
                    xr[(size_t)k * kLines + b] = s.real() - tdi;
                    xi[(size_t)k * kLines + b] = s.imag() + tdr;
                }
            }
            pl.run(xr.data(), xi.data(), yr.data(), yi.data(), nb);
            for (int b = 0; b < nb; ++b) {
                R *dst = out + (r0 + b) * N;
                for (long e = 0; e < M; ++e) {
                    dst[2 * e] = xr[(size_t)e * kLines + b];
                    dst[2 * e + 1] = xi[(size_t)e * kLines + b];
                }
            }
        }
    }
}

}  // namespace lc_fast

#endif
