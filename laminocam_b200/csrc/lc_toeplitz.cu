// PSF generation (closed form, FP64) and the fused-FFT Toeplitz apply.
#include <algorithm>
#include <array>
#include <cmath>
#include <cstdlib>
#include <tuple>

#include "lc_regfft.cuh"
#include "lc_toeplitz.hpp"

namespace lc {

namespace {

// sum_{m=0}^{n-1} exp(i u (2 pi/n)(m - (n-1)/2)) = sin(pi u) / sin(pi u / n)
__device__ __forceinline__ double dirichlet(double u, int n) {
    double v = u / (double)n;
    double sv = sinpi(v);
    if (fabs(sv) < 1e-13) {
        // u/n is (numerically) an integer: limit n cos(pi u) / cos(pi u / n)
        return (double)n * cospi(u) / cospi(v);
    }
    return sinpi(u) / sv;
}

// Per-angle coefficients of the fast PSF generator: uX = a . k, uY = b . k
// (k = (kx, ky, kz)), and (4 sin^2(t/2), sin t) for the steps h = a0, a0 / nx,
// b0, b0 / ny of sin(pi uX), sin(pi uX / nx), ... from one kx to the next,
// reduced to t = pi (h - round(h)).
struct PsfAngle {
    double a[3], b[3];
    double2 stepA, stepB, stepC, stepD;
};

// sin(pi (u0 + s h)), s = 0, 1, ..., by Reinsch's modification of the
// three-term recurrence.  The step is first reduced to |h'| <= 1/2,
// h' = h - round(h), using sin(pi (u0 + s h)) = (-1)^(s round(h)) sin(pi (u0 + s h'))
// (|h| <= 1 here, so round(h) is odd exactly when |h| > 1/2).  With t = pi h',
// lambda = 4 sin^2(t/2) and d_s = e_s - e_(s-1) for e_s = sin(pi (u0 + s h')):
//   d_(s+1) = d_s - lambda e_s,   e_(s+1) = e_s + d_(s+1).
// lambda carries t to full relative precision, which the plain recurrence
// (2 cos t) loses for small t (a phase drift of ~eps/t per step).  Over 16
// steps the error stays below 5e-16 for |h| <= 0.004 and 5e-15 for |h| <= 1
// (checked against exact values), one FMA and one add per step.
template <bool FLIP>
struct SinSeq {
    double cur, d, lam, flipf;
    // step = (4 sin^2(t/2), sin t) of the reduced step; h = the unreduced step
    __device__ __forceinline__ void init(double u0, double2 step, double h) {
        double s0, c0;
        sincospi(u0, &s0, &c0);
        cur = s0;
        lam = step.x;
        d = fma(0.5 * step.x, s0, c0 * step.y);  // e_0 - e_(-1) = s0 (1 - cos t) + c0 sin t
        flipf = (FLIP && fabs(h) > 0.5) ? -1.0 : 1.0;
    }
    // sin(pi (u0 + s h)) at the current step s
    __device__ __forceinline__ double val(int s) const { return (FLIP && (s & 1)) ? cur * flipf : cur; }
    __device__ __forceinline__ void advance() {
        d = fma(-lam, cur, d);
        cur += d;
    }
};

// Below this |sin(pi u / n)| a Dirichlet term is evaluated in closed form.
// Above it the recurrences' absolute error (~5e-16) gives a term a relative
// error of at most ~5e-10, and the kernel stays within ~1e-11 of the exact sum
// (the spectrum is then stored in FP32).  A larger threshold sends most warps
// through the closed form (0.07 % of the terms at 1e-3 already put 9 % of the
// warp steps there) and costs several times the whole sum.
constexpr double kDenMin = 1e-6;

// Dirichlet term sin(pi u) / sin(pi u / n) from the two sines, or from the
// closed form near its poles
__device__ __forceinline__ double dirichlet_term(double num, double den, double u, int n) {
    return fabs(den) > kDenMin ? num / den : dirichlet(u, n);
}

__device__ __forceinline__ int mirror_index(int j, int P) {
    // index of -k for mode index j (k = j - P/2); -1 when -k is outside the grid
    if (P % 2 == 0) return j == 0 ? -1 : P - j;
    return P - 1 - j;
}

// Rows of K (all kx of one (kz, ky)) in segments of S values of kx, 3D.  The
// sum over angles uses the Dirichlet closed form, with sin(pi u) and
// sin(pi u / n) advanced along kx by the three-term sine recurrence (FP64) and
// evaluated in closed form whenever the denominator is small.
// Only the half space kz <= 0 is summed; K(-k) = K(k) fills the rest.  With
// `mirror` the angle set is also closed under the reflection that negates the
// kz coefficients, K(kx, ky, -kz) = K(k), and a quarter of the grid is summed:
// rows with ky <= 0 of each plane kz <= 0, and K(-kx, -ky, kz), K(-k),
// K(kx, ky, -kz) from them (a per-angle pair whose a and b differ only in the
// sign of their kz coefficient).
template <int S, bool ONE_GROUP>
__global__ void __launch_bounds__(128, ONE_GROUP ? 3 : 1) psf_rows_kernel(const PsfAngle *__restrict__ angles, int ntheta,
                                                      const int *__restrict__ groups, int ngroups,
                                                      int nx, int ny, int P1, int P2, int P3, int mirror,
                                                      int zlo, double *__restrict__ K) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    PsfAngle *ang = reinterpret_cast<PsfAngle *>(smem_raw);
    int *gst = reinterpret_cast<int *>(ang + ntheta);
    for (int i = threadIdx.x; i < ntheta; i += blockDim.x) ang[i] = angles[i];
    for (int i = threadIdx.x; i <= ngroups; i += blockDim.x) gst[i] = groups[i];
    __syncthreads();
    const int nseg = (P3 + S - 1) / S;
    // rows of the half space: jz <= P1/2, all jy (jy <= P2/2 with the mirror);
    // only the planes zlo .. P1/2 of the half, the rest is not needed
    const int rows_per_plane = mirror ? P2 / 2 + 1 : P2;
    const long nrows_half = (long)(P1 / 2 + 1 - zlo) * rows_per_plane;
    const long items = nrows_half * nseg;
    const double inv_nx = 1.0 / (double)nx, inv_ny = 1.0 / (double)ny;
    for (long it = (long)blockIdx.x * blockDim.x + threadIdx.x; it < items;
         it += (long)gridDim.x * blockDim.x) {
        const long row = it / nseg;
        const int seg = (int)(it - row * nseg);
        const int pz = (int)(row / rows_per_plane);
        const int jy = (int)(row - (long)pz * rows_per_plane);
        const int jz = zlo + pz;
        const int jx0 = seg * S;
        const double kx0 = (double)(jx0 - P3 / 2);
        const double ky = (double)(jy - P2 / 2);
        const double kz = (double)(jz - P1 / 2);
        // one group (every angle of equal beta and gamma): acc is formed from ay
        // after the angle sum, so the two arrays are never live together
        double acc[S];
        if constexpr (!ONE_GROUP) {
#pragma unroll
            for (int s = 0; s < S; ++s) acc[s] = 0.0;
        }
        // uX = a . k does not depend on theta (a is the first column of
        // transpose(Rx(theta) Ry(beta) Rz(gamma)), which Rx leaves alone), so
        // within a group of angles of equal (beta, gamma) the sum factors:
        // K = sum_groups D_nx(uX) * sum_{theta in group} D_ny(uY).  Four
        // (then two, then one) angles share one division.
        for (int gi = 0; gi < (ONE_GROUP ? 1 : ngroups); ++gi) {
            const int i0 = gst[gi], i1 = gst[gi + 1];
            double ay[S];
#pragma unroll
            for (int s = 0; s < S; ++s) ay[s] = 0.0;
            int i = i0;
            // four angles per division:
            // a/b + c/d + e/f + g/h = ((a d + c b) f h + (e h + g f) b d) / (b d f h)
            for (; i + 3 < i1; i += 4) {
                const PsfAngle &A = ang[i], &B = ang[i + 1], &C = ang[i + 2], &D = ang[i + 3];
                const double uA = A.b[0] * kx0 + A.b[1] * ky + A.b[2] * kz;
                const double uB = B.b[0] * kx0 + B.b[1] * ky + B.b[2] * kz;
                const double uC = C.b[0] * kx0 + C.b[1] * ky + C.b[2] * kz;
                const double uD = D.b[0] * kx0 + D.b[1] * ky + D.b[2] * kz;
                SinSeq<true> nA, nB, nC, nD;
                SinSeq<false> dA, dB, dC, dD;
                nA.init(uA, A.stepC, A.b[0]);
                dA.init(uA * inv_ny, A.stepD, A.b[0] * inv_ny);
                nB.init(uB, B.stepC, B.b[0]);
                dB.init(uB * inv_ny, B.stepD, B.b[0] * inv_ny);
                nC.init(uC, C.stepC, C.b[0]);
                dC.init(uC * inv_ny, C.stepD, C.b[0] * inv_ny);
                nD.init(uD, D.stepC, D.b[0]);
                dD.init(uD * inv_ny, D.stepD, D.b[0] * inv_ny);
#pragma unroll
                for (int s = 0; s < S; ++s) {
                    if (fabs(dA.cur) > kDenMin && fabs(dB.cur) > kDenMin && fabs(dC.cur) > kDenMin &&
                        fabs(dD.cur) > kDenMin) {
                        const double pab = fma(nA.val(s), dB.cur, nB.val(s) * dA.cur), qab = dA.cur * dB.cur;
                        const double pcd = fma(nC.val(s), dD.cur, nD.val(s) * dC.cur), qcd = dC.cur * dD.cur;
                        ay[s] += fma(pab, qcd, pcd * qab) / (qab * qcd);
                    } else {
                        const double sd = (double)s;
                        ay[s] += dirichlet_term(nA.val(s), dA.cur, uA + sd * A.b[0], ny) +
                                 dirichlet_term(nB.val(s), dB.cur, uB + sd * B.b[0], ny) +
                                 dirichlet_term(nC.val(s), dC.cur, uC + sd * C.b[0], ny) +
                                 dirichlet_term(nD.val(s), dD.cur, uD + sd * D.b[0], ny);
                    }
                    nA.advance();
                    dA.advance();
                    nB.advance();
                    dB.advance();
                    nC.advance();
                    dC.advance();
                    nD.advance();
                    dD.advance();
                }
            }
            for (; i + 1 < i1; i += 2) {
                const PsfAngle &A = ang[i], &B = ang[i + 1];
                const double uA = A.b[0] * kx0 + A.b[1] * ky + A.b[2] * kz;
                const double uB = B.b[0] * kx0 + B.b[1] * ky + B.b[2] * kz;
                SinSeq<true> nA, nB;
                SinSeq<false> dA, dB;
                nA.init(uA, A.stepC, A.b[0]);
                dA.init(uA * inv_ny, A.stepD, A.b[0] * inv_ny);
                nB.init(uB, B.stepC, B.b[0]);
                dB.init(uB * inv_ny, B.stepD, B.b[0] * inv_ny);
#pragma unroll
                for (int s = 0; s < S; ++s) {
                    if (fabs(dA.cur) > kDenMin && fabs(dB.cur) > kDenMin) {
                        ay[s] += fma(nA.val(s), dB.cur, nB.val(s) * dA.cur) / (dA.cur * dB.cur);
                    } else {
                        ay[s] += dirichlet_term(nA.val(s), dA.cur, uA + (double)s * A.b[0], ny) +
                                 dirichlet_term(nB.val(s), dB.cur, uB + (double)s * B.b[0], ny);
                    }
                    nA.advance();
                    dA.advance();
                    nB.advance();
                    dB.advance();
                }
            }
            if (i < i1) {
                const PsfAngle &A = ang[i];
                const double uA = A.b[0] * kx0 + A.b[1] * ky + A.b[2] * kz;
                SinSeq<true> nA;
                SinSeq<false> dA;
                nA.init(uA, A.stepC, A.b[0]);
                dA.init(uA * inv_ny, A.stepD, A.b[0] * inv_ny);
#pragma unroll
                for (int s = 0; s < S; ++s) {
                    ay[s] += dirichlet_term(nA.val(s), dA.cur, uA + (double)s * A.b[0], ny);
                    nA.advance();
                    dA.advance();
                }
            }
            const PsfAngle &A = ang[i0];
            const double uX0 = A.a[0] * kx0 + A.a[1] * ky + A.a[2] * kz;
            SinSeq<true> nX;
            SinSeq<false> dX;
            nX.init(uX0, A.stepA, A.a[0]);
            dX.init(uX0 * inv_nx, A.stepB, A.a[0] * inv_nx);
#pragma unroll
            for (int s = 0; s < S; ++s) {
                const double tX = dirichlet_term(nX.val(s), dX.cur, uX0 + (double)s * A.a[0], nx);
                acc[s] = ONE_GROUP ? tX * ay[s] : fma(tX, ay[s], acc[s]);
                nX.advance();
                dX.advance();
            }
        }
        const long plane = (long)P2 * P3;
        const int mz = mirror_index(jz, P1);
        const int my = mirror_index(jy, P2);
        auto put = [&](int z, int y, int x, double v) { K[(long)z * plane + (long)y * P3 + x] = v; };
        if (!mirror) {
            const bool self_plane = mz == jz;
#pragma unroll
            for (int s = 0; s < S; ++s) {
                const int jx = jx0 + s;
                if (jx >= P3) break;
                put(jz, jy, jx, acc[s]);
                if (self_plane) continue;  // its mirror is summed by another row of the half space
                const int mx = mirror_index(jx, P3);
                if (mz < 0 || my < 0 || mx < 0) continue;
                put(mz, my, mx, acc[s]);
            }
        } else {
            // (jz, jy, jx) summed; (jz, my, mx), (mz, my, mx), (mz, jy, jx) copied.
            // A copy that lands on a summed row or plane is left to the sum.
#pragma unroll
            for (int s = 0; s < S; ++s) {
                const int jx = jx0 + s;
                if (jx >= P3) break;
                const int mx = mirror_index(jx, P3);
                put(jz, jy, jx, acc[s]);
                if (my != jy && my >= 0 && mx >= 0) put(jz, my, mx, acc[s]);
                if (mz != jz && mz >= 0) put(mz, jy, jx, acc[s]);
                if (mz != jz && my != jy && mz >= 0 && my >= 0 && mx >= 0) put(mz, my, mx, acc[s]);
            }
        }
    }
}

// ---- 2D kernel: K(kx, ky) = sum_theta D_nx(cos(theta) kx + sin(theta) ky) ----
// Rows ky <= 0 in segments of S values of kx (with the mirror, kx <= 0 only;
// with the quarter-turn closure, mirror == 2, only kx <= ky; the other
// entries are copies).  G lanes of one warp share a segment: each sums a
// contiguous share of the angle quads (the last lane also the 1 to 3 angles
// left over), and a butterfly of shuffles adds the shares, so that every lane
// of the group holds the same total.  The summation order depends on G, and
// G on the grid size and the angle count alone, so a kernel does not depend
// on what else runs beside it.  Small grids (a few hundred segments) split
// the angle sum over up to 32 lanes and still fill the GPU.
template <int S>
__device__ __forceinline__ void psf2d_sum_quads(const PsfAngle *ang, int i0, int i1, double kx0, double ky, int nx,
                                                double inv_nx, double (&acc)[S]) {
    for (int i = i0; i < i1; i += 4) {
        const PsfAngle &A = ang[i], &B = ang[i + 1], &C = ang[i + 2], &D = ang[i + 3];
        const double uA = A.a[0] * kx0 + A.a[1] * ky;
        const double uB = B.a[0] * kx0 + B.a[1] * ky;
        const double uC = C.a[0] * kx0 + C.a[1] * ky;
        const double uD = D.a[0] * kx0 + D.a[1] * ky;
        SinSeq<true> nA, nB, nC, nD;
        SinSeq<false> dA, dB, dC, dD;
        nA.init(uA, A.stepA, A.a[0]);
        dA.init(uA * inv_nx, A.stepB, A.a[0] * inv_nx);
        nB.init(uB, B.stepA, B.a[0]);
        dB.init(uB * inv_nx, B.stepB, B.a[0] * inv_nx);
        nC.init(uC, C.stepA, C.a[0]);
        dC.init(uC * inv_nx, C.stepB, C.a[0] * inv_nx);
        nD.init(uD, D.stepA, D.a[0]);
        dD.init(uD * inv_nx, D.stepB, D.a[0] * inv_nx);
#pragma unroll
        for (int s = 0; s < S; ++s) {
            if (fabs(dA.cur) > kDenMin && fabs(dB.cur) > kDenMin && fabs(dC.cur) > kDenMin &&
                fabs(dD.cur) > kDenMin) {
                const double pab = fma(nA.val(s), dB.cur, nB.val(s) * dA.cur), qab = dA.cur * dB.cur;
                const double pcd = fma(nC.val(s), dD.cur, nD.val(s) * dC.cur), qcd = dC.cur * dD.cur;
                acc[s] += fma(pab, qcd, pcd * qab) / (qab * qcd);
            } else {
                const double sd = (double)s;
                acc[s] += dirichlet_term(nA.val(s), dA.cur, uA + sd * A.a[0], nx) +
                          dirichlet_term(nB.val(s), dB.cur, uB + sd * B.a[0], nx) +
                          dirichlet_term(nC.val(s), dC.cur, uC + sd * C.a[0], nx) +
                          dirichlet_term(nD.val(s), dD.cur, uD + sd * D.a[0], nx);
            }
            nA.advance();
            dA.advance();
            nB.advance();
            dB.advance();
            nC.advance();
            dC.advance();
            nD.advance();
            dD.advance();
        }
    }
}

template <int S>
__device__ __forceinline__ void psf2d_sum_tail(const PsfAngle *ang, int i, int ntheta, double kx0, double ky, int nx,
                                               double inv_nx, double (&acc)[S]) {
    for (; i < ntheta; ++i) {
        const PsfAngle &A = ang[i];
        const double uA = A.a[0] * kx0 + A.a[1] * ky;
        SinSeq<true> nA;
        SinSeq<false> dA;
        nA.init(uA, A.stepA, A.a[0]);
        dA.init(uA * inv_nx, A.stepB, A.a[0] * inv_nx);
#pragma unroll
        for (int s = 0; s < S; ++s) {
            acc[s] += dirichlet_term(nA.val(s), dA.cur, uA + (double)s * A.a[0], nx);
            nA.advance();
            dA.advance();
        }
    }
}

// Segments of 16 summed in rows 0 .. J-1: with mirror == 2 row jy holds
// jy / 16 + 1 of them (kx <= ky), otherwise nseg.
__host__ __device__ __forceinline__ long psf2d_first_seg(long J, long nseg, int mirror) {
    if (mirror != 2) return J * nseg;
    const long A = J / 16, R = J % 16;
    return J + 16 * A * (A - 1) / 2 + R * A;
}

template <int S, int G>
__global__ void __launch_bounds__(128) psf2d_kernel(const PsfAngle *__restrict__ angles, int ntheta, int nx, int P2,
                                                    int P3, int mirror, double *__restrict__ K) {
    static_assert(S == 16, "psf2d_first_seg counts segments of 16");
    static_assert(G >= 1 && G <= 32 && (G & (G - 1)) == 0, "G lanes per segment: a power of two up to 32");
    extern __shared__ __align__(16) unsigned char smem_raw[];
    PsfAngle *ang = reinterpret_cast<PsfAngle *>(smem_raw);
    for (int i = threadIdx.x; i < ntheta; i += blockDim.x) ang[i] = angles[i];
    __syncthreads();
    const int xend = mirror ? P3 / 2 + 1 : P3;
    const int nseg = (xend + S - 1) / S;
    const int nrows = P2 / 2 + 1;
    const long items = psf2d_first_seg(nrows, nseg, mirror);
    const double inv_nx = 1.0 / (double)nx;
    constexpr int IPW = 32 / G;  // segments per warp
    const int lane = threadIdx.x & 31, sub = lane % G;
    const long warp = ((long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const long nwarps = ((long)gridDim.x * blockDim.x) >> 5;
    // this lane's angle quads; the angles after the last quad go to lane G - 1
    const int nq = ntheta / 4;
    const int i0 = 4 * (int)((long)sub * nq / G), i1 = 4 * (int)((long)(sub + 1) * nq / G);
    // the loop is warp-uniform: every lane reaches the shuffles
    for (long base = warp * IPW; base < items; base += nwarps * IPW) {
        const long it = base + lane / G;
        const bool active = it < items;
        // row of segment it: the last row whose first segment is <= it
        int jy = 0, seg = 0;
        if (active) {
            int lo = 0, hi = nrows - 1;
            while (lo < hi) {
                const int mid = (lo + hi + 1) >> 1;
                if (psf2d_first_seg(mid, nseg, mirror) <= it) lo = mid;
                else hi = mid - 1;
            }
            jy = lo;
            seg = (int)(it - psf2d_first_seg(jy, nseg, mirror));
        }
        const int jx0 = seg * S;
        const double kx0 = (double)(jx0 - P3 / 2);
        const double ky = (double)(jy - P2 / 2);
        double acc[S];
#pragma unroll
        for (int s = 0; s < S; ++s) acc[s] = 0.0;
        if (active) {
            psf2d_sum_quads<S>(ang, i0, i1, kx0, ky, nx, inv_nx, acc);
            if (sub == G - 1) psf2d_sum_tail<S>(ang, 4 * nq, ntheta, kx0, ky, nx, inv_nx, acc);
        }
#pragma unroll
        for (int off = G / 2; off >= 1; off >>= 1) {
#pragma unroll
            for (int s = 0; s < S; ++s) acc[s] += __shfl_xor_sync(0xffffffffu, acc[s], off);
        }
        if (!active) continue;
        const int my = mirror_index(jy, P2);
        auto put = [&](int y, int x, double v) { K[(long)y * P3 + x] = v; };
        if (!mirror) {
            const bool self_row = my == jy;
#pragma unroll
            for (int s = 0; s < S; ++s) {
                const int jx = jx0 + s;
                if (s % G != sub) continue;
                if (jx >= P3) break;
                put(jy, jx, acc[s]);
                if (self_row) continue;  // its mirror is summed in this row
                const int mx = mirror_index(jx, P3);
                if (my < 0 || mx < 0) continue;
                put(my, mx, acc[s]);
            }
        } else {
            // (jy, jx <= P3/2) summed; (jy, mx), (my, mx), (my, jx) copied, and
            // with mirror == 2 (jx <= jy summed) the same four transposed
#pragma unroll
            for (int s = 0; s < S; ++s) {
                const int jx = jx0 + s;
                if (s % G != sub) continue;
                if (jx >= xend || (mirror == 2 && jx > jy)) break;
                const int mx = mirror_index(jx, P3);
                const double v = acc[s];
                auto four = [&](int r, int c, int mr, int mc) {
                    put(r, c, v);
                    if (mc != c && mc >= 0) put(r, mc, v);
                    if (mr != r && mr >= 0) {
                        put(mr, c, v);
                        if (mc >= 0) put(mr, mc, v);
                    }
                };
                four(jy, jx, my, mx);
                if (mirror == 2 && jx != jy) four(jx, jy, mx, my);
            }
        }
    }
}

// ---- tabulated 3D kernel for one tilt and beta = 0 (laminography) ----
// With beta = 0 and one gamma for every angle, a = (cg, -sg, 0) and
// b_theta = (ct sg, ct cg, -st), so
//     K(k) = D_nx(w) * S(u, kz),  w = cg kx - sg ky,  u = sg kx + cg ky,
//     S(u, kz) = sum_theta D_ny(ct u - st kz).
// Each Dirichlet term is a sum of exponentials of u with frequencies below pi,
// so S(., kz) is band-limited: it is summed exactly (FP64, the recurrences of
// psf_rows_kernel) on a grid of u of spacing 1/32 for every needed kz <= 0
// and interpolated with ten equispaced points (Lagrange, barycentric form).
// The interpolation error is below (pi h)^10 |omega| / 10! of the kernel's
// peak, about 1e-14 at h = 1/32.  With the kz mirror S(u, -kz) = S(u, kz).
struct TabAngle {
    double ct, st;
    double2 stepN, stepD;  // (4 sin^2(t/2), sin t) of the u steps ct h and ct h / ny
};

constexpr int kTabSeg = 16;     // table samples per thread (one recurrence run)
constexpr int kTabPoints = 10;  // interpolation stencil

// table[r * nu + j] = S(u0 + j h, -r), r < nr, j < nu
__global__ void __launch_bounds__(128) psf_table_kernel(const TabAngle *__restrict__ angles, int ntheta, int ny,
                                                        double u0, double h, int nu, int nr,
                                                        double *__restrict__ table) {
    extern __shared__ __align__(16) unsigned char tab_smem[];
    TabAngle *ang = reinterpret_cast<TabAngle *>(tab_smem);
    for (int i = threadIdx.x; i < ntheta; i += blockDim.x) ang[i] = angles[i];
    __syncthreads();
    constexpr int S = kTabSeg;
    const int nseg = (nu + S - 1) / S;
    const double inv_ny = 1.0 / (double)ny;
    for (long it = (long)blockIdx.x * blockDim.x + threadIdx.x; it < (long)nr * nseg;
         it += (long)gridDim.x * blockDim.x) {
        const int r = (int)(it / nseg), seg = (int)(it - (long)r * nseg);
        const int j0 = seg * S;
        const double kz = -(double)r;
        const double ub = u0 + (double)j0 * h;
        double acc[S];
#pragma unroll
        for (int q = 0; q < S; ++q) acc[q] = 0.0;
        int i = 0;
        for (; i + 3 < ntheta; i += 4) {
            const TabAngle &A = ang[i], &B = ang[i + 1], &C = ang[i + 2], &D = ang[i + 3];
            const double vA = A.ct * ub - A.st * kz, vB = B.ct * ub - B.st * kz;
            const double vC = C.ct * ub - C.st * kz, vD = D.ct * ub - D.st * kz;
            SinSeq<false> nA, nB, nC, nD, dA, dB, dC, dD;
            nA.init(vA, A.stepN, A.ct * h);
            dA.init(vA * inv_ny, A.stepD, A.ct * h * inv_ny);
            nB.init(vB, B.stepN, B.ct * h);
            dB.init(vB * inv_ny, B.stepD, B.ct * h * inv_ny);
            nC.init(vC, C.stepN, C.ct * h);
            dC.init(vC * inv_ny, C.stepD, C.ct * h * inv_ny);
            nD.init(vD, D.stepN, D.ct * h);
            dD.init(vD * inv_ny, D.stepD, D.ct * h * inv_ny);
#pragma unroll
            for (int q = 0; q < S; ++q) {
                if (fabs(dA.cur) > kDenMin && fabs(dB.cur) > kDenMin && fabs(dC.cur) > kDenMin &&
                    fabs(dD.cur) > kDenMin) {
                    const double pab = fma(nA.cur, dB.cur, nB.cur * dA.cur), qab = dA.cur * dB.cur;
                    const double pcd = fma(nC.cur, dD.cur, nD.cur * dC.cur), qcd = dC.cur * dD.cur;
                    acc[q] += fma(pab, qcd, pcd * qab) / (qab * qcd);
                } else {
                    const double qd = (double)q * h;
                    acc[q] += dirichlet_term(nA.cur, dA.cur, vA + qd * A.ct, ny) +
                              dirichlet_term(nB.cur, dB.cur, vB + qd * B.ct, ny) +
                              dirichlet_term(nC.cur, dC.cur, vC + qd * C.ct, ny) +
                              dirichlet_term(nD.cur, dD.cur, vD + qd * D.ct, ny);
                }
                nA.advance();
                dA.advance();
                nB.advance();
                dB.advance();
                nC.advance();
                dC.advance();
                nD.advance();
                dD.advance();
            }
        }
        for (; i < ntheta; ++i) {
            const TabAngle &A = ang[i];
            const double vA = A.ct * ub - A.st * kz;
            SinSeq<false> nA, dA;
            nA.init(vA, A.stepN, A.ct * h);
            dA.init(vA * inv_ny, A.stepD, A.ct * h * inv_ny);
#pragma unroll
            for (int q = 0; q < S; ++q) {
                acc[q] += dirichlet_term(nA.cur, dA.cur, vA + (double)q * h * A.ct, ny);
                nA.advance();
                dA.advance();
            }
        }
#pragma unroll
        for (int q = 0; q < S; ++q)
            if (j0 + q < nu) table[(long)r * nu + j0 + q] = acc[q];
    }
}

// K from the table on the planes zs .. zs + nzc - 1, rows ky <= 0, and by the
// symmetries of the scan on the rest: K(-kx, -ky, kz) = K(k) always (u and w
// change sign, and S(-u, kz) = S(u, -kz) = S(u, kz)), and with zmirror the
// planes P1 - jz as well (K(kx, ky, -kz) = K(k)).  A copy that lands on a
// computed entry is left to it, so every entry has one writer.
//   K = D_nx(cg kx - sg ky) * S(sg kx + cg ky, -|kz|)
// The ten Lagrange weights are formed as c_q prod_{m != q} (t - m) from prefix
// and suffix products: no division, and exact at the nodes.
__global__ void __launch_bounds__(256) psf_interp_kernel(const double *__restrict__ table, double u0, double inv_h,
                                                         int nu, int nr, double sg, double cg, int nx, int P1, int P2,
                                                         int P3, int zs, int nzc, int zmirror, double *__restrict__ K) {
    // 1 / prod_{m != q} (q - m) = (-1)^(9-q) / (q! (9-q)!)
    constexpr double c[kTabPoints] = {-1.0 / 362880.0, 1.0 / 40320.0, -1.0 / 10080.0, 1.0 / 4320.0,
                                      -1.0 / 2880.0,   1.0 / 2880.0, -1.0 / 4320.0,  1.0 / 10080.0,
                                      -1.0 / 40320.0,  1.0 / 362880.0};
    const int rows = P2 / 2 + 1;
    const long plane = (long)P2 * P3, half = (long)rows * P3, total = (long)nzc * half;
    for (long idx = (long)blockIdx.x * blockDim.x + threadIdx.x; idx < total;
         idx += (long)gridDim.x * blockDim.x) {
        const int pz = (int)(idx / half);
        const long rem = idx - (long)pz * half;
        const int jy = (int)(rem / P3), jx = (int)(rem - (long)jy * P3);
        const int jz = zs + pz;
        const double kx = (double)(jx - P3 / 2), ky = (double)(jy - P2 / 2);
        const int r = abs(jz - P1 / 2);
        const double u = sg * kx + cg * ky, w = cg * kx - sg * ky;
        const double t = (u - u0) * inv_h;
        const int j = (int)floor(t) - 4;
        const double tt = t - (double)j;  // in [4, 5)
        const double *row = table + (long)min(r, nr - 1) * nu + j;
        double d[kTabPoints], pre[kTabPoints];
#pragma unroll
        for (int q = 0; q < kTabPoints; ++q) d[q] = tt - (double)q;
        pre[0] = 1.0;
#pragma unroll
        for (int q = 1; q < kTabPoints; ++q) pre[q] = pre[q - 1] * d[q - 1];
        double suf = 1.0, sv = 0.0;
#pragma unroll
        for (int q = kTabPoints - 1; q >= 0; --q) {
            sv = fma(c[q] * pre[q] * suf, row[q], sv);
            suf *= d[q];
        }
        const double v = dirichlet(w, nx) * sv;
        const int my = mirror_index(jy, P2), mx = mirror_index(jx, P3);
        const bool ycopy = my != jy && my >= 0 && mx >= 0;
        K[(long)jz * plane + rem] = v;
        if (ycopy) K[(long)jz * plane + (long)my * P3 + mx] = v;
        if (zmirror) {
            const int mz = mirror_index(jz, P1);
            if (mz != jz && mz >= 0) {
                K[(long)mz * plane + rem] = v;
                if (ycopy) K[(long)mz * plane + (long)my * P3 + mx] = v;
            }
        }
    }
}

// Zero the planes of mode -P/2 (index 0 in mode order) along every axis of even
// length.  Their values are never reached by the cropped convolution
// (|i - j| <= n - 1 < P/2), and without them the zero-centred kernel is
// exactly point-symmetric, so its spectrum is real.
__global__ void fill_ones_kernel(float2 *__restrict__ c, long n) {
    for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x)
        c[i] = make_float2(1.f, 0.f);
}

__global__ void widen_kernel(const float *__restrict__ a, double *__restrict__ b, long n) {
    for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x)
        b[i] = (double)a[i];
}

__global__ void zero_unpaired_kernel(double *__restrict__ K, int P1, int P2, int P3, int z0, int nz) {
    const long plane = (long)P2 * P3, end = (long)(z0 + nz) * plane;
    for (long idx = (long)z0 * plane + (long)blockIdx.x * blockDim.x + threadIdx.x; idx < end;
         idx += (long)gridDim.x * blockDim.x) {
        int jz = (int)(idx / plane);
        long r = idx - (long)jz * plane;
        int jy = (int)(r / P3), jx = (int)(r - (long)jy * P3);
        if ((P1 % 2 == 0 && jz == 0) || (P2 % 2 == 0 && jy == 0) || (P3 % 2 == 0 && jx == 0))
            K[idx] = 0.0;
    }
}

// taps[d][c] = L * Re b[(z0 + d)][c], d < n: the planes of the kernel after
// its x and y transforms at z offsets 0..n-1 (plane z0 of b holds offset 0)
__global__ void zdirect_taps_kernel(const double2 *__restrict__ b, float *__restrict__ taps, long plane, int n,
                                    int L, int z0) {
    const long total = (long)n * plane;
    for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (long)gridDim.x * blockDim.x) {
        const long d = i / plane, c = i - d * plane;
        taps[i] = (float)((double)L * b[(z0 + d) * plane + c].x);
    }
}

__global__ void d2f_kernel(const double *__restrict__ in, float *__restrict__ out, long n) {
    for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x)
        out[i] = (float)in[i];
}

// y += mu * (-laplacian(x)) with the zero-padded central-difference gradient and
// divergence of the reference GPU build (src/gpu/finitediff.cu:28-222):
// per axis  lap_a(x)[i] = 0.5*(g[i+1] - g[i-1]),  g[k] = 0.5*(x[k+1] - x[k-1]),
// g = 0 outside the volume and x = 0 outside the volume.
// One thread per voxel on a (32 x 8) x n1 grid of CTAs: (k, j) from the CTA
// and thread indices, i = blockIdx.z, so no index division; 32-bit offsets
// (the launcher checks n1 n2 n3 < 2^31).
__global__ void __launch_bounds__(256) neg_lap_axpy_kernel(const float *__restrict__ x,
                                                           float *__restrict__ y, int n1, int n2,
                                                           int n3, float mu) {
    const int k = blockIdx.x * 32 + threadIdx.x;
    const int j = blockIdx.y * 8 + threadIdx.y;
    const int i = blockIdx.z;
    if (k >= n3 || j >= n2) return;
    const int idx = (i * n2 + j) * n3 + k;
    const float c = x[idx];
    float lap = 0.f;
    {  // axis k (n3), stride 1
        const float p2 = (k + 2 < n3) ? x[idx + 2] : 0.f;
        const float m2 = (k >= 2) ? x[idx - 2] : 0.f;
        const float gp = (k + 1 < n3) ? 0.5f * (p2 - c) : 0.f;
        const float gm = (k >= 1) ? 0.5f * (c - m2) : 0.f;
        lap += 0.5f * (gp - gm);
    }
    {  // axis j (n2)
        const int s = n3;
        const float p2 = (j + 2 < n2) ? x[idx + 2 * s] : 0.f;
        const float m2 = (j >= 2) ? x[idx - 2 * s] : 0.f;
        const float gp = (j + 1 < n2) ? 0.5f * (p2 - c) : 0.f;
        const float gm = (j >= 1) ? 0.5f * (c - m2) : 0.f;
        lap += 0.5f * (gp - gm);
    }
    {  // axis i (n1)
        const int s = n2 * n3;
        const float p2 = (i + 2 < n1) ? x[idx + 2 * s] : 0.f;
        const float m2 = (i >= 2) ? x[idx - 2 * s] : 0.f;
        const float gp = (i + 1 < n1) ? 0.5f * (p2 - c) : 0.f;
        const float gm = (i >= 1) ? 0.5f * (c - m2) : 0.f;
        lap += 0.5f * (gp - gm);
    }
    y[idx] = fmaf(-mu, lap, y[idx]);
}

inline unsigned grid_for(long n, int threads, int sms) {
    long b = (n + threads - 1) / threads;
    return (unsigned)std::max<long>(1, std::min<long>(b, (long)sms * 32));
}

}  // namespace

void launch_neg_laplacian_axpy(Context &ctx, const float *x, float *y, const long dims[3], float mu) {
    long n = dims[0] * dims[1] * dims[2];
    ProfScope ps(ctx, PS_NEG_LAP, 12.0 * n);
    LC_REQUIRE(n < (1L << 31) && dims[0] < 65536 && dims[1] < 65536 * 8,
               "negative Laplacian: volume too large for 32-bit indexing");
    const dim3 block(32, 8, 1);
    const dim3 grid((unsigned)((dims[2] + 31) / 32), (unsigned)((dims[1] + 7) / 8), (unsigned)dims[0]);
    neg_lap_axpy_kernel<<<grid, block, 0, ctx.stream()>>>(x, y, (int)dims[0], (int)dims[1],
                                                          (int)dims[2], mu);
    LC_CHECK_LAUNCH();
}

static int next_fast_dim(long n) { return (int)next_smooth23(n); }

// false when the environment sets LC_PSF_TABLE=0 (the direct sum everywhere)
static bool psf_table_enabled() {
    static const bool on = [] {
        const char *e = std::getenv("LC_PSF_TABLE");
        return !(e && e[0] == '0');
    }();
    return on;
}

Toeplitz::Toeplitz(Context &ctx, const PolarGeometry &g, const long dims[3], bool three_d, bool psf_fp32)
    : three_d_(three_d), g_(&g) {
    for (int d = 0; d < 3; ++d) n_[d] = dims[d];
    LC_REQUIRE(n_[0] > 0 && n_[1] > 0 && n_[2] > 0, "Toeplitz: dims must be positive");
    if (three_d) {
        LC_REQUIRE(g.pts.dim == 3, "Toeplitz3D needs a 3D geometry");
        for (int d = 0; d < 3; ++d) P_[d] = next_fast_dim(2 * n_[d] - 1);
        for (int d = 0; d < 3; ++d) Ph_[d] = P_[d] / 2 + 1;
        scale_ = 1.0 / ((double)P_[0] * P_[1] * P_[2] * (double)n_[1] * (double)n_[2]);
    } else {
        LC_REQUIRE(g.pts.dim == 2, "Toeplitz2D needs a 2D geometry");
        P_[0] = 1;
        P_[1] = P_[2] = next_fast_dim(2 * n_[2] - 1);
        Ph_[0] = 1;
        Ph_[1] = Ph_[2] = P_[2] / 2 + 1;
        scale_ = 1.0 / ((double)P_[1] * P_[2] * (double)n_[2]);
    }
    cudaStream_t st = ctx.stream();
    psf_fp32_ = psf_fp32;
    // The direct z stage (3D, kernel even in z, n1 small) needs only the
    // kernel planes |dz| < n1 after the x and y transforms: those are summed
    // and transformed, and the full spectrum is built when it is asked for.
    // Otherwise the spectrum is built here.
    const bool try_direct = three_d && !psf_fp32 && zdirect_enabled() && n_[0] <= zdirect_max_rows();
    if (try_direct) {
        DevBuf<double> K;
        build_kernel(ctx, K, (int)n_[0]);
        if (kernel_mirror_) {
            ProfScope ps(ctx, PS_PSF_FFT, 0.0);
            const int P1 = P_[0], P2 = P_[1], P3 = P_[2], P3h = Ph_[2];
            // planes P1/2 .. P1/2 + n1 - 1 hold dz = 0 .. n1 - 1 (the kernel is
            // even in dz, so these are all the taps)
            const int nz = (int)n_[0];
            DevBuf<double2> a((long)nz * P2 * P3h, st), b((long)nz * P2 * P3h, st);
            kernel_xy_fft(ctx, K.get() + (long)(P1 / 2) * P2 * P3, nz, a.get(), b.get());
            K.release();
            a.release();
            const long plane = (long)P2 * P3h;
            Kz_ = std::make_shared<DevBuf<float>>(n_[0] * plane, st);
            zdirect_taps_kernel<<<grid_for(n_[0] * plane, 256, ctx.num_sms()), 256, 0, st>>>(
                b.get(), Kz_->get(), plane, (int)n_[0], P1, 0);
            LC_CHECK_LAUNCH();
            zfold_ = true;
        } else {
            // not even in z: the whole kernel and the FFT z stage
            build_spectrum(ctx, &K);
        }
    } else {
        build_spectrum(ctx, nullptr);
    }
    // the spectrum is complete in the order of st; callers that hand it to
    // other streams synchronise first (buffers here are freed in stream order)
    // work buffers
    if (three_d) {
        t1_.alloc(n_[0] * n_[1] * Ph_[2], st);
        t2_.alloc(n_[0] * (long)P_[1] * Ph_[2], st);
    } else {
        t1_.alloc(n_[0] * n_[1] * Ph_[2], st);
    }
}

// x (real to half spectrum) and y transforms, FP64, of nz kernel planes of
// {P2, P3} in mode order: K -> a -> b ({nz, P2, P3/2+1} complex)
void Toeplitz::kernel_xy_fft(Context &ctx, const double *K, int nz, double2 *a, double2 *b) {
    const int P2 = P_[1], P3 = P_[2], P3h = Ph_[2];
    {
        AxisFFT x;
        x.in = K;
        x.in_t = E_F64;
        x.out = a;
        x.out_t = E_C128;
        x.fp64 = true;
        x.n_outer = (long)nz * P2;
        x.n_inner = 1;
        x.in_ostride = P3;
        x.out_ostride = P3h;
        x.n_in = P3;
        x.in_map = IN_MODES;
        x.L = P3;
        x.n_out = P3h;
        x.sign = -1;
        launch_axis_fft(ctx, x);
    }
    {
        AxisFFT y;
        y.in = a;
        y.in_t = E_C128;
        y.fp64 = true;
        y.n_outer = nz;
        y.n_inner = P3h;
        y.in_ostride = (long)P2 * P3h;
        y.out_ostride = (long)P2 * P3h;
        y.n_in = P2;
        y.in_map = IN_MODES;
        y.L = P2;
        y.n_out = P2;
        y.sign = -1;
        y.out = b;
        y.out_t = E_C128;
        launch_axis_fft(ctx, y);
    }
}

// The real spectrum R_ of the whole kernel (built here unless *Kin holds it)
void Toeplitz::build_spectrum(Context &ctx, DevBuf<double> *Kin) {
    cudaStream_t st = ctx.stream();
    DevBuf<double> Kown;
    DevBuf<double> &K = Kin ? *Kin : Kown;
    if (!Kin) {
        if (psf_fp32_) build_kernel_nufft32(ctx, K);
        else build_kernel(ctx, K, 0);  // unpaired -P/2 planes already zeroed
    }
    // Spectrum of the zero-centred kernel: FFT with the mode placement k -> k mod P.
    // It is real and point-symmetric; keep x in [0, P3/2] (the R2C half) and all
    // of y and z, i.e. a real {P1, P2, P3/2+1} array.
    ProfScope ps(ctx, PS_PSF_FFT, 0.0);
    DevBuf<double2> a, b;
    DevBuf<double> Rd(spectrum_elems(), st);
    const int P1 = P_[0], P2 = P_[1], P3h = Ph_[2];
    a.alloc((long)P1 * P2 * P3h, st);
    if (three_d_) {
        b.alloc((long)P1 * P2 * P3h, st);
        kernel_xy_fft(ctx, K.get(), P1, a.get(), b.get());
        K.release();
        a.release();
        AxisFFT z;
        z.in = b.get();
        z.in_t = E_C128;
        z.out = Rd.get();
        z.out_t = E_F64;
        z.fp64 = true;
        z.n_outer = 1;
        z.n_inner = (long)P2 * P3h;
        z.in_ostride = 0;
        z.out_ostride = 0;
        z.n_in = P1;
        z.in_map = IN_MODES;
        z.L = P1;
        z.n_out = P1;
        z.sign = -1;
        launch_axis_fft(ctx, z);
    } else {
        const int P3 = P_[2];
        AxisFFT x;
        x.in = K.get();
        x.in_t = E_F64;
        x.out = a.get();
        x.out_t = E_C128;
        x.fp64 = true;
        x.n_outer = (long)P1 * P2;
        x.n_inner = 1;
        x.in_ostride = P3;
        x.out_ostride = P3h;
        x.n_in = P3;
        x.in_map = IN_MODES;
        x.L = P3;
        x.n_out = P3h;
        x.sign = -1;
        launch_axis_fft(ctx, x);
        K.release();
        AxisFFT y;
        y.in = a.get();
        y.in_t = E_C128;
        y.fp64 = true;
        y.n_outer = P1;
        y.n_inner = P3h;
        y.in_ostride = (long)P2 * P3h;
        y.out_ostride = (long)P2 * P3h;
        y.n_in = P2;
        y.in_map = IN_MODES;
        y.L = P2;
        y.n_out = P2;
        y.sign = -1;
        y.out = Rd.get();
        y.out_t = E_F64;
        launch_axis_fft(ctx, y);
    }
    // an FFT along z of a kernel even in kz is even in f1: keep the planes
    // f1 <= P1/2 (a prefix of the plane-major array)
    zfold_ = three_d_ && kernel_mirror_;
    long nR = stored_spectrum_elems();
    R_ = std::make_shared<DevBuf<float>>(nR, st);
    d2f_kernel<<<grid_for(nR, 256, ctx.num_sms()), 256, 0, st>>>(Rd.get(), R_->get(), nR);
    LC_CHECK_LAUNCH();
}

void Toeplitz::ensure_spectrum(Context &ctx) {
    if (R_) return;
    LC_REQUIRE(g_ != nullptr, "PSF spectrum export needs the PSF's own geometry");
    build_spectrum(ctx, nullptr);
}

static void psf_sizes(const long dims[3], bool three_d, long P[3], long Ph[3]) {
    if (three_d) {
        for (int d = 0; d < 3; ++d) P[d] = next_smooth23(2 * dims[d] - 1);
    } else {
        P[0] = 1;
        P[1] = P[2] = next_smooth23(2 * dims[2] - 1);
    }
    for (int d = 0; d < 3; ++d) Ph[d] = (three_d || d > 0) ? P[d] / 2 + 1 : 1;
}

size_t Toeplitz::work_bytes(const long dims[3], bool three_d) {
    long P[3], Ph[3];
    psf_sizes(dims, three_d, P, Ph);
    const size_t t1 = (size_t)dims[0] * dims[1] * Ph[2];
    const size_t t2 = three_d ? (size_t)dims[0] * P[1] * Ph[2] : 0;
    return (t1 + t2) * sizeof(float2);
}

size_t Toeplitz::build_peak_bytes(const long dims[3], bool three_d) {
    long P[3], Ph[3];
    psf_sizes(dims, three_d, P, Ph);
    // FP64 kernel, two complex FP64 FFT buffers, FP64 and FP32 real spectra,
    // and the direct z-stage taps (3D, at most n1 planes)
    const size_t full = (size_t)P[0] * P[1] * P[2];
    const size_t half = (size_t)P[0] * P[1] * Ph[2];
    const size_t taps = three_d ? (size_t)dims[0] * P[1] * Ph[2] : 0;
    return full * sizeof(double) + 2 * half * sizeof(double2) + half * (sizeof(double) + sizeof(float)) +
           taps * sizeof(float);
}

Toeplitz::Toeplitz(Context &ctx, const Toeplitz &src, bool work)
    : three_d_(src.three_d_), kernel_mirror_(src.kernel_mirror_), zfold_(src.zfold_), g_(nullptr), R_(src.R_),
      Kz_(src.Kz_), scale_(src.scale_) {
    for (int d = 0; d < 3; ++d) {
        n_[d] = src.n_[d];
        P_[d] = src.P_[d];
        Ph_[d] = src.Ph_[d];
    }
    if (!work) return;
    cudaStream_t st = ctx.stream();
    t1_.alloc(n_[0] * n_[1] * Ph_[2], st);
    if (three_d_) t2_.alloc(n_[0] * (long)P_[1] * Ph_[2], st);
}

// The kernel as the reference GPU path builds it (include/gpu/toeplitz2d.h:84-115,
// include/gpu/toeplitz.h:80-110): Re of a type-1 NUFFT of unit weights at every
// grid point onto the P grid, here in FP32 at tol 1e-6 (cuFINUFFT's float
// path runs at 1.2e-6), widened to FP64 for the spectrum FFTs that follow.
void Toeplitz::build_kernel_nufft32(Context &ctx, DevBuf<double> &K) {
    cudaStream_t st = ctx.stream();
    ProfScope ps(ctx, PS_PSF_GEN, 0.0);
    const int P1 = P_[0], P2 = P_[1], P3 = P_[2];
    const long total = (long)P1 * P2 * P3;
    const int modes[3] = {P3, P2, three_d_ ? P1 : 1};
    NufftPlan plan(ctx, *g_, modes, 1e-6);
    DevBuf<float2> ones(g_->pts.M, st);
    fill_ones_kernel<<<grid_for(g_->pts.M, 256, ctx.num_sms()), 256, 0, st>>>(ones.get(), g_->pts.M);
    LC_CHECK_LAUNCH();
    DevBuf<float> K32(total, st);
    plan.type1_real(ctx, ones.get(), 1, K32.get(), 1.0f, PT_PLAIN);
    K.alloc(total, st);
    widen_kernel<<<grid_for(total, 256, ctx.num_sms()), 256, 0, st>>>(K32.get(), K.get(), total);
    LC_CHECK_LAUNCH();
    kernel_mirror_ = false;
    zero_unpaired_kernel<<<grid_for(total, 256, ctx.num_sms()), 256, 0, st>>>(K.get(), P1, P2, P3, 0, P1);
    LC_CHECK_LAUNCH();
}

void Toeplitz::build_kernel(Context &ctx, DevBuf<double> &K, int zkeep) {
    cudaStream_t st = ctx.stream();
    ProfScope ps(ctx, PS_PSF_GEN, 0.0);
    const int nth = g_->pts.ntheta;
    const double pi = 3.14159265358979323846;
    std::vector<PsfAngle> tab(nth);
    int nx, ny;
    for (int i = 0; i < nth; ++i) {
        PsfAngle &A = tab[i];
        if (three_d_) {
            // columns of transpose(Rx(theta) Ry(beta) Rz(gamma)) (include/rotation.h:28-56):
            // uX = (R00, R10, R20) . k, uY = (R01, R11, R21) . k
            double ct = std::cos(g_->theta[i]), st_ = std::sin(g_->theta[i]);
            double cb = std::cos(g_->beta[i]), sb = std::sin(g_->beta[i]);
            double cg = std::cos(g_->gamma[i]), sg = std::sin(g_->gamma[i]);
            A.a[0] = cb * cg;
            A.a[1] = -cb * sg;
            A.a[2] = sb;
            A.b[0] = ct * sg + st_ * sb * cg;
            A.b[1] = ct * cg - st_ * sb * sg;
            A.b[2] = -st_ * cb;
        } else {
            A.a[0] = std::cos(g_->theta[i]);
            A.a[1] = std::sin(g_->theta[i]);
            A.a[2] = 0.0;
            A.b[0] = A.b[1] = A.b[2] = 0.0;
        }
    }
    if (three_d_) {
        nx = g_->pts.ncols;
        ny = g_->pts.nrows;
    } else {
        nx = g_->pts.nr;
        ny = 1;
    }
    // (4 sin^2(t/2), sin t) for t = pi h', h' = h - round(h) (|h| <= 1)
    auto step = [&](double h) {
        const double hr = h > 0.5 ? h - 1.0 : (h < -0.5 ? h + 1.0 : h);
        const double q = std::sin(0.5 * pi * hr);
        return make_double2(4.0 * q * q, std::sin(pi * hr));
    };
    for (auto &A : tab) {
        A.stepA = step(A.a[0]);
        A.stepB = step(A.a[0] / nx);
        A.stepC = step(A.b[0]);
        A.stepD = step(A.b[0] / ny);
    }
    // Is the angle set closed under the reflection that makes K even in one
    // more axis?  3D: (a, b) -> (a, b) with the kz coefficients negated;
    // 2D: a -> a with the kx coefficient negated.  The multisets of keys
    // (rounded to 1e-10) are compared; a key on a rounding boundary only costs
    // the saving, never the result.
    bool mirror = nth > 0;
    bool quarter_turn = false;
    {
        // Dirichlet kernels are even, so a and -a (b and -b) give the same term:
        // each vector is compared with the sign of its first nonzero component
        // made positive
        using Key = std::array<long long, 6>;
        auto key = [](const PsfAngle &A, bool refl, bool three) {
            auto q = [](double v) { return (long long)std::llround(v * 1e10); };
            auto canon = [&](double x, double y, double z, long long *out) {
                long long v[3] = {q(x), q(y), q(z)};
                const long long lead = v[0] != 0 ? v[0] : (v[1] != 0 ? v[1] : v[2]);
                for (int i = 0; i < 3; ++i) out[i] = lead < 0 ? -v[i] : v[i];
            };
            Key k{};
            if (three) {
                canon(A.a[0], A.a[1], refl ? -A.a[2] : A.a[2], &k[0]);
                canon(A.b[0], A.b[1], refl ? -A.b[2] : A.b[2], &k[3]);
            } else {
                canon(refl ? -A.a[0] : A.a[0], A.a[1], 0.0, &k[0]);
            }
            return k;
        };
        std::vector<Key> k0(nth), k1(nth);
        for (int i = 0; i < nth; ++i) {
            k0[i] = key(tab[i], false, three_d_);
            k1[i] = key(tab[i], true, three_d_);
        }
        std::sort(k0.begin(), k0.end());
        std::sort(k1.begin(), k1.end());
        mirror = mirror && k0 == k1;
        if (mirror && !three_d_ && P_[1] == P_[2]) {
            // 2D: also closed under theta -> theta + pi/2, a -> (-a1, a0)?
            std::vector<Key> k2(nth);
            for (int i = 0; i < nth; ++i) {
                PsfAngle r = tab[i];
                r.a[0] = -tab[i].a[1];
                r.a[1] = tab[i].a[0];
                k2[i] = key(r, false, false);
            }
            std::sort(k2.begin(), k2.end());
            quarter_turn = k0 == k2;
        }
    }
    kernel_mirror_ = mirror;
    // group the angles by their theta-independent vector a (equal beta and gamma)
    std::vector<int> order(nth);
    for (int i = 0; i < nth; ++i) order[i] = i;
    std::stable_sort(order.begin(), order.end(), [&](int p, int q) {
        const PsfAngle &x = tab[p], &y = tab[q];
        return std::tie(x.a[0], x.a[1], x.a[2]) < std::tie(y.a[0], y.a[1], y.a[2]);
    });
    std::vector<PsfAngle> sorted(nth);
    std::vector<int> groups{0};
    for (int r = 0; r < nth; ++r) {
        sorted[r] = tab[order[r]];
        if (r > 0) {
            const PsfAngle &x = sorted[r - 1], &y = sorted[r];
            if (x.a[0] != y.a[0] || x.a[1] != y.a[1] || x.a[2] != y.a[2]) groups.push_back(r);
        }
    }
    groups.push_back(nth);
    const int ngroups = three_d_ ? (int)groups.size() - 1 : 0;
    if (!three_d_) groups.assign(1, 0);
    DevBuf<PsfAngle> dtab;
    dtab.upload(three_d_ ? sorted.data() : tab.data(), tab.size(), st);
    DevBuf<int> dgroups;
    dgroups.upload(groups.data(), groups.size(), st);
    const int P1 = P_[0], P2 = P_[1], P3 = P_[2];
    long total = (long)P1 * P2 * P3;
    K.alloc(total, st);
    constexpr int S = 16;
    const long nseg = ((!three_d_ && mirror ? P3 / 2 + 1 : P3) + S - 1) / S;
    // with zkeep > 0 and the kz mirror, only the planes 0 <= kz < zkeep are
    // set (the direct sum sums -zkeep < kz <= 0 and mirrors them); the other
    // planes are left unset
    const bool zpart = three_d_ && mirror && zkeep > 0;
    const int zlo = zpart ? std::max(0, P1 / 2 - (zkeep - 1)) : 0;
    const int zbeg = zpart ? P1 / 2 : 0, zcnt = zpart ? std::min(zkeep, P1 - P1 / 2) : P1;
    const long items =
        (three_d_ ? (long)(P1 / 2 + 1 - zlo) * (mirror ? P2 / 2 + 1 : P2) : (long)(P2 / 2 + 1)) * nseg;
    size_t smem = sizeof(PsfAngle) * nth + sizeof(int) * groups.size();
    LC_REQUIRE(smem <= 220 * 1024, "Toeplitz: too many angles for one PSF launch");
    unsigned blocks = (unsigned)std::max<long>(1, std::min<long>((items + 127) / 128, (long)ctx.num_sms() * 16));
    // laminography (one tilt, beta = 0, the kz mirror): the tabulated form
    bool tabulated = three_d_ && ngroups == 1 && mirror && psf_table_enabled();
    for (int i = 0; tabulated && i < nth; ++i) tabulated = sorted[i].a[2] == 0.0;
    if (tabulated) {
        const double cg = sorted[0].a[0], sg = -sorted[0].a[1];
        const double h = 1.0 / 32.0;
        // u over the grid's corners, with the stencil's margin
        double umin = 1e300, umax = -1e300;
        for (int cx = 0; cx < 2; ++cx)
            for (int cy = 0; cy < 2; ++cy) {
                const double kx = cx ? (double)(P3 - 1 - P3 / 2) : (double)(-P3 / 2);
                const double ky = cy ? (double)(P2 - 1 - P2 / 2) : (double)(-P2 / 2);
                const double u = sg * kx + cg * ky;
                umin = std::min(umin, u);
                umax = std::max(umax, u);
            }
        const double u0 = umin - 6.0 * h;
        const int nu = (int)std::ceil((umax - u0) / h) + 8;
        // the planes 0 <= kz < zkeep, or kz <= 0 and their mirrors
        const int zs = zkeep > 0 ? P1 / 2 : 0;
        const int nzc = zkeep > 0 ? std::min(zkeep, P1 - P1 / 2) : P1 / 2 + 1;
        const int nr = zkeep > 0 ? nzc : P1 / 2 + 1;
        std::vector<TabAngle> ta(nth);
        for (int i = 0; i < nth; ++i) {
            // b = (ct sg, ct cg, -st): ct from the ky coefficient over cg, or the kx one over sg
            const PsfAngle &A = sorted[i];
            const double ct = std::fabs(cg) >= std::fabs(sg) ? A.b[1] / cg : A.b[0] / sg;
            ta[i].ct = ct;
            ta[i].st = -A.b[2];
            ta[i].stepN = step(ct * h);
            ta[i].stepD = step(ct * h / ny);
        }
        DevBuf<TabAngle> dta;
        dta.upload(ta.data(), ta.size(), st);
        DevBuf<double> table((long)nr * nu, st);
        const size_t tsm = sizeof(TabAngle) * nth;
        LC_REQUIRE(tsm <= 220 * 1024, "Toeplitz: too many angles for one PSF launch");
        allow_max_dynamic_smem(ctx, psf_table_kernel);
        const long titems = (long)nr * ((nu + kTabSeg - 1) / kTabSeg);
        const unsigned tb = (unsigned)std::max<long>(1, std::min<long>((titems + 127) / 128, (long)ctx.num_sms() * 16));
        psf_table_kernel<<<tb, 128, tsm, st>>>(dta.get(), nth, ny, u0, h, nu, nr, table.get());
        LC_CHECK_LAUNCH();
        const long npts = (long)nzc * (P2 / 2 + 1) * P3;
        psf_interp_kernel<<<grid_for(npts, 256, ctx.num_sms()), 256, 0, st>>>(
            table.get(), u0, 1.0 / h, nu, nr, sg, cg, nx, P1, P2, P3, zs, nzc, zkeep > 0 ? 0 : 1, K.get());
        LC_CHECK_LAUNCH();
    } else if (three_d_) {
        auto kern = ngroups == 1 ? psf_rows_kernel<S, true> : psf_rows_kernel<S, false>;
        allow_max_dynamic_smem(ctx, kern);
        kern<<<blocks, 128, smem, st>>>(dtab.get(), nth, dgroups.get(), ngroups, nx, ny, P1, P2, P3,
                                        mirror ? 1 : 0, zlo, K.get());
    } else {
        // lanes per segment: the fewest that give about 1024 threads per SM,
        // at least one angle quad per lane
        const int m2 = mirror ? (quarter_turn ? 2 : 1) : 0;
        const long nseg2 = ((mirror ? P3 / 2 + 1 : P3) + S - 1) / S;
        const long segs = psf2d_first_seg(P2 / 2 + 1, nseg2, m2);
        int G = 1;
        while (G < 32 && segs * G < (long)ctx.num_sms() * 1024 && 2 * G <= nth / 4) G *= 2;
        const size_t smem2 = sizeof(PsfAngle) * nth;
        LC_REQUIRE(smem2 <= 220 * 1024, "Toeplitz: too many angles for one PSF launch");
        const unsigned blocks2 =
            (unsigned)std::max<long>(1, std::min<long>((segs * G + 127) / 128, (long)ctx.num_sms() * 16));
        auto launch = [&](auto kern) {
            allow_max_dynamic_smem(ctx, kern);
            kern<<<blocks2, 128, smem2, st>>>(dtab.get(), nth, nx, P2, P3, m2, K.get());
        };
        switch (G) {
        case 1: launch(psf2d_kernel<S, 1>); break;
        case 2: launch(psf2d_kernel<S, 2>); break;
        case 4: launch(psf2d_kernel<S, 4>); break;
        case 8: launch(psf2d_kernel<S, 8>); break;
        case 16: launch(psf2d_kernel<S, 16>); break;
        default: launch(psf2d_kernel<S, 32>); break;
        }
    }
    LC_CHECK_LAUNCH();
    // planes of mode -P/2 have no mirror inside the grid; they are not needed
    zero_unpaired_kernel<<<grid_for((long)zcnt * P2 * P3, 256, ctx.num_sms()), 256, 0, st>>>(K.get(), P1, P2, P3,
                                                                                         zbeg, zcnt);
    LC_CHECK_LAUNCH();
    // the angle table is freed in the order of st; the host tables were
    // staged by their uploads
}

void Toeplitz::kernel_fp64(Context &ctx, double *host_out) {
    LC_REQUIRE(g_ != nullptr, "PSF kernel export needs the PSF's own geometry");
    DevBuf<double> K;
    build_kernel(ctx, K, 0);
    long total = three_d_ ? (long)P_[0] * P_[1] * P_[2] : (long)P_[2] * P_[2];
    LC_CUDA(cudaMemcpyAsync(host_out, K.get(), total * sizeof(double), cudaMemcpyDeviceToHost,
                            ctx.stream()));
    LC_CUDA(cudaStreamSynchronize(ctx.stream()));
}

double Toeplitz::algorithmic_bytes() const {
    // read x, write y, read the real spectrum octant (or the z taps) once
    return 8.0 * (double)nvox() + 4.0 * (double)(Kz_ ? (long)Kz_->size() : stored_spectrum_elems());
}

unsigned Toeplitz::cg_caps() const {
    const int P3 = P_[2];
    return (P3 % 2 == 0 && line_kernels_enabled() && line_plan_exists(P3 / 2)) ? (kFusedUpdate | kFusedDot)
                                                                                   : 0u;
}

long Toeplitz::cg_partials() const { return row_fft_ctas(n_[0] * n_[1]); }

void Toeplitz::apply(Context &ctx, const float *x, float *y, const CGFusion *f, unsigned parts, long pitch) {
    LC_REQUIRE((parts & ~cg_caps()) == 0, "Toeplitz: CG fusion not available for this size");
    const long n1 = n_[0], n2 = n_[1], n3 = n_[2];
    if (pitch <= 0) pitch = n3;
    LC_REQUIRE(pitch >= n3, "Toeplitz: row pitch below the row length");
    const int P1 = P_[0], P2 = P_[1], P3 = P_[2];
    const int P3h = Ph_[2];
    const double N = (double)n1 * n2 * n3;
    const double T1 = (double)n1 * n2 * P3h * 8.0;      // half-spectrum rows, complex
    const double T2 = (double)n1 * P2 * P3h * 8.0;      // after the y transform
    const double Rb = 4.0 * (double)stored_spectrum_elems();
    // x rows: real -> half spectrum
    {
        ProfScope ps(ctx, PS_TOEP_X_FWD, 4.0 * N + T1);
        AxisFFT a;
        a.in = x;
        a.in_t = E_F32;
        a.out = t1_.get();
        a.out_t = E_C64;
        a.n_outer = n1 * n2;
        a.n_inner = 1;
        a.in_ostride = pitch;
        a.out_ostride = P3h;
        a.n_in = (int)n3;
        a.L = P3;
        a.n_out = P3h;
        a.sign = -1;
        if (P3 % 2 == 0) {
            // real rows as half-length complex transforms (even/odd packing)
            a.L = P3 / 2;
            a.in_map = IN_REAL_PACKED;
            a.out_map = OUT_R2C_UNPACK;
        }
        a.cg = f;
        a.cg_parts = parts & kFusedUpdate;
        launch_axis_fft(ctx, a);
    }
    if (!three_d_) {
        ProfScope ps(ctx, PS_TOEP_Y_MID, 2.0 * T1 + Rb);
        AxisFFT a;
        a.in = t1_.get();
        a.in_t = E_C64;
        a.out = t1_.get();
        a.out_t = E_C64;
        a.n_outer = n1;
        a.n_inner = P3h;
        a.in_ostride = n2 * P3h;
        a.out_ostride = n2 * P3h;
        a.n_in = (int)n2;
        a.L = P2;
        a.n_out = (int)n2;
        a.out_map = OUT_WINDOW;
        a.out_off = 0;
        a.sign = -1;
        a.mid = R_->get();
        a.mid_ra = P3h;
        a.sign2 = +1;
        launch_axis_fft(ctx, a);
    } else {
        {
            ProfScope ps(ctx, PS_TOEP_Y_FWD, T1 + T2);
            AxisFFT a;
            a.in = t1_.get();
            a.in_t = E_C64;
            a.out = t2_.get();
            a.out_t = E_C64;
            a.n_outer = n1;
            a.n_inner = P3h;
            a.in_ostride = n2 * P3h;
            a.out_ostride = (long)P2 * P3h;
            a.n_in = (int)n2;
            a.L = P2;
            a.n_out = P2;
            a.sign = -1;
            launch_axis_fft(ctx, a);
        }
        if (Kz_) {
            ProfScope ps(ctx, PS_TOEP_Z_MID, 2.0 * T2 + 4.0 * (double)Kz_->size());
            launch_zdirect(ctx.stream(), t2_.get(), (long)P2 * P3h, (int)n1, Kz_->get());
        } else if (ProfScope ps(ctx, PS_TOEP_Z_MID, 2.0 * T2 + Rb);
            !(line_kernels_enabled() &&
              launch_zconv(ctx.stream(), t2_.get(), (long)P2 * P3h, P1, (int)n1, (int)n1, R_->get(),
                           zfold_))) {
            AxisFFT a;
            a.in = t2_.get();
            a.in_t = E_C64;
            a.out = t2_.get();
            a.out_t = E_C64;
            a.n_outer = 1;
            a.n_inner = (long)P2 * P3h;
            a.in_ostride = 0;
            a.out_ostride = 0;
            a.n_in = (int)n1;
            a.L = P1;
            a.n_out = (int)n1;
            a.out_map = OUT_WINDOW;
            a.out_off = 0;
            a.sign = -1;
            a.mid = R_->get();
            a.mid_ra = (long)P2 * P3h;
            a.mid_fold = zfold_;
            a.sign2 = +1;
            launch_axis_fft(ctx, a);
        }
        {
            ProfScope ps(ctx, PS_TOEP_Y_INV, T1 + T2);
            AxisFFT a;
            a.in = t2_.get();
            a.in_t = E_C64;
            a.out = t1_.get();
            a.out_t = E_C64;
            a.n_outer = n1;
            a.n_inner = P3h;
            a.in_ostride = (long)P2 * P3h;
            a.out_ostride = n2 * P3h;
            a.n_in = P2;
            a.L = P2;
            a.n_out = (int)n2;
            a.out_map = OUT_WINDOW;
            a.out_off = 0;
            a.sign = +1;
            launch_axis_fft(ctx, a);
        }
    }
    {
        ProfScope ps(ctx, PS_TOEP_X_INV, T1 + 4.0 * N);
        AxisFFT a;
        a.in = t1_.get();
        a.in_t = E_C64;
        a.out = y;
        a.out_t = E_F32;
        a.n_outer = n1 * n2;
        a.n_inner = 1;
        a.in_ostride = P3h;
        a.out_ostride = pitch;
        a.n_in = P3h;
        a.in_map = IN_HERM;
        a.L = P3;
        a.n_out = (int)n3;
        a.out_map = OUT_WINDOW;
        a.out_off = 0;
        a.sign = +1;
        a.scale = scale_;
        if (P3 % 2 == 0) {
            a.L = P3 / 2;
            a.in_map = IN_C2R_PACK;
            a.out_map = OUT_REAL_UNPACK;
        }
        a.cg = f;
        a.cg_parts = parts & kFusedDot;
        launch_axis_fft(ctx, a);
    }
}

void Toeplitz::apply_reg(Context &ctx, const float *x, float *y, float mu) {
    apply(ctx, x, y);
    if (mu != 0.0f) launch_neg_laplacian_axpy(ctx, x, y, n_, mu);
}

}  // namespace lc
