// Bin-sorted ES-kernel spreading (type 1) and tile-staged interpolation
// (type 2) on polar grids, plus the pruned fine-grid FFT passes.
#include <algorithm>
#include <cmath>
#include <memory>
#include <numeric>

#include "lc_nufft.hpp"

namespace lc {

// ---------------------------------------------------------------------------
// geometry
// ---------------------------------------------------------------------------
void geometry_init_2d(Context &ctx, PolarGeometry &g, const double *theta, int ntheta, int nr) {
    LC_REQUIRE(ntheta > 0 && nr > 0, "geometry: ntheta and nradial must be positive");
    LC_REQUIRE((long)ntheta * nr < (1L << 31), "geometry: too many points");
    g.theta.assign(theta, theta + ntheta);
    std::vector<double2> cs(ntheta);
    for (int i = 0; i < ntheta; ++i) cs[i] = make_double2(std::cos(theta[i]), std::sin(theta[i]));
    g.cs.upload(cs.data(), ntheta, ctx.stream());
    LC_CUDA(cudaStreamSynchronize(ctx.stream()));
    g.pts = PolarPts{};
    g.pts.dim = 2;
    g.pts.ntheta = ntheta;
    g.pts.nr = nr;
    g.pts.M = (long)ntheta * nr;
    g.pts.cs = g.cs.get();
    g.pts.div_angle = make_fastdiv((unsigned)nr);
}

void geometry_init_3d(Context &ctx, PolarGeometry &g, const double *theta, const double *gamma,
                      const double *beta, const float *shifts, int ntheta, int nrows, int ncols) {
    LC_REQUIRE(ntheta > 0 && nrows > 0 && ncols > 0, "geometry: sizes must be positive");
    LC_REQUIRE((long)ntheta * nrows * ncols < (1L << 31), "geometry: too many points");
    g.theta.assign(theta, theta + ntheta);
    g.gamma.assign(gamma, gamma + ntheta);
    g.beta.assign(beta, beta + ntheta);
    std::vector<double> rot(6 * (size_t)ntheta);
    for (int i = 0; i < ntheta; ++i) {
        // transpose(Rx(theta) Ry(beta) Rz(gamma)), columns 0 and 1 (q has no z part)
        double ct = std::cos(theta[i]), st = std::sin(theta[i]);
        double cb = std::cos(beta[i]), sb = std::sin(beta[i]);
        double cg = std::cos(gamma[i]), sg = std::sin(gamma[i]);
        double *r = &rot[6 * (size_t)i];
        r[0] = cb * cg;                 // R00
        r[1] = ct * sg + st * sb * cg;  // R01
        r[2] = -cb * sg;                // R10
        r[3] = ct * cg - st * sb * sg;  // R11
        r[4] = sb;                      // R20
        r[5] = -st * cb;                // R21
    }
    g.rot.upload(rot.data(), rot.size(), ctx.stream());
    g.shifts.assign(2 * (size_t)ntheta, 0.0f);
    if (shifts) std::copy(shifts, shifts + 2 * (size_t)ntheta, g.shifts.begin());
    g.dshifts.upload(reinterpret_cast<const float2 *>(g.shifts.data()), ntheta, ctx.stream());
    LC_CUDA(cudaStreamSynchronize(ctx.stream()));
    g.pts = PolarPts{};
    g.pts.dim = 3;
    g.pts.ntheta = ntheta;
    g.pts.nrows = nrows;
    g.pts.ncols = ncols;
    g.pts.M = (long)ntheta * nrows * ncols;
    g.pts.rot = g.rot.get();
    g.pts.div_angle = make_fastdiv((unsigned)nrows * (unsigned)ncols);
    g.pts.div_col = make_fastdiv((unsigned)ncols);
}

// ---------------------------------------------------------------------------
// ES kernel parameters and deapodisation
// ---------------------------------------------------------------------------
int es_width_for_tol(double tol) {
    LC_REQUIRE(tol > 0 && tol < 1, "NUFFT tolerance must be in (0, 1)");
    int w = (int)std::ceil(std::log10(1.0 / tol)) + 1;
    return std::min(12, std::max(4, w));
}

double es_beta_for_width(int w) { return 2.30 * w; }

// Gauss-Legendre nodes on [-1, 1] by Newton iteration on P_n.
static void gauss_legendre(int n, std::vector<double> &x, std::vector<double> &wt) {
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

std::vector<double> es_correction(int n, int nf, int w, double beta) {
    std::vector<double> x, wt;
    gauss_legendre(4 * w + 60, x, wt);
    std::vector<double> phi(x.size());
    for (size_t q = 0; q < x.size(); ++q) phi[q] = std::exp(beta * (std::sqrt(1.0 - x[q] * x[q]) - 1.0));
    std::vector<double> out(n);
    const double pi = 3.14159265358979323846;
    for (int j = 0; j < n; ++j) {
        double k = (double)(j - n / 2);
        double xi = k * w * pi / nf;
        double s = 0;
        for (size_t q = 0; q < x.size(); ++q) s += wt[q] * phi[q] * std::cos(xi * x[q]);
        out[j] = 2.0 / (w * s);
    }
    return out;
}

// ---------------------------------------------------------------------------
// device helpers
// ---------------------------------------------------------------------------
namespace {

constexpr double kInv2Pi = 0.15915494309189533577;
constexpr double kPi = 3.14159265358979323846;

struct GridCfg {
    int nf[3];
    int bs[3];
    int nb[3];
    int hw[3];
    int td[3];   // tile extent per dim
    double inv_nf[3];
    FastDiv div_tx, div_ty;  // by the tile extents along x and y
    float beta_l2e;          // ES beta times log2(e)
};

__device__ __forceinline__ unsigned fast_div(unsigned n, FastDiv f) { return (__umulhi(n, f.m) + n) >> f.s; }

struct PointInfo {
    double c[3];  // x, y, z
    double qX, qY;
    int angle;
};

__device__ __forceinline__ void point_at(const PolarPts &p, long j, PointInfo &pi) {
    const unsigned jj = (unsigned)j;  // M < 2^31
    if (p.dim == 2) {
        const int i = (int)fast_div(jj, p.div_angle);
        const int m = (int)(jj - (unsigned)i * (unsigned)p.nr);
        double r = ((double)m + 0.5) * (2.0 * kPi / p.nr) - kPi;
        double2 cs = p.cs[i];
        pi.c[0] = cs.x * r;
        pi.c[1] = cs.y * r;
        pi.c[2] = 0.0;
        pi.angle = i;
        pi.qX = r;
        pi.qY = 0.0;
    } else {
        const unsigned i = fast_div(jj, p.div_angle);
        const unsigned rem = jj - i * ((unsigned)p.nrows * (unsigned)p.ncols);
        const unsigned ua = fast_div(rem, p.div_col);
        const int a = (int)ua, b = (int)(rem - ua * (unsigned)p.ncols);
        double qX = ((double)b + 0.5) * (2.0 * kPi / p.ncols) - kPi;
        double qY = ((double)a + 0.5) * (2.0 * kPi / p.nrows) - kPi;
        const double *R = p.rot + 6 * (long)i;
        pi.c[0] = R[0] * qX + R[1] * qY;
        pi.c[1] = R[2] * qX + R[3] * qY;
        pi.c[2] = R[4] * qX + R[5] * qY;
        pi.qX = qX;
        pi.qY = qY;
        pi.angle = (int)i;
    }
}

__device__ __forceinline__ bool in_band(const PointInfo &pi) {
    return fabs(pi.c[0]) <= kPi && fabs(pi.c[1]) <= kPi && fabs(pi.c[2]) <= kPi;
}

// wrapped fine-grid coordinate u in [0, nf), its cell, first covered cell l0
// and the float offset u - l0 (inv_nf = 1 / nf; a quotient one off is
// corrected, so the result equals the wrap by exact division)
__device__ __forceinline__ void place(double x, int nf, double inv_nf, int W, int &cell, int &l0,
                                      float &off) {
    double u = x * (double)nf * kInv2Pi;
    u -= (double)nf * floor(u * inv_nf);
    if (u < 0.0) u += (double)nf;
    if (u >= (double)nf) u -= (double)nf;
    if (u < 0.0) u = 0.0;
    cell = (int)floor(u);
    if (cell >= nf) cell = nf - 1;
    double lo = ceil(u - 0.5 * (double)W);
    l0 = (int)lo;
    off = (float)(u - lo);
}

// v wrapped into [0, n) for v in [-n, 3n)
__device__ __forceinline__ int wrap_near(int v, int n) {
    if (v >= n) v -= n;
    if (v >= n) v -= n;
    if (v < 0) v += n;
    return v;
}

// fine-grid offset of tile cell rr (x fastest) of the tile starting at S
template <int DIM>
__device__ __forceinline__ long tile_cell_to_grid(int rr, const GridCfg &g, const int (&S)[3]) {
    const unsigned q = fast_div((unsigned)rr, g.div_tx);  // row of the tile: iy + ty iz
    const int ix = rr - (int)q * g.td[0];
    const unsigned iz = DIM == 3 ? fast_div(q, g.div_ty) : 0u;
    const int iy = (int)q - (int)iz * g.td[1];
    long gi = (long)wrap_near(S[0] + ix, g.nf[0]) + (long)wrap_near(S[1] + iy, g.nf[1]) * g.nf[0];
    if (DIM == 3) gi += (long)wrap_near(S[2] + (int)iz, g.nf[2]) * ((long)g.nf[0] * g.nf[1]);
    return gi;
}

template <int DIM>
__device__ __forceinline__ int bin_of(const PointInfo &pi, const GridCfg &g, int W) {
    int b = 0, mul = 1;
#pragma unroll
    for (int d = 0; d < DIM; ++d) {
        int cell, l0;
        float off;
        place(pi.c[d], g.nf[d], g.inv_nf[d], W, cell, l0, off);
        b += (cell / g.bs[d]) * mul;
        mul *= g.nb[d];
    }
    return b;
}

template <int DIM>
__global__ void bin_count_kernel(PolarPts pts, GridCfg g, int W, int *counts) {
    for (long j = (long)blockIdx.x * blockDim.x + threadIdx.x; j < pts.M;
         j += (long)gridDim.x * blockDim.x) {
        PointInfo pi;
        point_at(pts, j, pi);
        int b = bin_of<DIM>(pi, g, W);
        unsigned act = __activemask();
        unsigned peers = __match_any_sync(act, b);
        int lane = threadIdx.x & 31;
        int leader = __ffs(peers) - 1;
        if (lane == leader) atomicAdd(&counts[b], __popc(peers));
    }
}

// the bin of a point and its footprint corner in the bin's tile (x fastest):
// l0 - S per axis, S = bin start - hw, as the spreading kernel places it
template <int DIM>
__device__ __forceinline__ int bin_corner_of(const PointInfo &pi, const GridCfg &g, int W, int &corner) {
    int b = 0, mul = 1, stride = 1;
    corner = 0;
#pragma unroll
    for (int d = 0; d < DIM; ++d) {
        int cell, l0;
        float off;
        place(pi.c[d], g.nf[d], g.inv_nf[d], W, cell, l0, off);
        const int bd = cell / g.bs[d];
        b += bd * mul;
        mul *= g.nb[d];
        corner += (l0 - (bd * g.bs[d] - g.hw[d])) * stride;
        stride *= g.td[d];
    }
    return b;
}

// perm[k] = the point at sorted position k; corners[k] its footprint corner
// in its bin's tile (read by the footprint bound and the spreading's
// bucketing)
template <int DIM>
__global__ void bin_scatter_kernel(PolarPts pts, GridCfg g, int W, int *cursor, int *perm,
                                   unsigned short *corners) {
    for (long j = (long)blockIdx.x * blockDim.x + threadIdx.x; j < pts.M;
         j += (long)gridDim.x * blockDim.x) {
        PointInfo pi;
        point_at(pts, j, pi);
        int corner;
        int b = bin_corner_of<DIM>(pi, g, W, corner);
        unsigned act = __activemask();
        unsigned peers = __match_any_sync(act, b);
        int lane = threadIdx.x & 31;
        int leader = __ffs(peers) - 1;
        int rank = __popc(peers & ((1u << lane) - 1u));
        int base = 0;
        if (lane == leader) base = atomicAdd(&cursor[b], __popc(peers));
        base = __shfl_sync(peers, base, leader);
        perm[base + rank] = (int)j;
        corners[base + rank] = (unsigned short)corner;
    }
}

// ---- spreading ----------------------------------------------------------
// One thread spreads one point over its W^DIM footprint with shared-memory
// atomics into a planar tile.  All lanes of a warp issue each atomic
// instruction at the same footprint step, so two lanes conflict exactly when
// their footprint corners fall in the same shared-memory bank (corner index
// mod 32).  The points of a subproblem are bucketed by corner bank and spread
// in passes in which the unrotated points hold distinct banks:
//   * full rounds (every bank still holds a point): lane b takes the next
//     point of bank b;
//   * tail rounds (some banks have run out; round r holds the banks with more
//     than r points, so the sets shrink with r), 3D: the lowest round left
//     takes the highest round left along on its free lanes when some rotation
//     fits.  A rotated point visits its footprint planes in an order shifted
//     by rho modulo W, so at every step it sits at bank b + d1 or b + d2 of
//     the unrotated frame, d1 = rho P and d2 = (rho - W) P mod 32 with P the
//     plane stride; the rotation fits when both banks of every point of the
//     high round are clear of the low round's banks.  The pairing depends on
//     the bank counts alone, so every warp walks it and spreads the passes
//     that fall to it.  (2D tiles run the tail rounds one by one.)
// The accumulation is exact and order-free (below): the schedule decides the
// speed, never the result.
//
// The tile accumulates in exact fixed point with 32-bit integer atomics,
// which run about four times faster than float atomics in shared memory, one
// 32-bit word per real and imaginary part of a cell.  Each bin has its own
// scale F_b = 2^e_b from two bounds over all of its points: m_b, the largest
// |Re c| + |Im c| of their values (weights are at most 1, and a unit phase
// keeps each part below |c|), measured per launch, and W_b, a bound on the
// summed kernel weights of the bin's footprints over one tile cell, measured
// with the plan (the corner histogram of the bin's points, box-summed along
// each axis with the largest weight each footprint offset can take).
// Both depend on the bin's point set alone, not on how the bin is cut into
// subproblems (the cut follows the bin sort's atomic order), so every
// contribution is rounded the same way in every plan of the geometry.  A
// contribution v (a float) is rounded to the integer nearest v F_b by adding
// 1.5 * 2^23, which places it in the low mantissa bits (|v F_b| < 2^22), and
// the float's bits are added as they are: every contribution then carries
// the bias 0x4B400000, and the flush subtracts K_cell times it (modulo 2^32)
// with K_cell the footprints over the cell.  With F_b m_b <= 2^21 and
// K_b m_b F_b < 2^30 a tile cell's sum stays below 2^31, so the word holds it
// exactly.  The flush adds each sum, shifted to one scale F_G = 2^e_G for
// the whole launch (e_b <= e_G, so the shift is exact), to a 64-bit integer
// per part of the fine grid, and a conversion pass forms the float grid.
// Every sum is an exact integer, so the fine grid depends neither on the
// order of the atomics nor on the schedule: a backprojection is bit-for-bit
// repeatable.  The rounding step 1 / F_b is at most max(W_b 2^-29, 2^-20) m_b:
// a cell summed from K footprints is within about sqrt(K / 12) of that of its
// exact value.
constexpr int kSpreadThreads = 256;
constexpr float kRoundMagic = 12582912.0f;  // 1.5 * 2^23
constexpr unsigned kRoundMagicBits = 0x4B400000u;

// Exponents of the fixed-point scales.  Launch: F_G = 2^e_G with
// kmax m F_G < 2^61 (kmax bounds the footprints over one fine-grid cell, m
// the values), so a cell's 64-bit sum stays below 2^62.  Bin: F_b = 2^e_b
// with F_b m_b <= 2^21 (rounding by 1.5 2^23) and W_b m_b F_b < 2^30, W_b a
// bound on the sum of the weights of the bin's footprints over one cell, so
// a tile cell's sum (plus at most 1024 rounding halves) stays below 2^31;
// and e_b <= e_G.
__host__ __device__ __forceinline__ int fix_exponent_grid(float m, long kmax) {
    if (!(m > 0.f)) return 0;
    int e3;
    frexp((double)kmax * (double)m, &e3);  // kmax m < 2^e3
    return 61 - e3;
}

__device__ __forceinline__ int fix_exponent_tile(float mb, float wb, int eg) {
    int e1, e2;
    frexp((double)mb, &e1);               // m_b < 2^e1
    frexp((double)wb * (double)mb, &e2);  // W_b m_b < 2^e2
    const int a = 21 - e1, b = 30 - e2;
    const int e = a < b ? a : b;
    return e < eg ? e : eg;
}

// m = max |Re c| + |Im c| over n values, as the bits of a non-negative float
// (integer order equals float order); *bits must start at 0
__global__ void value_bound_kernel(const float2 *__restrict__ c, long n, int *bits) {
    float m = 0.f;
    for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
        const float2 v = c[i];
        m = fmaxf(m, fabsf(v.x) + fabsf(v.y));
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
    if ((threadIdx.x & 31) == 0 && m > 0.f) atomicMax(bits, __float_as_int(m));
}

// fine grid <- T / F_G from the two 64-bit fixed-point sums per cell
__global__ void fix_to_float_kernel(const long long *__restrict__ fix, float2 *__restrict__ grid, long n,
                                    const int *__restrict__ mbits, long kmax) {
    const double unscale = ldexp(1.0, -fix_exponent_grid(__int_as_float(*mbits), kmax));
    const longlong2 *f2 = reinterpret_cast<const longlong2 *>(fix);
    for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
        const longlong2 t = f2[i];
        grid[i] = make_float2((float)((double)t.x * unscale), (float)((double)t.y * unscale));
    }
}

// shared-memory atomic add without return at a 32-bit shared address plus a
// compile-time byte offset, so one address register serves a footprint row
template <int OFF>
__device__ __forceinline__ void red_shared(unsigned addr, int v) {
    asm volatile("red.shared.add.u32 [%0+%2], %1;" ::"r"(addr), "r"(v), "n"(OFF) : "memory");
}

// word += round(a b) + B (B = 0x4B400000, the bits of 1.5 2^23), |a b| < 2^22,
// at cell DX of the row starting at the shared address `row`
template <int DX>
__device__ __forceinline__ void fixed_add(unsigned row, float a, float b) {
    red_shared<4 * DX>(row, __float_as_int(fmaf(a, b, kRoundMagic)));
}

// one footprint row of W cells, real and imaginary parts
template <int W, int DX = 0>
__device__ __forceinline__ void spread_row(unsigned re, unsigned im, float vr, float vi, const float (&wx)[W]) {
    if constexpr (DX < W) {
        fixed_add<DX>(re, vr, wx[DX]);
        fixed_add<DX>(im, vi, wx[DX]);
        spread_row<W, DX + 1>(re, im, vr, vi, wx);
    }
}

// cnt[q] <- sum of cnt[q - d], d in [0, w), along one axis of a tile of
// tx x ty x tz cells (in place: a thread walks each of its lines downwards
// with a sliding window, so the values it still reads are the original ones)
__device__ __forceinline__ void box_sum_axis(int *cnt, int axis, int w, int tx, int ty, int tz) {
    const int plane = tx * ty;
    const int n = axis == 0 ? tx : (axis == 1 ? ty : tz);
    const int stride = axis == 0 ? 1 : (axis == 1 ? tx : plane);
    const int nlines = axis == 0 ? ty * tz : (axis == 1 ? tx * tz : plane);
    for (int line = threadIdx.x; line < nlines; line += blockDim.x) {
        const int base = axis == 0 ? line * tx : (axis == 1 ? (line % tx) + (line / tx) * plane : line);
        int win = 0;
        for (int q = max(0, n - w); q < n; ++q) win += cnt[base + q * stride];
        for (int q = n - 1; q >= 0; --q) {
            const int cq = cnt[base + q * stride];
            cnt[base + q * stride] = win;
            win += (q - w >= 0 ? cnt[base + (q - w) * stride] : 0) - cq;
        }
    }
}

// position of the k-th (from 0) set bit of m, k < popc(m)
__device__ __forceinline__ int kth_bit(unsigned m, int k) {
    int pos = 0;
#pragma unroll
    for (int w = 16; w > 0; w >>= 1) {
        const int c = __popc(m & ((1u << w) - 1u));
        if (k >= c) {
            k -= c;
            m >>= w;
            pos += w;
        }
    }
    return pos;
}

// Bank offsets (mod 32) that a point of a 3D tile whose footprint planes are
// visited rotated by rot (1 <= rot < W) occupies relative to the unrotated lanes
template <int W>
__device__ __forceinline__ void rot_banks(int rot, int plane, int &d1, int &d2) {
    d1 = (plane * rot) & 31;
    d2 = (plane * (rot - W)) & 31;
}

// Spreads point j; in 3D its footprint planes are visited in the order rotated
// by rot (0: in order).
template <int DIM, int W>
__device__ __forceinline__ void spread_point(const PolarPts &pts, const GridCfg &g,
                                             const float2 *__restrict__ c, long cstride, int nvol, int j,
                                             int mode, const float2 *__restrict__ shifts, const int (&S)[3],
                                             int tx, int plane, int tsize, unsigned sm_re,
                                             unsigned plane_bytes, float fscale, int rot) {
    const float inv_hw = 2.0f / (float)W;
    PointInfo pi;
    point_at(pts, j, pi);
    float2 mult = make_float2(fscale, 0.f);
    if (mode == PT_SHIFT) {
        const float2 sh = shifts[pi.angle];
        const double ph = pi.qX * (double)sh.x + pi.qY * (double)sh.y;
        double sn, cs;
        sincos(ph, &sn, &cs);
        mult = make_float2((float)cs * fscale, (float)-sn * fscale);
    }
    // wk[d][m]: weight of the cell at offset m along axis d (3D z: (m + rot) mod W)
    float wk[DIM][W];
    int corner = 0;
    {
        const int stride[3] = {1, tx, plane};
#pragma unroll
        for (int d = 0; d < DIM; ++d) {
            int cell, l0;
            float off;
            place(pi.c[d], g.nf[d], g.inv_nf[d], W, cell, l0, off);
            corner += (l0 - S[d]) * stride[d];
            const int r = d == 2 ? rot : 0;
#pragma unroll
            for (int m = 0; m < W; ++m) {
                int mm = m + r;
                if (mm >= W) mm -= W;
                wk[d][m] = es_eval2f(((float)mm - off) * inv_hw, g.beta_l2e);
            }
        }
    }
    for (int s = 0; s < nvol; ++s) {
        float2 v = c[(long)s * cstride + j];
        v = mode == PT_SHIFT ? cmul(v, mult) : make_float2(v.x * fscale, v.y * fscale);
        // 32-bit shared addresses of the footprint corner in the two planes
        const unsigned ar = sm_re + 4u * (unsigned)(s * tsize + corner);
        const unsigned ai = ar + plane_bytes;
        if constexpr (DIM == 2) {
#pragma unroll
            for (int dy = 0; dy < W; ++dy) {
                const float vr = v.x * wk[1][dy], vi = v.y * wk[1][dy];
                const unsigned row = 4u * (unsigned)(dy * tx);
                spread_row<W>(ar + row, ai + row, vr, vi, wk[0]);
            }
        } else {
#pragma unroll 1
            for (int dz = 0; dz < W; ++dz) {
                float wz = wk[2][0];
#pragma unroll
                for (int m = 1; m < W; ++m)
                    if (dz == m) wz = wk[2][m];
                int zz = dz + rot;
                if (zz >= W) zz -= W;
                const float zr = v.x * wz, zi = v.y * wz;
                const unsigned zo = 4u * (unsigned)(zz * plane);
#pragma unroll
                for (int dy = 0; dy < W; ++dy) {
                    const float vr = zr * wk[1][dy], vi = zi * wk[1][dy];
                    const unsigned row = zo + 4u * (unsigned)(dy * tx);
                    spread_row<W>(ar + row, ai + row, vr, vi, wk[0]);
                }
            }
        }
    }
}

// Largest kernel weight of each footprint offset m < W (over every position
// of the point), rounded up, for the weighted footprint bound
struct OffsetWeights {
    float w[16];
};

// Plan: W_b of every bin (one CTA per bin, float bits): the corner histogram
// of all the bin's points on its tile, summed along each axis with the
// offset weights (cell q gets sum_d om[d] h[q - d]), and its maximum.  Every
// line is summed by one thread in a fixed order, so the bound depends on the
// bin's point set alone.
template <int DIM, int W>
__global__ void __launch_bounds__(256) bin_footprint_kernel(GridCfg g, OffsetWeights om,
                                                            const unsigned short *__restrict__ corners,
                                                            const int2 *__restrict__ bins, int *kbin) {
    extern __shared__ int hist[];
    __shared__ int kmx;
    const int2 br = bins[blockIdx.x];  // (first position in perm, points)
    if (br.y == 0) {
        if (threadIdx.x == 0) kbin[blockIdx.x] = 0;
        return;
    }
    const int tx = g.td[0], ty = g.td[1], tz = DIM == 3 ? g.td[2] : 1;
    const int plane = tx * ty, tsize = plane * tz;
    for (int i = threadIdx.x; i < tsize; i += blockDim.x) hist[i] = 0;
    if (threadIdx.x == 0) kmx = 0;
    __syncthreads();
    for (int p = threadIdx.x; p < br.y; p += blockDim.x) atomicAdd(&hist[corners[br.x + p]], 1);
    __syncthreads();
    // weighted sums along x, y, z in place, one thread per line with the
    // last W inputs in registers
    float *acc = reinterpret_cast<float *>(hist);
    for (int i = threadIdx.x; i < tsize; i += blockDim.x) acc[i] = (float)hist[i];
    __syncthreads();
#pragma unroll 1
    for (int d = 0; d < DIM; ++d) {
        const int n = d == 0 ? tx : (d == 1 ? ty : tz);
        const int stride = d == 0 ? 1 : (d == 1 ? tx : plane);
        const int nlines = tsize / n;
        for (int line = threadIdx.x; line < nlines; line += blockDim.x) {
            const int base = d == 0 ? line * tx : (d == 1 ? (line % tx) + (line / tx) * plane : line);
            float r[W];
#pragma unroll
            for (int k = 0; k < W; ++k) r[k] = 0.f;
            for (int q = 0; q < n; ++q) {
#pragma unroll
                for (int k = W - 1; k > 0; --k) r[k] = r[k - 1];
                r[0] = acc[base + q * stride];
                float v = 0.f;
#pragma unroll
                for (int k = 0; k < W; ++k) v = fmaf(om.w[k], r[k], v);
                acc[base + q * stride] = v;
            }
        }
        __syncthreads();
    }
    float km = 0.f;
    for (int i = threadIdx.x; i < tsize; i += blockDim.x) km = fmaxf(km, acc[i]);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) km = fmaxf(km, __shfl_xor_sync(0xffffffffu, km, o));
    if ((threadIdx.x & 31) == 0) atomicMax(&kmx, __float_as_int(km));
    __syncthreads();
    // float rounding of the sums (relative 2^-24 per step): a margin of 1e-4
    if (threadIdx.x == 0) kbin[blockIdx.x] = __float_as_int(__int_as_float(kmx) * 1.0001f);
}

// Per launch: m_b of every bin (float bits, binm zeroed first) over all
// values of the bin's points (one CTA per subproblem)
__global__ void __launch_bounds__(256) bin_value_bound_kernel(const float2 *__restrict__ c, long cstride,
                                                              int nvol, const int *__restrict__ perm,
                                                              const int4 *__restrict__ subs, int *binm) {
    const int4 sp = subs[blockIdx.x];
    float m = 0.f;
    for (int p = threadIdx.x; p < sp.z; p += blockDim.x) {
        const int j = perm[sp.y + p];
        for (int s = 0; s < nvol; ++s) {
            const float2 v = c[(long)s * cstride + j];
            m = fmaxf(m, fabsf(v.x) + fabsf(v.y));
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
    if ((threadIdx.x & 31) == 0 && m > 0.f) atomicMax(&binm[sp.x], __float_as_int(m));
}

#ifndef LC_SPREAD_MIN_BLOCKS
#define LC_SPREAD_MIN_BLOCKS 3  // CTAs per SM the spreading kernel's registers are sized for
#endif

template <int DIM, int W>
__global__ void __launch_bounds__(kSpreadThreads, LC_SPREAD_MIN_BLOCKS)
    spread_kernel(PolarPts pts, GridCfg g, const float2 *__restrict__ c, long cstride, int nvol,
                  const int *__restrict__ perm, const unsigned short *__restrict__ corners,
                  const int4 *__restrict__ subs,
                  unsigned long long *__restrict__ fix, long gstride, int mode,
                  const float2 *__restrict__ shifts, const int *__restrict__ mbits, long kmax,
                  const int *__restrict__ kbin, const int *__restrict__ binm) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ int cnt[32], start[32], mincnt, maxcnt;
    const int4 sp = subs[blockIdx.x];
    int bcoord[3] = {0, 0, 0};
    {
        int rr = sp.x;
#pragma unroll
        for (int d = 0; d < DIM; ++d) {
            bcoord[d] = rr % g.nb[d];
            rr /= g.nb[d];
        }
    }
    int S[3] = {0, 0, 0};
#pragma unroll
    for (int d = 0; d < DIM; ++d) S[d] = bcoord[d] * g.bs[d] - g.hw[d];
    const int tx = g.td[0], ty = g.td[1], tz = DIM == 3 ? g.td[2] : 1;
    const int plane = tx * ty;
    const int tsize = plane * tz;
    const long acc_n = (long)nvol * tsize;
    int *are = reinterpret_cast<int *>(smem_raw);  // real parts
    int *aim = are + acc_n;                        // imaginary parts
    int *kcnt = aim + acc_n;  // footprint corners per cell, then footprints per cell
    unsigned short *order = reinterpret_cast<unsigned short *>(kcnt + tsize);  // points by bank
    constexpr int kKeys = 8;  // points per thread in the bucketing pass (maxpts <= 8 * threads)
    int key[kKeys];
    const int tid = threadIdx.x;
    for (long idx = tid; idx < 2 * acc_n + tsize; idx += blockDim.x) are[idx] = 0;
    if (tid < 32) cnt[tid] = 0;
    __syncthreads();

    // ---- bucket the points by the bank of their footprint corner ----
#pragma unroll
    for (int q = 0; q < kKeys; ++q) {
        const int p = tid + q * (int)blockDim.x;
        key[q] = -1;
        if (p >= sp.z) continue;
        bool use = true;
        if (mode != PT_PLAIN) {
            PointInfo pi;
            point_at(pts, perm[sp.y + p], pi);
            use = in_band(pi);
        }
        int k = -1;
        if (use) {
            const int corner = corners[sp.y + p];  // from the bin sort
            const int b = corner & 31;
            k = (b << 16) | atomicAdd(&cnt[b], 1);
            atomicAdd(&kcnt[corner], 1);
        }
        key[q] = k;
    }
    __syncthreads();
    if (tid < 32) {
        const int v = cnt[tid];
        int incl = v, mn = v, mx = v;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int t = __shfl_up_sync(0xffffffffu, incl, o);
            if (tid >= o) incl += t;
            mn = min(mn, __shfl_xor_sync(0xffffffffu, mn, o));
            mx = max(mx, __shfl_xor_sync(0xffffffffu, mx, o));
        }
        start[tid] = incl - v;
        if (tid == 0) {
            mincnt = mn;
            maxcnt = mx;
        }
    }
    __syncthreads();
#pragma unroll
    for (int q = 0; q < kKeys; ++q) {
        const int k = key[q];
        if (k >= 0) order[start[k >> 16] + (k & 0xffff)] = (unsigned short)(tid + q * (int)blockDim.x);
    }
    // footprints per cell: box sums of the corner histogram along each axis
    __syncthreads();
#pragma unroll
    for (int d = 0; d < DIM; ++d) {
        box_sum_axis(kcnt, d, W, tx, ty, tz);
        __syncthreads();
    }
    const float mb = __int_as_float(binm[sp.x]);
    if (!(mb > 0.f)) return;  // every value of the bin is zero: nothing to add (uniform over the CTA)
    // the bin's fixed-point scale F_b = 2^e_b, and the launch's e_G
    const int eg = fix_exponent_grid(__int_as_float(*mbits), kmax);
    const int eb = fix_exponent_tile(mb, __int_as_float(kbin[sp.x]), eg);
    const float fscale = ldexpf(1.f, eb);

    const int lane = tid & 31, warp = tid >> 5, nwarps = blockDim.x >> 5;
    const unsigned sm_re = (unsigned)__cvta_generic_to_shared(are);
    const unsigned plane_bytes = 4u * (unsigned)acc_n;  // bytes between the real and imaginary planes
    const int mycnt = cnt[lane], mystart = start[lane], nrounds = maxcnt, nfull = mincnt;
    // ---- rounds 0 .. nrounds-1 in passes; round r holds the banks with more
    // than r points, so the sets shrink with r.  Rounds below nfull hold every
    // bank.  In 3D the lowest tail round left (banks A_lo) takes the highest
    // round left (A_hi) along when some plane rotation keeps both banks of
    // every A_hi point clear of A_lo; the points of A_hi then fill the free
    // lanes in bank order.  Every warp walks the same pairing of the tail and
    // spreads the passes that fall to it (one call site keeps the unrolled
    // footprint code in the instruction cache once).
    int od1 = 0, od2 = 0;  // lane o tests the plane rotation o + 1
    if (DIM == 3 && lane < W - 1) rot_banks<W>(lane + 1, plane, od1, od2);
    int wi = nfull, wj = nrounds - 1, wpass = nfull;  // tail walk: next pass and its rounds
    for (int pass = warp;; pass += nwarps) {
        int i = pass, j = 0, rot = 0;
        unsigned alo = 0xffffffffu, ahi = 0;
        if (pass >= nfull) {
            bool found = false;
            while (wi <= wj) {
                const unsigned lo = __ballot_sync(0xffffffffu, mycnt > wi);
                unsigned hi = 0;
                int r = 0;
                if (DIM == 3 && wi < wj) {
                    hi = __ballot_sync(0xffffffffu, mycnt > wj);
                    const bool ok = lane < W - 1 && __popc(lo) + __popc(hi) <= 32 &&
                                    !(__funnelshift_l(hi, hi, od1) & lo) && !(__funnelshift_l(hi, hi, od2) & lo);
                    const unsigned m = __ballot_sync(0xffffffffu, ok);
                    if (m) r = __ffs(m);
                    else hi = 0;
                }
                if (wpass++ == pass) {
                    i = wi;
                    j = wj;
                    alo = lo;
                    ahi = hi;
                    rot = r;
                    found = true;
                }
                ++wi;
                if (hi) --wj;
                if (found) break;
            }
            if (!found) break;
        }
        int p = -1, prot = 0;
        if ((alo >> lane) & 1u) {
            p = order[mystart + i];
        } else if (ahi) {
            const int k = __popc(~alo & ((1u << lane) - 1u));  // rank among the free lanes
            if (k < __popc(ahi)) {
                p = order[start[kth_bit(ahi, k)] + j];
                prot = rot;
            }
        }
        if (p >= 0)
            spread_point<DIM, W>(pts, g, c, cstride, nvol, perm[sp.y + p], mode, shifts, S, tx, plane, tsize,
                                 sm_re, plane_bytes, fscale, prot);
    }
    __syncthreads();
    // flush the tile's exact sums at the launch's scale (halos overlap
    // neighbouring bins, so add atomically; integer sums make the order
    // irrelevant)
    const int sh = eg - eb;
    for (int s = 0; s < nvol; ++s) {
        for (int rr = tid; rr < tsize; rr += blockDim.x) {
            const int k = kcnt[rr];
            if (k == 0) continue;
            const unsigned kb = (unsigned)k * kRoundMagicBits;
            const int idx = s * tsize + rr;
            const int t1 = (int)((unsigned)are[idx] - kb), t2 = (int)((unsigned)aim[idx] - kb);
            if ((t1 | t2) == 0) continue;
            unsigned long long *cell = fix + 2 * ((long)s * gstride + tile_cell_to_grid<DIM>(rr, g, S));
            // two's-complement sums: shift the 64-bit patterns (sh <= 40)
            if (t1) atomicAdd(cell, (unsigned long long)(long long)t1 << sh);
            if (t2) atomicAdd(cell + 1, (unsigned long long)(long long)t2 << sh);
        }
    }
}

// ---- interpolation --------------------------------------------------------
template <int DIM, int W>
__global__ void __launch_bounds__(256) interp_kernel(PolarPts pts, GridCfg g,
                                                     const float2 *__restrict__ grid, long gstride,
                                                     int nvol, const int *__restrict__ perm,
                                                     const int4 *__restrict__ subs,
                                                     float2 *__restrict__ c, long cstride, int mode) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    float2 *tile = reinterpret_cast<float2 *>(smem_raw);
    const int4 sp = subs[blockIdx.x];
    const int bin = sp.x;
    int bcoord[3] = {0, 0, 0};
    {
        int r = bin;
#pragma unroll
        for (int d = 0; d < DIM; ++d) {
            bcoord[d] = r % g.nb[d];
            r /= g.nb[d];
        }
    }
    int S[3] = {0, 0, 0};
#pragma unroll
    for (int d = 0; d < DIM; ++d) S[d] = bcoord[d] * g.bs[d] - g.hw[d];
    const int tx = g.td[0], ty = g.td[1], tz = DIM == 3 ? g.td[2] : 1;
    const int tsize = tx * ty * tz;
    for (int s = 0; s < nvol; ++s)
        for (int r = threadIdx.x; r < tsize; r += blockDim.x)
            tile[s * tsize + r] = __ldg(grid + (long)s * gstride + tile_cell_to_grid<DIM>(r, g, S));
    __syncthreads();
    const float inv_hw = 2.0f / (float)W;
    for (int p = threadIdx.x; p < sp.z; p += blockDim.x) {
        const int j = perm[sp.y + p];
        PointInfo pi;
        point_at(pts, j, pi);
        if (mode != PT_PLAIN && !in_band(pi)) {
            for (int s = 0; s < nvol; ++s) c[(long)s * cstride + j] = make_float2(0.f, 0.f);
            continue;
        }
        float wk[2][W];
        int lo[3] = {0, 0, 0};
        float offz = 0.f;
#pragma unroll
        for (int d = 0; d < DIM; ++d) {
            int cell, l0;
            float off;
            place(pi.c[d], g.nf[d], g.inv_nf[d], W, cell, l0, off);
            lo[d] = l0 - S[d];
            if (d < 2) {
#pragma unroll
                for (int m = 0; m < W; ++m) wk[d][m] = es_eval2f(((float)m - off) * inv_hw, g.beta_l2e);
            } else {
                offz = off;
            }
        }
        for (int s = 0; s < nvol; ++s) {
            const float2 *ts = tile + (long)s * tsize;
            float ar = 0.f, ai = 0.f;
            if constexpr (DIM == 2) {
#pragma unroll
                for (int dy = 0; dy < W; ++dy) {
                    const float2 *row = ts + (lo[1] + dy) * tx + lo[0];
                    float rr = 0.f, ri = 0.f;
#pragma unroll
                    for (int dx = 0; dx < W; ++dx) {
                        float2 v = row[dx];
                        rr = fmaf(v.x, wk[0][dx], rr);
                        ri = fmaf(v.y, wk[0][dx], ri);
                    }
                    ar = fmaf(rr, wk[1][dy], ar);
                    ai = fmaf(ri, wk[1][dy], ai);
                }
            } else {
                for (int dz = 0; dz < W; ++dz) {
                    float zr = 0.f, zi = 0.f;
#pragma unroll
                    for (int dy = 0; dy < W; ++dy) {
                        const float2 *row = ts + ((lo[2] + dz) * ty + (lo[1] + dy)) * tx + lo[0];
                        float rr = 0.f, ri = 0.f;
#pragma unroll
                        for (int dx = 0; dx < W; ++dx) {
                            float2 v = row[dx];
                            rr = fmaf(v.x, wk[0][dx], rr);
                            ri = fmaf(v.y, wk[0][dx], ri);
                        }
                        zr = fmaf(rr, wk[1][dy], zr);
                        zi = fmaf(ri, wk[1][dy], zi);
                    }
                    const float wz = es_eval2f(((float)dz - offz) * inv_hw, g.beta_l2e);
                    ar = fmaf(zr, wz, ar);
                    ai = fmaf(zi, wz, ai);
                }
            }
            c[(long)s * cstride + j] = make_float2(ar, ai);
        }
    }
}

template <int DIM, int W>
void launch_spread_w(const Context &ctx, dim3 grid, size_t smem, cudaStream_t st, const PolarPts &pts,
                     const GridCfg &g, const float2 *c, long cstride, int nvol, const int *perm,
                     const unsigned short *corners, const int4 *subs, unsigned long long *out, long gstride,
                     int mode, const float2 *shifts, const int *mbits, long kmax, const int *kbin,
                     const int *binm) {
    auto kern = spread_kernel<DIM, W>;
    allow_max_dynamic_smem(ctx, kern);
    kern<<<grid, kSpreadThreads, smem, st>>>(pts, g, c, cstride, nvol, perm, corners, subs, out, gstride,
                                             mode, shifts, mbits, kmax, kbin, binm);
    LC_CHECK_LAUNCH();
}

template <int DIM, int W>
void launch_footprint_w(const Context &ctx, unsigned nbins, size_t smem, cudaStream_t st, const GridCfg &g,
                        const OffsetWeights &om, const unsigned short *corners, const int2 *bins, int *kbin) {
    auto kern = bin_footprint_kernel<DIM, W>;
    allow_max_dynamic_smem(ctx, kern);
    kern<<<nbins, 256, smem, st>>>(g, om, corners, bins, kbin);
    LC_CHECK_LAUNCH();
}

template <int DIM, int W>
void launch_interp_w(const Context &ctx, dim3 grid, int threads, size_t smem, cudaStream_t st,
                     const PolarPts &pts, const GridCfg &g, const float2 *gr, long gstride, int nvol,
                     const int *perm, const int4 *subs, float2 *c, long cstride, int mode) {
    auto kern = interp_kernel<DIM, W>;
    allow_max_dynamic_smem(ctx, kern);
    kern<<<grid, threads, smem, st>>>(pts, g, gr, gstride, nvol, perm, subs, c, cstride, mode);
    LC_CHECK_LAUNCH();
}

#define LC_W_SWITCH(W, CALL)                           \
    switch (W) {                                       \
        case 4: { constexpr int WW = 4; CALL; } break; \
        case 5: { constexpr int WW = 5; CALL; } break; \
        case 6: { constexpr int WW = 6; CALL; } break; \
        case 7: { constexpr int WW = 7; CALL; } break; \
        case 8: { constexpr int WW = 8; CALL; } break; \
        case 9: { constexpr int WW = 9; CALL; } break; \
        case 10: { constexpr int WW = 10; CALL; } break; \
        case 11: { constexpr int WW = 11; CALL; } break; \
        case 12: { constexpr int WW = 12; CALL; } break; \
        default: throw Error(1, "unsupported ES kernel width"); \
    }

GridCfg make_cfg(int dim, const int nf[3], const int bs[3], const int nb[3], int w, double beta) {
    GridCfg g{};
    // A point in cell c covers cells [c - floor(w/2), c + ceil(w/2)] (first
    // covered cell ceil(u - w/2) for u in [c, c+1)), so a bin of bs cells
    // needs a tile of bs + w cells starting floor(w/2) cells before it.
    const int lo = w / 2;
    for (int d = 0; d < 3; ++d) {
        g.nf[d] = nf[d];
        g.bs[d] = bs[d];
        g.nb[d] = nb[d];
        g.hw[d] = d < dim ? lo : 0;
        g.td[d] = d < dim ? bs[d] + w : 1;
        g.inv_nf[d] = 1.0 / (double)nf[d];
    }
    g.div_tx = make_fastdiv((unsigned)g.td[0]);
    g.div_ty = make_fastdiv((unsigned)g.td[1]);
    g.beta_l2e = (float)(beta * 1.4426950408889634074);
    return g;
}

}  // namespace

// ---------------------------------------------------------------------------
// plan
// ---------------------------------------------------------------------------
NufftPlan::NufftPlan(Context &ctx, const PolarGeometry &g, const int modes[3], double tol) {
    dim_ = g.pts.dim;
    pts_ = g.pts;
    shifts_ = g.dshifts.get();
    w_ = es_width_for_tol(tol);
    beta_ = es_beta_for_width(w_);
    for (int d = 0; d < 3; ++d) {
        modes_[d] = d < dim_ ? modes[d] : 1;
        LC_REQUIRE(modes_[d] >= 1, "NUFFT: mode counts must be positive");
        nf_[d] = d < dim_ ? (int)next_smooth23(std::max(2 * modes_[d], 2 * w_)) : 1;
    }
    const int bs2[3] = {32, 32, 1};
    const int bs3[3] = {16, 8, 8};
    maxsub_ = dim_ == 2 ? 1024 : 2048;
    for (int d = 0; d < 3; ++d) {
        bs_[d] = std::min(dim_ == 2 ? bs2[d] : bs3[d], nf_[d]);
        nb_[d] = (nf_[d] + bs_[d] - 1) / bs_[d];
    }
    cudaStream_t st = ctx.stream();
    for (int d = 0; d < dim_; ++d) {
        auto c = es_correction(modes_[d], nf_[d], w_, beta_);
        std::vector<float> cf(c.begin(), c.end());
        corr_[d].upload(cf.data(), cf.size(), st);
    }
    if (dim_ == 3) {
        auto cx_ = es_correction(modes_[0], nf_[0], w_, beta_);
        auto cy_ = es_correction(modes_[1], nf_[1], w_, beta_);
        std::vector<float> xy((size_t)modes_[0] * modes_[1]);
        for (int y = 0; y < modes_[1]; ++y)
            for (int x = 0; x < modes_[0]; ++x) xy[(size_t)y * modes_[0] + x] = (float)(cy_[y] * cx_[x]);
        corr_xy_.upload(xy.data(), xy.size(), st);
    }
    LC_CUDA(cudaStreamSynchronize(st));
    sort_points(ctx);
}

void NufftPlan::sort_points(Context &ctx) {
    cudaStream_t st = ctx.stream();
    long nbins = (long)nb_[0] * nb_[1] * nb_[2];
    GridCfg g = make_cfg(dim_, nf_, bs_, nb_, w_, beta_);
    DevBuf<int> counts(nbins, st);
    counts.zero(st);
    int threads = 256;
    long blocks = std::min<long>((pts_.M + threads - 1) / threads, (long)ctx.num_sms() * 16);
    blocks = std::max<long>(blocks, 1);
    if (dim_ == 2) bin_count_kernel<2><<<(unsigned)blocks, threads, 0, st>>>(pts_, g, w_, counts.get());
    else bin_count_kernel<3><<<(unsigned)blocks, threads, 0, st>>>(pts_, g, w_, counts.get());
    LC_CHECK_LAUNCH();
    std::vector<int> hc(nbins);
    LC_CUDA(cudaMemcpyAsync(hc.data(), counts.get(), nbins * sizeof(int), cudaMemcpyDeviceToHost, st));
    LC_CUDA(cudaStreamSynchronize(st));
    std::vector<int> off(nbins);
    long acc = 0;
    const int maxsub = maxsub_;
    std::vector<int4> subs;
    for (long b = 0; b < nbins; ++b) {
        off[b] = (int)acc;
        for (int s = 0; s < hc[b]; s += maxsub)
            subs.push_back(make_int4((int)b, (int)(acc + s), std::min(maxsub, hc[b] - s), 0));
        acc += hc[b];
    }
    LC_REQUIRE(acc == pts_.M, "NUFFT: bin sort lost points");
    // footprints over one cell: a footprint reaches at most w/2 + 1 <= bs
    // cells beyond its point's cell, so only points of the bin and of its
    // neighbours (wrapped, each counted once) can cover a cell of the bin;
    // the neighbourhood sums are separable box sums of the bin counts
    {
        std::vector<long> a(hc.begin(), hc.end()), t(nbins);
        const long stride[3] = {1, nb_[0], (long)nb_[0] * nb_[1]};
        for (int k = 0; k < 3; ++k) {
            const int n = nb_[k];
            const int lo = n >= 3 ? -1 : 0, hi = n >= 2 ? 1 : 0;  // distinct wrapped offsets
            for (long b = 0; b < nbins; ++b) {
                const int c = (int)((b / stride[k]) % n);
                long sum = 0;
                for (int d = lo; d <= hi; ++d) sum += a[b + (long)(((c + d + n) % n) - c) * stride[k]];
                t[b] = sum;
            }
            a.swap(t);
        }
        kmax_ = std::max<long>(1, *std::max_element(a.begin(), a.end()));
    }
    nsub_ = (int)subs.size();
    LC_REQUIRE(nsub_ > 0, "NUFFT: no points");
    subs_.upload(subs.data(), subs.size(), st);
    DevBuf<int> cursor;
    cursor.upload(off.data(), off.size(), st);
    perm_.alloc(pts_.M, st);
    corner_.alloc(pts_.M, st);
    LC_REQUIRE((long)g.td[0] * g.td[1] * g.td[2] <= 65536, "NUFFT: bin tile too large for 16-bit corners");
    if (dim_ == 2)
        bin_scatter_kernel<2><<<(unsigned)blocks, threads, 0, st>>>(pts_, g, w_, cursor.get(), perm_.get(),
                                                                    corner_.get());
    else
        bin_scatter_kernel<3><<<(unsigned)blocks, threads, 0, st>>>(pts_, g, w_, cursor.get(), perm_.get(),
                                                                    corner_.get());
    LC_CHECK_LAUNCH();
    // K_b of every bin, over all of its points
    {
        std::vector<int2> br(nbins);
        for (long b = 0; b < nbins; ++b) br[b] = make_int2(off[b], hc[b]);
        DevBuf<int2> dbr;
        dbr.upload(br.data(), br.size(), st);
        kbin_.alloc(nbins, st);
        binm_.alloc(nbins, st);
        LC_REQUIRE(nbins < (1L << 31), "NUFFT: too many bins");
        const size_t hsm = (size_t)g.td[0] * g.td[1] * g.td[2] * sizeof(int);
        LC_REQUIRE(hsm <= ctx.max_smem(), "NUFFT: bin tile does not fit shared memory");
        LC_REQUIRE(w_ <= 16, "NUFFT: kernel too wide");
        // Offset m of a footprint sees the point at x = (m - off) 2 / w with
        // off in (w/2 - 1, w/2]: the weight is at most the kernel at the end
        // of [(m - w/2) 2/w, (m - w/2 + 1) 2/w] nearest 0 (1 when it holds 0),
        // raised by 1e-3 for the device's exp2 and rounded up to 2^-12.
        OffsetWeights om{};
        for (int m = 0; m < w_; ++m) {
            const double a = (m - 0.5 * w_) * 2.0 / w_, b = (m - 0.5 * w_ + 1.0) * 2.0 / w_;
            const double x = (a <= 0.0 && b >= 0.0) ? 0.0 : std::min(std::fabs(a), std::fabs(b));
            const double phi = x < 1.0 ? std::exp(beta_ * (std::sqrt(1.0 - x * x) - 1.0)) : 0.0;
            om.w[m] = (float)(std::ceil(phi * 1.001 * 4096.0) / 4096.0);
        }
        if (dim_ == 2) {
            LC_W_SWITCH(w_, (launch_footprint_w<2, WW>(ctx, (unsigned)nbins, hsm, st, g, om, corner_.get(),
                                                      dbr.get(), kbin_.get())));
        } else {
            LC_W_SWITCH(w_, (launch_footprint_w<3, WW>(ctx, (unsigned)nbins, hsm, st, g, om, corner_.get(),
                                                      dbr.get(), kbin_.get())));
        }
        LC_CHECK_LAUNCH();
        LC_CUDA(cudaStreamSynchronize(st));
    }
}

void NufftPlan::spread(Context &ctx, const float2 *c, int nvol, float2 *grid, PtMode mode) {
    GridCfg g = make_cfg(dim_, nf_, bs_, nb_, w_, beta_);
    const long gvol = (long)nf_[0] * nf_[1] * nf_[2];
    cudaStream_t st = ctx.stream();
    // values read once, fine grid written once (plus the permutation)
    ProfScope ps(ctx, PS_SPREAD, (double)nvol * (8.0 * pts_.M + 8.0 * gvol) + 4.0 * pts_.M);
    // two 32-bit fixed-point accumulators per cell (real and imaginary parts)
    // per volume, a footprint count per cell and the bucketed point order (16
    // bits per point)
    const size_t tile_bytes = (size_t)g.td[0] * g.td[1] * g.td[2] * 2 * sizeof(int);
    const size_t bucket_bytes = (size_t)g.td[0] * g.td[1] * g.td[2] * sizeof(int) +
                                (size_t)maxsub_ * sizeof(unsigned short);
    LC_REQUIRE(maxsub_ <= 8 * kSpreadThreads, "NUFFT spread: subproblem larger than the bucketing pass");
    LC_REQUIRE(maxsub_ <= 2048, "NUFFT spread: subproblem too large for the fixed-point sums");
    // one fixed-point scale for the fine grid of the launch: bound the values first
    mbits_.ensure(1, st);
    fix_.ensure(2 * gvol * nvol, st);
    LC_CUDA(cudaMemsetAsync(mbits_.get(), 0, sizeof(int), st));
    LC_CUDA(cudaMemsetAsync(fix_.get(), 0, 2 * gvol * nvol * sizeof(long long), st));
    {
        const long n = (long)nvol * pts_.M;
        const long blocks = std::max<long>(1, std::min<long>((n + 255) / 256, (long)ctx.num_sms() * 8));
        value_bound_kernel<<<(unsigned)blocks, 256, 0, st>>>(c, n, mbits_.get());
        LC_CHECK_LAUNCH();
    }
    unsigned long long *fix = reinterpret_cast<unsigned long long *>(fix_.get());
    const int vchunk = (int)std::max<size_t>(1, (96 * 1024) / tile_bytes);
    for (int v0 = 0; v0 < nvol; v0 += vchunk) {
        const int nv = std::min(vchunk, nvol - v0);
        const size_t smem = tile_bytes * nv + bucket_bytes;
        LC_REQUIRE(smem <= ctx.max_smem(), "NUFFT spread: tile does not fit shared memory");
        const float2 *cv = c + (long)v0 * pts_.M;
        unsigned long long *fv = fix + 2 * (long)v0 * gvol;
        dim3 gd(nsub_);
        // the bins' value bounds over this chunk of volumes
        LC_CUDA(cudaMemsetAsync(binm_.get(), 0, binm_.size() * sizeof(int), st));
        bin_value_bound_kernel<<<gd, 256, 0, st>>>(cv, pts_.M, nv, perm_.get(), subs_.get(), binm_.get());
        LC_CHECK_LAUNCH();
        if (dim_ == 2) {
            LC_W_SWITCH(w_, (launch_spread_w<2, WW>(ctx, gd, smem, st, pts_, g, cv, pts_.M, nv,
                                                   perm_.get(), corner_.get(), subs_.get(), fv, gvol, mode, shifts_,
                                                   mbits_.get(), kmax_, kbin_.get(), binm_.get())));
        } else {
            LC_W_SWITCH(w_, (launch_spread_w<3, WW>(ctx, gd, smem, st, pts_, g, cv, pts_.M, nv,
                                                   perm_.get(), corner_.get(), subs_.get(), fv, gvol, mode, shifts_,
                                                   mbits_.get(), kmax_, kbin_.get(), binm_.get())));
        }
    }
    {
        const long n = gvol * nvol;
        const long blocks = std::max<long>(1, std::min<long>((n + 255) / 256, (long)ctx.num_sms() * 8));
        fix_to_float_kernel<<<(unsigned)blocks, 256, 0, st>>>(fix_.get(), grid, n, mbits_.get(), kmax_);
        LC_CHECK_LAUNCH();
    }
}

void NufftPlan::interp(Context &ctx, const float2 *grid, int nvol, float2 *c, PtMode mode) {
    GridCfg g = make_cfg(dim_, nf_, bs_, nb_, w_, beta_);
    const long gvol = (long)nf_[0] * nf_[1] * nf_[2];
    ProfScope ps(ctx, PS_INTERP, (double)nvol * (8.0 * pts_.M + 8.0 * gvol) + 4.0 * pts_.M);
    const size_t tile_bytes = (size_t)g.td[0] * g.td[1] * g.td[2] * sizeof(float2);
    int vchunk = (int)std::max<size_t>(1, (96 * 1024) / tile_bytes);
    for (int v0 = 0; v0 < nvol; v0 += vchunk) {
        int nv = std::min(vchunk, nvol - v0);
        size_t smem = tile_bytes * nv;
        const float2 *gv = grid + (long)v0 * gvol;
        float2 *cv = c + (long)v0 * pts_.M;
        dim3 gd(nsub_);
        if (dim_ == 2) {
            LC_W_SWITCH(w_, (launch_interp_w<2, WW>(ctx, gd, 256, smem, ctx.stream(), pts_, g, gv, gvol, nv,
                                                   perm_.get(), subs_.get(), cv, pts_.M, mode)));
        } else {
            LC_W_SWITCH(w_, (launch_interp_w<3, WW>(ctx, gd, 256, smem, ctx.stream(), pts_, g, gv, gvol, nv,
                                                   perm_.get(), subs_.get(), cv, pts_.M, mode)));
        }
    }
}

void NufftPlan::type1_real(Context &ctx, const float2 *c, int nvol, float *out, float scale,
                           PtMode mode) {
    cudaStream_t st = ctx.stream();
    const long gvol = (long)nf_[0] * nf_[1] * nf_[2];
    grid_.ensure(gvol * nvol, st);
    spread(ctx, c, nvol, grid_.get(), mode);
    const int n3 = modes_[0], n2 = modes_[1], n1 = modes_[2];
    const int fx = nf_[0], fy = nf_[1], fz = nf_[2];
    ProfScope ps(ctx, PS_NUFFT_FFT,
                 (double)nvol * 8.0 * ((double)gvol + 2.0 * fz * fy * n3 + 2.0 * fz * n2 * n3) +
                     (double)nvol * 4.0 * n1 * n2 * n3);
    // x pass: fine rows -> n3 modes
    h1_.ensure((long)nvol * fz * fy * n3, st);
    {
        AxisFFT a;
        a.in = grid_.get();
        a.in_t = E_C64;
        a.out = h1_.get();
        a.out_t = E_C64;
        a.n_outer = (long)nvol * fz * fy;
        a.n_inner = 1;
        a.in_ostride = fx;
        a.out_ostride = n3;
        a.n_in = fx;
        a.L = fx;
        a.n_out = n3;
        a.out_map = OUT_MODES;
        a.sign = +1;
        a.post = corr_[0].get();
        launch_axis_fft(ctx, a);
    }
    if (dim_ == 2) {
        AxisFFT a;
        a.in = h1_.get();
        a.in_t = E_C64;
        a.out = out;
        a.out_t = E_F32;
        a.n_outer = nvol;
        a.n_inner = n3;
        a.in_ostride = (long)fy * n3;
        a.out_ostride = (long)n2 * n3;
        a.n_in = fy;
        a.L = fy;
        a.n_out = n2;
        a.out_map = OUT_MODES;
        a.sign = +1;
        a.post = corr_[1].get();
        a.scale = scale;
        launch_axis_fft(ctx, a);
        return;
    }
    h2_.ensure((long)nvol * fz * n2 * n3, st);
    {
        AxisFFT a;
        a.in = h1_.get();
        a.in_t = E_C64;
        a.out = h2_.get();
        a.out_t = E_C64;
        a.n_outer = (long)nvol * fz;
        a.n_inner = n3;
        a.in_ostride = (long)fy * n3;
        a.out_ostride = (long)n2 * n3;
        a.n_in = fy;
        a.L = fy;
        a.n_out = n2;
        a.out_map = OUT_MODES;
        a.sign = +1;
        a.post = corr_[1].get();
        launch_axis_fft(ctx, a);
    }
    {
        AxisFFT a;
        a.in = h2_.get();
        a.in_t = E_C64;
        a.out = out;
        a.out_t = E_F32;
        a.n_outer = nvol;
        a.n_inner = (long)n2 * n3;
        a.in_ostride = (long)fz * n2 * n3;
        a.out_ostride = (long)n1 * n2 * n3;
        a.n_in = fz;
        a.L = fz;
        a.n_out = n1;
        a.out_map = OUT_MODES;
        a.sign = +1;
        a.post = corr_[2].get();
        a.scale = scale;
        launch_axis_fft(ctx, a);
    }
}

void NufftPlan::type2_real(Context &ctx, const float *in, int nvol, float2 *c, PtMode mode) {
    cudaStream_t st = ctx.stream();
    const int n3 = modes_[0], n2 = modes_[1], n1 = modes_[2];
    const int fx = nf_[0], fy = nf_[1], fz = nf_[2];
    const long gvol = (long)fx * fy * fz;
    grid_.ensure(gvol * nvol, st);
    h1_.ensure((long)nvol * fz * fy * n3, st);
    std::unique_ptr<ProfScope> ps(new ProfScope(
        ctx, PS_NUFFT_FFT,
        (double)nvol * 8.0 * ((double)gvol + 2.0 * fz * fy * n3 + 2.0 * fz * n2 * n3) +
            (double)nvol * 4.0 * n1 * n2 * n3));
    if (dim_ == 2) {
        AxisFFT a;
        a.in = in;
        a.in_t = E_F32;
        a.out = h1_.get();
        a.out_t = E_C64;
        a.n_outer = nvol;
        a.n_inner = n3;
        a.in_ostride = (long)n2 * n3;
        a.out_ostride = (long)fy * n3;
        a.n_in = n2;
        a.in_map = IN_MODES;
        a.L = fy;
        a.n_out = fy;
        a.sign = -1;
        a.pre = corr_[1].get();
        a.linefac = corr_[0].get();
        launch_axis_fft(ctx, a);
    } else {
        h2_.ensure((long)nvol * fz * n2 * n3, st);
        {
            AxisFFT a;
            a.in = in;
            a.in_t = E_F32;
            a.out = h2_.get();
            a.out_t = E_C64;
            a.n_outer = nvol;
            a.n_inner = (long)n2 * n3;
            a.in_ostride = (long)n1 * n2 * n3;
            a.out_ostride = (long)fz * n2 * n3;
            a.n_in = n1;
            a.in_map = IN_MODES;
            a.L = fz;
            a.n_out = fz;
            a.sign = -1;
            a.pre = corr_[2].get();
            a.linefac = corr_xy_.get();
            launch_axis_fft(ctx, a);
        }
        {
            AxisFFT a;
            a.in = h2_.get();
            a.in_t = E_C64;
            a.out = h1_.get();
            a.out_t = E_C64;
            a.n_outer = (long)nvol * fz;
            a.n_inner = n3;
            a.in_ostride = (long)n2 * n3;
            a.out_ostride = (long)fy * n3;
            a.n_in = n2;
            a.in_map = IN_MODES;
            a.L = fy;
            a.n_out = fy;
            a.sign = -1;
            launch_axis_fft(ctx, a);
        }
    }
    {
        AxisFFT a;
        a.in = h1_.get();
        a.in_t = E_C64;
        a.out = grid_.get();
        a.out_t = E_C64;
        a.n_outer = (long)nvol * fz * fy;
        a.n_inner = 1;
        a.in_ostride = n3;
        a.out_ostride = fx;
        a.n_in = n3;
        a.in_map = IN_MODES;
        a.L = fx;
        a.n_out = fx;
        a.sign = -1;
        launch_axis_fft(ctx, a);
    }
    ps.reset();
    interp(ctx, grid_.get(), nvol, c, mode);
}

}  // namespace lc
