// Non-uniform FFTs on the polar Fourier grids of LaminoCam, FINUFFT semantics:
//   type 1 (iflag +1):  f_k = sum_j c_j exp(+i k.x_j)
//   type 2 (iflag -1):  c_j = sum_k f_k exp(-i k.x_j)
// with modes k in [-floor(N/2), floor((N-1)/2)] in increasing order and x the
// fastest dimension (include/nufft.h:37-95 of the reference).
//
// Non-uniform points are never stored: they are regenerated in FP64 from the
// grid description (polar radius/angle in 2D, rotated detector lattice in 3D)
// wherever a kernel needs them.  Only a permutation that sorts point indices
// by fine-grid bin is kept per (geometry, fine grid).
#pragma once

#include <vector>

#include "lc_fft.hpp"

namespace lc {

// n / d for 0 <= n < 2^31 by a multiply and a shift (Granlund and Montgomery,
// "Division by invariant integers using multiplication", PLDI 1994): with
// 2^(s-1) < d <= 2^s and m = floor(2^32 (2^s - d) / d) + 1,
// n / d = (umulhi(n, m) + n) >> s  (the sum stays below 2^32 for n < 2^31).
struct FastDiv {
    unsigned m = 1, s = 0;
};

inline FastDiv make_fastdiv(unsigned d) {
    FastDiv f;
    while ((1ull << f.s) < d) ++f.s;
    f.m = (unsigned)(((1ull << 32) * ((1ull << f.s) - d)) / d + 1);
    return f;
}

// Polar grid description.  2D: x = r cos(theta), y = r sin(theta),
// r_m = (m+1/2) 2pi/nr - pi (include/polar_grid2d.h:50-65).  3D: rows of the
// detector lattice rotated by transpose(Rx(theta) Ry(beta) Rz(gamma))
// (include/polar_grid.h:52-94, include/rotation.h:28-56).
struct PolarPts {
    int dim = 2;
    long M = 0;  // below 2^31 (the bin sort stores point indices as int)
    int ntheta = 0;
    // 2D
    int nr = 0;
    const double2 *cs = nullptr;  // (cos theta, sin theta) per angle
    // 3D
    int nrows = 0, ncols = 0;
    const double *rot = nullptr;  // R00 R01 R10 R11 R20 R21 per angle
    // point index -> angle (by nr in 2D, nrows * ncols in 3D) and, in 3D, row (by ncols)
    FastDiv div_angle, div_col;
};

struct PolarGeometry {
    PolarPts pts;
    std::vector<double> theta, gamma, beta;
    std::vector<float> shifts;  // 2 per angle (dx, dy), 3D only
    DevBuf<double2> cs;
    DevBuf<double> rot;
    DevBuf<float2> dshifts;
};

void geometry_init_2d(Context &ctx, PolarGeometry &g, const double *theta, int ntheta, int nr);
void geometry_init_3d(Context &ctx, PolarGeometry &g, const double *theta, const double *gamma,
                      const double *beta, const float *shifts, int ntheta, int nrows, int ncols);

// kernel width and shape for a requested tolerance (upsampling factor 2)
int es_width_for_tol(double tol);
double es_beta_for_width(int w);
// deapodisation factors 2/(w*phihat(k*w*pi/nf)) for the n modes k = j - n/2
std::vector<double> es_correction(int n, int nf, int w, double beta);

// Pointwise handling of the non-uniform values inside spread / interp.
enum PtMode {
    PT_PLAIN = 0,   // values used as given
    PT_MASK = 1,    // multiply by the 3D |q|<=pi mask w_j
    PT_SHIFT = 2,   // 3D: mask and exp(-i(qX dx + qY dy)) per projection
};

// NUFFT plan for one geometry and one mode box (x, y[, z] = n3, n2[, n1]).
class NufftPlan {
  public:
    NufftPlan(Context &ctx, const PolarGeometry &g, const int modes[3], double tol);
    // type 1: c [nvol][M] complex -> out real [nvol][n1][n2][n3] = Re(f) * scale
    void type1_real(Context &ctx, const float2 *c, int nvol, float *out, float scale,
                    PtMode mode);
    // type 2: real in [nvol][...modes] -> c [nvol][M]
    void type2_real(Context &ctx, const float *in, int nvol, float2 *c, PtMode mode);

    int dim() const { return dim_; }
    long M() const { return pts_.M; }
    const int *nf() const { return nf_; }
    int width() const { return w_; }

  private:
    void sort_points(Context &ctx);
    void spread(Context &ctx, const float2 *c, int nvol, float2 *grid, PtMode mode);
    void interp(Context &ctx, const float2 *grid, int nvol, float2 *c, PtMode mode);

    int dim_;
    PolarPts pts_;
    const float2 *shifts_ = nullptr;
    int modes_[3];
    int nf_[3];
    int w_;
    double beta_;
    int bs_[3];
    int nb_[3];
    DevBuf<float> corr_[3];
    DevBuf<float> corr_xy_;  // corr_y (x) corr_x, 3D type 2
    DevBuf<int> perm_;
    DevBuf<unsigned short> corner_;  // per sorted point: footprint corner in its bin's tile
    DevBuf<int4> subs_;
    int nsub_ = 0;
    int maxsub_ = 1024;  // most points of one spreading subproblem
    long kmax_ = 1;      // bound on the footprints that cover one fine-grid cell
    DevBuf<float2> grid_, h1_, h2_;
    DevBuf<long long> fix_;  // 64-bit fixed-point fine grid of the spreading (re, im)
    DevBuf<int> mbits_;      // bound on the spread values (float bits)
    DevBuf<int> kbin_;       // per bin: bound on the summed weights over one tile cell (float bits)
    DevBuf<int> binm_;       // per bin: bound on its spread values (float bits), per call
};

}  // namespace lc
