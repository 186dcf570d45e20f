// Toeplitz normal operator A^T A as a convolution with the point-spread
// function of the polar grid (include/toeplitz.h:61-129 and
// include/toeplitz2d.h:81-125 of the reference).
//
// The PSF is K(k) = Re sum_j exp(i k.x_j) on the P-grid, P = next 2^p3^q >=
// 2n-1 per axis, with unit weights at every grid point (no mask).  On a polar
// grid the sum over the radial samples of one angle is a Dirichlet kernel,
//     sum_m exp(i u r_m) = sin(pi u) / sin(pi u / n),
// so K is generated exactly, in FP64, as a sum over angles of products of
// Dirichlet kernels (one factor in 2D, two in 3D) instead of a type-1 NUFFT of
// ones.  K(-k) = K(k).  After zeroing the unpaired planes k = -P/2 (never reached
// by the cropped convolution) the zero-centred kernel K0 is point-symmetric, so
// its spectrum is real; the R2C half {P1, P2, P3/2+1} is kept in FP32 (half the
// bytes of the reference's complex half spectrum).  Convolving with K0 and
// cropping at offset 0 equals the reference's convolution with the centred
// kernel cropped at P/2.
#pragma once

#include "lc_nufft.hpp"

namespace lc {

class Toeplitz {
  public:
    // dims = {n1, n2, n3}: volume (3D) or stack of n1 independent n2 x n3
    // slices (2D, n2 == n3 required by the reference API).  The spectrum is
    // built in the order of ctx.stream() and may still be in flight on
    // return.
    // psf_fp32: the kernel K from a FP32 type-1 NUFFT of ones (tol 1e-6), the
    // reference GPU's construction, in place of the exact FP64 closed form
    Toeplitz(Context &ctx, const PolarGeometry &g, const long dims[3], bool three_d, bool psf_fp32 = false);
    // shares src's spectrum (read-only) and, with `work`, owns fresh work
    // buffers on ctx's stream: concurrent jobs on one geometry use one
    // spectrum.  Without work buffers the copy only holds the spectrum (a
    // cache entry) and cannot be applied.
    Toeplitz(Context &ctx, const Toeplitz &src, bool work = true);
    // y = A^T A x.  With f, the parts of `parts` (a subset of cg_caps()) of the
    // surrounding CG iteration are fused into the x passes: x is then the
    // direction f->p, updated in place.
    // pitch: the row stride of x and y (>= n3; 0 = n3); y's values past n3
    // are not written
    void apply(Context &ctx, const float *x, float *y, const CGFusion *f = nullptr, unsigned parts = 0,
               long pitch = 0);
    // CG work the apply can fuse (its x passes run the register-plan row kernel)
    unsigned cg_caps() const;
    // CTAs whose partials a fused dot product writes
    long cg_partials() const;
    // y = A^T A x + mu * (-laplacian(x))
    void apply_reg(Context &ctx, const float *x, float *y, float mu);

    const long *dims() const { return n_; }
    const int *P() const { return P_; }
    bool three_d() const { return three_d_; }
    long nvox() const { return n_[0] * n_[1] * n_[2]; }
    // elements of the real spectrum {P1, P2, P3/2+1}
    long spectrum_elems() const { return (long)P_[0] * P_[1] * Ph_[2]; }
    // the planes of it kept on the device: all P1, or only f1 <= P1/2 when
    // the kernel is even in kz (then R(P1 - f1) = R(f1), spectrum_zfold())
    long stored_spectrum_elems() const { return (long)(zfold_ ? P_[0] / 2 + 1 : P_[0]) * P_[1] * Ph_[2]; }
    bool spectrum_zfold() const { return zfold_; }
    // the spectrum (built on first use when the z stage is direct: that
    // needs the PSF's own geometry, as kernel_fp64 does)
    void ensure_spectrum(Context &ctx);
    const float *spectrum() const { return R_ ? R_->get() : nullptr; }
    // factor of the last pass: 1 / (P1 P2 P3 n2 n3) (3D) or 1 / (P^2 n) (2D)
    double scale() const { return scale_; }
    size_t device_bytes() const {
        return spectrum_bytes() + (t1_.size() + t2_.size()) * sizeof(float2);
    }
    // the spectrum and, when the z stage runs in direct form, its taps
    size_t spectrum_bytes() const {
        return ((R_ ? R_->size() : 0) + (Kz_ ? Kz_->size() : 0)) * sizeof(float);
    }
    // the z stage runs as the direct Toeplitz product (kernel even in z,
    // n1 <= zdirect_max_rows()); its taps are {n1, P2, P3/2+1} floats
    bool z_direct() const { return (bool)Kz_; }
    // device bytes, for given dims, of the work buffers of one apply and of
    // the peak of a spectrum construction
    static size_t work_bytes(const long dims[3], bool three_d);
    static size_t build_peak_bytes(const long dims[3], bool three_d);
    // FP64 PSF K on the P-grid in mode order (k = j - P/2), for tests
    void kernel_fp64(Context &ctx, double *host_out);
    // bytes the apply must move at minimum (algorithmic traffic)
    double algorithmic_bytes() const;

  private:
    // zkeep > 0: with the kz mirror, only the planes 0 <= kz < zkeep are set
    void build_kernel(Context &ctx, DevBuf<double> &K, int zkeep);
    void build_kernel_nufft32(Context &ctx, DevBuf<double> &K);
    void kernel_xy_fft(Context &ctx, const double *K, int nz, double2 *a, double2 *b);
    void build_spectrum(Context &ctx, DevBuf<double> *K);
    bool psf_fp32_ = false;
    bool three_d_;
    bool kernel_mirror_ = false;  // the last kernel built is even in its mirror axis (kz in 3D)
    bool zfold_ = false;          // spectrum stored for f1 <= P1/2 only
    long n_[3];
    int P_[3];
    int Ph_[3];
    const PolarGeometry *g_;
    std::shared_ptr<DevBuf<float>> R_;
    std::shared_ptr<DevBuf<float>> Kz_;  // direct z-stage taps L b(dz), dz < n1 (or null)
    DevBuf<float2> t1_, t2_;
    double scale_;
};

void launch_neg_laplacian_axpy(Context &ctx, const float *x, float *y, const long dims[3], float mu);

}  // namespace lc
