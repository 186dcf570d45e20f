// CG and Split-Bregman (isotropic TV) on the device.
//
// Algorithms follow src/conjgrad.cpp:33-76 / src/gpu/conjgrad.cu:45-108 and
// src/bregman.cpp:36-94 / src/gpu/bregman.cu:88-165 of the reference.  All
// solver scalars (alpha, beta, r.r, p.Ap, the norms and the stopping tests)
// live in device memory and are computed in FP64 by the last CTA of each
// fused reduction, so an iteration never waits on the host.  Once a stopping
// test fires, a device flag turns the remaining update kernels into no-ops.
#pragma once

#include <functional>

#include "lc_cgstate.hpp"
#include "lc_runtime.hpp"

namespace lc {

struct SolverParams {
    int max_iters = 50;   // CG iterations, or Split-Bregman outer iterations
    int inner_iters = 1;  // CG iterations per Split-Bregman outer iteration
    float tol = 1e-5f;
    float xtol = 1e-5f;
    float lambda = 0.1f;
    float mu = 10.0f;
    int fp32_scalars = 0;  // 1: float accumulation of dots (the reference GPU path)
    int poll_every = 8;    // iterations between host checks of the stop flag (0: never)
    int use_graph = 0;     // 1: replay CG iterations (Split-Bregman: outer iterations) as CUDA graphs
    // Split-Bregman: recompute the operator product A x of the warm-started
    // residual every this many outer iterations (1: every one); in between it
    // is carried by the CG updates
    int residual_refresh = 1;
};

struct SolverStats {
    int iters = 0;          // CG iterations, or outer iterations for Split-Bregman
    int cg_iters_total = 0;
    double residual = 0;    // ||r|| / (||y|| + 1e-8) of the last CG iteration
    double dx = 0;          // last CG relative step, or Split-Bregman relative change
    int stop_reason = 0;    // 0 max iters, 1 residual, 2 step, 3 |pAp| tiny
};

using Operator = std::function<void(const float *in, float *out)>;

// An operator that can take over CG work around its own passes (see
// CGFusion): caps says which parts apply() performs.
struct FusedOperator {
    unsigned caps = 0;   // kFusedUpdate | kFusedDot
    long partials = 0;   // CTAs whose partials a fused dot writes
    std::function<void(const float *in, float *out, const CGFusion &f)> apply;
};

class Solver {
  public:
    Solver(Context &ctx, long n);
    ~Solver();
    Solver(const Solver &) = delete;
    long size() const { return n_; }
    Solver &operator=(const Solver &) = delete;
    // x (in: x0, out: solution); y = right-hand side
    // With F, each iteration applies F (fusing the direction update and the
    // dot product when F can) instead of A.
    void cg(Context &ctx, const Operator &A, const float *y, float *x, const SolverParams &p,
            SolverStats *stats, const FusedOperator *F = nullptr);
    // A is the normal operator A^T A alone; mu * (-laplacian) is added here.
    // pitch: the row stride of x, yT and of the vectors AtA gets and returns
    // (>= dims[2], the values past dims[2] zero; 0 = dims[2]); the solver's
    // size is dims[0] * dims[1] * pitch.  A multiple of 4 lets the stencil
    // kernels take four voxels per thread.
    void split_bregman(Context &ctx, const Operator &AtA, const long dims[3], const float *yT,
                       float *x, const SolverParams &p, SolverStats *stats, long pitch = 0);

  private:
    void cg_run(Context &ctx, const Operator &A, const float *y, float *x, int iters, float tol,
                float xtol, int fp32, int poll_every, bool graph, const FusedOperator *F);
    // one CG iteration: Ap = A p, the fused scalar/vector updates, p = r + beta p
    // (with F: p = r + beta p first, then Ap = A p with what F fuses)
    void cg_iter(Context &ctx, const Operator &A, float *x, float tol, float xtol, int fp32,
                 const FusedOperator *F);
    // records body into graph_ on the context's private stream
    void capture(Context &ctx, const std::function<void()> &body);
    CapturedGraph graph_;
    long n_;
    int nblk_;
    DevBuf<float> r_, p_, ap_, xold_;
    DevBuf<float> q_[3], b_[3], ax_;  // q = d - b (Split-Bregman), b, carried A x
    DevBuf<double> part_;
    DevBuf<unsigned> counter_;
    DevBuf<CGState> st_;
    CGState *host_st_ = nullptr;  // the context's pinned scratch, set per solve
};

}  // namespace lc
