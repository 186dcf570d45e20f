// Device-resident CG state, and the CG work an operator may fuse into its own
// passes.
#pragma once

namespace lc {

// device-resident solver state
struct CGState {
    double rs_old, pAp, alpha, beta;
    double y2;
    double res, dx;
    int iters, done, reason, pad;
    // Split-Bregman: |x - x_old|^2 and |x_old|^2 of the outer iteration (when
    // the CG update forms them), the relative change
    double sb_diff2, sb_old2, sb_rel;
    int sb_iters, sb_done;
};

// CG work that an operator applied to the direction p can take over:
//   kFusedUpdate  p = r + beta p (beta from st, skipped once st->done is set)
//                 while its first pass loads p
//   kFusedDot     p.Ap, then alpha = r.r / p.Ap and the |p.Ap| < 1e-10 stop
//                 (st->pAp, st->alpha, st->done, st->reason) while its last
//                 pass stores Ap; per-CTA partials go to part, the last CTA
//                 (ticket counter) sums them in a fixed order
constexpr unsigned kFusedUpdate = 1u, kFusedDot = 2u;

struct CGFusion {
    float *p = nullptr;
    const float *r = nullptr;
    CGState *st = nullptr;
    double *part = nullptr;
    unsigned *counter = nullptr;
    int fp32 = 0;  // float accumulation of the dot (the reference GPU path)
};

}  // namespace lc
