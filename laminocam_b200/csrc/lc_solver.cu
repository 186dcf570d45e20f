// Fused solver kernels: CG updates with FP64 reductions finished by the last
// CTA (deterministic fixed-order sum of per-CTA partials), and the
// Split-Bregman stencil kernels (right-hand side, shrinkage + Bregman update).
#include <algorithm>
#include <cstdint>
#include <cstdlib>
#include <memory>

#include "lc_solver.hpp"
#include "lc_toeplitz.hpp"

namespace lc {

namespace {

constexpr int kThreads = 256;
constexpr int kParts = 4;  // partial sums per CTA

template <typename A>
__device__ __forceinline__ A warp_sum(A v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    return v;
}

// Block-reduce up to kParts sums and store them as this CTA's partials.
// Returns true in every thread of the CTA that finished last.
template <typename A, int K>
__device__ bool block_partials(A (&v)[K], double *part, unsigned *counter) {
    __shared__ A sh[K][kThreads / 32];
    __shared__ bool last;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
    for (int k = 0; k < K; ++k) {
        A s = warp_sum(v[k]);
        if (lane == 0) sh[k][wid] = s;
    }
    __syncthreads();
    if (threadIdx.x < 32) {
#pragma unroll
        for (int k = 0; k < K; ++k) {
            A s = lane < (int)(blockDim.x >> 5) ? sh[k][lane] : A(0);
            s = warp_sum(s);
            if (lane == 0) part[(long)blockIdx.x * kParts + k] = (double)s;
        }
    }
    __threadfence();
    if (threadIdx.x == 0) {
        unsigned t = atomicAdd(counter, 1u);
        last = (t == gridDim.x - 1);
    }
    __syncthreads();
    return last;
}

// Fixed-order total of partial k over all CTAs (called by the last CTA).
template <typename A>
__device__ double total(const double *part, int k, int nblk) {
    __shared__ A sh[kThreads / 32];
    A s = A(0);
    for (int b = threadIdx.x; b < nblk; b += blockDim.x) s += (A)part[(long)b * kParts + k];
    s = warp_sum(s);
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    if (lane == 0) sh[wid] = s;
    __syncthreads();
    A t = A(0);
    if (threadIdx.x < 32) {
        t = lane < (int)(blockDim.x >> 5) ? sh[lane] : A(0);
        t = warp_sum(t);
    }
    __shared__ A res;
    if (threadIdx.x == 0) res = t;
    __syncthreads();
    double out = (double)res;
    __syncthreads();
    return out;
}

// r = y - r(=A x0);  p = r;  partials y.y, r.r
template <typename A>
__global__ void __launch_bounds__(kThreads) cg_init_kernel(const float *__restrict__ y, float *__restrict__ r,
                                                          float *__restrict__ p, long n, double *part,
                                                          unsigned *counter, CGState *st) {
    if (st->sb_done) {
        if (blockIdx.x == 0 && threadIdx.x == 0) st->done = 1;
        return;
    }
    A v[2] = {A(0), A(0)};
    for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
        float yi = y[i];
        float ri = yi - r[i];
        r[i] = ri;
        p[i] = ri;
        v[0] += (A)yi * (A)yi;
        v[1] += (A)ri * (A)ri;
    }
    if (block_partials<A, 2>(v, part, counter)) {
        double y2 = total<A>(part, 0, gridDim.x);
        double r2 = total<A>(part, 1, gridDim.x);
        if (threadIdx.x == 0) {
            st->y2 = y2;
            st->rs_old = r2;
            st->beta = 0.0;  // p = r + 0 p: a direction update ahead of the first iteration keeps p
            st->iters = 0;
            st->done = 0;
            st->reason = 0;
            st->res = 0;
            st->dx = 0;
            *counter = 0;
        }
    }
}

template <typename A>
__global__ void __launch_bounds__(kThreads) dot_pap_kernel(const float *__restrict__ p,
                                                          const float *__restrict__ ap, long n,
                                                          double *part, unsigned *counter,
                                                          CGState *st) {
    if (st->done) return;
    A v[1] = {A(0)};
    for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x)
        v[0] += (A)p[i] * (A)ap[i];
    if (block_partials<A, 1>(v, part, counter)) {
        double pap = total<A>(part, 0, gridDim.x);
        if (threadIdx.x == 0) {
            st->pAp = pap;
            if (fabs(pap) < 1e-10) {
                st->done = 1;
                st->reason = 3;
            } else {
                st->alpha = (double)((A)st->rs_old / (A)pap);
            }
            *counter = 0;
        }
    }
}

// x += a p; r -= a Ap; partials r.r, |a p|^2, x.x; then beta, stopping tests.
// AX: also carry the operator product, ax += a Ap (Split-Bregman keeps A x up
// to date this way between exact recomputations).  STORE_R: false when no
// later kernel reads r (one CG iteration per outer iteration, where p and r
// may then share a buffer: both are only read then, which the restrict
// qualifiers allow).  SB_CHANGE (one CG iteration per Split-Bregman outer
// iteration, which is then the whole change of x): the second and third sums
// are |x_new - x_old|^2 and |x_old|^2 of the stored floats, kept in
// st->sb_diff2 and st->sb_old2 for the outer change test, in place of the
// CG step test.
template <typename A, bool AX = false, bool STORE_R = true, bool SB_CHANGE = false>
__global__ void __launch_bounds__(kThreads)
    cg_update_kernel(float *__restrict__ x, float *__restrict__ r, const float *__restrict__ p,
                     const float *__restrict__ ap, float *__restrict__ ax, long n, double *part,
                     unsigned *counter, CGState *st, float tol, float xtol) {
    if (st->done) return;
    const float a = (float)st->alpha;
    A v[3] = {A(0), A(0), A(0)};
    auto one = [&](float api, float pi, float xo, float ro, float axo, float &xi, float &ri, float &axn) {
        const float step = a * pi;
        xi = xo + step;
        ri = fmaf(-a, api, ro);
        axn = fmaf(a, api, axo);
        v[0] += (A)ri * (A)ri;
        if constexpr (SB_CHANGE) {
            const float df = xi - xo;
            v[1] += (A)df * (A)df;
            v[2] += (A)xo * (A)xo;
        } else {
            v[1] += (A)step * (A)step;
            v[2] += (A)xi * (A)xi;
        }
    };
    const long tid = (long)blockIdx.x * blockDim.x + threadIdx.x, nth = (long)gridDim.x * blockDim.x;
    // float4 accesses (four times the bytes in flight per load) when every
    // vector is 16-byte aligned and n is a multiple of 4
    const unsigned long al = (unsigned long)x | (unsigned long)r | (unsigned long)p | (unsigned long)ap |
                             (AX ? (unsigned long)ax : 0ul);
    if ((al & 15ul) == 0 && (n & 3) == 0) {
        const long n4 = n >> 2;
        for (long i = tid; i < n4; i += nth) {
            const float4 apv = reinterpret_cast<const float4 *>(ap)[i];
            const float4 pv = reinterpret_cast<const float4 *>(p)[i];
            const float4 xv = reinterpret_cast<const float4 *>(x)[i];
            const float4 rv = reinterpret_cast<const float4 *>(r)[i];
            const float4 av = AX ? reinterpret_cast<const float4 *>(ax)[i] : make_float4(0.f, 0.f, 0.f, 0.f);
            float4 xn, rn, an;
            one(apv.x, pv.x, xv.x, rv.x, av.x, xn.x, rn.x, an.x);
            one(apv.y, pv.y, xv.y, rv.y, av.y, xn.y, rn.y, an.y);
            one(apv.z, pv.z, xv.z, rv.z, av.z, xn.z, rn.z, an.z);
            one(apv.w, pv.w, xv.w, rv.w, av.w, xn.w, rn.w, an.w);
            reinterpret_cast<float4 *>(x)[i] = xn;
            if constexpr (STORE_R) reinterpret_cast<float4 *>(r)[i] = rn;
            if constexpr (AX) reinterpret_cast<float4 *>(ax)[i] = an;
        }
    } else {
        for (long i = tid; i < n; i += nth) {
            float xi, ri, axn;
            one(ap[i], p[i], x[i], r[i], AX ? ax[i] : 0.f, xi, ri, axn);
            x[i] = xi;
            if constexpr (STORE_R) r[i] = ri;
            if constexpr (AX) ax[i] = axn;
        }
    }
    if (block_partials<A, 3>(v, part, counter)) {
        double rs_new = total<A>(part, 0, gridDim.x);
        double s2 = total<A>(part, 1, gridDim.x);
        double x2 = total<A>(part, 2, gridDim.x);
        if (threadIdx.x == 0) {
            st->beta = (double)((A)rs_new / (A)st->rs_old);
            st->rs_old = rs_new;
            double res = sqrt(rs_new) / (sqrt(st->y2) + 1e-8);
            st->res = res;
            st->iters += 1;
            if constexpr (SB_CHANGE) {
                // the CG ends after this iteration; the outer test uses the change
                st->sb_diff2 = s2;
                st->sb_old2 = x2;
            } else {
                double dx = sqrt(s2) / (sqrt(x2) + 1e-8);
                st->dx = dx;
                if (res < (double)tol) {
                    st->done = 1;
                    st->reason = 1;
                } else if (dx < (double)xtol) {
                    st->done = 1;
                    st->reason = 2;
                }
            }
            *counter = 0;
        }
    }
}

__global__ void __launch_bounds__(kThreads) p_update_kernel(float *__restrict__ p, const float *__restrict__ r,
                                                           long n, const CGState *st) {
    if (st->done) return;
    const float b = (float)st->beta;
    for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x)
        p[i] = fmaf(b, p[i], r[i]);
}

// n3 values of a row, stored at a row pitch p3 >= n3 (the values past n3 are
// kept zero)
struct Dims {
    int n1, n2, n3, p3;
};

// The stencil kernels walk the volume in tiles of 32 (along n3) x kTileRows
// (along n2) voxels of one plane, each thread taking kTileRows / 8 voxels 8
// rows apart (two per thread measured slower than one: more registers, fewer
// CTAs); a persistent grid of CTAs strides over the tiles, so one partial sum per CTA feeds the fused reductions.  The stride
// (the grid size) is pre-split into whole planes, tile rows and tiles, so a
// CTA steps from tile to tile without dividing.  Offsets are 32-bit (the host
// checks the size).
constexpr int kTileRows = 8;

struct Tiles {
    int tk, tj;      // tiles along n3 and n2
    int count;       // tk * tj * n1
    int qi, qj, qk;  // grid size = qi (tk tj) + qj tk + qk
};

struct TileGrid {
    Tiles tl;
    int blocks;
};

// body(i, j, k) for every voxel of this thread's tiles
template <typename F>
__device__ __forceinline__ void for_voxels(const Tiles &tl, const Dims &dm, F &&body) {
    const int per = tl.tk * tl.tj;
    int t = (int)blockIdx.x;
    int i = t / per;
    int jb = (t - i * per) / tl.tk;
    int kb = t - i * per - jb * tl.tk;
    const int ty = (int)(threadIdx.x >> 5), tx = (int)(threadIdx.x & 31);
    for (; t < tl.count; t += (int)gridDim.x) {
        const int k = kb * 32 + tx;
        if (k < dm.n3) {
#pragma unroll
            for (int u = 0; u < kTileRows / 8; ++u) {
                const int j = jb * kTileRows + ty + 8 * u;
                if (j < dm.n2) body(i, j, k);
            }
        }
        kb += tl.qk;
        if (kb >= tl.tk) {
            kb -= tl.tk;
            ++jb;
        }
        jb += tl.qj;
        if (jb >= tl.tj) {
            jb -= tl.tj;
            ++i;
        }
        i += tl.qi;
    }
}

// per-axis term of the negative-Laplacian stencil (src/gpu/finitediff.cu:28-222):
// 0.5 (g[i+1] - g[i-1]) with g[k] = 0.5 (x[k+1] - x[k-1]) and x = g = 0 outside
__device__ __forceinline__ float lap_term(const float *__restrict__ x, int idx, int pos, int n, int s,
                                          float c) {
    const float p2 = (pos + 2 < n) ? x[idx + 2 * s] : 0.f;
    const float m2 = (pos >= 2) ? x[idx - 2 * s] : 0.f;
    const float gp = (pos + 1 < n) ? 0.5f * (p2 - c) : 0.f;
    const float gm = (pos >= 1) ? 0.5f * (c - m2) : 0.f;
    return 0.5f * (gp - gm);
}

__device__ __forceinline__ float lap_at(const float *__restrict__ x, int idx, int i, int j, int k,
                                        const Dims &dm) {
    const float c = x[idx];
    float lap = 0.f;
    lap += lap_term(x, idx, k, dm.n3, 1, c);
    lap += lap_term(x, idx, j, dm.n2, dm.p3, c);
    lap += lap_term(x, idx, i, dm.n1, dm.n2 * dm.p3, c);
    return lap;
}

// Start of a Split-Bregman outer iteration (src/bregman.cpp:36-94):
//   rhs = yT - mu div(q),  q = d - b as stored by sb_shrink_diff
//                          (div = sum over axes of the zero-padded central
//                          difference; rhs is not stored)
//   ax  = tx - mu lap(x)       when tx (= A^T A x) is given, else the carried ax
//   r = rhs - ax,  p = r (when p is given);  partials rhs.rhs, r.r
// i.e. the warm-started CG initialisation of src/conjgrad.cpp:33-76.
template <typename A>
__global__ void __launch_bounds__(kThreads)
    sb_begin_kernel(const float *__restrict__ yT, const float *__restrict__ q0, const float *__restrict__ q1,
                    const float *__restrict__ q2, const float *__restrict__ tx, const float *__restrict__ x,
                    float *__restrict__ ax, float *__restrict__ r, float *__restrict__ p, Dims dm, Tiles tl,
                    float mu, double *part, unsigned *counter, CGState *st) {
    if (st->sb_done) {
        if (blockIdx.x == 0 && threadIdx.x == 0) st->done = 1;
        return;
    }
    A v[2] = {A(0), A(0)};
    const int sj = dm.p3, si = dm.n2 * dm.p3;
    for_voxels(tl, dm, [&](int i, int j, int k) {
        const int idx = i * si + j * sj + k;
        const float dk = (k + 1 < dm.n3 ? q0[idx + 1] : 0.f) - (k >= 1 ? q0[idx - 1] : 0.f);
        const float dj = (j + 1 < dm.n2 ? q1[idx + sj] : 0.f) - (j >= 1 ? q1[idx - sj] : 0.f);
        const float di = (i + 1 < dm.n1 ? q2[idx + si] : 0.f) - (i >= 1 ? q2[idx - si] : 0.f);
        const float rhs = fmaf(-mu, 0.5f * dk + 0.5f * dj + 0.5f * di, yT[idx]);
        float a;
        if (tx) {
            a = fmaf(-mu, lap_at(x, idx, i, j, k, dm), tx[idx]);
            ax[idx] = a;
        } else {
            a = ax[idx];
        }
        const float ri = rhs - a;
        r[idx] = ri;
        if (p) p[idx] = ri;
        v[0] += (A)rhs * (A)rhs;
        v[1] += (A)ri * (A)ri;
    });
    if (block_partials<A, 2>(v, part, counter)) {
        double y2 = total<A>(part, 0, gridDim.x);
        double r2 = total<A>(part, 1, gridDim.x);
        if (threadIdx.x == 0) {
            st->y2 = y2;
            st->rs_old = r2;
            st->iters = 0;
            st->done = 0;
            st->reason = 0;
            st->res = 0;
            st->dx = 0;
            st->sb_diff2 = 0;  // an update skipped by the |p.Ap| stop leaves x unchanged
            st->sb_old2 = 0;
            *counter = 0;
        }
    }
}

// ap = tp - mu lap(p) in place (tp = A^T A p on entry), then p.Ap and alpha:
// the operator (A^T A + mu (-lap)) of the Split-Bregman CG and its dot product
// in one pass
template <typename A>
__global__ void __launch_bounds__(kThreads) lap_dot_kernel(const float *__restrict__ p, float *__restrict__ ap, Dims dm,
                                                          Tiles tl, float mu, double *part,
                                                          unsigned *counter, CGState *st) {
    if (st->done) return;
    A v[1] = {A(0)};
    const int sj = dm.p3, si = dm.n2 * dm.p3;
    for_voxels(tl, dm, [&](int i, int j, int k) {
        const int idx = i * si + j * sj + k;
        const float a = fmaf(-mu, lap_at(p, idx, i, j, k, dm), ap[idx]);
        const float pc = p[idx];
        ap[idx] = a;
        v[0] += (A)pc * (A)a;
    });
    if (block_partials<A, 1>(v, part, counter)) {
        double pap = total<A>(part, 0, gridDim.x);
        if (threadIdx.x == 0) {
            st->pAp = pap;
            if (fabs(pap) < 1e-10) {
                st->done = 1;
                st->reason = 3;
            } else {
                st->alpha = (double)((A)st->rs_old / (A)pap);
            }
            *counter = 0;
        }
    }
}

// End of an outer iteration: g = grad x; t = g + b; s = |t|;
// d = max(0, s - lam/mu) t / (s + 1e-8); b += g - d; then the relative change
// |x - xold| / |xold| (partials) and xold = x.  d is read only as d - b (the
// next sb_begin), so q = d - b is stored in its place: the same float as the
// difference of the stored d and b.
// Without XOLD the change sums come from the CG update (st->sb_diff2,
// st->sb_old2) and xold is not touched.
template <typename A, bool XOLD>
__global__ void __launch_bounds__(kThreads)
    sb_shrink_diff_kernel(const float *__restrict__ x, float *__restrict__ xold, float *__restrict__ q0,
                          float *__restrict__ q1, float *__restrict__ q2, float *__restrict__ b0,
                          float *__restrict__ b1, float *__restrict__ b2, Dims dm, Tiles tl, float thresh,
                          double *part, unsigned *counter, CGState *st, float xtol) {
    if (st->sb_done) return;
    A v[2] = {A(0), A(0)};
    const int sj = dm.p3, si = dm.n2 * dm.p3;
    for_voxels(tl, dm, [&](int i, int j, int k) {
        const int idx = i * si + j * sj + k;
        // every load first (the buffers are distinct), then the stores
        const float xi = x[idx], xo = XOLD ? xold[idx] : 0.f;
        const float c0 = b0[idx], c1 = b1[idx], c2 = b2[idx];
        const float g0 = 0.5f * ((k + 1 < dm.n3 ? x[idx + 1] : 0.f) - (k >= 1 ? x[idx - 1] : 0.f));
        const float g1 = 0.5f * ((j + 1 < dm.n2 ? x[idx + sj] : 0.f) - (j >= 1 ? x[idx - sj] : 0.f));
        const float g2 = 0.5f * ((i + 1 < dm.n1 ? x[idx + si] : 0.f) - (i >= 1 ? x[idx - si] : 0.f));
        const float t0 = g0 + c0, t1 = g1 + c1, t2 = g2 + c2;
        const float s = sqrtf(t0 * t0 + t1 * t1 + t2 * t2);
        const float m = fmaxf(0.f, s - thresh);
        const float inv = 1.0f / (s + 1e-8f);
        const float e0 = m * (t0 * inv), e1 = m * (t1 * inv), e2 = m * (t2 * inv);
        const float n0 = c0 + (g0 - e0), n1 = c1 + (g1 - e1), n2 = c2 + (g2 - e2);
        q0[idx] = e0 - n0;
        q1[idx] = e1 - n1;
        q2[idx] = e2 - n2;
        b0[idx] = n0;
        b1[idx] = n1;
        b2[idx] = n2;
        if constexpr (XOLD) {
            const float df = xi - xo;
            v[0] += (A)df * (A)df;
            v[1] += (A)xo * (A)xo;
            xold[idx] = xi;
        }
    });
    if (block_partials<A, 2>(v, part, counter)) {
        double d2s = XOLD ? total<A>(part, 0, gridDim.x) : st->sb_diff2;
        double o2 = XOLD ? total<A>(part, 1, gridDim.x) : st->sb_old2;
        if (threadIdx.x == 0) {
            double rel = sqrt(d2s) / (sqrt(o2) + 1e-8);
            st->sb_rel = rel;
            st->sb_iters += 1;
            if (rel < (double)xtol) st->sb_done = 1;
            *counter = 0;
        }
    }
}

// ---- the same three stencil kernels on four voxels per thread ----
// With the row pitch a multiple of 4 every row starts 16-byte aligned: a
// thread takes the four voxels k0 .. k0+3 of its row as one float4 (a warp
// one row segment of 128 voxels, a CTA eight rows), their neighbours along
// k come from the next lanes by shuffles (the warp's end lanes load the one
// or two values past the segment), and those along n2 and n1 are float4
// loads of the neighbouring rows.  The arithmetic per voxel is that of the
// scalar kernels; values at k >= n3 are stored as 0 and left out of the sums.
struct Quad {
    float v[4];
};

__device__ __forceinline__ Quad ld4(const float *__restrict__ a, long idx) {
    const float4 t = *reinterpret_cast<const float4 *>(a + idx);
    return Quad{{t.x, t.y, t.z, t.w}};
}

__device__ __forceinline__ void st4(float *__restrict__ a, long idx, const Quad &q) {
    *reinterpret_cast<float4 *>(a + idx) = make_float4(q.v[0], q.v[1], q.v[2], q.v[3]);
}

// values at k - 1 and k + 1 (and k - 2, k + 2 with TWO) of the four values c
// at k0 .. k0+3 of a row (row-relative k0; zero before the row and past its
// pitch).  Every lane of the warp calls it (shuffles).
template <bool TWO>
__device__ __forceinline__ void k_neighbours(const float *__restrict__ row, int k0, int p3, const Quad &c,
                                             Quad &m1, Quad &p1, Quad &m2, Quad &p2) {
    const int lane = (int)(threadIdx.x & 31);
    float w3 = __shfl_up_sync(0xffffffffu, c.v[3], 1);
    float n0 = __shfl_down_sync(0xffffffffu, c.v[0], 1);
    float w2 = 0.f, n1 = 0.f;
    if constexpr (TWO) {
        w2 = __shfl_up_sync(0xffffffffu, c.v[2], 1);
        n1 = __shfl_down_sync(0xffffffffu, c.v[1], 1);
    }
    if (lane == 0) {
        w3 = k0 >= 1 && k0 - 1 < p3 ? row[k0 - 1] : 0.f;
        if constexpr (TWO) w2 = k0 >= 2 && k0 - 2 < p3 ? row[k0 - 2] : 0.f;
    }
    if (lane == 31) {
        n0 = k0 + 4 < p3 ? row[k0 + 4] : 0.f;
        if constexpr (TWO) n1 = k0 + 5 < p3 ? row[k0 + 5] : 0.f;
    }
    m1 = Quad{{w3, c.v[0], c.v[1], c.v[2]}};
    p1 = Quad{{c.v[1], c.v[2], c.v[3], n0}};
    if constexpr (TWO) {
        m2 = Quad{{w2, w3, c.v[0], c.v[1]}};
        p2 = Quad{{c.v[2], c.v[3], n0, n1}};
    }
}

// per-axis term of the negative Laplacian (lap_term) from the values at
// pos - 2, pos, pos + 2 along an axis of length n
__device__ __forceinline__ float lap_term_v(float m2, float c, float p2, int pos, int n) {
    const float pp = (pos + 2 < n) ? p2 : 0.f;
    const float mm = (pos >= 2) ? m2 : 0.f;
    const float gp = (pos + 1 < n) ? 0.5f * (pp - c) : 0.f;
    const float gm = (pos >= 1) ? 0.5f * (c - mm) : 0.f;
    return 0.5f * (gp - gm);
}

// body(i, j, k0, act): every (row, four-voxel group) of this thread's tiles;
// act is false for lanes past the row's pitch (they still join the shuffles)
template <typename F>
__device__ __forceinline__ void for_quads(const Tiles &tl, const Dims &dm, F &&body) {
    const int per = tl.tk * tl.tj;
    int t = (int)blockIdx.x;
    int i = t / per;
    int jb = (t - i * per) / tl.tk;
    int kb = t - i * per - jb * tl.tk;
    const int ty = (int)(threadIdx.x >> 5), tx = (int)(threadIdx.x & 31);
    for (; t < tl.count; t += (int)gridDim.x) {
        const int j = jb * kTileRows + ty;
        const int k0 = (kb * 32 + tx) * 4;
        if (j < dm.n2) body(i, j, k0, k0 < dm.p3);  // uniform over the warp but for act
        kb += tl.qk;
        if (kb >= tl.tk) {
            kb -= tl.tk;
            ++jb;
        }
        jb += tl.qj;
        if (jb >= tl.tj) {
            jb -= tl.tj;
            ++i;
        }
        i += tl.qi;
    }
}

__device__ __forceinline__ Quad lap4(const float *__restrict__ x, long idx, int i, int j, int k0, const Dims &dm,
                                     const Quad &c, const Quad &m2k, const Quad &p2k) {
    const int sj = dm.p3, si = dm.n2 * dm.p3;
    const Quad jm = j >= 2 ? ld4(x, idx - 2 * sj) : Quad{{0.f, 0.f, 0.f, 0.f}};
    const Quad jp = j + 2 < dm.n2 ? ld4(x, idx + 2 * sj) : Quad{{0.f, 0.f, 0.f, 0.f}};
    const Quad im = i >= 2 ? ld4(x, idx - 2 * si) : Quad{{0.f, 0.f, 0.f, 0.f}};
    const Quad ip = i + 2 < dm.n1 ? ld4(x, idx + 2 * si) : Quad{{0.f, 0.f, 0.f, 0.f}};
    Quad out;
#pragma unroll
    for (int e = 0; e < 4; ++e) {
        float lap = 0.f;
        lap += lap_term_v(m2k.v[e], c.v[e], p2k.v[e], k0 + e, dm.n3);
        lap += lap_term_v(jm.v[e], c.v[e], jp.v[e], j, dm.n2);
        lap += lap_term_v(im.v[e], c.v[e], ip.v[e], i, dm.n1);
        out.v[e] = lap;
    }
    return out;
}

#ifndef LC_SB_BEGIN_MIN_BLOCKS
#define LC_SB_BEGIN_MIN_BLOCKS 4  // CTAs per SM sb_begin4's registers are sized for
#endif

template <typename A>
__global__ void __launch_bounds__(kThreads, LC_SB_BEGIN_MIN_BLOCKS)
    sb_begin4_kernel(const float *__restrict__ yT, const float *__restrict__ q0, const float *__restrict__ q1,
                     const float *__restrict__ q2, const float *__restrict__ tx, const float *__restrict__ x,
                     float *__restrict__ ax, float *__restrict__ r, float *__restrict__ p, Dims dm, Tiles tl,
                     float mu, double *part, unsigned *counter, CGState *st) {
    if (st->sb_done) {
        if (blockIdx.x == 0 && threadIdx.x == 0) st->done = 1;
        return;
    }
    A v[2] = {A(0), A(0)};
    const int sj = dm.p3, si = dm.n2 * dm.p3;
    const Quad zero{{0.f, 0.f, 0.f, 0.f}};
    for_quads(tl, dm, [&](int i, int j, int k0, bool act) {
        const long base = (long)i * si + (long)j * sj;
        const long idx = base + k0;
        const Quad c0 = act ? ld4(q0, idx) : zero;
        Quad m1, p1, m2, p2;
        k_neighbours<false>(q0 + base, k0, dm.p3, c0, m1, p1, m2, p2);
        Quad xc = zero, xm2 = zero, xp2 = zero, xm1, xp1;
        if (tx) {
            xc = act ? ld4(x, idx) : zero;
            k_neighbours<true>(x + base, k0, dm.p3, xc, xm1, xp1, xm2, xp2);
        }
        if (!act) return;
        const Quad jm = j >= 1 ? ld4(q1, idx - sj) : zero, jp = j + 1 < dm.n2 ? ld4(q1, idx + sj) : zero;
        const Quad im = i >= 1 ? ld4(q2, idx - si) : zero, ip = i + 1 < dm.n1 ? ld4(q2, idx + si) : zero;
        const Quad y = ld4(yT, idx);
        Quad a = tx ? ld4(tx, idx) : ld4(ax, idx);
        if (tx) {
            const Quad lp = lap4(x, idx, i, j, k0, dm, xc, xm2, xp2);
#pragma unroll
            for (int e = 0; e < 4; ++e) a.v[e] = k0 + e < dm.n3 ? fmaf(-mu, lp.v[e], a.v[e]) : 0.f;
            st4(ax, idx, a);
        }
        Quad rr;
#pragma unroll
        for (int e = 0; e < 4; ++e) {
            const float dk = p1.v[e] - m1.v[e];
            const float dj = jp.v[e] - jm.v[e];
            const float di = ip.v[e] - im.v[e];
            const float rhs = fmaf(-mu, 0.5f * dk + 0.5f * dj + 0.5f * di, y.v[e]);
            const float ri = rhs - a.v[e];
            const bool in = k0 + e < dm.n3;
            rr.v[e] = in ? ri : 0.f;
            if (in) {
                v[0] += (A)rhs * (A)rhs;
                v[1] += (A)ri * (A)ri;
            }
        }
        st4(r, idx, rr);
        if (p) st4(p, idx, rr);
    });
    if (block_partials<A, 2>(v, part, counter)) {
        double y2 = total<A>(part, 0, gridDim.x);
        double r2 = total<A>(part, 1, gridDim.x);
        if (threadIdx.x == 0) {
            st->y2 = y2;
            st->rs_old = r2;
            st->iters = 0;
            st->done = 0;
            st->reason = 0;
            st->res = 0;
            st->dx = 0;
            st->sb_diff2 = 0;  // an update skipped by the |p.Ap| stop leaves x unchanged
            st->sb_old2 = 0;
            *counter = 0;
        }
    }
}

template <typename A>
__global__ void __launch_bounds__(kThreads) lap_dot4_kernel(const float *__restrict__ p, float *__restrict__ ap,
                                                           Dims dm, Tiles tl, float mu, double *part,
                                                           unsigned *counter, CGState *st) {
    if (st->done) return;
    A v[1] = {A(0)};
    const int sj = dm.p3, si = dm.n2 * dm.p3;
    const Quad zero{{0.f, 0.f, 0.f, 0.f}};
    for_quads(tl, dm, [&](int i, int j, int k0, bool act) {
        const long base = (long)i * si + (long)j * sj;
        const long idx = base + k0;
        const Quad c = act ? ld4(p, idx) : zero;
        Quad m1, p1, m2, p2;
        k_neighbours<true>(p + base, k0, dm.p3, c, m1, p1, m2, p2);
        if (!act) return;
        const Quad lp = lap4(p, idx, i, j, k0, dm, c, m2, p2);
        Quad a = ld4(ap, idx);
#pragma unroll
        for (int e = 0; e < 4; ++e) {
            const bool in = k0 + e < dm.n3;
            a.v[e] = in ? fmaf(-mu, lp.v[e], a.v[e]) : 0.f;
            if (in) v[0] += (A)c.v[e] * (A)a.v[e];
        }
        st4(ap, idx, a);
    });
    if (block_partials<A, 1>(v, part, counter)) {
        double pap = total<A>(part, 0, gridDim.x);
        if (threadIdx.x == 0) {
            st->pAp = pap;
            if (fabs(pap) < 1e-10) {
                st->done = 1;
                st->reason = 3;
            } else {
                st->alpha = (double)((A)st->rs_old / (A)pap);
            }
            *counter = 0;
        }
    }
}

template <typename A, bool XOLD>
__global__ void __launch_bounds__(kThreads)
    sb_shrink4_kernel(const float *__restrict__ x, float *__restrict__ xold, float *__restrict__ q0,
                      float *__restrict__ q1, float *__restrict__ q2, float *__restrict__ b0,
                      float *__restrict__ b1, float *__restrict__ b2, Dims dm, Tiles tl, float thresh,
                      double *part, unsigned *counter, CGState *st, float xtol) {
    if (st->sb_done) return;
    A v[2] = {A(0), A(0)};
    const int sj = dm.p3, si = dm.n2 * dm.p3;
    const Quad zero{{0.f, 0.f, 0.f, 0.f}};
    for_quads(tl, dm, [&](int i, int j, int k0, bool act) {
        const long base = (long)i * si + (long)j * sj;
        const long idx = base + k0;
        const Quad xc = act ? ld4(x, idx) : zero;
        Quad m1, p1, m2, p2;
        k_neighbours<false>(x + base, k0, dm.p3, xc, m1, p1, m2, p2);
        if (!act) return;
        const Quad xo = XOLD ? ld4(xold, idx) : zero;
        const Quad c0 = ld4(b0, idx), c1 = ld4(b1, idx), c2 = ld4(b2, idx);
        const Quad jm = j >= 1 ? ld4(x, idx - sj) : zero, jp = j + 1 < dm.n2 ? ld4(x, idx + sj) : zero;
        const Quad im = i >= 1 ? ld4(x, idx - si) : zero, ip = i + 1 < dm.n1 ? ld4(x, idx + si) : zero;
        Quad o0, o1, o2, n0, n1, n2;
#pragma unroll
        for (int e = 0; e < 4; ++e) {
            const bool in = k0 + e < dm.n3;
            const float g0 = 0.5f * ((k0 + e + 1 < dm.n3 ? p1.v[e] : 0.f) - (k0 + e >= 1 ? m1.v[e] : 0.f));
            const float g1 = 0.5f * (jp.v[e] - jm.v[e]);
            const float g2 = 0.5f * (ip.v[e] - im.v[e]);
            const float t0 = g0 + c0.v[e], t1 = g1 + c1.v[e], t2 = g2 + c2.v[e];
            const float s = sqrtf(t0 * t0 + t1 * t1 + t2 * t2);
            const float m = fmaxf(0.f, s - thresh);
            const float inv = 1.0f / (s + 1e-8f);
            const float e0 = m * (t0 * inv), e1 = m * (t1 * inv), e2 = m * (t2 * inv);
            const float d0 = c0.v[e] + (g0 - e0), d1 = c1.v[e] + (g1 - e1), d2 = c2.v[e] + (g2 - e2);
            o0.v[e] = in ? e0 - d0 : 0.f;
            o1.v[e] = in ? e1 - d1 : 0.f;
            o2.v[e] = in ? e2 - d2 : 0.f;
            n0.v[e] = in ? d0 : 0.f;
            n1.v[e] = in ? d1 : 0.f;
            n2.v[e] = in ? d2 : 0.f;
            if constexpr (XOLD) {
                if (in) {
                    const float df = xc.v[e] - xo.v[e];
                    v[0] += (A)df * (A)df;
                    v[1] += (A)xo.v[e] * (A)xo.v[e];
                }
            }
        }
        st4(q0, idx, o0);
        st4(q1, idx, o1);
        st4(q2, idx, o2);
        st4(b0, idx, n0);
        st4(b1, idx, n1);
        st4(b2, idx, n2);
        if constexpr (XOLD) st4(xold, idx, xc);
    });
    if (block_partials<A, 2>(v, part, counter)) {
        double d2s = XOLD ? total<A>(part, 0, gridDim.x) : st->sb_diff2;
        double o2 = XOLD ? total<A>(part, 1, gridDim.x) : st->sb_old2;
        if (threadIdx.x == 0) {
            double rel = sqrt(d2s) / (sqrt(o2) + 1e-8);
            st->sb_rel = rel;
            st->sb_iters += 1;
            if (rel < (double)xtol) st->sb_done = 1;
            *counter = 0;
        }
    }
}

__global__ void reset_state_kernel(CGState *st) {
    CGState z{};
    *st = z;
}

}  // namespace

Solver::Solver(Context &ctx, long n) : n_(n) {
    cudaStream_t s = ctx.stream();
    // the 1D vector kernels: one full wave of the CTAs that fit at once
    int per_sm = 8;
    for (const void *k : {(const void *)cg_update_kernel<double>, (const void *)cg_update_kernel<double, true, false, true>,
                          (const void *)cg_init_kernel<double>, (const void *)dot_pap_kernel<double>,
                          (const void *)p_update_kernel}) {
        int b = 0;
        LC_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, k, kThreads, 0));
        per_sm = std::min(per_sm, std::max(b, 1));
    }
    nblk_ = (int)std::max<long>(1, std::min<long>((n + kThreads - 1) / kThreads, (long)ctx.num_sms() * per_sm));
    r_.alloc(n, s);
    p_.alloc(n, s);
    ap_.alloc(n, s);
    part_.alloc((long)nblk_ * kParts, s);
    counter_.alloc(1, s);
    counter_.zero(s);
    st_.alloc(1, s);
}

Solver::~Solver() { graph_.reset(); }

void Solver::capture(Context &ctx, const std::function<void()> &body) {
    // Capturing records the launches without running them.  It happens on the
    // context's private stream (the caller's stream may be the legacy default
    // stream, which cannot capture); the replays go to the caller's stream.
    const cudaStream_t user = ctx.stream();
    const cudaStream_t side = ctx.capture_stream();
    ctx.set_stream(side);
    try {
        graph_.capture(side, body);
    } catch (...) {
        ctx.set_stream(user);
        throw;
    }
    ctx.set_stream(user);
}

void Solver::cg_iter(Context &ctx, const Operator &A, float *x, float tol, float xtol, int fp32,
                     const FusedOperator *F) {
    cudaStream_t s = ctx.stream();
    if (F) {
        // p = r + beta p ahead of the operator (beta = 0 in the first
        // iteration), inside its first pass when it can; p.Ap inside its last
        CGFusion f;
        f.p = p_.get();
        f.r = r_.get();
        f.st = st_.get();
        f.part = part_.get();
        f.counter = counter_.get();
        f.fp32 = fp32;
        if (!(F->caps & kFusedUpdate)) {
            p_update_kernel<<<nblk_, kThreads, 0, s>>>(p_.get(), r_.get(), n_, st_.get());
            LC_CHECK_LAUNCH();
        }
        F->apply(p_.get(), ap_.get(), f);
        ProfScope ps(ctx, PS_CG_VEC, 4.0 * n_ * ((F->caps & kFusedDot) ? 5.0 : 7.0));
        if (!(F->caps & kFusedDot)) {
            if (fp32)
                dot_pap_kernel<float><<<nblk_, kThreads, 0, s>>>(p_.get(), ap_.get(), n_, part_.get(),
                                                                 counter_.get(), st_.get());
            else
                dot_pap_kernel<double><<<nblk_, kThreads, 0, s>>>(p_.get(), ap_.get(), n_, part_.get(),
                                                                  counter_.get(), st_.get());
            LC_CHECK_LAUNCH();
        }
        if (fp32)
            cg_update_kernel<float><<<nblk_, kThreads, 0, s>>>(x, r_.get(), p_.get(), ap_.get(), nullptr, n_,
                                                               part_.get(), counter_.get(), st_.get(), tol, xtol);
        else
            cg_update_kernel<double><<<nblk_, kThreads, 0, s>>>(x, r_.get(), p_.get(), ap_.get(), nullptr, n_,
                                                                part_.get(), counter_.get(), st_.get(), tol, xtol);
        LC_CHECK_LAUNCH();
        return;
    }
    A(p_.get(), ap_.get());
    ProfScope ps(ctx, PS_CG_VEC, 4.0 * n_ * 10.0);
    if (fp32) {
        dot_pap_kernel<float><<<nblk_, kThreads, 0, s>>>(p_.get(), ap_.get(), n_, part_.get(),
                                                         counter_.get(), st_.get());
        LC_CHECK_LAUNCH();
        cg_update_kernel<float><<<nblk_, kThreads, 0, s>>>(x, r_.get(), p_.get(), ap_.get(), nullptr,
                                                           n_, part_.get(), counter_.get(),
                                                           st_.get(), tol, xtol);
        LC_CHECK_LAUNCH();
    } else {
        dot_pap_kernel<double><<<nblk_, kThreads, 0, s>>>(p_.get(), ap_.get(), n_, part_.get(),
                                                          counter_.get(), st_.get());
        LC_CHECK_LAUNCH();
        cg_update_kernel<double><<<nblk_, kThreads, 0, s>>>(x, r_.get(), p_.get(), ap_.get(), nullptr,
                                                            n_, part_.get(), counter_.get(),
                                                            st_.get(), tol, xtol);
        LC_CHECK_LAUNCH();
    }
    p_update_kernel<<<nblk_, kThreads, 0, s>>>(p_.get(), r_.get(), n_, st_.get());
    LC_CHECK_LAUNCH();
}

void Solver::cg_run(Context &ctx, const Operator &A, const float *y, float *x, int iters,
                    float tol, float xtol, int fp32, int poll_every, bool graph, const FusedOperator *F) {
    cudaStream_t s = ctx.stream();
    A(x, ap_.get());
    // r <- A x0 (moved), then r = y - r, p = r
    LC_CUDA(cudaMemcpyAsync(r_.get(), ap_.get(), n_ * sizeof(float), cudaMemcpyDeviceToDevice, s));
    if (fp32)
        cg_init_kernel<float><<<nblk_, kThreads, 0, s>>>(y, r_.get(), p_.get(), n_, part_.get(),
                                                         counter_.get(), st_.get());
    else
        cg_init_kernel<double><<<nblk_, kThreads, 0, s>>>(y, r_.get(), p_.get(), n_, part_.get(),
                                                          counter_.get(), st_.get());
    LC_CHECK_LAUNCH();
    const bool poll = poll_every > 0;
    // With graphs one replay covers `chunk` iterations (the polling interval
    // when the host polls); a remainder runs as ordinary launches.  Iterations
    // after the stop flag are no-ops on the device either way.
    int chunk = 0;
    if (graph && iters > 1) {
        chunk = poll ? std::min(poll_every, iters) : std::min(iters, 8);
        capture(ctx, [&] {
            for (int k = 0; k < chunk; ++k) cg_iter(ctx, A, x, tol, xtol, fp32, F);
        });
    }
    int it = 0;
    while (it < iters) {
        if (chunk > 0 && iters - it >= chunk) {
            graph_.launch(s);
            it += chunk;
        } else {
            cg_iter(ctx, A, x, tol, xtol, fp32, F);
            it += 1;
        }
        const bool boundary = chunk > 0 || it % std::max(poll_every, 1) == 0;
        if (poll && boundary && it < iters) {
            LC_CUDA(cudaMemcpyAsync(host_st_, st_.get(), sizeof(CGState), cudaMemcpyDeviceToHost, s));
            LC_CUDA(cudaStreamSynchronize(s));
            if (host_st_->done) break;
        }
    }
}

void Solver::cg(Context &ctx, const Operator &A, const float *y, float *x, const SolverParams &p,
                SolverStats *stats, const FusedOperator *F) {
    cudaStream_t s = ctx.stream();
    host_st_ = static_cast<CGState *>(ctx.pinned_scratch(sizeof(CGState)));
    if (F && (F->caps & kFusedDot)) part_.ensure((long)std::max<long>(nblk_, F->partials) * kParts, s);
    reset_state_kernel<<<1, 1, 0, s>>>(st_.get());
    LC_CHECK_LAUNCH();
    int poll = (p.tol > 0 || p.xtol > 0) ? p.poll_every : 0;
    const bool graph = p.use_graph != 0 && !ctx.prof.on;
    cg_run(ctx, A, y, x, p.max_iters, p.tol, p.xtol, p.fp32_scalars, poll, graph, F);
    graph_.reset();
    LC_CUDA(cudaMemcpyAsync(host_st_, st_.get(), sizeof(CGState), cudaMemcpyDeviceToHost, s));
    LC_CUDA(cudaStreamSynchronize(s));
    if (stats) {
        stats->iters = host_st_->iters;
        stats->cg_iters_total = host_st_->iters;
        stats->residual = host_st_->res;
        stats->dx = host_st_->dx;
        stats->stop_reason = host_st_->reason;
    }
}

bool sb_vec4_enabled() {
    static const bool on = [] {
        const char *e = std::getenv("LC_SB_VEC4");
        return !(e && e[0] == '0');
    }();
    return on;
}

void Solver::split_bregman(Context &ctx, const Operator &AtA, const long dims[3], const float *yT,
                           float *x, const SolverParams &p, SolverStats *stats, long pitch) {
    cudaStream_t s = ctx.stream();
    if (pitch <= 0) pitch = dims[2];
    LC_REQUIRE(pitch >= dims[2], "split_bregman: row pitch below the row length");
    LC_REQUIRE(dims[0] * dims[1] * pitch == n_, "split_bregman: dims do not match the solver size");
    LC_REQUIRE(n_ < (1L << 31) && dims[1] < (1L << 24) && pitch < (1L << 24),
               "split_bregman: volume too large for 32-bit indexing");
    // four voxels per thread when every row starts 16-byte aligned
    const bool vec4 = pitch % 4 == 0 && sb_vec4_enabled() &&
                      ((reinterpret_cast<uintptr_t>(x) | reinterpret_cast<uintptr_t>(yT)) & 15) == 0;
    host_st_ = static_cast<CGState *>(ctx.pinned_scratch(sizeof(CGState)));
    const int inner = std::max(0, p.inner_iters);
    for (int a = 0; a < 3; ++a) {
        q_[a].ensure(n_, s);
        b_[a].ensure(n_, s);
        q_[a].zero(s);
        b_[a].zero(s);
    }
    ax_.ensure(n_, s);
    // with one CG iteration per outer iteration the CG update forms the change
    // sums; more need the iterate of the previous outer iteration
    const bool keep_xold = inner > 1;
    if (keep_xold) {
        xold_.ensure(n_, s);
        LC_CUDA(cudaMemcpyAsync(xold_.get(), x, n_ * sizeof(float), cudaMemcpyDeviceToDevice, s));
    }
    reset_state_kernel<<<1, 1, 0, s>>>(st_.get());
    LC_CHECK_LAUNCH();
    const float mu = p.mu;
    const Dims dm{(int)dims[0], (int)dims[1], (int)dims[2], (int)pitch};
    // the values past the row length stay zero in every work vector
    if (pitch != dims[2]) {
        ap_.zero(s);
        r_.zero(s);
        ax_.zero(s);
        if (inner > 1) p_.zero(s);
    }
    Tiles tl;
    tl.tk = vec4 ? (int)((pitch / 4 + 31) / 32) : (int)((dims[2] + 31) / 32);
    tl.tj = (int)((dims[1] + kTileRows - 1) / kTileRows);
    const long ntiles = (long)tl.tk * tl.tj * dims[0];
    LC_REQUIRE(ntiles < (1L << 31), "split_bregman: too many tiles");
    tl.count = (int)ntiles;
    // Each stencil kernel gets one full wave: its persistent grid is as large
    // as the number of its CTAs that fit on the device at once (a partial
    // second wave would repeat a whole CTA's share of tiles on a few SMs).
    auto grid_for_kernel = [&](const void *k) {
        int b = 0;
        LC_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, k, kThreads, 0));
        TileGrid g;
        g.tl = tl;
        g.blocks = (int)std::max<long>(1, std::min<long>(ntiles, (long)ctx.num_sms() * std::max(b, 1)));
        g.tl.qi = g.blocks / (tl.tk * tl.tj);
        g.tl.qj = (g.blocks - g.tl.qi * tl.tk * tl.tj) / tl.tk;
        g.tl.qk = g.blocks - g.tl.qi * tl.tk * tl.tj - g.tl.qj * tl.tk;
        return g;
    };
    const bool f32 = p.fp32_scalars != 0;
    const void *k_begin = vec4 ? (f32 ? (const void *)sb_begin4_kernel<float> : (const void *)sb_begin4_kernel<double>)
                               : (f32 ? (const void *)sb_begin_kernel<float> : (const void *)sb_begin_kernel<double>);
    const void *k_lap = vec4 ? (f32 ? (const void *)lap_dot4_kernel<float> : (const void *)lap_dot4_kernel<double>)
                             : (f32 ? (const void *)lap_dot_kernel<float> : (const void *)lap_dot_kernel<double>);
    const void *k_shrink =
        vec4 ? (f32 ? (keep_xold ? (const void *)sb_shrink4_kernel<float, true> : (const void *)sb_shrink4_kernel<float, false>)
                    : (keep_xold ? (const void *)sb_shrink4_kernel<double, true> : (const void *)sb_shrink4_kernel<double, false>))
             : (f32 ? (keep_xold ? (const void *)sb_shrink_diff_kernel<float, true> : (const void *)sb_shrink_diff_kernel<float, false>)
                    : (keep_xold ? (const void *)sb_shrink_diff_kernel<double, true>
                                 : (const void *)sb_shrink_diff_kernel<double, false>));
    const TileGrid g_begin = grid_for_kernel(k_begin);
    const TileGrid g_lap = grid_for_kernel(k_lap);
    const TileGrid g_shrink = grid_for_kernel(k_shrink);
    const int sblk = std::max(g_begin.blocks, std::max(g_lap.blocks, g_shrink.blocks));
    part_.ensure((long)std::max(sblk, nblk_) * kParts, s);
    // With one CG iteration per outer iteration its direction is the residual
    // itself, so p and r share a buffer and r is not stored after the update.
    float *pp = inner > 1 ? p_.get() : r_.get();
    const bool fp32 = p.fp32_scalars != 0;
    // One outer iteration: rhs and the warm-started residual, `inner` CG
    // iterations, shrinkage and the change test.  The operator product A x of
    // the warm start is recomputed when `exact` is set and otherwise carried
    // from the previous iteration's CG updates (ax += alpha A p), which equals
    // it up to rounding.  Launches go to ctx.stream() as it is when the lambda
    // runs (the capture stream while a graph is recorded).
    auto outer = [&](bool exact) {
        const cudaStream_t os = ctx.stream();
        if (exact) AtA(x, ap_.get());
        {
            // yT, q[3] and A x (carried: read; exact: A^T A x and x read, A x written), r written
            ProfScope ps(ctx, PS_SB_VEC, 4.0 * n_ * (exact ? 8.0 : 6.0) + (inner > 1 ? 4.0 * n_ : 0.0));
            const float *tx = exact ? ap_.get() : nullptr;
            float *pinit = inner > 1 ? p_.get() : nullptr;
            if (fp32)
                (vec4 ? sb_begin4_kernel<float> : sb_begin_kernel<float>)<<<g_begin.blocks, kThreads, 0, os>>>(
                    yT, q_[0].get(), q_[1].get(), q_[2].get(), tx, x,
                    ax_.get(), r_.get(), pinit, dm, g_begin.tl, mu, part_.get(), counter_.get(), st_.get());
            else
                (vec4 ? sb_begin4_kernel<double> : sb_begin_kernel<double>)<<<g_begin.blocks, kThreads, 0, os>>>(
                    yT, q_[0].get(), q_[1].get(), q_[2].get(), tx, x,
                    ax_.get(), r_.get(), pinit, dm, g_begin.tl, mu, part_.get(), counter_.get(), st_.get());
            LC_CHECK_LAUNCH();
        }
        for (int it = 0; it < inner; ++it) {
            AtA(pp, ap_.get());
            ProfScope ps(ctx, PS_CG_VEC, 4.0 * n_ * (inner > 1 ? 13.0 : 10.0));
            if (fp32) {
                (vec4 ? lap_dot4_kernel<float> : lap_dot_kernel<float>)<<<g_lap.blocks, kThreads, 0, os>>>(pp, ap_.get(), dm, g_lap.tl, mu, part_.get(),
                                                                counter_.get(), st_.get());
                LC_CHECK_LAUNCH();
                if (inner > 1)
                    cg_update_kernel<float, true, true><<<nblk_, kThreads, 0, os>>>(
                        x, r_.get(), pp, ap_.get(), ax_.get(), n_, part_.get(), counter_.get(), st_.get(), p.tol,
                        p.xtol);
                else
                    cg_update_kernel<float, true, false, true><<<nblk_, kThreads, 0, os>>>(
                        x, r_.get(), pp, ap_.get(), ax_.get(), n_, part_.get(), counter_.get(), st_.get(), p.tol,
                        p.xtol);
            } else {
                (vec4 ? lap_dot4_kernel<double> : lap_dot_kernel<double>)<<<g_lap.blocks, kThreads, 0, os>>>(pp, ap_.get(), dm, g_lap.tl, mu, part_.get(),
                                                                 counter_.get(), st_.get());
                LC_CHECK_LAUNCH();
                if (inner > 1)
                    cg_update_kernel<double, true, true><<<nblk_, kThreads, 0, os>>>(
                        x, r_.get(), pp, ap_.get(), ax_.get(), n_, part_.get(), counter_.get(), st_.get(), p.tol,
                        p.xtol);
                else
                    cg_update_kernel<double, true, false, true><<<nblk_, kThreads, 0, os>>>(
                        x, r_.get(), pp, ap_.get(), ax_.get(), n_, part_.get(), counter_.get(), st_.get(), p.tol,
                        p.xtol);
            }
            LC_CHECK_LAUNCH();
            if (it + 1 < inner) {
                p_update_kernel<<<nblk_, kThreads, 0, os>>>(p_.get(), r_.get(), n_, st_.get());
                LC_CHECK_LAUNCH();
            }
        }
        // x and b[3] read, q[3] and b[3] written (and xold read and written)
        ProfScope ps(ctx, PS_SB_VEC, 4.0 * n_ * (keep_xold ? 12.0 : 10.0));
        float *xo = keep_xold ? xold_.get() : nullptr;
        const float th = p.lambda / p.mu;
        if (fp32) {
            if (keep_xold)
                (vec4 ? sb_shrink4_kernel<float, true> : sb_shrink_diff_kernel<float, true>)<<<g_shrink.blocks, kThreads, 0, os>>>(
                    x, xo, q_[0].get(), q_[1].get(), q_[2].get(), b_[0].get(), b_[1].get(), b_[2].get(), dm,
                    g_shrink.tl, th, part_.get(), counter_.get(), st_.get(), p.xtol);
            else
                (vec4 ? sb_shrink4_kernel<float, false> : sb_shrink_diff_kernel<float, false>)<<<g_shrink.blocks, kThreads, 0, os>>>(
                    x, xo, q_[0].get(), q_[1].get(), q_[2].get(), b_[0].get(), b_[1].get(), b_[2].get(), dm,
                    g_shrink.tl, th, part_.get(), counter_.get(), st_.get(), p.xtol);
        } else {
            if (keep_xold)
                (vec4 ? sb_shrink4_kernel<double, true> : sb_shrink_diff_kernel<double, true>)<<<g_shrink.blocks, kThreads, 0, os>>>(
                    x, xo, q_[0].get(), q_[1].get(), q_[2].get(), b_[0].get(), b_[1].get(), b_[2].get(), dm,
                    g_shrink.tl, th, part_.get(), counter_.get(), st_.get(), p.xtol);
            else
                (vec4 ? sb_shrink4_kernel<double, false> : sb_shrink_diff_kernel<double, false>)<<<g_shrink.blocks, kThreads, 0, os>>>(
                    x, xo, q_[0].get(), q_[1].get(), q_[2].get(), b_[0].get(), b_[1].get(), b_[2].get(), dm,
                    g_shrink.tl, th, part_.get(), counter_.get(), st_.get(), p.xtol);
        }
        LC_CHECK_LAUNCH();
    };
    // exact operator products every `every` outer iterations (and always in
    // the first one, which also sets up ax)
    const int every = std::max(1, p.residual_refresh);
    auto exact_at = [&](int it) { return it % every == 0; };
    const bool graph = p.use_graph != 0 && !ctx.prof.on && p.max_iters > 1;
    if (graph) {
        // the first outer iteration runs eagerly (it also fills the plan and
        // launch-tuner caches the recorded launches rely on); the graph holds
        // the iteration that the other iterations, but the exact ones, replay
        outer(true);
        capture(ctx, [&] { outer(every == 1); });
    }
    const int poll = p.xtol > 0 ? std::max(1, p.poll_every) : 0;
    for (int it = graph ? 1 : 0; it < p.max_iters; ++it) {
        if (graph && (every == 1 || !exact_at(it)))
            graph_.launch(s);
        else
            outer(exact_at(it));
        if (poll > 0 && (it + 1) % poll == 0 && it + 1 < p.max_iters) {
            LC_CUDA(cudaMemcpyAsync(host_st_, st_.get(), sizeof(CGState), cudaMemcpyDeviceToHost, s));
            LC_CUDA(cudaStreamSynchronize(s));
            if (host_st_->sb_done) break;
        }
    }
    graph_.reset();
    LC_CUDA(cudaMemcpyAsync(host_st_, st_.get(), sizeof(CGState), cudaMemcpyDeviceToHost, s));
    LC_CUDA(cudaStreamSynchronize(s));
    if (stats) {
        stats->iters = host_st_->sb_iters;
        // outer iterations after the stop flag run no CG work
        stats->cg_iters_total = host_st_->sb_iters * inner;
        stats->residual = host_st_->res;
        stats->dx = host_st_->sb_rel;
        stats->stop_reason = host_st_->sb_done ? 2 : 0;
    }
}

}  // namespace lc
