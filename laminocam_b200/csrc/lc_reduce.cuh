// Deterministic grid reductions shared by the solver kernels and the kernels
// that fuse a solver reduction into their epilogue: every CTA stores FP64
// partials, and the CTA that finishes last (atomic ticket) sums them in a
// fixed order.
#pragma once

#include "lc_common.cuh"

namespace lc {

constexpr int kRedParts = 4;  // partial sums per CTA

template <typename A>
__device__ __forceinline__ A warp_sum_red(A v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    return v;
}

// Block-reduce K (<= kRedParts) sums of any CTA size up to 1024 threads and
// store them as partial slot `slot` of `nslots` (one per CTA taking part).
// Returns true in every thread of the CTA that finished last.  Every thread of
// the CTA must call it.
template <typename A, int K>
__device__ bool red_block_partials_at(A (&v)[K], double *part, unsigned *counter, long slot, long nslots) {
    __shared__ A sh[K][32];
    __shared__ bool last;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const int nw = (int)((blockDim.x + 31) >> 5);
#pragma unroll
    for (int k = 0; k < K; ++k) {
        A s = warp_sum_red(v[k]);
        if (lane == 0) sh[k][wid] = s;
    }
    __syncthreads();
    if (threadIdx.x < 32) {
#pragma unroll
        for (int k = 0; k < K; ++k) {
            A s = lane < nw ? sh[k][lane] : A(0);
            s = warp_sum_red(s);
            if (lane == 0) part[slot * kRedParts + k] = (double)s;
        }
    }
    __threadfence();
    if (threadIdx.x == 0) {
        unsigned t = atomicAdd(counter, 1u);
        last = ((long)t == nslots - 1);
    }
    __syncthreads();
    return last;
}

// The same over the whole grid: one slot per CTA
template <typename A, int K>
__device__ bool red_block_partials(A (&v)[K], double *part, unsigned *counter) {
    return red_block_partials_at<A, K>(v, part, counter, (long)blockIdx.x, (long)gridDim.x);
}

// Fixed-order total of partial k over all CTAs (called by the last CTA, all
// of its threads)
template <typename A>
__device__ double red_total(const double *part, int k, int nblk) {
    __shared__ A sh[32];
    __shared__ A res;
    A s = A(0);
    for (int b = threadIdx.x; b < nblk; b += blockDim.x) s += (A)part[(long)b * kRedParts + k];
    s = warp_sum_red(s);
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const int nw = (int)((blockDim.x + 31) >> 5);
    if (lane == 0) sh[wid] = s;
    __syncthreads();
    if (threadIdx.x < 32) {
        A t = lane < nw ? sh[lane] : A(0);
        t = warp_sum_red(t);
        if (lane == 0) res = t;
    }
    __syncthreads();
    const double out = (double)res;
    __syncthreads();
    return out;
}

}  // namespace lc
