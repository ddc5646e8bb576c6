// Deterministic device reductions: per-block partials in a fixed thread
// order, then the last block to finish sums the partials by block index.
#pragma once

#include <cuda_runtime.h>

namespace fvmb {

constexpr int kRedBlocks = 296;   // 2 x 148 SMs
constexpr int kRedThreads = 256;

static __device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    return v;
}

// block-wide sum of v; valid in thread 0
static __device__ __forceinline__ double block_sum(double v) {
    __shared__ double red[32];
    v = warp_sum(v);
    __syncthreads();
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
    __syncthreads();
    double t = 0.0;
    if (threadIdx.x < 32) {
        t = threadIdx.x < (blockDim.x >> 5) ? red[threadIdx.x] : 0.0;
        t = warp_sum(t);
    }
    return t;
}

// every block calls this after writing partial[blockIdx.x * nv + v]; the
// last block to arrive writes out[v] = sum_b partial[b * nv + v] and
// re-arms the counter.  One warp per value: lane l sums blocks l, l+32, ...
// in order, then a fixed shuffle tree combines the lanes, so the result
// does not depend on which block finished last.
static __device__ __forceinline__ void last_block_reduce(double* partial, int nv,
                                                         unsigned* counter, double* out) {
    __shared__ bool last;
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) {
        unsigned t = atomicAdd(counter, 1u);
        last = (t == gridDim.x - 1);
    }
    __syncthreads();
    if (!last) return;
    __threadfence();
    // partials of the other blocks are read through L2 (ld.cg), a lane
    // keeping 8 of them in flight; summed in ascending block order per lane
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
    const int nblk = (int)gridDim.x;
    for (int v = warp; v < nv; v += nw) {
        double s = 0.0;
        for (int b0 = 0; b0 < nblk; b0 += 32 * 8) {
            double x[8];
#pragma unroll
            for (int i = 0; i < 8; ++i) {
                const int b = b0 + lane + 32 * i;
                x[i] = b < nblk ? __ldcg(partial + (size_t)b * nv + v) : 0.0;
            }
#pragma unroll
            for (int i = 0; i < 8; ++i) s += x[i];
        }
        s = warp_sum(s);
        if (lane == 0) out[v] = s;
    }
    __syncthreads();
    if (threadIdx.x == 0) *counter = 0u;
}

} // namespace fvmb
