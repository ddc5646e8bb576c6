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
// last block to arrive writes out[v] = sum_b partial[b * nv + v] in block
// order and re-arms the counter
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
    for (int v = threadIdx.x; v < nv; v += blockDim.x) {
        double s = 0.0;
        for (int b = 0; b < (int)gridDim.x; ++b) s += ((volatile double*)partial)[(size_t)b * nv + v];
        out[v] = s;
    }
    __syncthreads();
    if (threadIdx.x == 0) *counter = 0u;
}

} // namespace fvmb
