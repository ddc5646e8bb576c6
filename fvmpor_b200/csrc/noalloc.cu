// fvm_wrms_noalloc: the WRMS norm of fvm_wrms without any device
// allocation, for callers that cannot call cudaMalloc -- for example a host
// integrator that owns all device memory through its own pool and calls the
// norm from inside its step loop, where a library allocation would
// synchronise the device or is not permitted at all.
//
// The reduction's scratch (one partial sum per block and the completion
// counter of the last-block reduction) lives in a file-scope __device__
// array of fixed size, so the largest vector is bounded: one block reduces
// kNoAllocChunk elements, and at most kNoAllocBlocks blocks fit the scratch.
#include "ctx.cuh"
#include "reduce.cuh"

#include <mutex>

namespace fvmb {

constexpr int kNoAllocBlocks = 4096;   // partial sums held in the static scratch
constexpr int kNoAllocThreads = 256;
constexpr int kNoAllocChunk = 2048;    // elements per block (8 per thread)
constexpr long kNoAllocMaxN = (long)kNoAllocBlocks * kNoAllocChunk;   // 8,388,608

// [0, kNoAllocBlocks): per-block partial sums; [kNoAllocBlocks]: counter;
// [kNoAllocBlocks + 8]: the finished sum.  4,128 doubles (33,024 bytes),
// which every GPU that loads the library holds until exit.
static __device__ __align__(256) double g_noalloc_scratch[kNoAllocBlocks + 32];

// per-block sums of (x w)^2 into scratch[block]; the last block to finish
// adds them in block order into scratch[kNoAllocBlocks + 8]
__global__ void k_wrms_noalloc(long n, const double* __restrict__ x, const double* __restrict__ w,
                               double* scratch) {
    double s = 0.0;
    long base = (long)blockIdx.x * kNoAllocChunk;
    long end = min(n, base + (long)kNoAllocChunk);
    for (long k = base + threadIdx.x; k < end; k += blockDim.x) {
        double v = w ? x[k] * w[k] : x[k];
        s += v * v;
    }
    double t = block_sum(s);
    if (threadIdx.x == 0) scratch[blockIdx.x] = t;
    unsigned* counter = reinterpret_cast<unsigned*>(scratch + kNoAllocBlocks);
    last_block_reduce(scratch, 1, counter, scratch + kNoAllocBlocks + 8);
}

__global__ void k_wrms_noalloc_finish(long n, const double* scratch, double* __restrict__ result) {
    *result = sqrt(scratch[kNoAllocBlocks + 8] / (double)n);
}

// per-device address of the static scratch, looked up once per device and
// kept for the life of the process (a cudaDeviceReset may reload the module
// elsewhere; the header tells callers not to call again after one)
static std::mutex g_noalloc_mutex;
static double* g_noalloc_ptr[64] = {};

static double* noalloc_scratch(int device) {
    if (device < 0 || device >= 64) throw Error("fvm_wrms_noalloc: device index out of range");
    std::lock_guard<std::mutex> lock(g_noalloc_mutex);
    if (!g_noalloc_ptr[device]) {
        void* ptr = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&ptr, g_noalloc_scratch);
        if (e != cudaSuccess || !ptr)
            throw Error(std::string("fvm_wrms_noalloc: cudaGetSymbolAddress failed: ") + cudaGetErrorString(e), -2);
        g_noalloc_ptr[device] = static_cast<double*>(ptr);
    }
    return g_noalloc_ptr[device];
}

} // namespace fvmb

using namespace fvmb;

extern "C" long fvm_wrms_noalloc_max_n(void) { return kNoAllocMaxN; }

extern "C" int fvm_wrms_noalloc(const double* x, const double* ewt, long n, double* result, void* stream) {
    try {
        if (!x || !result) throw Error("fvm_wrms_noalloc: null argument");
        if (n <= 0) throw Error("fvm_wrms_noalloc: n must be positive");
        if (n > kNoAllocMaxN)
            throw Error("fvm_wrms_noalloc: n = " + std::to_string(n) + " exceeds the static scratch limit of " +
                        std::to_string(kNoAllocMaxN) + " elements");
        int dev = 0;
        FVM_CUDA(cudaGetDevice(&dev));
        double* scratch = noalloc_scratch(dev);
        cudaStream_t s = static_cast<cudaStream_t>(stream);
        // the counter must start at zero whatever the previous call left
        FVM_CUDA(cudaMemsetAsync(scratch + kNoAllocBlocks, 0, 8 * sizeof(double), s));
        int blocks = (int)((n + kNoAllocChunk - 1) / kNoAllocChunk);
        k_wrms_noalloc<<<blocks, kNoAllocThreads, 0, s>>>(n, x, ewt, scratch);
        k_wrms_noalloc_finish<<<1, 1, 0, s>>>(n, scratch, result);
        FVM_CUDA(cudaGetLastError());
        return 0;
    } catch (const Error& ex) {
        set_error(ex.what());
        return ex.code;
    } catch (const std::exception& ex) {
        set_error(ex.what());
        return -1;
    }
}
