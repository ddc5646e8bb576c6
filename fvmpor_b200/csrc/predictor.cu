// Learned Newton initial iterate: a per-node MLP 8 -> 64 -> 64 -> 64 -> 1
// with GELU, BF16 weights and activations, FP32 accumulation on the sm_100a
// tensor cores (tcgen05.mma, accumulators in TMEM), trained on the device
// with hand-written forward and backward kernels and Adam.
//
// The reference has no counterpart (its Newton iterate is IDAS's BDF
// predictor).  The network's iterate is judged by the FP64 nonlinear
// residual: on every step where it is tried, y_pred + w * MLP(x) is kept
// only if its residual norm is below the BDF predictor's, otherwise the
// plain BDF extrapolation is used.
//
// Tile shape: one CTA of 128 threads owns a tile of 128 nodes; thread t
// owns row t, which is TMEM lane t (warp w reads lanes 32w..32w+31).  One
// elected thread issues the MMAs (M = 128, N = 64, K = 16 per instruction;
// the first layer pads its 8 inputs to K = 16), commits them to an
// mbarrier, and all threads read the FP32 accumulators back with
// tcgen05.ld for the bias + GELU epilogue, which writes the next layer's
// BF16 operand straight into shared memory.  Backward: dA = dZ W runs on
// the tensor cores (the forward weight tile read as an MN-major operand);
// the rank-128 weight-gradient updates dW += dZ^T A run on the CUDA cores
// in FP32 and are reduced across CTAs in a fixed order.
#include "predictor.cuh"
#include "krylov.cuh"
#include "reduce.cuh"
#include "tc05.cuh"

#include <cuda_bf16.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

namespace fvmb {

using namespace tc05;

constexpr int kTile = 128;
// bf16 operand layouts inside the packed weight buffer (in 16-bit units)
constexpr int kW1s = 0;                       // 64 x 16
constexpr int kW2s = kW1s + kMlpH * kMlpK0;   // 64 x 64
constexpr int kW3s = kW2s + kMlpH * kMlpH;    // 64 x 64
constexpr int kWsz = kW3s + kMlpH * kMlpH;    // 9216 halves = 18432 B

constexpr uint32_t kIdescFwd = idesc_bf16_f32(128, 64, false, false);
constexpr uint32_t kIdescBwd = idesc_bf16_f32(128, 64, false, true);

struct Predictor {
    DevBuf<float> p;          // [kNParam] FP32 master parameters
    DevBuf<float> m, v;       // Adam moments
    DevBuf<unsigned short> wl;
    DevBuf<float> partial;    // per-CTA gradients [nblk][kNTrain + 1]
    DevBuf<float> gsum;       // [kNTrain + 1] (last = loss sum)
    DevBuf<float> X, out;     // features / network output for all nodes
    DevBuf<double> yg, ypg, Fg;
    DevBuf<int> err;
    long adam_t = 0;
    bool ready = false;
    int train_blocks = 0;
};

__device__ __forceinline__ float gelu(float x) { return 0.5f * x * (1.0f + erff(x * 0.70710678118654752f)); }
__device__ __forceinline__ float gelu_grad(float x) {
    // d/dx [x Phi(x)] = Phi(x) + x phi(x)
    float cdf = 0.5f * (1.0f + erff(x * 0.70710678118654752f));
    float pdf = 0.39894228040143268f * __expf(-0.5f * x * x);
    return cdf + x * pdf;
}

__device__ __forceinline__ unsigned short bf16_bits(float x) {
    __nv_bfloat16 b = __float2bfloat16_rn(x);
    return *reinterpret_cast<unsigned short*>(&b);
}
__device__ __forceinline__ float bf16_val(unsigned short u) {
    return __bfloat162float(*reinterpret_cast<__nv_bfloat16*>(&u));
}

// FP32 masters -> BF16 operand tiles
__global__ void k_pack_weights(const float* __restrict__ P, unsigned short* __restrict__ wl) {
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t < kMlpH * kMlpK0) {
        int n = t / kMlpK0, k = t % kMlpK0;
        float v = k < kMlpIn ? P[kOffW1 + n * kMlpIn + k] : 0.0f;
        wl[kW1s + il_off(n, k, kMlpK0) / 2] = bf16_bits(v);
    }
    if (t < kMlpH * kMlpH) {
        int n = t / kMlpH, k = t % kMlpH;
        wl[kW2s + il_off(n, k, kMlpH) / 2] = bf16_bits(P[kOffW2 + n * kMlpH + k]);
        wl[kW3s + il_off(n, k, kMlpH) / 2] = bf16_bits(P[kOffW3 + n * kMlpH + k]);
    }
}

// shared-memory carve-up common to the forward and training kernels
struct MlpSmem {
    unsigned short* W;   // packed weight tiles
    unsigned short* A0;  // 128 x 16
    unsigned short* A1;  // 128 x 64
    unsigned short* A2;  // 128 x 64 (training)
    unsigned short* dZ;  // 128 x 64 (training)
    float* prm;          // b1, b2, b3, w4, b4, mu, sd (FP32 copies)
    float* red;          // [4][64 + 1] per-warp reduction scratch (training)
    float* grad;         // [kNTrain + 1] CTA gradient accumulators (training)
    uint64_t* bar;
    uint32_t* tbase;
};

constexpr int kPrmB1 = 0, kPrmB2 = 64, kPrmB3 = 128, kPrmW4 = 192, kPrmB4 = 256, kPrmMu = 260, kPrmSd = 268,
              kPrmN = 276;

__host__ __device__ constexpr size_t mlp_smem_bytes(bool train) {
    return (size_t)kWsz * 2 + 128 * 16 * 2 + 128 * 64 * 2 + (train ? 2 * 128 * 64 * 2 : 0) + kPrmN * 4 +
           (train ? (4 * 65 + kNTrain + 1) * 4 : 0) + 64;
}

__device__ MlpSmem carve(unsigned char* base, bool train) {
    MlpSmem s;
    unsigned char* p = base;
    s.W = (unsigned short*)p; p += kWsz * 2;
    s.A0 = (unsigned short*)p; p += 128 * 16 * 2;
    s.A1 = (unsigned short*)p; p += 128 * 64 * 2;
    if (train) {
        s.A2 = (unsigned short*)p; p += 128 * 64 * 2;
        s.dZ = (unsigned short*)p; p += 128 * 64 * 2;
    } else {
        s.A2 = s.A1;
        s.dZ = nullptr;
    }
    s.prm = (float*)p; p += kPrmN * 4;
    if (train) {
        s.red = (float*)p; p += 4 * 65 * 4;
        s.grad = (float*)p; p += (kNTrain + 1) * 4;
    } else {
        s.red = nullptr;
        s.grad = nullptr;
    }
    p = (unsigned char*)(((uintptr_t)p + 15) & ~(uintptr_t)15);
    s.bar = (uint64_t*)p; p += 16;
    s.tbase = (uint32_t*)p;
    return s;
}

__device__ void load_params(const MlpSmem& s, const float* __restrict__ P, const unsigned short* __restrict__ wl) {
    const uint4* src = reinterpret_cast<const uint4*>(wl);
    uint4* dst = reinterpret_cast<uint4*>(s.W);
    for (int i = threadIdx.x; i < kWsz * 2 / 16; i += blockDim.x) dst[i] = src[i];
    for (int i = threadIdx.x; i < 64; i += blockDim.x) {
        s.prm[kPrmB1 + i] = P[kOffB1 + i];
        s.prm[kPrmB2 + i] = P[kOffB2 + i];
        s.prm[kPrmB3 + i] = P[kOffB3 + i];
        s.prm[kPrmW4 + i] = P[kOffW4 + i];
    }
    if (threadIdx.x == 0) s.prm[kPrmB4] = P[kOffB4];
    if (threadIdx.x < 8) {
        s.prm[kPrmMu + threadIdx.x] = P[kOffMu + threadIdx.x];
        float sd = P[kOffSd + threadIdx.x];
        s.prm[kPrmSd + threadIdx.x] = sd > 0.0f ? sd : 1.0f;
    }
}

// normalised features of one row into the layer-1 operand
__device__ void write_features(const MlpSmem& s, const float* __restrict__ X, long row, long n) {
    float f[8];
    if (row < n) {
        const float4* x4 = reinterpret_cast<const float4*>(X + row * 8);
        float4 a = x4[0], b = x4[1];
        f[0] = a.x; f[1] = a.y; f[2] = a.z; f[3] = a.w; f[4] = b.x; f[5] = b.y; f[6] = b.z; f[7] = b.w;
    } else {
#pragma unroll
        for (int k = 0; k < 8; ++k) f[k] = 0.0f;
    }
    unsigned short h[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) {
        float v = row < n ? (f[k] - s.prm[kPrmMu + k]) / s.prm[kPrmSd + k] : 0.0f;
        h[k] = bf16_bits(v);
    }
    int r = threadIdx.x;
    uint4 lo = make_uint4(h[0] | (h[1] << 16), h[2] | (h[3] << 16), h[4] | (h[5] << 16), h[6] | (h[7] << 16));
    *reinterpret_cast<uint4*>((unsigned char*)s.A0 + il_off(r, 0, 16)) = lo;
    *reinterpret_cast<uint4*>((unsigned char*)s.A0 + il_off(r, 8, 16)) = make_uint4(0, 0, 0, 0);
}

// bias + GELU epilogue of a hidden layer: TMEM columns [col, col+64) of this
// thread's lane -> BF16 row of `dst`; optionally keeps the pre-activation
__device__ void epilogue_hidden(uint32_t tmem, int col, const float* bias, unsigned short* dst) {
    int w = threadIdx.x >> 5, r = threadIdx.x;
#pragma unroll
    for (int c = 0; c < 4; ++c) {
        float v[16];
        tmem_ld16(tmem + ((uint32_t)(w * 32) << 16) + col + c * 16, v);
#pragma unroll
        for (int g = 0; g < 2; ++g) {
            unsigned short h[8];
#pragma unroll
            for (int j = 0; j < 8; ++j) h[j] = bf16_bits(gelu(v[g * 8 + j] + bias[c * 16 + g * 8 + j]));
            *reinterpret_cast<uint4*>((unsigned char*)dst + il_off(r, c * 16 + g * 8, 64)) =
                make_uint4(h[0] | (h[1] << 16), h[2] | (h[3] << 16), h[4] | (h[5] << 16), h[6] | (h[7] << 16));
        }
    }
}

// one layer of MMAs: D(tmem col) = A (128 x K, K-major) x W (64 x K)^T
__device__ void issue_layer(uint32_t dtm, const unsigned short* A, const unsigned short* W, int K) {
    uint32_t a = smem_u32(A), b = smem_u32(W);
    for (int s = 0; s < K / 16; ++s)
        mma_bf16(dtm, smem_desc(a + s * 256, 128, K * 16), smem_desc(b + s * 256, 128, K * 16), kIdescFwd, s > 0);
}

struct Phase {
    uint32_t ph = 0;
};

// waits for the MMAs committed by thread 0; false (and the error flag) on timeout
__device__ bool sync_mma(const MlpSmem& s, Phase& ph, int* err) {
    bool ok = mbar_wait(s.bar, ph.ph & 1u);
    if (!ok) {
        atomicExch(err, 1);
        ok = mbar_wait(s.bar, ph.ph & 1u);   // give in-flight work a second bounded chance
    }
    ph.ph++;
    fence_after_sync();
    // every thread leaves with the same verdict, so the tile loop stays uniform
    return __syncthreads_and(ok ? 1 : 0) != 0;
}

__device__ void commit_from_thread0(const MlpSmem& s) {
    if (threadIdx.x == 0) mma_commit(s.bar);
}

// ------------------------------------------------------------------ inference
__global__ void __launch_bounds__(128) k_mlp_forward(const float* __restrict__ X, long n,
                                                     const float* __restrict__ P,
                                                     const unsigned short* __restrict__ wl,
                                                     float* __restrict__ out, int* err) {
    extern __shared__ __align__(128) unsigned char smem[];
    MlpSmem s = carve(smem, false);
    load_params(s, P, wl);
    if (threadIdx.x < 32) tmem_alloc(s.tbase, 64);
    if (threadIdx.x == 0) {
        mbar_init(s.bar, 1);
        asm volatile("fence.mbarrier_init.release.cluster;");
    }
    fence_before_sync();
    __syncthreads();
    fence_after_sync();
    const uint32_t tmem = *s.tbase;
    Phase ph;
    bool ok = true;
    const long ntiles = (n + kTile - 1) / kTile;
    for (long tile = blockIdx.x; tile < ntiles && ok; tile += gridDim.x) {
        long row = tile * kTile + threadIdx.x;
        write_features(s, X, row, n);
        fence_smem_async();
        __syncthreads();
        if (threadIdx.x == 0) {
            fence_after_sync();
            issue_layer(tmem, s.A0, s.W + kW1s, 16);
        }
        commit_from_thread0(s);
        ok = sync_mma(s, ph, err);
        epilogue_hidden(tmem, 0, s.prm + kPrmB1, s.A1);
        fence_before_sync();
        fence_smem_async();
        __syncthreads();
        if (threadIdx.x == 0) {
            fence_after_sync();
            issue_layer(tmem, s.A1, s.W + kW2s, 64);
        }
        commit_from_thread0(s);
        ok = sync_mma(s, ph, err) && ok;
        epilogue_hidden(tmem, 0, s.prm + kPrmB2, s.A1);
        fence_before_sync();
        fence_smem_async();
        __syncthreads();
        if (threadIdx.x == 0) {
            fence_after_sync();
            issue_layer(tmem, s.A1, s.W + kW3s, 64);
        }
        commit_from_thread0(s);
        ok = sync_mma(s, ph, err) && ok;
        // output layer on the CUDA cores: y = gelu(z3 + b3) . w4 + b4
        int w = threadIdx.x >> 5;
        float acc = s.prm[kPrmB4];
#pragma unroll
        for (int c = 0; c < 4; ++c) {
            float v[16];
            tmem_ld16(tmem + ((uint32_t)(w * 32) << 16) + c * 16, v);
#pragma unroll
            for (int j = 0; j < 16; ++j) acc += gelu(v[j] + s.prm[kPrmB3 + c * 16 + j]) * s.prm[kPrmW4 + c * 16 + j];
        }
        if (row < n) out[row] = acc;
        fence_before_sync();
        __syncthreads();
    }
    __syncthreads();
    if (threadIdx.x < 32) {
        fence_after_sync();
        tmem_dealloc(tmem, 64);
    }
}

// ------------------------------------------------------------------ training
// per-row value -> per-CTA sum of 128 rows in fixed order, accumulated into
// grad[idx + j] for j < cols (each row contributes v[j])
__device__ void reduce_rows_add(const MlpSmem& s, const float* v, int cols, float* gdst) {
    int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    for (int j = 0; j < cols; ++j) {
        float x = v[j];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
        if (lane == 0) s.red[w * 65 + j] = x;
    }
    __syncthreads();
    for (int j = threadIdx.x; j < cols; j += blockDim.x)
        gdst[j] += ((s.red[j] + s.red[65 + j]) + s.red[130 + j]) + s.red[195 + j];
    __syncthreads();
}

// dW[o][i] += sum_r dZ[r][o] * A[r][i] for o < 64, i < K (FP32, CUDA cores);
// thread t owns o = t / 2 and half of the i range
__device__ void weight_grad(const MlpSmem& s, const unsigned short* A, int K, int Kstore, float* gW) {
    int o = threadIdx.x >> 1;
    int i0 = (threadIdx.x & 1) * (K / 2), ni = K / 2;
    float acc[32];
#pragma unroll
    for (int j = 0; j < 32; ++j) acc[j] = 0.0f;
    for (int r = 0; r < 128; ++r) {
        float dz = bf16_val(s.dZ[il_off(r, o, 64) / 2]);
        for (int j = 0; j < ni; ++j) acc[j] += dz * bf16_val(A[il_off(r, i0 + j, Kstore) / 2]);
    }
    for (int j = 0; j < ni; ++j) gW[o * K + i0 + j] += acc[j];
}

// backward epilogue: dz = dA(tmem col) * gelu'(z) with z = D(zcol) + bias;
// writes BF16 dZ row and returns dz in v (64 values)
__device__ void backward_dz(uint32_t tmem, int dacol, int zcol, const float* bias, unsigned short* dZ, float* dz,
                            const float* dh_in) {
    int w = threadIdx.x >> 5, r = threadIdx.x;
#pragma unroll
    for (int c = 0; c < 4; ++c) {
        float z[16], d[16];
        tmem_ld16(tmem + ((uint32_t)(w * 32) << 16) + zcol + c * 16, z);
        if (dh_in) {
#pragma unroll
            for (int j = 0; j < 16; ++j) d[j] = dh_in[c * 16 + j];
        } else {
            tmem_ld16(tmem + ((uint32_t)(w * 32) << 16) + dacol + c * 16, d);
        }
#pragma unroll
        for (int j = 0; j < 16; ++j) dz[c * 16 + j] = d[j] * gelu_grad(z[j] + bias[c * 16 + j]);
    }
#pragma unroll
    for (int g = 0; g < 8; ++g) {
        unsigned short h[8];
#pragma unroll
        for (int j = 0; j < 8; ++j) h[j] = bf16_bits(dz[g * 8 + j]);
        *reinterpret_cast<uint4*>((unsigned char*)dZ + il_off(r, g * 8, 64)) =
            make_uint4(h[0] | (h[1] << 16), h[2] | (h[3] << 16), h[4] | (h[5] << 16), h[6] | (h[7] << 16));
    }
}

// dA(tmem dcol) = dZ (128 x 64, K-major) x W (64 x 64 weight tile read as the
// MN-major operand of W^T)
__device__ void issue_backward(uint32_t dtm, const unsigned short* dZ, const unsigned short* W) {
    uint32_t a = smem_u32(dZ), b = smem_u32(W);
    for (int s2 = 0; s2 < 4; ++s2)
        mma_bf16(dtm, smem_desc(a + s2 * 256, 128, 1024), smem_desc(b + s2 * 2048, 1024, 128), kIdescBwd, s2 > 0);
}

// one pass over rows [begin, end) of (X, Y): loss = mean (mlp(x) - y)^2;
// writes this CTA's gradient (scaled by 1/count) and loss sum to partial
__global__ void __launch_bounds__(128, 1) k_mlp_train(const float* __restrict__ X, const float* __restrict__ Y,
                                                      long begin, long end, long tiles_per_cta,
                                                      const float* __restrict__ P,
                                                      const unsigned short* __restrict__ wl,
                                                      float* __restrict__ partial, int* err) {
    extern __shared__ __align__(128) unsigned char smem[];
    MlpSmem s = carve(smem, true);
    load_params(s, P, wl);
    for (int j = threadIdx.x; j < kNTrain + 1; j += blockDim.x) s.grad[j] = 0.0f;
    if (threadIdx.x < 32) tmem_alloc(s.tbase, 256);
    if (threadIdx.x == 0) {
        mbar_init(s.bar, 1);
        asm volatile("fence.mbarrier_init.release.cluster;");
    }
    fence_before_sync();
    __syncthreads();
    fence_after_sync();
    const uint32_t tmem = *s.tbase;
    const uint32_t D1 = tmem, D2 = tmem + 64, D3 = tmem + 128, DA = tmem + 192;
    const float inv_count = 1.0f / (float)max(1l, end - begin);
    Phase ph;
    bool ok = true;
    const int w = threadIdx.x >> 5;
    for (long t = 0; t < tiles_per_cta && ok; ++t) {
        long tile = (long)blockIdx.x * tiles_per_cta + t;
        long row = begin + tile * kTile + threadIdx.x;
        bool valid = row < end;
        // ---- forward
        write_features(s, X, row, end);
        fence_smem_async();
        __syncthreads();
        if (threadIdx.x == 0) { fence_after_sync(); issue_layer(D1, s.A0, s.W + kW1s, 16); }
        commit_from_thread0(s);
        ok = sync_mma(s, ph, err) && ok;
        epilogue_hidden(D1, 0, s.prm + kPrmB1, s.A1);
        fence_before_sync(); fence_smem_async(); __syncthreads();
        if (threadIdx.x == 0) { fence_after_sync(); issue_layer(D2, s.A1, s.W + kW2s, 64); }
        commit_from_thread0(s);
        ok = sync_mma(s, ph, err) && ok;
        epilogue_hidden(D2, 0, s.prm + kPrmB2, s.A2);
        fence_before_sync(); fence_smem_async(); __syncthreads();
        if (threadIdx.x == 0) { fence_after_sync(); issue_layer(D3, s.A2, s.W + kW3s, 64); }
        commit_from_thread0(s);
        ok = sync_mma(s, ph, err) && ok;
        float h3[64];
        float outv = s.prm[kPrmB4];
#pragma unroll
        for (int c = 0; c < 4; ++c) {
            float v[16];
            tmem_ld16(D3 + ((uint32_t)(w * 32) << 16) + c * 16, v);
#pragma unroll
            for (int j = 0; j < 16; ++j) {
                h3[c * 16 + j] = gelu(v[j] + s.prm[kPrmB3 + c * 16 + j]);
                outv += h3[c * 16 + j] * s.prm[kPrmW4 + c * 16 + j];
            }
        }
        float e = valid ? outv - Y[row] : 0.0f;
        float dout = 2.0f * e * inv_count;
        // ---- output layer gradients
        float tmp[65];
#pragma unroll
        for (int j = 0; j < 64; ++j) tmp[j] = dout * h3[j];
        tmp[64] = dout;
        reduce_rows_add(s, tmp, 65, s.grad + kOffW4);   // w4 then b4 (contiguous)
        {
            float l = e * e;
            reduce_rows_add(s, &l, 1, s.grad + kNTrain);
        }
        // ---- layer 3
        float dh[64], dz[64];
#pragma unroll
        for (int j = 0; j < 64; ++j) dh[j] = dout * s.prm[kPrmW4 + j];
        backward_dz(tmem, 0, 128, s.prm + kPrmB3, s.dZ, dz, dh);
        fence_before_sync(); fence_smem_async(); __syncthreads();
        if (threadIdx.x == 0) { fence_after_sync(); issue_backward(DA, s.dZ, s.W + kW3s); }
        commit_from_thread0(s);
        reduce_rows_add(s, dz, 64, s.grad + kOffB3);
        weight_grad(s, s.A2, 64, 64, s.grad + kOffW3);
        ok = sync_mma(s, ph, err) && ok;
        __syncthreads();
        // ---- layer 2
        backward_dz(tmem, 192, 64, s.prm + kPrmB2, s.dZ, dz, nullptr);
        fence_before_sync(); fence_smem_async(); __syncthreads();
        if (threadIdx.x == 0) { fence_after_sync(); issue_backward(DA, s.dZ, s.W + kW2s); }
        commit_from_thread0(s);
        reduce_rows_add(s, dz, 64, s.grad + kOffB2);
        weight_grad(s, s.A1, 64, 64, s.grad + kOffW2);
        ok = sync_mma(s, ph, err) && ok;
        __syncthreads();
        // ---- layer 1
        backward_dz(tmem, 192, 0, s.prm + kPrmB1, s.dZ, dz, nullptr);
        fence_before_sync(); fence_smem_async(); __syncthreads();
        reduce_rows_add(s, dz, 64, s.grad + kOffB1);
        weight_grad(s, s.A0, 8, 16, s.grad + kOffW1);
        __syncthreads();
    }
    for (int j = threadIdx.x; j < kNTrain + 1; j += blockDim.x) partial[(size_t)blockIdx.x * (kNTrain + 1) + j] = s.grad[j];
    fence_before_sync();
    __syncthreads();
    if (threadIdx.x < 32) {
        fence_after_sync();
        tmem_dealloc(tmem, 256);
    }
}

// sums the per-CTA gradients in CTA order
__global__ void k_grad_reduce(const float* __restrict__ partial, int nblk, float* __restrict__ g) {
    int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j > kNTrain) return;
    float s = 0.0f;
    for (int b = 0; b < nblk; ++b) s += partial[(size_t)b * (kNTrain + 1) + j];
    g[j] = s;
}

__global__ void k_adam(float* __restrict__ P, float* __restrict__ m, float* __restrict__ v,
                       const float* __restrict__ g, float lr, float b1, float b2, float eps, float bc1,
                       float bc2) {
    int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= kNTrain) return;
    float gj = g[j];
    float mj = b1 * m[j] + (1.0f - b1) * gj;
    float vj = b2 * v[j] + (1.0f - b2) * gj * gj;
    m[j] = mj;
    v[j] = vj;
    P[j] -= lr * (mj / bc1) / (sqrtf(vj / bc2) + eps);
}

// ------------------------------------------------------------------ features
__global__ void k_features(int N, const double* __restrict__ h_n, const double* __restrict__ h_prev,
                           const double* __restrict__ ypred, float ldt, const float* __restrict__ statf,
                           float* __restrict__ X) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N) return;
    double h = h_n[i];
    float4 a = make_float4((float)h, (float)(h - h_prev[i]), (float)(ypred[i] - h), ldt);
    float4 b = make_float4(statf[i], statf[(size_t)N + i], statf[(size_t)2 * N + i], 0.0f);
    float4* x4 = reinterpret_cast<float4*>(X + (size_t)i * 8);
    x4[0] = a;
    x4[1] = b;
}

// guess = y_pred + w * mlp on free rows; y' follows the corrector relation
__global__ void k_apply_guess(int N, const float* __restrict__ out, const double* __restrict__ ypred,
                              const double* __restrict__ yppred, const double* __restrict__ h_n,
                              const unsigned char* __restrict__ ntype, double rtol, double atol, double cj,
                              double* __restrict__ yg, double* __restrict__ ypg) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N) return;
    double d = ntype[i] ? 0.0 : (rtol * fabs(h_n[i]) + atol) * (double)out[i];
    yg[i] = ypred[i] + d;
    ypg[i] = yppred[i] + cj * d;
}

// y = y_pred + a (y_guess - y_pred), y' likewise; e = y - y_pred
__global__ void k_take_guess(int N, double a, const double* __restrict__ yg, const double* __restrict__ ypg,
                             const double* __restrict__ ypred, const double* __restrict__ yppred,
                             double* __restrict__ y, double* __restrict__ yp, double* __restrict__ e) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N) return;
    const double d = a == 1.0 ? yg[i] - ypred[i] : a * (yg[i] - ypred[i]);
    y[i] = a == 1.0 ? yg[i] : ypred[i] + d;
    yp[i] = a == 1.0 ? ypg[i] : yppred[i] + a * (ypg[i] - yppred[i]);
    e[i] = d;
}

// out = (F0.F0, F0.F1, F1.F1), fixed-order reduction
__global__ void k_dot3(int N, const double* __restrict__ F0, const double* __restrict__ F1, double* partial,
                       unsigned* counter, double* out) {
    double s0 = 0.0, s1 = 0.0, s2 = 0.0;
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < N; k += gridDim.x * blockDim.x) {
        const double a = F0[k], b = F1[k];
        s0 += a * a;
        s1 += a * b;
        s2 += b * b;
    }
    __shared__ double red[3][32];
    s0 = warp_sum(s0);
    s1 = warp_sum(s1);
    s2 = warp_sum(s2);
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
    if (lane == 0) { red[0][w] = s0; red[1][w] = s1; red[2][w] = s2; }
    __syncthreads();
    if (w < 3) {
        double t = lane < nw ? red[w][lane] : 0.0;
        t = warp_sum(t);
        if (lane == 0) partial[(size_t)blockIdx.x * 3 + w] = t;
    }
    last_block_reduce(partial, 3, counter, out);
}

__global__ void k_record(int N, int stride, int offset, const float* __restrict__ Xall,
                         const double* __restrict__ y_new, const double* __restrict__ ypred,
                         const double* __restrict__ h_n, const unsigned char* __restrict__ ntype, double rtol,
                         double atol, long base, long cap, float* __restrict__ X, float* __restrict__ Y) {
    long q = blockIdx.x * (long)blockDim.x + threadIdx.x;
    long i = offset + q * stride;
    if (i >= N) return;
    long slot = base + q;
    if (slot >= cap) return;
    for (int k = 0; k < 8; ++k) X[slot * 8 + k] = Xall[i * 8 + k];
    double w = rtol * fabs(h_n[i]) + atol;
    Y[slot] = ntype[i] ? 0.0f : (float)((y_new[i] - ypred[i]) / w);
}

// ------------------------------------------------------------------ host side
Predictor* predictor_get(fvm_ctx* c) {
    if (!c->pred) {
        Predictor* p = new Predictor();
        p->p.alloc(kNParam);
        p->m.alloc(kNTrain);
        p->v.alloc(kNTrain);
        p->wl.alloc(kWsz);
        p->gsum.alloc(kNTrain + 1);
        p->err.alloc(1);
        p->err.zero(c->stream);
        p->m.zero(c->stream);
        p->v.zero(c->stream);
        p->X.alloc((size_t)c->N * 8);
        p->out.alloc(c->N);
        p->yg.alloc(c->N);
        p->ypg.alloc(c->N);
        p->Fg.alloc(c->N);
        c->pred = p;
        raise_smem_limit(k_mlp_forward, mlp_smem_bytes(false));
        raise_smem_limit(k_mlp_train, mlp_smem_bytes(true));
    }
    return c->pred;
}

Predictor* predictor_of(fvm_ctx* c) { return (c->pred && c->pred->ready) ? c->pred : nullptr; }
bool predictor_ready(Predictor* p) { return p && p->ready; }

static void pack(fvm_ctx* c, Predictor* p) {
    fvm_launch(c, k_pack_weights, (kMlpH * kMlpH + 255) / 256, 256, 0, c->stream, p->p.p, p->wl.p);
}

void predictor_features(fvm_ctx* c, const double* h_n, const double* h_prev, const double* ypred, double dt,
                        float* X) {
    fvm_launch(c, k_features, grid_for(c->N, 256), 256, 0, c->stream, c->N, h_n, h_prev, ypred,
               (float)std::log10(std::max(dt, 1e-30)), c->statf.p, X);
}

void predictor_forward(fvm_ctx* c, Predictor* p, const float* X, int n, float* out) {
    long ntiles = ((long)n + kTile - 1) / kTile;
    int grid = (int)std::min<long>(ntiles, 148 * 4);
    if (grid < 1) return;
    fvm_launch(c, k_mlp_forward, grid, 128, mlp_smem_bytes(false), c->stream, X, (long)n, p->p.p, p->wl.p, out,
               p->err.p);
}

// squared residual-norm ratio below which the learned iterate is kept
constexpr double kGuessKeep = 0.25;

bool predictor_apply(fvm_ctx* c, Predictor* p, double rtol, double atol, double dt, double cj, const double* h_n,
                     const double* h_prev, const double* ypred, const double* yppred, double* y, double* yp,
                     double* e, double* F) {
    const int N = c->N;
    c->tm.begin(TM_PRED, c->stream);
    struct EndTimer {
        fvm_ctx* c;
        ~EndTimer() { c->tm.end(TM_PRED, c->stream); }
    } end_timer{c};
    c->tm.begin(TM_MLP, c->stream);
    predictor_features(c, h_n, h_prev, ypred, dt, p->X.p);
    predictor_forward(c, p, p->X.p, N, p->out.p);
    c->tm.end(TM_MLP, c->stream);
    fvm_launch(c, k_apply_guess, grid_for(N, 256), 256, 0, c->stream, N, p->out.p, ypred, yppred, h_n, c->ntype.p,
               rtol, atol, cj, p->yg.p, p->ypg.p);
    Perturb none;
    launch_residual(c, p->yg.p, p->ypg.p, none, nullptr, p->Fg.p);
    launch_residual(c, ypred, yppred, none, nullptr, F);
    // The residual is close to linear over one Newton correction, so along
    // y(a) = y_pred + a (y_guess - y_pred) its squared norm is the quadratic
    // through F0 = F(y_pred) and F1 = F(y_guess):
    //   |F(a)|^2 ~ A + 2a (B - A) + a^2 (A - 2B + C),  A = F0.F0, B = F0.F1, C = F1.F1.
    // Take its minimiser on [0, 1]; keep the BDF predictor when the learned
    // direction does not lower the residual.
    Krylov* K = krylov_scratch(c);
    fvm_launch(c, k_dot3, kRedBlocks, kRedThreads, 0, c->stream, N, F, p->Fg.p, K->partial.p, K->counter.p,
               K->res.p);
    FVM_CUDA(cudaMemcpyAsync(K->host, K->res.p, 3 * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    ctx_sync(c);
    const double A = K->host[0], B = K->host[1], Cc = K->host[2];
    const double curv = A - 2.0 * B + Cc;   // |F1 - F0|^2
    if (!std::isfinite(A) || !std::isfinite(Cc) || !(curv > 0.0)) return false;
    double a = (A - B) / curv;
    a = std::min(1.0, a);
    const double pred = A + 2.0 * a * (B - A) + a * a * curv;
    // A learned start that lowers the residual only a little leaves Newton
    // converging (within its tolerance) to a point biased toward the guess,
    // which inflates the BDF error estimate: on the 3D benchmark, accepting
    // guesses at a 2 % residual drop raised the step count by 16 %.  Keep
    // the guess only when it halves the residual norm.
    if (!(a > 0.05) || !(pred < kGuessKeep * A)) return false;
    fvm_launch(c, k_take_guess, grid_for(N, 256), 256, 0, c->stream, N, a, p->yg.p, p->ypg.p, ypred, yppred, y, yp,
               e);
    if (a == 1.0) FVM_CUDA(cudaMemcpyAsync(F, p->Fg.p, sizeof(double) * N, cudaMemcpyDeviceToDevice, c->stream));
    else launch_residual(c, y, yp, none, nullptr, F);
    return true;
}

void recorder_push(fvm_ctx* c, Recorder* r, const float* Xall, const double* y_new, const double* ypred,
                   const double* h_n, double rtol, double atol) {
    if (!r || r->count >= r->cap) return;
    int offset = (int)(r->step % r->stride);
    long q = (c->N - offset + r->stride - 1) / r->stride;
    q = std::min(q, r->cap - r->count);
    if (q > 0)
        fvm_launch(c, k_record, grid_for(q, 256), 256, 0, c->stream, c->N, r->stride, offset, Xall, y_new, ypred, h_n,
                   c->ntype.p, rtol, atol, r->count, r->cap, r->X, r->Y);
    r->count += q;
    r->step++;
}

static void train_pass(fvm_ctx* c, Predictor* p, const float* X, const float* Y, long begin, long end, int* nblk_out) {
    long ntiles = (end - begin + kTile - 1) / kTile;
    int nblk = (int)std::min<long>(ntiles, 148);
    long per = (ntiles + nblk - 1) / nblk;
    nblk = (int)((ntiles + per - 1) / per);
    if ((long)p->partial.n < (long)nblk * (kNTrain + 1)) p->partial.alloc((size_t)nblk * (kNTrain + 1));
    fvm_launch(c, k_mlp_train, nblk, 128, mlp_smem_bytes(true), c->stream, X, Y, begin, end, per, p->p.p, p->wl.p,
               p->partial.p, p->err.p);
    fvm_launch(c, k_grad_reduce, grid_for(kNTrain + 1, 256), 256, 0, c->stream, p->partial.p, nblk, p->gsum.p);
    *nblk_out = nblk;
}

static int check_err(fvm_ctx* c, Predictor* p) {
    int h = 0;
    FVM_CUDA(cudaMemcpyAsync(&h, p->err.p, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
    FVM_CUDA(cudaStreamSynchronize(c->stream));
    return h;
}

} // namespace fvmb

using namespace fvmb;

void fvmb_destroy_predictor(fvmb::Predictor* p) { delete p; }

#define API_TRY try {
#define API_CATCH                        \
    }                                    \
    catch (const Error& ex) {            \
        set_error(ex.what());            \
        return ex.code;                  \
    }                                    \
    catch (const std::exception& ex) {   \
        set_error(ex.what());            \
        return -1;                       \
    }

extern "C" int fvm_mlp_nparams(void) { return kNParam; }

extern "C" int fvm_mlp_set_params(fvm_ctx* c, const float* params_host) {
    API_TRY
    if (!c || !params_host) throw Error("fvm_mlp_set_params: null argument");
    Predictor* p = predictor_get(c);
    FVM_CUDA(cudaMemcpyAsync(p->p.p, params_host, sizeof(float) * kNParam, cudaMemcpyHostToDevice, c->stream));
    pack(c, p);
    p->m.zero(c->stream);
    p->v.zero(c->stream);
    p->adam_t = 0;
    p->ready = true;
    FVM_CUDA(cudaStreamSynchronize(c->stream));
    return 0;
    API_CATCH
}

extern "C" int fvm_mlp_get_params(fvm_ctx* c, float* params_host) {
    API_TRY
    if (!c || !params_host || !c->pred) throw Error("fvm_mlp_get_params: no predictor");
    FVM_CUDA(cudaMemcpyAsync(params_host, c->pred->p.p, sizeof(float) * kNParam, cudaMemcpyDeviceToHost, c->stream));
    FVM_CUDA(cudaStreamSynchronize(c->stream));
    return 0;
    API_CATCH
}

extern "C" int fvm_mlp_forward(fvm_ctx* c, const float* X, int n, float* out) {
    API_TRY
    if (!c || !X || !out || !c->pred) throw Error("fvm_mlp_forward: no predictor or null argument");
    predictor_forward(c, c->pred, X, n, out);
    FVM_CUDA(cudaGetLastError());
    int e = check_err(c, c->pred);
    return e ? 2 : 0;
    API_CATCH
}

extern "C" int fvm_mlp_grad(fvm_ctx* c, const float* X, const float* Y, int n, float* grad_host,
                            float* loss) {
    API_TRY
    if (!c || !X || !Y || !c->pred) throw Error("fvm_mlp_grad: no predictor or null argument");
    int nb;
    train_pass(c, c->pred, X, Y, 0, n, &nb);
    std::vector<float> g(kNTrain + 1);
    FVM_CUDA(cudaMemcpyAsync(g.data(), c->pred->gsum.p, sizeof(float) * (kNTrain + 1), cudaMemcpyDeviceToHost,
                             c->stream));
    int e = check_err(c, c->pred);
    if (grad_host) std::copy(g.begin(), g.begin() + kNTrain, grad_host);
    if (loss) *loss = g[kNTrain] / std::max(1, n);
    return e ? 2 : 0;
    API_CATCH
}

extern "C" int fvm_mlp_train(fvm_ctx* c, const float* X, const float* Y, int n, int epochs, int batch, float lr,
                             float* loss_history) {
    API_TRY
    if (!c || !X || !Y || !c->pred || n <= 0 || epochs <= 0) throw Error("fvm_mlp_train: bad argument");
    Predictor* p = c->pred;
    if (batch <= 0) batch = 148 * 2 * kTile;
    const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
    std::vector<float> gl(kNTrain + 1);
    for (int ep = 0; ep < epochs; ++ep) {
        double lsum = 0.0;
        for (long b0 = 0; b0 < n; b0 += batch) {
            long b1e = std::min<long>(n, b0 + batch);
            int nb;
            train_pass(c, p, X, Y, b0, b1e, &nb);
            p->adam_t++;
            float bc1 = 1.0f - std::pow(b1, (float)p->adam_t), bc2 = 1.0f - std::pow(b2, (float)p->adam_t);
            fvm_launch(c, k_adam, grid_for(kNTrain, 256), 256, 0, c->stream, p->p.p, p->m.p, p->v.p, p->gsum.p, lr, b1,
                       b2, eps, bc1, bc2);
            pack(c, p);
            float ls = 0.0f;
            FVM_CUDA(cudaMemcpyAsync(&ls, p->gsum.p + kNTrain, sizeof(float), cudaMemcpyDeviceToHost, c->stream));
            FVM_CUDA(cudaStreamSynchronize(c->stream));
            lsum += ls;
        }
        if (loss_history) loss_history[ep] = (float)(lsum / n);
    }
    p->ready = true;
    return check_err(c, p) ? 2 : 0;
    API_CATCH
}
