// Device helpers of the cooperative Krylov kernels: the bounded grid
// barrier, fixed-order cross-block reductions and the row-quad basis passes
// of the CGS2 orthogonalisation (linalg.cu, arnoldi_fused.cu).
#pragma once

#include "ctx.cuh"
#include "reduce.cuh"

namespace fvmb {

// ---- fused Arnoldi orthogonalisation (one cooperative launch per step)
// Grid barrier of a cooperative launch: arrival counter plus generation
// word.  The wait is bounded; if it runs out the kernel records error 3 and
// every block leaves at its next barrier.
__device__ __forceinline__ bool grid_barrier(unsigned* count, unsigned* gen, int* err) {
    __syncthreads();
    if (threadIdx.x == 0) {
        volatile unsigned* vg = gen;
        const unsigned g = *vg;
        __threadfence();
        if (atomicAdd(count, 1u) == gridDim.x - 1) {
            *count = 0u;
            __threadfence();
            atomicAdd(gen, 1u);
        } else {
            long it = 0;
            while (*vg == g) {
                if (++it > (1l << 26)) { atomicExch(err, 3); break; }
            }
        }
        __threadfence();
    }
    __syncthreads();
    return *(volatile int*)err == 0;
}

// out[v] = sum over blocks b (ascending, lane-strided, fixed shuffle tree) of
// partial[b * nv + v] -- the order of last_block_reduce, so every block gets
// the same bits; written to shared memory.  The partials were written by
// other blocks before the grid barrier: they are read through L2 (ld.cg,
// never a stale L1 line), a warp taking 4 vectors and each lane 5 blocks at
// a time so that 20 loads per lane are in flight.
__device__ __forceinline__ void block_reduce_all(const double* partial, int nv, int nblk, double* out) {
    constexpr int kQ = 4, kI = 5;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
    for (int v0 = warp; v0 < nv; v0 += kQ * nw) {
        double s[kQ];
#pragma unroll
        for (int q = 0; q < kQ; ++q) s[q] = 0.0;
        for (int b0 = 0; b0 < nblk; b0 += 32 * kI) {
            double x[kI][kQ];
#pragma unroll
            for (int i = 0; i < kI; ++i) {
                const int b = b0 + lane + 32 * i;
#pragma unroll
                for (int q = 0; q < kQ; ++q) {
                    const int v = v0 + q * nw;
                    x[i][q] = (b < nblk && v < nv) ? __ldcg(partial + (size_t)b * nv + v) : 0.0;
                }
            }
#pragma unroll
            for (int i = 0; i < kI; ++i)
#pragma unroll
                for (int q = 0; q < kQ; ++q) s[q] += x[i][q];
        }
#pragma unroll
        for (int q = 0; q < kQ; ++q) {
            const double t = warp_sum(s[q]);
            const int v = v0 + q * nw;
            if (lane == 0 && v < nv) out[v] = t;
        }
    }
    __syncthreads();
}

// block_reduce_all for vector-major partials (partial[v * nblk + b]): a
// warp's lanes read consecutive blocks of one vector, so every load is
// coalesced; the same blocks in the same order, so the same bits
__device__ __forceinline__ void block_reduce_all_vmajor(const double* partial, int nv, int nblk, double* out) {
    constexpr int kQ = 4;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
    for (int v0 = warp; v0 < nv; v0 += kQ * nw) {
        double s[kQ];
#pragma unroll
        for (int q = 0; q < kQ; ++q) s[q] = 0.0;
        for (int b0 = 0; b0 < nblk; b0 += 32 * 5) {
            double x[5][kQ];
#pragma unroll
            for (int i = 0; i < 5; ++i) {
                const int b = b0 + lane + 32 * i;
#pragma unroll
                for (int q = 0; q < kQ; ++q) {
                    const int v = v0 + q * nw;
                    x[i][q] = (b < nblk && v < nv) ? __ldcg(partial + (size_t)v * nblk + b) : 0.0;
                }
            }
#pragma unroll
            for (int i = 0; i < 5; ++i)
#pragma unroll
                for (int q = 0; q < kQ; ++q) s[q] += x[i][q];
        }
#pragma unroll
        for (int q = 0; q < kQ; ++q) {
            const double t = warp_sum(s[q]);
            const int v = v0 + q * nw;
            if (lane == 0 && v < nv) out[v] = t;
        }
    }
    __syncthreads();
}

constexpr int kCgsThreads = 512;
constexpr int kCgsGroup = 8;   // basis vectors whose loads are in flight together

// rows per block of the fused orthogonalisation: ceil(N / nblk) rounded up
// to 4, so every block's rows start on a 4-row (16-byte FP32 / 32-byte
// FP64) boundary and each thread owns whole quads of rows
__host__ __device__ inline int cgs_chunk(int N, int nblk) {
    const int c = (N + nblk - 1) / nblk;
    return (c + 3) & ~3;
}

// four consecutive basis values starting at a 4-aligned row (the basis
// allocation is padded to a multiple of 64 rows and zeroed, so a quad that
// straddles row N reads zeros)
__device__ __forceinline__ void ld4(const float* p, double v[4]) {
    const float4 q = __ldg(reinterpret_cast<const float4*>(p));
    v[0] = q.x; v[1] = q.y; v[2] = q.z; v[3] = q.w;
}
__device__ __forceinline__ void ld4(const double* p, double v[4]) {
    const double2 a = __ldg(reinterpret_cast<const double2*>(p));
    const double2 b = __ldg(reinterpret_cast<const double2*>(p) + 1);
    v[0] = a.x; v[1] = a.y; v[2] = b.x; v[3] = b.y;
}
// through L2 only (ld.global.cg): for vectors written earlier in the same
// launch, which the read-only path could serve from a stale line
__device__ __forceinline__ void ld4_cg(const float* p, double v[4]) {
    const float4 q = __ldcg(reinterpret_cast<const float4*>(p));
    v[0] = q.x; v[1] = q.y; v[2] = q.z; v[3] = q.w;
}
__device__ __forceinline__ void ld4_cg(const double* p, double v[4]) {
    const double2 a = __ldcg(reinterpret_cast<const double2*>(p));
    const double2 b = __ldcg(reinterpret_cast<const double2*>(p) + 1);
    v[0] = a.x; v[1] = a.y; v[2] = b.x; v[3] = b.y;
}
// the basis, read by row quads: through the read-only path (the block's
// rows of the vectors stay in L1 between the three passes), or, with CG,
// through L2 only -- for a kernel that writes basis vectors and reads them
// back in the same launch
template <class B, bool CG = false>
struct BasisRows {
    const B* U;
    size_t ld;
    __device__ __forceinline__ void quad(int i, int r, double v[4]) const {
        if (CG) ld4_cg(U + ld * i + r, v);
        else ld4(U + ld * i + r, v);
    }
};

// block-local dot products <U_i, W> over rows [k0, k1) for i < nv, with the
// block's W rows in shared memory (Wl[k - k0]).  Each thread owns quads of
// rows; the vectors are taken kCgsGroup at a time so that many loads are in
// flight per thread.  Per vector: the thread's quads in row order, then the
// warp's lanes by a fixed shuffle tree, then the warps in warp order.  Row
// nv of the output (when with_norm) is sum W^2.  out[i] is valid in every
// thread after the call.  red holds kCgsGroup doubles per warp.
template <class B, bool CG>
__device__ __forceinline__ void block_dots(const BasisRows<B, CG>& U, const double* __restrict__ Wl, int k0, int k1,
                                           int nv, bool with_norm, double* red, double* out) {
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
    const int nvec = nv + (with_norm ? 1 : 0);
    // quads start on a 4-row boundary; rows of the quad outside [k0, k1)
    // enter as zeros (a block range that starts on a quad is unaffected)
    const int a0 = k0 & ~3;
    for (int i0 = 0; i0 < nvec; i0 += kCgsGroup) {
        double acc[kCgsGroup];
#pragma unroll
        for (int q = 0; q < kCgsGroup; ++q) acc[q] = 0.0;
        for (int r = a0 + 4 * threadIdx.x; r < k1; r += 4 * blockDim.x) {
            double w[4];
#pragma unroll
            for (int e = 0; e < 4; ++e) w[e] = (r + e >= k0 && r + e < k1) ? Wl[r + e - k0] : 0.0;
#pragma unroll
            for (int q = 0; q < kCgsGroup; ++q) {
                const int i = i0 + q;
                if (i < nv) {
                    double u[4];
                    U.quad(i, r, u);
                    acc[q] += u[0] * w[0] + u[1] * w[1] + u[2] * w[2] + u[3] * w[3];
                } else if (i == nv && with_norm) {
                    acc[q] += w[0] * w[0] + w[1] * w[1] + w[2] * w[2] + w[3] * w[3];
                }
            }
        }
#pragma unroll
        for (int q = 0; q < kCgsGroup; ++q) acc[q] = warp_sum(acc[q]);
        if (lane == 0) {
#pragma unroll
            for (int q = 0; q < kCgsGroup; ++q) red[warp * kCgsGroup + q] = acc[q];
        }
        __syncthreads();
        if (threadIdx.x < kCgsGroup && i0 + threadIdx.x < nvec) {
            double t = 0.0;
            for (int w2 = 0; w2 < nw; ++w2) t += red[w2 * kCgsGroup + threadIdx.x];
            out[i0 + threadIdx.x] = t;
        }
        __syncthreads();
    }
}

// acc[e] = sum_i coef[i] U_i[r + e], e < 4, vectors kCgsGroup at a time
template <class B, bool CG>
__device__ __forceinline__ void quad_combine(const BasisRows<B, CG>& U, const double* coef, int nv, int r,
                                             double acc[4]) {
    acc[0] = acc[1] = acc[2] = acc[3] = 0.0;
    for (int i0 = 0; i0 < nv; i0 += kCgsGroup) {
#pragma unroll
        for (int q = 0; q < kCgsGroup; ++q) {
            const int i = i0 + q;
            if (i < nv) {
                double u[4];
                U.quad(i, r, u);
                const double c = coef[i];
                acc[0] += c * u[0]; acc[1] += c * u[1]; acc[2] += c * u[2]; acc[3] += c * u[3];
            }
        }
    }
}

// Rows of a block held in shared memory quad-transposed: the block's row
// quads start at a0 = k0 & ~3, and row a0 + 4 q + e sits at e * nqp + q,
// so the lanes of a warp, each on its own quad, read consecutive doubles
// (no bank conflicts; row-major quads would put every fourth lane on the
// same banks).  Rows of the edge quads outside [k0, k1) hold zeros.
__device__ __forceinline__ int quad_pos(int k0, int nqp, int k) {
    const int t = k - (k0 & ~3);
    return (t & 3) * nqp + (t >> 2);
}

// Block-local dot products <U_i, W> over rows [k0, k1) for i < nv (and
// sum W^2 as entry nv when with_norm) for an FP32 basis, one warp per
// vector: the warp's lanes take the block's row quads in turn with eight
// quads' loads (float4, read-only path) in flight per lane, then one shuffle
// tree.  No block-wide reduction is needed, so vectors finish
// independently.  out[i] is valid in every thread after the call.  Wt is
// quad-transposed (quad_pos).
__device__ __forceinline__ void block_dots_by_warp(const float* __restrict__ U, size_t ld,
                                                   const double* __restrict__ Wt, int nqp, int k0, int k1, int nv,
                                                   bool with_norm, double* out) {
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
    const int a0 = k0 & ~3;
    const int nq = (k1 - a0 + 3) >> 2;
    const int nvec = nv + (with_norm ? 1 : 0);
    for (int i = warp; i < nvec; i += nw) {
        double acc = 0.0;
        const float* Ui = U + ld * (i < nv ? i : 0);
        for (int q0 = lane; q0 < nq; q0 += 32 * 8) {
            float4 u[8];
#pragma unroll
            for (int t = 0; t < 8; ++t) {
                const int q = q0 + 32 * t;
                u[t] = (i < nv && q < nq) ? __ldg(reinterpret_cast<const float4*>(Ui + a0 + 4 * q))
                                          : make_float4(0.f, 0.f, 0.f, 0.f);
            }
#pragma unroll
            for (int t = 0; t < 8; ++t) {
                const int q = q0 + 32 * t;
                if (q >= nq) continue;
                double w[4];
#pragma unroll
                for (int e = 0; e < 4; ++e) w[e] = Wt[e * nqp + q];
                if (i < nv)
                    acc += (double)u[t].x * w[0] + (double)u[t].y * w[1] + (double)u[t].z * w[2] +
                           (double)u[t].w * w[3];
                else
                    acc += w[0] * w[0] + w[1] * w[1] + w[2] * w[2] + w[3] * w[3];
            }
        }
        acc = warp_sum(acc);
        if (lane == 0) out[i] = acc;
    }
    __syncthreads();
}

// Two block-local dot-product sets in one pass over the basis (FP32, one
// warp per basis vector): out[i] = <U_i, A>, out[nb + i] = <U_i, B> for
// i < nb, then out[2 nb] = <A, A> and out[2 nb + 1] = <A, B>, with A and B
// the block's rows in shared memory (quad-transposed, quad_pos).  Each
// basis row quad is loaded once for both products.  out[] is valid in every
// thread after the call.
__device__ __forceinline__ void block_dots2_by_warp(const float* __restrict__ U, size_t ld,
                                                    const double* __restrict__ A, const double* __restrict__ Bv,
                                                    int nqp, int k0, int k1, int nb, double* out) {
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
    const int a0 = k0 & ~3;
    const int nq = (k1 - a0 + 3) >> 2;
    for (int i = warp; i < nb + 1; i += nw) {
        double sa = 0.0, sb = 0.0;
        const float* Ui = U + ld * (i < nb ? i : 0);
        for (int q0 = lane; q0 < nq; q0 += 32 * 8) {
            float4 u[8];
#pragma unroll
            for (int t = 0; t < 8; ++t) {
                const int q = q0 + 32 * t;
                u[t] = (i < nb && q < nq) ? __ldg(reinterpret_cast<const float4*>(Ui + a0 + 4 * q))
                                          : make_float4(0.f, 0.f, 0.f, 0.f);
            }
#pragma unroll
            for (int t = 0; t < 8; ++t) {
                const int q = q0 + 32 * t;
                if (q >= nq) continue;
                double va[4], vb[4];
#pragma unroll
                for (int e = 0; e < 4; ++e) {
                    va[e] = A[e * nqp + q];
                    vb[e] = Bv[e * nqp + q];
                }
                if (i < nb) {
                    sa += (double)u[t].x * va[0] + (double)u[t].y * va[1] + (double)u[t].z * va[2] +
                          (double)u[t].w * va[3];
                    sb += (double)u[t].x * vb[0] + (double)u[t].y * vb[1] + (double)u[t].z * vb[2] +
                          (double)u[t].w * vb[3];
                } else {
                    sa += va[0] * va[0] + va[1] * va[1] + va[2] * va[2] + va[3] * va[3];
                    sb += va[0] * vb[0] + va[1] * vb[1] + va[2] * vb[2] + va[3] * vb[3];
                }
            }
        }
        sa = warp_sum(sa);
        sb = warp_sum(sb);
        if (lane == 0) {
            if (i < nb) {
                out[i] = sa;
                out[nb + i] = sb;
            } else {
                out[2 * nb] = sa;
                out[2 * nb + 1] = sb;
            }
        }
    }
    __syncthreads();
}

// The same two dot-product sets (and the same out[] layout) with one thread
// per row quad: a thread reads its rows of A and B from shared memory once
// per kCgsGroup basis vectors and keeps that group's loads in flight
// together.  The warp's 2 kCgsGroup partial sums are reduced by a
// transposing butterfly: each exchange hands the partner the half of the
// values it keeps, so after offsets 16, 8, 4, 2 every lane holds one value
// (index b1 + 2 b2 + 4 b3 + 8 b4 of its lane bits) summed over 16 lanes, and
// offset 1 completes it; 16 exchanges instead of 5 per value.  The warps'
// sums are then added in warp order.  red holds 2 x (warps x 2 kCgsGroup)
// doubles (alternating groups, so one barrier per group).  keep receives
// the thread's first quad of the last group's vectors (from kept_first(nb)
// on, zeros past nb - 1), for a later pass over the same rows.
__host__ __device__ inline int kept_first(int nb) { return nb & ~(kCgsGroup - 1); }
__device__ __forceinline__ void block_dots2_by_quad(const float* __restrict__ U, size_t ld,
                                                    const double* __restrict__ A, const double* __restrict__ Bv,
                                                    int nqp, int k0, int k1, int nb, double* red, double* out,
                                                    float4 (&keep)[kCgsGroup]) {
    constexpr int G = kCgsGroup, NV = 2 * kCgsGroup;
    static_assert(NV == 16, "the butterfly below reduces 16 values per lane");
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
    const int a0 = k0 & ~3;
    const int nq = (k1 - a0 + 3) >> 2;
    const int idx = ((lane >> 1) & 1) | (((lane >> 2) & 1) << 1) | (((lane >> 3) & 1) << 2) | (((lane >> 4) & 1) << 3);
    int buf = 0;
    for (int i0 = 0; i0 <= nb; i0 += G, buf ^= 1) {
        double v[NV];
#pragma unroll
        for (int j = 0; j < NV; ++j) v[j] = 0.0;
        for (int q = threadIdx.x; q < nq; q += blockDim.x) {
            float4 u[G];
#pragma unroll
            for (int g = 0; g < G; ++g) {
                const int i = i0 + g;
                u[g] = i < nb ? __ldg(reinterpret_cast<const float4*>(U + ld * i + a0 + 4 * q))
                              : make_float4(0.f, 0.f, 0.f, 0.f);
            }
            if (i0 + G > nb && q == (int)threadIdx.x) {
#pragma unroll
                for (int g = 0; g < G; ++g) keep[g] = u[g];
            }
            double x[4], y[4];
#pragma unroll
            for (int e = 0; e < 4; ++e) {
                x[e] = A[e * nqp + q];
                y[e] = Bv[e * nqp + q];
            }
#pragma unroll
            for (int g = 0; g < G; ++g) {
                const int i = i0 + g;
                if (i < nb) {
                    const double u0 = u[g].x, u1 = u[g].y, u2 = u[g].z, u3 = u[g].w;
                    v[2 * g] += u0 * x[0] + u1 * x[1] + u2 * x[2] + u3 * x[3];
                    v[2 * g + 1] += u0 * y[0] + u1 * y[1] + u2 * y[2] + u3 * y[3];
                } else if (i == nb) {
                    v[2 * g] += x[0] * x[0] + x[1] * x[1] + x[2] * x[2] + x[3] * x[3];
                    v[2 * g + 1] += x[0] * y[0] + x[1] * y[1] + x[2] * y[2] + x[3] * y[3];
                }
            }
        }
#pragma unroll
        for (int s = 0; s < 4; ++s) {
            const int o = 16 >> s, c = NV >> (s + 1);
            const bool up = (lane & o) != 0;
#pragma unroll
            for (int j = 0; j < c; ++j) {
                const double send = up ? v[j] : v[j + c];
                const double mine = up ? v[j + c] : v[j];
                v[j] = mine + __shfl_xor_sync(0xffffffffu, send, o);
            }
        }
        v[0] += __shfl_xor_sync(0xffffffffu, v[0], 1);
        double* rb = red + buf * nw * NV;
        if (!(lane & 1)) rb[warp * NV + idx] = v[0];
        __syncthreads();
        if (threadIdx.x < NV) {
            const int i = i0 + (threadIdx.x >> 1);
            if (i <= nb) {
                double t = 0.0;
                for (int w2 = 0; w2 < nw; ++w2) t += rb[w2 * NV + threadIdx.x];
                if (i < nb) out[(threadIdx.x & 1) ? nb + i : i] = t;
                else out[2 * nb + (threadIdx.x & 1)] = t;
            }
        }
    }
    __syncthreads();
}

// quad_combine2 for a row quad whose vectors from kept_first(nv) on are
// already in registers (keep, from block_dots2_by_quad): those first, then
// the others loaded kCgsGroup at a time
template <class B, bool CG>
__device__ __forceinline__ void quad_combine2_kept(const BasisRows<B, CG>& U, const double* c1, const double* c2,
                                                   int nv, int r, const float4 (&keep)[kCgsGroup], double acc1[4],
                                                   double acc2[4]) {
    const int i1 = kept_first(nv);
#pragma unroll
    for (int e = 0; e < 4; ++e) acc1[e] = acc2[e] = 0.0;
#pragma unroll
    for (int q = 0; q < kCgsGroup; ++q) {
        const int i = i1 + q;
        if (i < nv) {
            const double u[4] = {keep[q].x, keep[q].y, keep[q].z, keep[q].w};
            const double a = c1[i], b = c2[i];
#pragma unroll
            for (int e = 0; e < 4; ++e) {
                acc1[e] += a * u[e];
                acc2[e] += b * u[e];
            }
        }
    }
    for (int i0 = 0; i0 < i1; i0 += kCgsGroup) {
#pragma unroll
        for (int q = 0; q < kCgsGroup; ++q) {
            const int i = i0 + q;
            double u[4];
            U.quad(i, r, u);
            const double a = c1[i], b = c2[i];
#pragma unroll
            for (int e = 0; e < 4; ++e) {
                acc1[e] += a * u[e];
                acc2[e] += b * u[e];
            }
        }
    }
}

// acc1[e] = sum_i c1[i] U_i[r + e], acc2[e] = sum_i c2[i] U_i[r + e] (e < 4)
// from one load of each basis row quad
template <class B, bool CG>
__device__ __forceinline__ void quad_combine2(const BasisRows<B, CG>& U, const double* c1, const double* c2, int nv,
                                              int r, double acc1[4], double acc2[4]) {
#pragma unroll
    for (int e = 0; e < 4; ++e) acc1[e] = acc2[e] = 0.0;
    for (int i0 = 0; i0 < nv; i0 += kCgsGroup) {
#pragma unroll
        for (int q = 0; q < kCgsGroup; ++q) {
            const int i = i0 + q;
            if (i < nv) {
                double u[4];
                U.quad(i, r, u);
                const double a = c1[i], b = c2[i];
#pragma unroll
                for (int e = 0; e < 4; ++e) {
                    acc1[e] += a * u[e];
                    acc2[e] += b * u[e];
                }
            }
        }
    }
}

} // namespace fvmb
