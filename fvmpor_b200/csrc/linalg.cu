// Reductions, WRMS norms and preconditioned restarted GMRES.
//
// Algorithm: restarted GMRES(m) with Arnoldi and the Givens least squares
// of decomp/gmres.c:26-201, :412-511 and decomp/linalg_dense.c:128-173,
// applied the way IDAS SPGMR applies it inside the Newton iteration (the
// solver the reference's hot path actually runs, ida_integrator.h:248-254):
// zero initial guess, LEFT preconditioning, scaling by D = diag(ewt), so
// the stopping test sees ||D P^-1 (b - J x)||_wrms -- a head-space quantity
// comparable with the Newton tolerance.  (decomp's stand-alone gmres.c is
// right-preconditioned; with the unscaled residual F of this problem that
// variant measures mass-flux units against head weights.)  J*v is the
// difference quotient of the residual with sigma = 1/||v||_wrms.
//
// B200 layout: the Arnoldi basis is kept as unnormalised vectors U_i with a
// per-vector scale s_i (V_i = s_i U_i), in FP64 or FP32 (mixed precision).
// Orthogonalisation is classical Gram-Schmidt with one re-orthogonalisation
// (CGS2) in three fused passes over the basis, so one Arnoldi step costs
// three basis reads instead of the 2(j+1) of modified Gram-Schmidt; every
// dot product accumulates in FP64 and is reduced in a fixed order (per-block
// partials, then the last block sums them by block index), so results are
// bitwise reproducible.  The Hessenberg matrix, Givens rotations and the
// stopping test run in FP64 on the host from j+2 numbers copied back per
// step.
#include "cgs.cuh"
#include "ctx.cuh"
#include "krylov.cuh"
#include "reduce.cuh"

#include <algorithm>
#include <cmath>

namespace fvmb {

// out[0] = sum_k (x_k w_k)^2 (w may be null -> 1)
__global__ void k_sumsq(int N, const double* __restrict__ x, const double* __restrict__ w,
                        double* partial, unsigned* counter, double* out) {
    double s = 0.0;
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < N; k += gridDim.x * blockDim.x) {
        double v = w ? x[k] * w[k] : x[k];
        s += v * v;
    }
    __shared__ double red[32];
    s = warp_sum(s);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x < 32) {
        double t = threadIdx.x < (blockDim.x >> 5) ? red[threadIdx.x] : 0.0;
        t = warp_sum(t);
        if (threadIdx.x == 0) partial[blockIdx.x] = t;
    }
    last_block_reduce(partial, 1, counter, out);
}

__global__ void k_dot(int N, const double* __restrict__ x, const double* __restrict__ y,
                      double* partial, unsigned* counter, double* out) {
    double s = 0.0;
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < N; k += gridDim.x * blockDim.x) s += x[k] * y[k];
    __shared__ double red[32];
    s = warp_sum(s);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x < 32) {
        double t = threadIdx.x < (blockDim.x >> 5) ? red[threadIdx.x] : 0.0;
        t = warp_sum(t);
        if (threadIdx.x == 0) partial[blockIdx.x] = t;
    }
    last_block_reduce(partial, 1, counter, out);
}

// sigma = 1 / ||z||_wrms for the difference-quotient J*v (IDAS picks the
// increment that makes the perturbation one weighted unit); 1 if z = 0
__global__ void k_sigma_from_sumsq(const double* sumsq, int N, double* sigma) {
    double n = sqrt(sumsq[0] / (double)N);
    *sigma = n > 0.0 ? 1.0 / n : 1.0;
}

// ------------------------------------------------------------------ CGS2
template <class B>
__device__ __forceinline__ double ldb(const B* U, size_t i) { return (double)U[i]; }

// pass 1: w~ = ewt * Jv (stored in W); a_i = <U_i, w~> for i < nv
template <class B>
__global__ void k_cgs_pass1(int N, int nv, const B* __restrict__ U, size_t ld,
                            const double* __restrict__ Jv, const double* __restrict__ ewt,
                            double* __restrict__ W, double* partial, unsigned* counter,
                            double* out) {
    int chunk = (N + gridDim.x - 1) / gridDim.x;
    int k0 = blockIdx.x * chunk, k1 = min(N, k0 + chunk);
    for (int k = k0 + threadIdx.x; k < k1; k += blockDim.x) W[k] = ewt[k] * Jv[k];
    __syncthreads();
    int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
    for (int i = warp; i < nv; i += nw) {
        const B* Ui = U + ld * i;
        double s = 0.0;
        for (int k = k0 + lane; k < k1; k += 32) s += ldb(Ui, k) * W[k];
        s = warp_sum(s);
        if (lane == 0) partial[(size_t)blockIdx.x * nv + i] = s;
    }
    last_block_reduce(partial, nv, counter, out);
}

// pass 2: W -= sum_i (a_i s_i^2) U_i ; b_i = <U_i, W>
template <class B>
__global__ void k_cgs_pass2(int N, int nv, const B* __restrict__ U, size_t ld,
                            const double* __restrict__ scale, const double* __restrict__ a,
                            double* __restrict__ W, double* partial, unsigned* counter,
                            double* out) {
    __shared__ double coef[64];
    for (int i = threadIdx.x; i < nv; i += blockDim.x) coef[i] = a[i] * scale[i] * scale[i];
    __syncthreads();
    int chunk = (N + gridDim.x - 1) / gridDim.x;
    int k0 = blockIdx.x * chunk, k1 = min(N, k0 + chunk);
    for (int k = k0 + threadIdx.x; k < k1; k += blockDim.x) {
        double acc = 0.0;
        for (int i = 0; i < nv; ++i) acc += coef[i] * ldb(U + ld * i, k);
        W[k] = W[k] - acc;
    }
    __syncthreads();
    int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
    for (int i = warp; i < nv; i += nw) {
        const B* Ui = U + ld * i;
        double s = 0.0;
        for (int k = k0 + lane; k < k1; k += 32) s += ldb(Ui, k) * W[k];
        s = warp_sum(s);
        if (lane == 0) partial[(size_t)blockIdx.x * nv + i] = s;
    }
    last_block_reduce(partial, nv, counter, out);
}

// pass 3: W -= sum_i (b_i s_i^2) U_i ; U_nv = store(W) ; out[0] = ||U_nv||^2
// and scale[nv] = 1/||U_nv|| written by the last block
template <class B>
__global__ void k_cgs_pass3(int N, int nv, B* __restrict__ U, size_t ld,
                            double* __restrict__ scale, const double* __restrict__ b,
                            const double* __restrict__ W, double* partial, unsigned* counter,
                            double* out) {
    __shared__ double coef[64];
    for (int i = threadIdx.x; i < nv; i += blockDim.x) coef[i] = b[i] * scale[i] * scale[i];
    __syncthreads();
    B* Un = U + ld * nv;
    double s = 0.0;
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < N; k += gridDim.x * blockDim.x) {
        double acc = 0.0;
        for (int i = 0; i < nv; ++i) acc += coef[i] * ldb(U + ld * i, k);
        B st = (B)(W[k] - acc);
        Un[k] = st;
        double d = (double)st;
        s += d * d;
    }
    __shared__ double red[32];
    s = warp_sum(s);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x < 32) {
        double t = threadIdx.x < (blockDim.x >> 5) ? red[threadIdx.x] : 0.0;
        t = warp_sum(t);
        if (threadIdx.x == 0) partial[blockIdx.x] = t;
    }
    last_block_reduce(partial, 1, counter, out);
}

// One Arnoldi step of the device-driven GMRES in one cooperative launch:
// CGS2 orthogonalisation of the new direction against the basis, the new
// basis vector and its scale, the next Krylov direction t = s_nv U_nv / ewt
// with its difference-quotient increment sigma = 1 / ||t||_wrms, and (block
// 0) the Hessenberg column, Givens rotations and stopping test
// (linalg_dense.c:128-173):
//   W = ewt Jv; a = U^T W;  W' = W - U diag(s^2) a;  b = U^T W';
//   U_nv = W' - U diag(s^2) b;  ||U_nv||^2 = ||W'||^2 - sum_i (s_i b_i)^2.
// The last line is Pythagoras on the re-orthogonalisation: b is a
// rounding-level correction, so the norm needs no third reduction.  Two grid
// barriers per step.  Every reduction is fixed-order (per-block partials in
// block order), so results are bitwise reproducible.  Block b owns rows
// [b c, min(N, (b+1) c)) with c = cgs_chunk(N, gridDim.x); its rows of W
// live in dynamic shared memory (c doubles).  Its rows of the basis are
// read three times, by row quads; they stay in L1 between the passes.
// (Staging them in shared memory by bulk copies was measured slower: 50 us
// against 45 us at 40 vectors, the 226 KB of shared memory leaving L1 too
// little for the rest.)
template <class B>
__global__ void __launch_bounds__(kCgsThreads) k_arnoldi_cgs2(int N, ArnState* st, B* __restrict__ U, size_t ld,
                                                              double* __restrict__ scale,
                                                              const double* __restrict__ Jv,
                                                              const double* __restrict__ ewt,
                                                              double* __restrict__ W, double* partial,
                                                              unsigned* bar, int* err,
                                                              double* __restrict__ t_next, double* sigma_next,
                                                              double* __restrict__ H, double* __restrict__ cs,
                                                              double* __restrict__ sn, double* __restrict__ g) {
    __shared__ double ca[64], cb[64], coef[64];
    __shared__ double red[(kCgsThreads / 32) * kCgsGroup];
    extern __shared__ double Ws[];   // this block's rows of W (the vector being orthogonalised)
    (void)W;
    // launched as a programmatic dependent of the preconditioner apply, and
    // lets the next step's node pass launch early in turn
    pdl_wait_and_trigger();
    if (st->done) return;            // the device-driven loop has finished
    const int j = st->j, nv = j + 1, m = st->m;
    const int nblk = gridDim.x;
    const int chunk = cgs_chunk(N, nblk);
    const int k0 = min(N, blockIdx.x * chunk), k1 = min(N, k0 + chunk);
    double* pa = partial;
    double* pb = partial + (size_t)nblk * 64;
    // pass 1: a = U^T W
    for (int k = k0 + threadIdx.x; k < k1; k += blockDim.x) Ws[k - k0] = ewt[k] * Jv[k];
    __syncthreads();
    const BasisRows<B> UR{U, ld};
    block_dots(UR, Ws, k0, k1, nv, false, red, ca);
    for (int i = threadIdx.x; i < nv; i += blockDim.x) pa[(size_t)blockIdx.x * nv + i] = ca[i];
    if (!grid_barrier(bar, bar + 1, err)) return;
    block_reduce_all(pa, nv, nblk, ca);
    for (int i = threadIdx.x; i < nv; i += blockDim.x) coef[i] = ca[i] * scale[i] * scale[i];
    __syncthreads();
    // pass 2: W' = W - U diag(s^2) a; b = U^T W', ||W'||^2
    for (int r = k0 + 4 * threadIdx.x; r < k1; r += 4 * blockDim.x) {
        double acc[4];
        quad_combine(UR, coef, nv, r, acc);
#pragma unroll
        for (int e = 0; e < 4; ++e)
            if (r + e < k1) Ws[r + e - k0] -= acc[e];
    }
    __syncthreads();
    block_dots(UR, Ws, k0, k1, nv, true, red, cb);
    for (int i = threadIdx.x; i <= nv; i += blockDim.x) pb[(size_t)blockIdx.x * (nv + 1) + i] = cb[i];
    if (!grid_barrier(bar, bar + 1, err)) return;
    block_reduce_all(pb, nv + 1, nblk, cb);
    double nrm2 = cb[nv];
    for (int i = 0; i < nv; ++i) {
        const double c = scale[i] * cb[i];
        nrm2 -= c * c;
    }
    nrm2 = nrm2 > 0.0 ? nrm2 : 0.0;
    const double snv = nrm2 > 0.0 ? 1.0 / sqrt(nrm2) : 0.0;
    for (int i = threadIdx.x; i < nv; i += blockDim.x) coef[i] = cb[i] * scale[i] * scale[i];
    __syncthreads();
    // pass 3: the new basis vector and the next direction
    B* Un = U + ld * nv;
    for (int r = k0 + 4 * threadIdx.x; r < k1; r += 4 * blockDim.x) {
        double acc[4];
        quad_combine(UR, coef, nv, r, acc);
#pragma unroll
        for (int e = 0; e < 4; ++e) {
            const int k = r + e;
            if (k < k1) {
                const B u = (B)(Ws[k - k0] - acc[e]);
                Un[k] = u;
                t_next[k] = snv * (double)u / ewt[k];
            }
        }
    }
    if (blockIdx.x != 0) return;
    // block 0: the Hessenberg column (in ca) and the earlier rotations are
    // loaded by the whole block into shared memory; one thread then applies
    // the rotations in sequence, carrying the running entry in a register
    __shared__ double rc[64], rs[64];
    for (int i = threadIdx.x; i < nv; i += blockDim.x) ca[i] = scale[i] * (ca[i] + cb[i]);
    for (int i = threadIdx.x; i < j; i += blockDim.x) { rc[i] = cs[i]; rs[i] = sn[i]; }
    __syncthreads();
    if (threadIdx.x != 0) return;
    scale[nv] = snv;
    // ||t||_wrms^2 = sum_k (s U_k)^2 / N
    const double tw = snv * snv * nrm2 / (double)N;
    *sigma_next = tw > 0.0 ? 1.0 / sqrt(tw) : 1.0;
    // Hessenberg column, rotations, least-squares residual
    double* hc = ca;
    const double hn = sqrt(nrm2);
    hc[nv] = hn;
    if (!isfinite(hn) || !isfinite(hc[j])) {
        st->done = 3;
        return;
    }
    double cur = hc[0];
    for (int i = 0; i < j; ++i) {
        const double nx = hc[i + 1];
        hc[i] = rc[i] * cur + rs[i] * nx;
        cur = -rs[i] * cur + rc[i] * nx;
    }
    hc[j] = cur;
    const double den = hypot(hc[j], hc[j + 1]);
    double cj_, sj_;
    if (den == 0.0) { cj_ = 1.0; sj_ = 0.0; }
    else { cj_ = hc[j] / den; sj_ = hc[j + 1] / den; }
    cs[j] = cj_;
    sn[j] = sj_;
    hc[j] = den;
    const double gj = g[j];
    g[j + 1] = -sj_ * gj;
    g[j] = cj_ * gj;
    for (int i = 0; i <= j; ++i) H[(size_t)i * m + j] = hc[i];
    const double rn = fabs(-sj_ * gj) / st->sqrtN;
    st->rnorm = rn;
    st->j = j + 1;
    if (rn <= st->tol || hn == 0.0) st->done = 1;
    else if (j + 1 == m) st->done = 2;
}

__global__ void k_set_scale(const double* nrm2, double* scale, int idx) {
    double n = sqrt(nrm2[0]);
    scale[idx] = n > 0.0 ? 1.0 / n : 0.0;
}

// t = s_j U_j / ewt  (unscaled Krylov direction fed to the preconditioner)
template <class B>
__global__ void k_unscale(int N, const B* __restrict__ Uj, const double* __restrict__ scale,
                          int j, const double* __restrict__ ewt, double* __restrict__ t) {
    int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= N) return;
    t[k] = scale[j] * ldb(Uj, k) / ewt[k];
}

// x += (sum_i y_i s_i U_i) / ewt
template <class B>
__global__ void k_combine(int N, int nv, const B* __restrict__ U, size_t ld,
                          const double* __restrict__ ys, const double* __restrict__ ewt,
                          double* __restrict__ x) {
    __shared__ double coef[64];
    for (int i = threadIdx.x; i < nv; i += blockDim.x) coef[i] = ys[i];
    __syncthreads();
    int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= N) return;
    double acc = 0.0;
    for (int i = 0; i < nv; ++i) acc += coef[i] * ldb(U + ld * i, k);
    x[k] += acc / ewt[k];
}

// r~ = ewt * (b - Jx) (Jx may be null -> b); U_0 = r~; out = ||r~||^2
template <class B>
__global__ void k_init_residual(int N, const double* __restrict__ b, const double* __restrict__ Jx,
                                const double* __restrict__ ewt, B* __restrict__ U0, double* partial,
                                unsigned* counter, double* out) {
    double s = 0.0;
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < N; k += gridDim.x * blockDim.x) {
        double r = Jx ? b[k] - Jx[k] : b[k];
        B st = (B)(ewt[k] * r);
        U0[k] = st;
        double d = (double)st;
        s += d * d;
    }
    __shared__ double red[32];
    s = warp_sum(s);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x < 32) {
        double t = threadIdx.x < (blockDim.x >> 5) ? red[threadIdx.x] : 0.0;
        t = warp_sum(t);
        if (threadIdx.x == 0) partial[blockIdx.x] = t;
    }
    last_block_reduce(partial, 1, counter, out);
}

__global__ void k_sub(int N, const double* __restrict__ a, const double* __restrict__ b,
                      double* __restrict__ out) {
    int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k < N) out[k] = a[k] - b[k];
}

// ------------------------------------------------------------------ Krylov
Krylov* krylov_get(fvm_ctx* c, int m, int precision) {
    precision = precision ? 1 : 0;
    Krylov* K = c->kry[precision];
    if (K && K->m >= m) return c->kry_last = K;
    if (K) {
        ctx_sync(c);
        fvmb_destroy_krylov_impl(K);
        c->kry[precision] = nullptr;
    }
    K = new Krylov();
    K->m = m;
    K->precision = precision;
    K->ld = ((size_t)c->N + 63) / 64 * 64;
    size_t bytes = (precision ? sizeof(float) : sizeof(double)) * K->ld * (m + 1);
    FVM_CUDA(cudaMalloc(&K->U, bytes));
    // rows N .. ld of every basis vector stay zero: the fused
    // orthogonalisation reads them in its last row quad
    FVM_CUDA(cudaMemsetAsync(K->U, 0, bytes, c->stream));
    K->scale.alloc(m + 2);
    K->W.alloc(c->N);
    K->t.alloc(c->N);
    K->z.alloc(c->N);
    K->Jv.alloc(c->N);
    K->partial.alloc((size_t)kRedBlocks * std::max(m + 2, 3 * 64));
    K->counter.alloc(1);
    K->counter.zero(c->stream);
    K->st.alloc(1);
    K->ls.alloc((size_t)(m + 1) * m + 3 * (size_t)m + 1);
    K->bar.alloc(2);
    K->bar.zero(c->stream);
    K->err.alloc(1);
    K->err.zero(c->stream);
    {
        // the fused orthogonalisation needs every block resident at once
        int dev = 0, coop = 0, nsm = 0, per_sm = 0;
        FVM_CUDA(cudaGetDevice(&dev));
        FVM_CUDA(cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, dev));
        FVM_CUDA(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
        // one block per SM: fewer arrivals at each grid barrier; the block's
        // rows of W (at most 48 KB) live in its shared memory
        const void* kfn = precision ? (const void*)k_arnoldi_cgs2<float> : (const void*)k_arnoldi_cgs2<double>;
        K->coop_smem = sizeof(double) * (size_t)cgs_chunk(c->N, nsm);
        const bool fits = K->coop_smem <= 48 * 1024;
        if (fits)
            FVM_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kfn, kCgsThreads, K->coop_smem));
        K->coop_grid = (coop && fits && per_sm > 0 && m + 1 <= 63) ? nsm : 0;
        // one thread per row quad, whole warps: at 214k rows a block has 362
        // quads, and 384 threads instead of 512 leave fewer idle warps at
        // each block barrier (30-day FP32 run 0.759 -> 0.752 s, same bits:
        // the extra warps only added zeros)
        const int quads = cgs_chunk(c->N, nsm) / 4;
        K->coop_threads = std::min(kCgsThreads, std::max(128, (quads + 31) / 32 * 32));
    }
    K->res.alloc(3 * (m + 2) + 8);
    K->sigma.alloc(1);
    // results of the three passes, the m+1 basis scales, a status word and
    // the device-driven Arnoldi state
    FVM_CUDA(cudaMallocHost(&K->host, sizeof(double) * (4 * (m + 2) + 8) + sizeof(ArnState)));
    FVM_CUDA(cudaMallocHost(&K->host_ls, sizeof(double) * ((size_t)(m + 1) * m + m + 1)));
    c->kry[precision] = K;
    return c->kry_last = K;
}

void fvmb_destroy_krylov_impl(Krylov* K) {
    if (!K) return;
    if (K->gexec) cudaGraphExecDestroy(K->gexec);
    if (K->graph) cudaGraphDestroy(K->graph);
    if (K->U) cudaFree(K->U);
    if (K->host) cudaFreeHost(K->host);
    if (K->host_ls) cudaFreeHost(K->host_ls);
    delete K;
}

// host-synchronous reductions used by the controller
double reduce_sumsq(fvm_ctx* c, const double* x, const double* w) {
    Krylov* K = krylov_scratch(c);
    fvm_launch(c, k_sumsq, kRedBlocks, kRedThreads, 0, c->stream, c->N, x, w, K->partial.p, K->counter.p, K->res.p);
    FVM_CUDA(cudaMemcpyAsync(K->host, K->res.p, sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    ctx_sync(c);
    return K->host[0];
}

double reduce_dot(fvm_ctx* c, const double* x, const double* y) {
    Krylov* K = krylov_scratch(c);
    fvm_launch(c, k_dot, kRedBlocks, kRedThreads, 0, c->stream, c->N, x, y, K->partial.p, K->counter.p, K->res.p);
    FVM_CUDA(cudaMemcpyAsync(K->host, K->res.p, sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    ctx_sync(c);
    return K->host[0];
}

// J*v into out, sigma = 1/||v||_wrms computed on the device (or already in
// K->sigma when have_sigma)
static void jv_dev(fvm_ctx* c, Krylov* K, double cj, const double* y, const double* yp,
                   const double* F0, const double* v, const double* ewt, double* out, bool have_sigma = false) {
    if (!have_sigma) {
        fvm_launch(c, k_sumsq, kRedBlocks, kRedThreads, 0, c->stream, c->N, v, ewt, K->partial.p, K->counter.p,
                   K->res.p);
        fvm_launch(c, k_sigma_from_sumsq, 1, 1, 0, c->stream, K->res.p, c->N, K->sigma.p);
    }
    Perturb pt;
    pt.mode = 1;
    pt.cj = cj;
    pt.v = v;
    pt.sigma_dev = K->sigma.p;
    launch_residual(c, y, yp, pt, F0, out);
}

__global__ void k_set_cj(double* cjd, double cj, double dcj) {
    cjd[0] = cj;
    cjd[1] = dcj;
}

template <class B>
static int gmres_impl(fvm_ctx* c, Krylov* K, double cj, const double* y, const double* yp,
                      const double* F0, const double* ewt, const double* b, double* x, int m,
                      int max_restarts, double tol, int* iters, double* res_norm,
                      GmresCounters* cnt, int op, bool sync_end) {
    cudaStream_t s = c->stream;
    const int N = c->N;
    B* U = reinterpret_cast<B*>(K->U);
    const size_t ld = K->ld;
    const double sqrtN = std::sqrt((double)N);
    std::vector<double> H((size_t)(m + 1) * m), cs(m), sn(m), g(m + 1), hcol(m + 2);
    FVM_CUDA(cudaMemsetAsync(x, 0, sizeof(double) * N, s));
    int total = 0;
    double rnorm = 0.0;
    bool have_x = false;
    for (int cycle = 0; cycle <= max_restarts; ++cycle) {
        // preconditioned residual of the current iterate: z = P^-1 (b - J x)
        if (have_x) {
            if (op) jacobian_apply(c, cj, x, K->Jv.p);
            else jv_dev(c, K, cj, y, yp, F0, x, ewt, K->Jv.p);
            if (cnt) cnt->njv++;
            fvm_launch(c, k_sub, grid_for(N, 256), 256, 0, s, N, b, K->Jv.p, K->t.p);
            psolve_dev(c, K->t.p, K->z.p);
        } else {
            psolve_dev(c, b, K->z.p);
        }
        if (cnt) cnt->nps++;
        fvm_launch(c, k_init_residual<B>, kRedBlocks, kRedThreads, 0, s, N, K->z.p, nullptr, ewt, U,
                                                              K->partial.p, K->counter.p, K->res.p);
        // the assembled operator with the FP32 factor and basis: the whole
        // cycle in one persistent launch (arnoldi_fused.cu), which also takes
        // the initial norm from K->res, sets the first scale and direction
        // and decides there whether any step is needed, so the host waits
        // once per cycle
        const bool fused = op && sizeof(B) == sizeof(float) && K->coop_grid > 0 && fused_prepare(c, m);
        if (!fused) fvm_launch(c, k_set_scale, 1, 1, 0, s, K->res.p, K->scale.p, 0);
        std::fill(g.begin(), g.end(), 0.0);
        if (!fused) {
            FVM_CUDA(cudaMemcpyAsync(K->host, K->res.p, sizeof(double), cudaMemcpyDeviceToHost, s));
            ctx_sync(c);
            const double beta = std::sqrt(K->host[0]);
            rnorm = beta / sqrtN;
            if (!std::isfinite(beta)) { *iters = total; *res_norm = rnorm; return 2; }
            if (rnorm <= tol) { *iters = total; *res_norm = rnorm; return 0; }
            g[0] = beta;
        }
        int j = 0;
        bool conv = false;
        if (fused) {
            ArnState* hst = reinterpret_cast<ArnState*>(K->host + 4 * (m + 2) + 8);
            *hst = ArnState{0, 0, m, 0, tol, sqrtN, 0.0};
            FVM_CUDA(cudaMemcpyAsync(K->st.p, hst, sizeof(ArnState), cudaMemcpyHostToDevice, s));
            double* H_d = K->ls.p;
            double* cs_d = H_d + (size_t)(m + 1) * m;
            double* sn_d = cs_d + m;
            double* g_d = sn_d + m;
            fused_cycle(c, K, cj, ewt, H_d, cs_d, sn_d, g_d);
            // state, status, least-squares data and scales in one wait
            int* herr = reinterpret_cast<int*>(K->host + 4 * (m + 2) + 7);
            double* hls = K->host_ls;
            FVM_CUDA(cudaMemcpyAsync(hst, K->st.p, sizeof(ArnState), cudaMemcpyDeviceToHost, s));
            FVM_CUDA(cudaMemcpyAsync(herr, K->err.p, sizeof(int), cudaMemcpyDeviceToHost, s));
            FVM_CUDA(cudaMemcpyAsync(hls, H_d, sizeof(double) * ((size_t)(m + 1) * m), cudaMemcpyDeviceToHost, s));
            FVM_CUDA(cudaMemcpyAsync(hls + (size_t)(m + 1) * m, g_d, sizeof(double) * (m + 1), cudaMemcpyDeviceToHost,
                                     s));
            FVM_CUDA(cudaMemcpyAsync(K->host + 3 * (m + 2), K->scale.p, sizeof(double) * (m + 1),
                                     cudaMemcpyDeviceToHost, s));
            ctx_sync(c);
            if (*herr != 0) {
                // a grid barrier, a flag wait or the factor copy gave up
                K->err.zero(s);
                K->bar.zero(s);
                *iters = total + hst->j;
                *res_norm = hst->rnorm;
                return 2;
            }
            j = hst->j;
            total += j;
            if (cnt) { cnt->njv += j; cnt->nps += j; }
            rnorm = hst->rnorm;
            if (hst->done == 3) { *iters = total; *res_norm = rnorm; return 2; }
            if (j == 0) { *iters = total; *res_norm = rnorm; return 0; }   // already within tol
            conv = hst->done == 1;
            std::copy(hls, hls + (size_t)(m + 1) * m, H.begin());
            std::copy(hls + (size_t)(m + 1) * m, hls + (size_t)(m + 1) * m + m + 1, g.begin());
        } else if (K->coop_grid > 0) {
            // Device-driven Arnoldi: each step is J*v, the preconditioner,
            // the fused CGS2 and the Givens update, all reading the step
            // index and the stop flag from device memory; steps are queued
            // in batches and the host looks at the state once per batch.
            // Steps queued after the stop are skipped by every kernel.
            ArnState* hst = reinterpret_cast<ArnState*>(K->host + 4 * (m + 2) + 8);
            *hst = ArnState{0, 0, m, 0, tol, sqrtN, rnorm};
            FVM_CUDA(cudaMemcpyAsync(K->st.p, hst, sizeof(ArnState), cudaMemcpyHostToDevice, s));
            double* H_d = K->ls.p;
            double* cs_d = H_d + (size_t)(m + 1) * m;
            double* sn_d = cs_d + m;
            double* g_d = sn_d + m;
            FVM_CUDA(cudaMemcpyAsync(g_d, g.data(), sizeof(double) * (m + 1), cudaMemcpyHostToDevice, s));
            const int* skip = &K->st.p->done;
            int queued = 0;
            // full batches from a CUDA graph (fvm_opts.graph): cj and the
            // operator's cj shift come from device memory so that one
            // capture serves every Newton solve with the same vectors
            const bool graph = c->use_graph && c->graph_ok && !c->tm.on && !schur_active(c);
            if (graph) {
                if (K->cjd.n < 2) K->cjd.alloc(2);
                fvm_launch(c, k_set_cj, 1, 1, 0, s, K->cjd.p, cj, cj - jacobian_cj_setup(c));
            }
            // first direction and its increment
            fvm_launch(c, k_unscale<B>, grid_for(N, 256), 256, 0, s, N, U, K->scale.p, 0, ewt, K->t.p);
            fvm_launch(c, k_sumsq, kRedBlocks, kRedThreads, 0, s, N, K->t.p, ewt, K->partial.p, K->counter.p,
                       K->res.p);
            fvm_launch(c, k_sigma_from_sumsq, 1, 1, 0, s, K->res.p, N, K->sigma.p);
            for (;;) {
                // 2 steps, then 8 per host look: steps queued after the stop
                // cost little (every kernel of the chain returns at once), a
                // host round trip costs the GPU idle time (30-day 3D run:
                // 771 ms with batches of 4, 764 ms with 8)
                const int batch = std::min(m - queued, queued < 2 ? 2 : 8);
                auto enqueue = [&](int nsteps, bool dev_cj) {
                for (int q = 0; q < nsteps; ++q) {
                    Perturb pt;
                    pt.mode = 1;
                    pt.cj = cj;
                    pt.cj_dev = dev_cj ? K->cjd.p : nullptr;
                    pt.v = K->t.p;
                    pt.sigma_dev = K->sigma.p;
                    pt.skip = skip;
                    if (op) jacobian_apply(c, cj, K->t.p, K->Jv.p, skip, dev_cj ? K->cjd.p + 1 : nullptr);
                    else launch_residual(c, y, yp, pt, F0, K->Jv.p);
                    psolve_dev(c, K->Jv.p, K->z.p, skip);
                    c->tm.begin(TM_CGS, s);
                    int Ni = N;
                    ArnState* stp = K->st.p;
                    B* Ub = U;
                    size_t ldv = ld;
                    double* scp = K->scale.p;
                    const double* jvp = K->z.p;
                    const double* ew = ewt;
                    double* Wp = K->W.p;
                    double* pp = K->partial.p;
                    unsigned* bp = K->bar.p;
                    int* ep = K->err.p;
                    double* tp = K->t.p;
                    double* sgp = K->sigma.p;
                    // cooperative (grid barriers) and a programmatic dependent
                    // of the apply: its blocks take their SM slots while the
                    // apply finishes, then wait for it at entry
                    cudaLaunchConfig_t cfg = {};
                    cfg.gridDim = dim3(K->coop_grid);
                    cfg.blockDim = dim3(K->coop_threads);
                    cfg.dynamicSmemBytes = K->coop_smem;
                    cfg.stream = s;
                    cudaLaunchAttribute attr[2];
                    attr[0].id = cudaLaunchAttributeCooperative;
                    attr[0].val.cooperative = 1;
                    attr[1].id = cudaLaunchAttributeProgrammaticStreamSerialization;
                    attr[1].val.programmaticStreamSerializationAllowed = 1;
                    cfg.attrs = attr;
                    cfg.numAttrs = 2;
                    FVM_CUDA(cudaLaunchKernelEx(&cfg, k_arnoldi_cgs2<B>, Ni, stp, Ub, ldv, scp, (const double*)jvp,
                                                (const double*)ew, Wp, pp, bp, ep, tp, sgp, H_d, cs_d, sn_d, g_d));
                    c->launches++;
                    c->tm.end(TM_CGS, s);
                }
                };
                if (graph && batch == 8) {
                    // the key: everything a captured launch bakes in
                    size_t key = 1469598103934665603ull;
                    auto mix = [&](size_t v) { key = (key ^ v) * 1099511628211ull; };
                    mix((size_t)op); mix((size_t)y); mix((size_t)yp); mix((size_t)F0); mix((size_t)ewt);
                    mix((size_t)c->ilu); mix((size_t)(ilu_factored(c) + 2)); mix((size_t)c->chunk_e);
                    mix((size_t)c->recompute); mix((size_t)K->coop_grid);
                    bool ready = K->gexec && K->gkey == key;
                    if (!ready) {
                        const long l0 = c->launches, r0 = c->n_residuals;
                        cudaGraph_t g = nullptr;
                        bool ok = cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal) == cudaSuccess;
                        if (ok) {
                            try {
                                enqueue(8, true);
                            } catch (...) {
                                ok = false;
                            }
                            ok = cudaStreamEndCapture(s, &g) == cudaSuccess && ok && g;
                        }
                        K->g_launches = c->launches - l0;
                        K->g_residuals = c->n_residuals - r0;
                        c->launches = l0;
                        c->n_residuals = r0;
                        if (ok) {
                            if (K->gexec) cudaGraphExecDestroy(K->gexec);
                            K->gexec = nullptr;
                            ok = cudaGraphInstantiate(&K->gexec, g, 0) == cudaSuccess;
                        }
                        if (K->graph) cudaGraphDestroy(K->graph);
                        K->graph = g;
                        if (!ok) {
                            // launch directly from now on
                            cudaGetLastError();
                            c->graph_ok = false;
                            if (K->gexec) cudaGraphExecDestroy(K->gexec);
                            K->gexec = nullptr;
                        } else {
                            K->gkey = key;
                            c->graph_captures++;
                        }
                        ready = ok;
                    }
                    if (ready) {
                        FVM_CUDA(cudaGraphLaunch(K->gexec, s));
                        c->graph_replays++;
                        c->launches += K->g_launches;
                        c->n_residuals += K->g_residuals;
                    } else {
                        enqueue(batch, false);
                    }
                } else {
                    enqueue(batch, false);
                }
                queued += batch;
                int* herr = reinterpret_cast<int*>(K->host + 4 * (m + 2) + 7);
                FVM_CUDA(cudaMemcpyAsync(hst, K->st.p, sizeof(ArnState), cudaMemcpyDeviceToHost, s));
                FVM_CUDA(cudaMemcpyAsync(herr, K->err.p, sizeof(int), cudaMemcpyDeviceToHost, s));
                ctx_sync(c);
                if (*herr != 0) {
                    // a grid barrier gave up: the step's numbers are not valid
                    K->err.zero(s);
                    K->bar.zero(s);
                    *iters = total + hst->j;
                    *res_norm = rnorm;
                    return 2;
                }
                if (hst->done || queued >= m) break;
            }
            j = hst->j;
            total += j;
            if (!op) c->n_residuals -= queued - j;   // evaluations queued after the stop were skipped
            if (cnt) { cnt->njv += j; cnt->nps += j; }
            if (hst->done == 3) { *iters = total; *res_norm = rnorm; return 2; }
            rnorm = hst->rnorm;
            conv = hst->done == 1;
            // least-squares data of the cycle for the back substitution
            FVM_CUDA(cudaMemcpyAsync(H.data(), H_d, sizeof(double) * (size_t)(m + 1) * m, cudaMemcpyDeviceToHost, s));
            FVM_CUDA(cudaMemcpyAsync(g.data(), g_d, sizeof(double) * (m + 1), cudaMemcpyDeviceToHost, s));
            FVM_CUDA(cudaMemcpyAsync(K->host + 3 * (m + 2), K->scale.p, sizeof(double) * std::max(j, 1),
                                     cudaMemcpyDeviceToHost, s));
            ctx_sync(c);
        }
        for (; K->coop_grid == 0 && j < m; ++j) {
            // w = D P^-1 J D^-1 V_j (left preconditioning, scaled by D = ewt)
            fvm_launch(c, k_unscale<B>, grid_for(N, 256), 256, 0, s, N, U + ld * j, K->scale.p, j, ewt, K->t.p);
            if (op) jacobian_apply(c, cj, K->t.p, K->Jv.p);
            else jv_dev(c, K, cj, y, yp, F0, K->t.p, ewt, K->Jv.p);
            if (cnt) cnt->njv++;
            psolve_dev(c, K->Jv.p, K->z.p);
            if (cnt) cnt->nps++;
            int nv = j + 1;
            double* ra = K->res.p;
            double* rb = K->res.p + (m + 2);
            double* rn = K->res.p + 2 * (m + 2);
            c->tm.begin(TM_CGS, s);
            {
                fvm_launch(c, k_cgs_pass1<B>, kRedBlocks, kRedThreads, 0, s, N, nv, U, ld, K->z.p, ewt, K->W.p, K->partial.p, K->counter.p, ra);
                fvm_launch(c, k_cgs_pass2<B>, kRedBlocks, kRedThreads, 0, s, N, nv, U, ld, K->scale.p, ra, K->W.p, K->partial.p, K->counter.p, rb);
                fvm_launch(c, k_cgs_pass3<B>, kRedBlocks, kRedThreads, 0, s, N, nv, U, ld, K->scale.p, rb, K->W.p, K->partial.p, K->counter.p, rn);
                fvm_launch(c, k_set_scale, 1, 1, 0, s, rn, K->scale.p, nv);
            }
            c->tm.end(TM_CGS, s);
            FVM_CUDA(cudaMemcpyAsync(K->host, K->res.p, sizeof(double) * 3 * (m + 2), cudaMemcpyDeviceToHost, s));
            FVM_CUDA(cudaMemcpyAsync(K->host + 3 * (m + 2), K->scale.p, sizeof(double) * (nv), cudaMemcpyDeviceToHost, s));
            ctx_sync(c);
            const double* ha = K->host;
            const double* hb = K->host + (m + 2);
            const double* hsc = K->host + 3 * (m + 2);
            double hn = std::sqrt(K->host[2 * (m + 2)]);
            for (int i = 0; i < nv; ++i) hcol[i] = hsc[i] * (ha[i] + hb[i]);
            hcol[nv] = hn;
            ++total;
            if (!std::isfinite(hn)) { *iters = total; *res_norm = rnorm; return 2; }
            // apply previous rotations, then a new one (linalg_dense.c:128-173)
            for (int i = 0; i < j; ++i) {
                double t0 = cs[i] * hcol[i] + sn[i] * hcol[i + 1];
                double t1 = -sn[i] * hcol[i] + cs[i] * hcol[i + 1];
                hcol[i] = t0;
                hcol[i + 1] = t1;
            }
            double den = std::hypot(hcol[j], hcol[j + 1]);
            if (den == 0.0) { cs[j] = 1.0; sn[j] = 0.0; }
            else { cs[j] = hcol[j] / den; sn[j] = hcol[j + 1] / den; }
            hcol[j] = den;
            hcol[j + 1] = 0.0;
            g[j + 1] = -sn[j] * g[j];
            g[j] = cs[j] * g[j];
            for (int i = 0; i <= j; ++i) H[(size_t)i * m + j] = hcol[i];
            rnorm = std::fabs(g[j + 1]) / sqrtN;
            if (rnorm <= tol || hn == 0.0) { ++j; conv = true; break; }
        }
        // back substitution H y = g
        int kdim = j;
        std::vector<double> yv(kdim);
        for (int i = kdim - 1; i >= 0; --i) {
            double sacc = g[i];
            for (int l = i + 1; l < kdim; ++l) sacc -= H[(size_t)i * m + l] * yv[l];
            double d = H[(size_t)i * m + i];
            yv[i] = d != 0.0 ? sacc / d : 0.0;
        }
        // x += D^-1 sum_i y_i V_i  (scales of V_0..V_{kdim-1} are in the last
        // batch copied back)
        for (int i = 0; i < kdim; ++i) K->host[i] = yv[i] * K->host[3 * (m + 2) + i];
        FVM_CUDA(cudaMemcpyAsync(K->res.p, K->host, sizeof(double) * kdim, cudaMemcpyHostToDevice, s));
        fvm_launch(c, k_combine<B>, grid_for(N, 256), 256, 0, s, N, kdim, U, ld, K->res.p, ewt, x);
        have_x = true;
        if (conv) {
            // x is complete once the stream reaches here; a caller that reads
            // device results next on the same stream (the integrator's Newton
            // update) need not wait
            if (sync_end) ctx_sync(c);
            *iters = total;
            *res_norm = rnorm;
            return 0;
        }
    }
    ctx_sync(c);
    *iters = total;
    *res_norm = rnorm;
    return 1;
}

int gmres_dev(fvm_ctx* c, double cj, const double* y, const double* yp, const double* F0,
              const double* ewt, const double* b, double* x, int m, int max_restarts,
              int precision, double tol, int* iters, double* res_norm, GmresCounters* cnt, int op, bool sync_end) {
    if (m < 1 || m > 60) throw Error("gmres: krylov dimension must be in [1, 60]");
    Krylov* K = krylov_get(c, m, precision);
    const int r = precision
                      ? gmres_impl<float>(c, K, cj, y, yp, F0, ewt, b, x, m, max_restarts, tol, iters, res_norm, cnt, op,
                                          sync_end)
                      : gmres_impl<double>(c, K, cj, y, yp, F0, ewt, b, x, m, max_restarts, tol, iters, res_norm, cnt, op,
                                           sync_end);
    // a timed-out barrier of the Schur-coupled apply voids the solve
    if (schur_status(c)) return 2;
    return r;
}

} // namespace fvmb

using namespace fvmb;

void fvmb_destroy_krylov(fvmb::Krylov* p) { fvmb_destroy_krylov_impl(p); }

extern "C" double fvm_wrms(fvm_ctx* c, const double* x, const double* ewt) {
    try {
        if (!c || !x) throw Error("fvm_wrms: null argument");
        return std::sqrt(reduce_sumsq(c, x, ewt) / c->N);
    } catch (const std::exception& ex) {
        set_error(ex.what());
        return NAN;
    }
}

extern "C" double fvm_dot(fvm_ctx* c, const double* x, const double* y) {
    try {
        if (!c || !x || !y) throw Error("fvm_dot: null argument");
        return reduce_dot(c, x, y);
    } catch (const std::exception& ex) {
        set_error(ex.what());
        return NAN;
    }
}

extern "C" int fvm_gmres(fvm_ctx* c, double t, double cj, const double* y, const double* yp,
                         const double* F0, const double* ewt, const double* b, double* x, int m,
                         int max_restarts, int precision, double tol, int* iters, double* res_norm) {
    try {
        (void)t;
        if (!c || !y || !yp || !F0 || !ewt || !b || !x || !iters || !res_norm) throw Error("fvm_gmres: null argument");
        if (!c->ilu || !ilu_ready(c)) throw Error("fvm_gmres: call fvm_psetup first");
        int r = gmres_dev(c, cj, y, yp, F0, ewt, b, x, m, max_restarts, precision, tol, iters, res_norm, nullptr);
        FVM_CUDA(cudaGetLastError());
        return r;
    } catch (const Error& ex) {
        set_error(ex.what());
        return ex.code;
    } catch (const std::exception& ex) {
        set_error(ex.what());
        return -1;
    }
}
