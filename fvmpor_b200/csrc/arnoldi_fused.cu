// One GMRES cycle in one persistent cooperative launch, for the assembled
// Krylov operator (fvm_opts.krylov_operator = 1) with the FP32 block-ILU(0)
// factor and FP32 basis.
//
// The Arnoldi step of decomp/gmres.c:412-511 (left-preconditioned and scaled
// by D = diag(ewt), as IDAS SPGMR runs it, ida_integrator.h:248-254) is
//   w = D P^-1 J D^-1 V_j,  CGS2 against V_0..V_j,  Givens update
// (linalg_dense.c:128-173).  With J assembled (the preconditioner set-up's
// difference-quotient Jacobian, shifted exactly to the current cj), every
// part of a step is local to the rows of one ILU block except the operator's
// reads of the direction at neighbouring nodes and the orthogonalisation's
// dot products.  So one CTA owns one ILU block for the whole cycle:
//   - its factor window and metadata are brought into shared memory ONCE per
//     cycle by bulk copies (the staged apply reloads them on every apply);
//   - per step it gathers the direction at its own and its halo nodes into
//     shared memory, forms its rows of J t from there (rows in factor order,
//     one warp per 32 rows, entry-major slices with 16-bit local columns)
//     straight into the shared-memory vector the triangular sweeps work on,
//     runs both sweeps there, scales by ewt, and
//     orthogonalises its rows (by delayed reorthogonalisation in two passes
//     over the basis, or by CGS2 in three; row quads, fixed-order reductions
//     through per-block partials);
//   - every block computes the Hessenberg column, the rotations and the
//     stopping test from the same reduced numbers, so all take the same
//     decision without another barrier; block 0 writes them out for the
//     host's back substitution.
// One bounded grid barrier per step with delayed reorthogonalisation, two
// with CGS2 (after each dot pass).  The next
// direction is published block by block: a block raises its flag once its
// rows are written, and a block starting the next step waits (bounded) only
// for the flags of the blocks its operator rows reach, plus its two
// neighbours in node order.  Nothing returns to the host until the cycle
// ends.  Replaces, for this operator, the five launches per step of the
// difference-quotient path (node pass, element pass, gather, apply, CGS2).
#include "cgs.cuh"
#include "ilu.cuh"
#include "krylov.cuh"

#include <algorithm>
#include <cmath>

namespace fvmb {

struct FusedArgs {
    int N, m, nr_max, nh_max;
    int nqp;                   // quads per block row array in shared memory (quad-transposed, quad_pos)
    size_t stage_max;          // shared bytes of the largest block's staged factor
    ArnState* st;
    float* U;
    size_t ld;
    double* scale;
    float* tdir;               // D^-1 V_j, FP32, node order (read at neighbours)
    const double* ewt;
    const int* slptr;          // [slices + 1] first entry of each slice
    const int* blksl;          // [nb + 1] first slice of each block
    const unsigned short* op_lcol;   // entry -> index in the block's node list
    const unsigned short* op_self;   // [N], factor order: the row's own index there
    const int* halo_ptr;       // [nb + 1] the block's node list: its rows and halo
    const int* halo_node;
    const int* nbr_ptr;        // [nb + 1] blocks whose flags a block waits for
    const int* nbr;
    unsigned* flags;           // [nb] last step whose direction rows a block wrote
    unsigned* sync;            // arrival counter of the cycle's grid barriers (cleared with the flags)
    const float* op_val;
    const float* op_dg;        // [N], factor order: ahh(h + d) on free rows, else 0
    float dcj;                 // cj - cj of the set-up
    const int* bstart;
    const int* lu_ptr;
    const unsigned short* lu_col;
    const unsigned short* meta;
    const int* meta_off;
    const int* blk_lvl;
    const int* blk_ulvl;
    const float* lu;
    const int* lu_row;
    const double* beta2;       // ||D P^-1 r||^2 of the cycle's start
    double* partial;
    int* err;
    double* H;
    double* cs;
    double* sn;
    double* g;
};

__device__ __forceinline__ unsigned ld_acquire_gpu(const unsigned* p) {
    unsigned v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void st_release_gpu(unsigned* p, unsigned v) {
    asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
__device__ __forceinline__ unsigned atom_add_release_gpu(unsigned* p, unsigned v) {
    unsigned old;
    asm volatile("atom.add.release.gpu.global.u32 %0, [%1], %2;" : "=r"(old) : "l"(p), "r"(v) : "memory");
    return old;
}

// Grid barrier of the cycle on a counter that only grows within a launch
// (cleared with the flags before it): a block adds 1 with release semantics
// and waits (acquire, bounded) until the counter reaches the next multiple
// of the grid size.  Its own arrival number says which multiple, so there is
// no generation word, no reset and no further step for the last block to
// arrive.  A block that gives up, or meets an error elsewhere, sets
// kSyncFail (far above any count of one launch): every block sees it at its
// next barrier and leaves, and err carries the reason to the host.
constexpr unsigned kSyncFail = 1u << 30;
__device__ __forceinline__ void fused_fail(unsigned* sync, int* err, int code) {
    atomicExch(err, code);
    atomicOr(sync, kSyncFail);
}
__device__ __forceinline__ bool fused_sync(unsigned* sync, int* err, int* s_ok) {
    __syncthreads();
    if (threadIdx.x == 0) {
        const unsigned old = atom_add_release_gpu(sync, 1u);
        bool ok = !(old & kSyncFail);
        if (ok) {
            const unsigned target = (old / gridDim.x + 1) * gridDim.x;
            long it = 0;
            unsigned v;
            while ((v = ld_acquire_gpu(sync)) < target) {
                if (++it > (1l << 26)) {
                    fused_fail(sync, err, 3);
                    break;
                }
            }
            ok = v >= target && !(v & kSyncFail);
        }
        *s_ok = ok ? 1 : 0;
    }
    __syncthreads();
    return *s_ok != 0;
}

// barrier among `count` threads (whole warps) of the block on barrier `id`
__device__ __forceinline__ void named_barrier(int id, int count) {
    asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(count) : "memory");
}

// at most 384 threads (one per row quad of a 1,536-row block; larger blocks
// loop), so a thread may hold up to 170 registers
constexpr int kFusedThreads = 384;

template <int KM, bool DEL>
__global__ void __launch_bounds__(kFusedThreads, 1) k_arnoldi_fused(FusedArgs a) {
    // ca holds up to 2 (m + 1) + 2 reduced numbers on the delayed variant
    __shared__ double ca[DEL ? 132 : 64], cb[64], coef[64], sc[64], rc[64], rs[64], gs[64];
    // delayed variant: first projection of the pending column, t, p, H t and
    // the two combine coefficient sets
    __shared__ double hp[DEL ? 64 : 1], tv[DEL ? 64 : 1], pv[DEL ? 64 : 1], htv[DEL ? 64 : 1],
        c1[DEL ? 64 : 1], c2[DEL ? 64 : 1];
    // warp partials of the delayed variant's dot pass (two alternating groups)
    __shared__ double red[DEL ? 2 * (kFusedThreads / 32) * 2 * kCgsGroup : 1];
    __shared__ int s_done, s_ok;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int b = blockIdx.x, nblk = gridDim.x;
    const int r0 = a.bstart[b], r1 = a.bstart[b + 1], nr = r1 - r0;
    const IluWindow w = ilu_window(a.lu_ptr[r0], a.lu_ptr[r1]);
    const int la = a.blk_lvl[b], nl = a.blk_lvl[b + 1] - la;
    const int ua = a.blk_ulvl[b], nu = a.blk_ulvl[b + 1] - ua;
    // staged factor (the layout of k_ilu_apply_smem), then the inverse of
    // the block's row order and its rows of W
    float* x = reinterpret_cast<float*>(smem_raw);
    float* val = reinterpret_cast<float*>(smem_raw + round16(sizeof(float) * nr));
    unsigned short* col = reinterpret_cast<unsigned short*>(val + w.wn);
    unsigned short* rp = col + w.wn;
    unsigned short* dg = rp + nr + 1;
    unsigned short* lrow = dg + nr;
    unsigned short* urow = lrow + nr;
    unsigned short* lptr = urow + nr;
    unsigned short* uptr = lptr + nl + 1;
    uint64_t* mbar = reinterpret_cast<uint64_t*>(smem_raw + ilu_stage_bytes(nr, w.wn, nl + nu + 2, sizeof(float)) - 16);
    unsigned short* inv = reinterpret_cast<unsigned short*>(smem_raw + a.stage_max);
    // the block's rows of W (and of the pending vector), quad-transposed
    const int nqp = a.nqp;
    double* Ws = reinterpret_cast<double*>(smem_raw + a.stage_max + round16(2 * (size_t)a.nr_max));
    float* tl = reinterpret_cast<float*>(reinterpret_cast<unsigned char*>(Ws) + 32 * (size_t)nqp);
    // delayed variant: the block's rows of the pending vector v_k, then the
    // unrotated Hessenberg matrix (column c at Hs[64 c ..])
    double* Vs = reinterpret_cast<double*>(reinterpret_cast<unsigned char*>(tl) + round16(4 * (size_t)a.nh_max));
    double* Hs = Vs + 4 * (size_t)nqp;
    // delayed variant: the block's rows of ewt (quad-transposed, 1 in the
    // edge quads' padding), read by every step's scaling of W and of the
    // next direction instead of going to L2 for them
    double* Es = Hs + 64 * 64;
    // delayed variant: the block's node list (its rows, then its halo), for
    // the gather of every step's direction
    int* Hn = reinterpret_cast<int*>(Es + 4 * (size_t)nqp);
    if (threadIdx.x == 0) {
        tc05::mbar_init(mbar, 1);
        asm volatile("fence.mbarrier_init.release.cluster;");
    }
    __syncthreads();
    const int mo = a.meta_off[b];
    ilu_stage_bulk(val, col, a.lu, a.lu_col, w, mbar, rp, a.meta + mo, a.meta_off[b + 1] - mo);
    for (int q = threadIdx.x; q < nr; q += blockDim.x) inv[a.lu_row[r0 + q] - r0] = (unsigned short)q;
    const int m = a.m;
    const double tol = a.st->tol, sqrtN = a.st->sqrtN;
    // the cycle's initial residual norm (||D P^-1 r||, left by the host's
    // launches in a.beta2) decides whether any step is needed
    const double beta = sqrt(*a.beta2);
    const double rn0 = beta / sqrtN;
    for (int i = threadIdx.x; i <= m; i += blockDim.x) gs[i] = i == 0 ? beta : 0.0;
    // the scale of U_0 (1 / beta), also for the host's back substitution
    const double s0 = beta > 0.0 ? 1.0 / beta : 0.0;
    if (threadIdx.x == 0) {
        sc[0] = s0;
        if (b == 0) a.scale[0] = s0;
    }
    if (!isfinite(beta) || rn0 <= tol) {
        if (b == 0 && threadIdx.x == 0) {
            a.st->rnorm = rn0;
            a.st->j = 0;
            a.st->done = isfinite(beta) ? 1 : 3;
        }
        tc05::mbar_wait(mbar, 0);   // the factor copies land before the block leaves
        return;
    }
    bool ok = tc05::mbar_wait(mbar, 0);
    if (!ok) ok = tc05::mbar_wait(mbar, 0);   // copies in flight get a second bounded chance
    if (!__syncthreads_and(ok ? 1 : 0) && threadIdx.x == 0) fused_fail(a.sync, a.err, 2);   // all blocks stop at the next barrier
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
    const int sl0 = a.blksl[b], nsl = a.blksl[b + 1] - sl0;
    // vector-major partials: pa[v * nblk + b]
    double* pa = a.partial;
    double* pb = a.partial + (size_t)nblk * 64;
    // the block reads only basis rows that were complete before its last
    // barrier (its own rows; the other rows of its edge quads are masked
    // out and belong to blocks it waits for), so the read-only path is safe
    const BasisRows<float, false> UR{a.U, a.ld};
    const int q0 = r0 & ~3;
    const int h0 = a.halo_ptr[b], nh = a.halo_ptr[b + 1] - h0;
    const int nb0 = a.nbr_ptr[b], nb1 = a.nbr_ptr[b + 1];
    // step 0's direction s_0 U_0 / ewt at the block's own and halo nodes
    // (U_0 was written before the launch)
    for (int k = threadIdx.x; k < nh; k += blockDim.x) {
        const int node = a.halo_node[h0 + k];
        if constexpr (DEL) Hn[k] = node;
        tl[k] = (float)(s0 * (double)__ldcg(a.U + node) / a.ewt[node]);
    }
    // the padding rows of the edge quads stay zero
    for (int k = threadIdx.x; k < 4 * nqp; k += blockDim.x) {
        Ws[k] = 0.0;
        if constexpr (DEL) {
            Vs[k] = 0.0;
            const int e = k / nqp, row = (r0 & ~3) + 4 * (k - e * nqp) + e;   // inverse of quad_pos
            Es[k] = row >= r0 && row < r1 ? a.ewt[row] : 1.0;
        }
    }
    __syncthreads();
    for (int j = 0;; ++j) {
        const int nv = j + 1;
        // operator: x = J(cj) t for the block's rows, in factor order; a
        // warp takes two slices at a time, eight entries of each in flight
        for (int sl = warp; sl < nsl; sl += 2 * nw) {
            const int slb = sl + nw < nsl ? sl + nw : sl;
            const int ea = a.slptr[sl0 + sl] + lane, ea1 = a.slptr[sl0 + sl + 1];
            const int eb = a.slptr[sl0 + slb] + lane, eb1 = slb != sl ? a.slptr[sl0 + slb + 1] : eb;
            float acc_a = 0.f, acc_b = 0.f;
            for (int k = 0; ea + 32 * k < ea1 || eb + 32 * k < eb1; k += 8) {
                float va[8], vb[8];
                unsigned short ca_[8], cb_[8];
#pragma unroll
                for (int t = 0; t < 8; ++t) {
                    const int e = ea + 32 * (k + t), f = eb + 32 * (k + t);
                    // streamed once per step through L2 only, so that L1
                    // keeps the block's basis rows between the passes
                    va[t] = e < ea1 ? __ldcg(a.op_val + e) : 0.f;
                    ca_[t] = e < ea1 ? __ldcg(a.op_lcol + e) : (unsigned short)0;
                    vb[t] = f < eb1 ? __ldcg(a.op_val + f) : 0.f;
                    cb_[t] = f < eb1 ? __ldcg(a.op_lcol + f) : (unsigned short)0;
                }
#pragma unroll
                for (int t = 0; t < 8; ++t) {
                    acc_a = fmaf(va[t], tl[ca_[t]], acc_a);
                    acc_b = fmaf(vb[t], tl[cb_[t]], acc_b);
                }
            }
            const int qa = 32 * sl + lane, qb = 32 * slb + lane;
            if (qa < nr) x[qa] = fmaf(-a.dcj * a.op_dg[r0 + qa], tl[a.op_self[r0 + qa]], acc_a);
            if (slb != sl && qb < nr) x[qb] = fmaf(-a.dcj * a.op_dg[r0 + qb], tl[a.op_self[r0 + qb]], acc_b);
        }
        __syncthreads();
        // preconditioner: both triangular sweeps in shared memory
        ilu_sweep<float, KM, false>(x, val, col, rp, dg, lrow, lptr, 1, nl);
        ilu_sweep<float, KM, true>(x, val, col, rp, dg, urow, uptr, 0, nu);
        for (int k = threadIdx.x; k < nr; k += blockDim.x) {
            const int qp = quad_pos(r0, nqp, r0 + k);
            Ws[qp] = (DEL ? Es[qp] : a.ewt[r0 + k]) * (double)x[inv[k]];
        }
        __syncthreads();
        // Hessenberg column finalised by this step (-1: none yet), the entry
        // below its diagonal, and the scale of the basis vector it finalises
        int hcol = j;
        double hn = 0.0;
        double newscale = 0.0;
        if constexpr (!DEL) {
        // pass 1: a = U^T W
        block_dots_by_warp(a.U, a.ld, Ws, nqp, r0, r1, nv, false, ca);
        for (int i = threadIdx.x; i < nv; i += blockDim.x) pa[(size_t)i * nblk + b] = ca[i];
        if (!fused_sync(a.sync, a.err, &s_ok)) return;
        block_reduce_all_vmajor(pa, nv, nblk, ca);
        for (int i = threadIdx.x; i < nv; i += blockDim.x) coef[i] = ca[i] * sc[i] * sc[i];
        __syncthreads();
        // pass 2: W' = W - U diag(s^2) a; b = U^T W', ||W'||^2
        for (int r = q0 + 4 * threadIdx.x; r < r1; r += 4 * blockDim.x) {
            double acc[4];
            quad_combine(UR, coef, nv, r, acc);
#pragma unroll
            for (int e = 0; e < 4; ++e)
                if (r + e >= r0 && r + e < r1) Ws[quad_pos(r0, nqp, r + e)] -= acc[e];
        }
        __syncthreads();
        block_dots_by_warp(a.U, a.ld, Ws, nqp, r0, r1, nv, true, cb);
        for (int i = threadIdx.x; i <= nv; i += blockDim.x) pb[(size_t)i * nblk + b] = cb[i];
        if (!fused_sync(a.sync, a.err, &s_ok)) return;
        block_reduce_all_vmajor(pb, nv + 1, nblk, cb);
        double nrm2 = cb[nv];
        for (int i = 0; i < nv; ++i) {
            const double c = sc[i] * cb[i];
            nrm2 -= c * c;
        }
        nrm2 = nrm2 > 0.0 ? nrm2 : 0.0;
        const double snv = nrm2 > 0.0 ? 1.0 / sqrt(nrm2) : 0.0;
        for (int i = threadIdx.x; i < nv; i += blockDim.x) coef[i] = cb[i] * sc[i] * sc[i];
        __syncthreads();
        // pass 3: the new basis vector (unnormalised, scale snv) and the
        // next direction D^-1 V_{j+1}
        float* Un = a.U + a.ld * nv;
        for (int r = q0 + 4 * threadIdx.x; r < r1; r += 4 * blockDim.x) {
            double acc[4];
            quad_combine(UR, coef, nv, r, acc);
#pragma unroll
            for (int e = 0; e < 4; ++e) {
                const int k = r + e;
                if (k >= r0 && k < r1) {
                    const float u = (float)(Ws[quad_pos(r0, nqp, k)] - acc[e]);
                    Un[k] = u;
                    a.tdir[k] = (float)(snv * (double)u / a.ewt[k]);
                }
            }
        }
        // the Hessenberg column of the two projections
        for (int i = threadIdx.x; i < nv; i += blockDim.x) ca[i] = sc[i] * (ca[i] + cb[i]);
        hn = sqrt(nrm2);
        newscale = snv;
        } else {
        // Delayed reorthogonalisation (DCGS2: Swirydowicz, Langou, Ananthan,
        // Yang & Thomas, Numer. Linear Algebra Appl. 28 (2021) e2343).  The
        // step's direction is v_k, the previous step's vector after one
        // projection; z = A v_k.  One pass over the basis gives
        // t = V^T v_k, p = V^T z, v_k.v_k and v_k.z, one grid barrier reduces
        // them.  Then q_k = (v_k - V t) / beta with beta^2 = v.v - t.t
        // finalises column k-1 of H (first projection of step k-1 plus t,
        // and beta below it); A q_k = (z - V_k H t) / beta by the Arnoldi
        // relation, so its first projection s and the next vector
        // v_{k+1} = A q_k - V_k s follow from the reduced numbers, and one
        // more pass over the basis writes both q_k (as U_k, scale 1/beta)
        // and v_{k+1}.  Two passes and one barrier per step instead of
        // four and two; the column of step k is final one step later.
        const int k = j;
        const int nbv = k == 0 ? 1 : k;   // basis vectors this step reads
        float4 kept[kCgsGroup];
        block_dots2_by_quad(a.U, a.ld, Vs, Ws, nqp, r0, r1, nbv, red, ca, kept);
        const int nred = 2 * nbv + 2;
        for (int i = threadIdx.x; i < nred; i += blockDim.x) pa[(size_t)i * nblk + b] = ca[i];
        if (!fused_sync(a.sync, a.err, &s_ok)) return;
        block_reduce_all_vmajor(pa, nred, nblk, ca);
        double beta = 1.0, ck = 0.0;
        if (k == 0) {
            // v_1 = z - V_0 p_0
            if (threadIdx.x == 0) {
                const double p0 = sc[0] * ca[1];
                hp[0] = p0;
                c1[0] = 0.0;
                c2[0] = sc[0] * p0;
            }
            hcol = -1;
        } else {
            double tt = 0.0;
            for (int i = 0; i < k; ++i) {
                const double t = sc[i] * ca[i];
                tt += t * t;
            }
            const double b2 = ca[2 * k] - tt;
            beta = b2 > 0.0 ? sqrt(b2) : 0.0;
            for (int i = threadIdx.x; i <= k; i += blockDim.x) {
                const double t = i < k ? sc[i] * ca[i] : 0.0;
                tv[i] = t;
                pv[i] = i < k ? sc[i] * ca[k + i] : 0.0;
                Hs[(size_t)(k - 1) * 64 + i] = i < k ? hp[i] + t : beta;
            }
            __syncthreads();
            // Ht = H[0..k][0..k-1] t (H[i][c] is zero below c + 1)
            for (int i = threadIdx.x; i <= k; i += blockDim.x) {
                double acc = 0.0;
                for (int c = i > 0 ? i - 1 : 0; c < k; ++c) acc += Hs[(size_t)c * 64 + i] * tv[c];
                htv[i] = acc;
            }
            __syncthreads();
            double tp = 0.0;
            for (int i = 0; i < k; ++i) tp += tv[i] * pv[i];
            const double rb = beta > 0.0 ? 1.0 / beta : 0.0;
            const double sk = (ca[2 * k + 1] - tp - beta * htv[k]) * rb * rb;
            ck = htv[k] * rb + sk;
            for (int i = threadIdx.x; i < k; i += blockDim.x) {
                const double si = (pv[i] - htv[i]) * rb;
                c1[i] = sc[i] * tv[i];
                c2[i] = sc[i] * (htv[i] * rb + si - ck * tv[i] * rb);
                hp[i] = si;
            }
            if (threadIdx.x == 0) {
                hp[k] = sk;
                sc[k] = rb;
            }
            hcol = k - 1;
            hn = beta;
            newscale = rb;
        }
        __syncthreads();
        // q_k = v_k - V t (k >= 1), v_{k+1} = z / beta - (c_k / beta) v_k - V c2,
        // and the next direction D^-1 v_{k+1}
        {
            float* Uk = a.U + a.ld * k;
            const double rb = k == 0 ? 1.0 : (beta > 0.0 ? 1.0 / beta : 0.0);
            const double vcoef = k == 0 ? 0.0 : ck * rb;
            for (int r = q0 + 4 * threadIdx.x; r < r1; r += 4 * blockDim.x) {
                double acc1[4], acc2[4];
                if (r == q0 + 4 * (int)threadIdx.x) quad_combine2_kept(UR, c1, c2, nbv, r, kept, acc1, acc2);
                else quad_combine2(UR, c1, c2, nbv, r, acc1, acc2);
#pragma unroll
                for (int e = 0; e < 4; ++e) {
                    const int q = r + e;
                    if (q >= r0 && q < r1) {
                        const int qp = quad_pos(r0, nqp, q);
                        const double vq = Vs[qp];
                        if (k >= 1) Uk[q] = (float)(vq - acc1[e]);
                        const double vn = Ws[qp] * rb - vcoef * vq - acc2[e];
                        Vs[qp] = vn;
                        a.tdir[q] = (float)(vn / Es[qp]);
                    }
                }
            }
        }
        }
        // publish this block's rows of the next direction
        __syncthreads();
        if (threadIdx.x == 0) st_release_gpu(a.flags + b, (unsigned)nv);   // release: the block's writes before the barrier
        __syncthreads();
        // rotations and stopping test for the finalised column, the same in
        // every block (the same reduced numbers, the same operations), on
        // thread 0 while the other warps wait for the next direction's rows
        // this block reads (bounded) and gather them into shared memory
        if (warp > 0) {
            if (warp == 1) {
                for (int kk = nb0 + lane; kk < nb1; kk += 32) {
                    const unsigned* f = a.flags + a.nbr[kk];
                    long it = 0;
                    while (ld_acquire_gpu(f) < (unsigned)nv) {
                        if (++it > (1l << 26)) { fused_fail(a.sync, a.err, 3); break; }
                    }
                }
            }
            named_barrier(1, blockDim.x - 32);
            for (int kk = threadIdx.x - 32; kk < nh; kk += blockDim.x - 32)
                tl[kk] = __ldcg(a.tdir + (DEL ? Hn[kk] : a.halo_node[h0 + kk]));
        } else if (threadIdx.x == 0) {
            int done = 0;
            if (hcol >= 0) {
                double* hc = ca;
                if constexpr (DEL) {
                    for (int i = 0; i <= hcol; ++i) hc[i] = Hs[(size_t)hcol * 64 + i];
                }
                hc[hcol + 1] = hn;
                if (!isfinite(hn) || !isfinite(hc[hcol])) {
                    done = 3;
                } else {
                    double cur = hc[0];
                    for (int i = 0; i < hcol; ++i) {
                        const double nx = hc[i + 1];
                        hc[i] = rc[i] * cur + rs[i] * nx;
                        cur = -rs[i] * cur + rc[i] * nx;
                    }
                    hc[hcol] = cur;
                    const double den = hypot(hc[hcol], hc[hcol + 1]);
                    double cj_, sj_;
                    if (den == 0.0) { cj_ = 1.0; sj_ = 0.0; }
                    else { cj_ = hc[hcol] / den; sj_ = hc[hcol + 1] / den; }
                    rc[hcol] = cj_;
                    rs[hcol] = sj_;
                    hc[hcol] = den;
                    const double gj = gs[hcol];
                    gs[hcol + 1] = -sj_ * gj;
                    gs[hcol] = cj_ * gj;
                    sc[hcol + 1] = newscale;
                    const double rn = fabs(gs[hcol + 1]) / sqrtN;
                    if (rn <= tol || hn == 0.0) done = 1;
                    else if (hcol + 1 == m) done = 2;
                    if (b == 0) {
                        for (int i = 0; i <= hcol; ++i) a.H[(size_t)i * m + hcol] = hc[i];
                        a.cs[hcol] = cj_;
                        a.sn[hcol] = sj_;
                        a.g[hcol] = gs[hcol];
                        a.g[hcol + 1] = gs[hcol + 1];
                        a.scale[hcol + 1] = newscale;
                        a.st->rnorm = rn;
                        a.st->j = hcol + 1;
                    }
                }
            }
            if (b == 0) a.st->done = done;
            s_done = done;
        }
        __syncthreads();
        if (s_done) return;
    }
}

static int fused_sync_slot(int nb) { return ((nb + 31) & ~31) + 32; }

static const void* fused_kernel(int lanes, int variant) {
    if (lanes == 8) return variant ? (const void*)k_arnoldi_fused<8, true> : (const void*)k_arnoldi_fused<8, false>;
    return variant ? (const void*)k_arnoldi_fused<4, true> : (const void*)k_arnoldi_fused<4, false>;
}

// Gram-Schmidt of the fused cycle on this context: 0 CGS2 (two projections,
// two grid barriers per step), 1 delayed reorthogonalisation (DCGS2)
static int fused_variant(const fvm_ctx* c) { return c->krylov_variant ? 1 : 0; }

// values of the operator's slices from the set-up's Jacobian (FP64 CSR) and
// the cj coefficient of its diagonal, in factor order
__global__ void k_op_refresh(long ne, const int* __restrict__ src, const double* __restrict__ J, float* __restrict__ v,
                             int N, const int* __restrict__ lu_row, const double* __restrict__ ahhp,
                             const unsigned char* __restrict__ ntype, float* __restrict__ dgq) {
    const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t < ne) {
        const int p = src[t];
        v[t] = p >= 0 ? (float)J[p] : 0.f;
    }
    if (t < N) {
        const int row = lu_row[t];
        dgq[t] = ntype[row] ? 0.f : (float)ahhp[row];
    }
}

// Host side: the slice layout (once per pattern), the launch checks, and the
// per-set-up refresh.  Returns false when the fused cycle cannot run on this
// context (FP32 staged factor does not fit, or the blocks cannot all be
// resident at once); the caller then uses the separate kernels.
bool fused_prepare(fvm_ctx* c, int m) {
    BlockILU* P = c->ilu;
    // the cycle inlines the block-Jacobi apply; the Schur-coupled apply
    // runs as its own cooperative launch between the separate kernels
    if (!P || !P->built || P->factored != 1 || m + 2 > 64 || P->schur_iters >= 0) return false;
    cudaStream_t s = c->stream;
    if (!P->op_built) {
        P->op_built = true;
        P->fused_ok = false;
        const int nb = P->nb;
        if (!P->smem_stage[1]) return false;
        std::vector<int> slptr(1, 0), blksl(1, 0), opcol, opsrc;
        std::vector<int> halo_ptr(1, 0), halo_node, nbr_ptr(1, 0), nbr;
        std::vector<unsigned short> lcol, self(c->N);
        std::vector<int> where(c->N, -1);
        int nr_max = 0, nh_max = 0;
        for (int b = 0; b < nb; ++b) {
            const int r0 = P->h_bstart[b], r1 = P->h_bstart[b + 1];
            nr_max = std::max(nr_max, r1 - r0);
            const size_t ebase = opcol.size();
            for (int q0 = r0; q0 < r1; q0 += 32) {
                const int n = std::min(32, r1 - q0);
                int width = 0;
                for (int l = 0; l < n; ++l) {
                    const int row = P->h_lu_row[q0 + l];
                    width = std::max(width, P->h_rowptr[row + 1] - P->h_rowptr[row]);
                }
                const size_t base = opcol.size();
                opcol.resize(base + 32 * (size_t)width);
                opsrc.resize(base + 32 * (size_t)width);
                for (int l = 0; l < 32; ++l) {
                    const int row = l < n ? P->h_lu_row[q0 + l] : P->h_lu_row[q0];
                    const int p0 = P->h_rowptr[row], len = l < n ? P->h_rowptr[row + 1] - p0 : 0;
                    for (int k = 0; k < width; ++k) {
                        opcol[base + 32 * (size_t)k + l] = k < len ? P->h_col[p0 + k] : row;
                        opsrc[base + 32 * (size_t)k + l] = k < len ? p0 + k : -1;
                    }
                }
                if (opcol.size() >= (size_t)INT32_MAX) return false;
                slptr.push_back((int)opcol.size());
            }
            blksl.push_back((int)slptr.size() - 1);
            // the block's node list (its operator columns, sorted), local
            // column indices, and the blocks owning those nodes
            std::vector<int> nodes(opcol.begin() + ebase, opcol.end());
            std::sort(nodes.begin(), nodes.end());
            nodes.erase(std::unique(nodes.begin(), nodes.end()), nodes.end());
            if (nodes.size() >= 65535) return false;
            nh_max = std::max(nh_max, (int)nodes.size());
            for (size_t k = 0; k < nodes.size(); ++k) where[nodes[k]] = (int)k;
            for (size_t e = ebase; e < opcol.size(); ++e) lcol.push_back((unsigned short)where[opcol[e]]);
            for (int q = r0; q < r1; ++q) self[q] = (unsigned short)where[P->h_lu_row[q]];
            std::vector<int> nbs;
            if (b > 0) nbs.push_back(b - 1);
            if (b + 1 < nb) nbs.push_back(b + 1);
            for (int v : nodes) {
                const int ob = (int)(std::upper_bound(P->h_bstart.begin(), P->h_bstart.end(), v) - P->h_bstart.begin()) - 1;
                if (ob != b) nbs.push_back(ob);
            }
            std::sort(nbs.begin(), nbs.end());
            nbs.erase(std::unique(nbs.begin(), nbs.end()), nbs.end());
            nbr.insert(nbr.end(), nbs.begin(), nbs.end());
            nbr_ptr.push_back((int)nbr.size());
            halo_node.insert(halo_node.end(), nodes.begin(), nodes.end());
            halo_ptr.push_back((int)halo_node.size());
            for (int v : nodes) where[v] = -1;
        }
        P->op_slptr.upload(slptr, s);
        P->op_blksl.upload(blksl, s);
        P->op_lcol.upload(lcol, s);
        P->op_self.upload(self, s);
        P->op_src.upload(opsrc, s);
        {
            // the slice position of every Jacobian entry, for fd_gather
            std::vector<int> opdst(P->nnz, 0);
            for (size_t e = 0; e < opsrc.size(); ++e)
                if (opsrc[e] >= 0) opdst[opsrc[e]] = (int)e;
            P->op_dst.upload(opdst, s);
        }
        P->halo_ptr.upload(halo_ptr, s);
        P->halo_node.upload(halo_node, s);
        P->nbr_ptr.upload(nbr_ptr, s);
        P->nbr.upload(nbr, s);
        // the blocks' flags, then the barrier counter on its own 128-byte line
        P->flags.alloc(fused_sync_slot(nb) + 32);
        P->op_val.alloc(opcol.size());
        P->op_val.zero(s);   // the padding entries stay zero
        P->op_dg.alloc(c->N);
        P->fused_nrmax = nr_max;
        P->fused_nhmax = nh_max;
        P->fused_stage = round16(P->smem_stage[1]);
        // CGS2: staged factor | row order | rows of W | direction at the
        // block's nodes; the delayed variant adds the pending vector's rows
        // and the unrotated Hessenberg matrix (64 x 64), then the block's
        // rows of ewt and its node list
        // block row arrays quad-transposed: nqp quads cover any block's rows
        // from its first quad boundary
        P->fused_nqp = nr_max / 4 + 2;
        const size_t rows = 32 * (size_t)P->fused_nqp;
        const size_t base = P->fused_stage + round16(2 * (size_t)nr_max) + rows;
        P->fused_smem = base + 4 * (size_t)nh_max;
        P->fused_smem_d = base + round16(4 * (size_t)nh_max) + rows + 8 * 64 * 64 + rows + round16(4 * (size_t)nh_max);
        // one thread per row quad of the largest block, whole warps
        P->fused_threads = std::min(kFusedThreads, std::max(128, ((nr_max + 3) / 4 + 1 + 31) / 32 * 32));
        int dev = 0, coop = 0, nsm = 0;
        FVM_CUDA(cudaGetDevice(&dev));
        FVM_CUDA(cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, dev));
        FVM_CUDA(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
        for (int v = 0; v < 2; ++v) {
            const size_t smem = v ? P->fused_smem_d : P->fused_smem;
            P->fused_var_ok[v] = false;
            if (smem > kMaxDynSmem) continue;
            const void* kfn = fused_kernel(P->lanes, v);
            raise_smem_limit(kfn, smem);
            // the smallest shared-memory carveout that holds the block's
            // shared data (dynamic + static, about 1 KB reserved), so that
            // the rest of the SM's 256 KB stays L1 for the block's basis rows
            cudaFuncAttributes fa;
            FVM_CUDA(cudaFuncGetAttributes(&fa, kfn));
            const double need = (double)(smem + fa.sharedSizeBytes + 1024);
            const int pct = std::min(100, (int)std::ceil(100.0 * need / (228.0 * 1024.0)));
            FVM_CUDA(cudaFuncSetAttribute(kfn, cudaFuncAttributePreferredSharedMemoryCarveout, pct));
            int per_sm = 0;
            FVM_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kfn, P->fused_threads, smem));
            P->fused_var_ok[v] = coop && per_sm > 0 && nb <= per_sm * nsm;
        }
        P->fused_ok = P->fused_var_ok[0] || P->fused_var_ok[1];
    }
    if (!P->fused_ok || !P->fused_var_ok[fused_variant(c)]) return false;
    if (P->op_setup_id != P->setup_id) {
        // the values come from fd_gather once the layout exists; the first
        // set-up after the layout was built copies them here
        const long ne = P->op_vals_setup == P->setup_id ? 0 : (long)P->op_val.n;
        const long nt = std::max(ne, (long)c->N);
        fvm_launch(c, k_op_refresh, grid_for(nt, 256), 256, 0, s, ne, P->op_src.p, P->J.p, P->op_val.p, c->N,
                   P->lu_row.p, P->ahhp.p, c->ntype.p, P->op_dg.p);
        P->op_setup_id = P->setup_id;
    }
    return true;
}

// one cycle: the Arnoldi state (j = 0), g[0] and U_0 with its scale are in
// place; runs until convergence, a full basis or a breakdown
void fused_cycle(fvm_ctx* c, Krylov* K, double cj, const double* ewt, double* H_d, double* cs_d, double* sn_d,
                 double* g_d) {
    BlockILU* P = c->ilu;
    cudaStream_t s = c->stream;
    float* U = reinterpret_cast<float*>(K->U);
    if (K->tdir.n < (size_t)c->N) K->tdir.alloc(c->N);
    FusedArgs a;
    a.N = c->N;
    a.m = K->m;
    a.nr_max = P->fused_nrmax;
    a.nqp = P->fused_nqp;
    a.nh_max = P->fused_nhmax;
    a.stage_max = P->fused_stage;
    a.st = K->st.p;
    a.U = U;
    a.ld = K->ld;
    a.scale = K->scale.p;
    a.tdir = K->tdir.p;
    a.ewt = ewt;
    a.slptr = P->op_slptr.p;
    a.blksl = P->op_blksl.p;
    a.op_lcol = P->op_lcol.p;
    a.op_self = P->op_self.p;
    a.halo_ptr = P->halo_ptr.p;
    a.halo_node = P->halo_node.p;
    a.nbr_ptr = P->nbr_ptr.p;
    a.nbr = P->nbr.p;
    a.flags = P->flags.p;
    a.sync = P->flags.p + fused_sync_slot(P->nb);
    a.op_val = P->op_val.p;
    a.op_dg = P->op_dg.p;
    a.dcj = (float)(cj - P->cj_setup);
    a.bstart = P->bstart.p;
    a.lu_ptr = P->lu_ptr.p;
    a.lu_col = P->lu_col.p;
    a.meta = P->meta.p;
    a.meta_off = P->meta_off.p;
    a.blk_lvl = P->blk_lvl.p;
    a.blk_ulvl = P->blk_ulvl.p;
    a.lu = P->lu32.p;
    a.lu_row = P->lu_row.p;
    a.beta2 = K->res.p;
    a.partial = K->partial.p;
    a.err = K->err.p;
    a.H = H_d;
    a.cs = cs_d;
    a.sn = sn_d;
    a.g = g_d;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(P->nb);
    cfg.blockDim = dim3(P->fused_threads);
    const int var = fused_variant(c);
    cfg.dynamicSmemBytes = var ? P->fused_smem_d : P->fused_smem;
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    P->flags.zero(s);
    c->tm.begin(TM_CGS, s);
    if (P->lanes == 8) {
        if (var) FVM_CUDA(cudaLaunchKernelEx(&cfg, k_arnoldi_fused<8, true>, a));
        else FVM_CUDA(cudaLaunchKernelEx(&cfg, k_arnoldi_fused<8, false>, a));
    } else {
        if (var) FVM_CUDA(cudaLaunchKernelEx(&cfg, k_arnoldi_fused<4, true>, a));
        else FVM_CUDA(cudaLaunchKernelEx(&cfg, k_arnoldi_fused<4, false>, a));
    }
    c->tm.end(TM_CGS, s);
    c->launches++;
}

} // namespace fvmb
