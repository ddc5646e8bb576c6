// Preconditioner: coloured finite-difference Jacobian + block-ILU(0).
//
// Set-up follows Preconditioner::setup (examples/fvmporMinlin/
// preconditioner_dss.cpp:284-373): the node-graph pattern of
// column_pattern (:107-142), the greedy distance-2 colouring of
// sequential_vertex_colouring (:61-94, neighbourhoods from
// dependent_columns :36-59), the shift
//   d_j = sqrt(eps) * max(|y_j|, |h y'_j|, 1 / w_j)          (:322-329)
// and one perturbed residual per colour (y + d on the colour's columns,
// y' + cj d) to fill J = dF/dy + cj dF/dy' column group by column group.
// The reference stores (F0 - F_shift)/d = -J; here the values are
// (F_shift - F0)/d = +J.  GMRES with a right preconditioner is unaffected
// by the sign of P, which the tests check.
//
// The reference factors that matrix with MKL DSS on the host (:368) and
// solves on the host with two PCIe copies per apply (:375-405).  Here it is
// factored on the device with ILU(0) restricted to diagonal blocks of
// contiguous node ranges (block Jacobi ILU(0), the local B_i factor of
// decomp/schur.c:887-987 without the interface Schur system).  The
// factorisation is the row-wise IKJ ILU(0) of decomp/ILU.c:12-115 with the
// pivot of row i inverted after row i is eliminated (the block branch,
// :105-107; the scalar branch at :65 indexes the pivot by the last column
// k instead of i, which is an upstream slip and not reproduced).  One CTA
// owns one block; rows are processed by dependency levels (rows of one
// level only depend on rows of earlier levels), with a barrier between
// levels, for both the factorisation and the triangular solves
// (decomp/ILU.c:133-223).
#include "ctx.cuh"
#include "krylov.cuh"

#include <algorithm>
#include <cfloat>
#include <cmath>

namespace fvmb {

struct BlockILU {
    bool built = false;
    int nnz = 0, ncol = 0;
    std::vector<int> h_rowptr, h_col, h_cptr, h_colour;
    DevBuf<int> rowof, col;
    DevBuf<double> J;
    DevBuf<int> colour, cnnz;
    DevBuf<double> shift, Fc;
    int nb = 0, maxb = 0;
    DevBuf<int> bstart, lu_ptr, lu_src, lu_diag;
    DevBuf<unsigned short> lu_col;
    DevBuf<int> lvl_ptr, lvl_rows, blk_lvl, ulvl_ptr, ulvl_rows, blk_ulvl;
    DevBuf<double> lu64;
    DevBuf<float> lu32;
    int factored = -1;        // precision of the current factor, -1 none
    DevBuf<int> status;
    int* h_status = nullptr;  // pinned
    int nlevels_max = 0;
    size_t smem_stage[2] = {0, 0};   // staged apply: shared bytes for FP64 / FP32, 0 = not possible
};

// largest dynamic shared-memory carve-out a CTA may request on sm_100
constexpr size_t kMaxDynSmem = 227 * 1024;

// ------------------------------------------------------------------ kernels
__global__ void k_shift(int N, const double* __restrict__ y, const double* __restrict__ yp,
                        const double* __restrict__ ewt, double h, double eps,
                        double* __restrict__ shift) {
    int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= N) return;
    double a = fabs(y[j]), b = fabs(h * yp[j]), w = 1.0 / ewt[j];
    shift[j] = eps * fmax(a, fmax(b, w));
}

__global__ void k_fd_scatter(int count, const int* __restrict__ list, const int* __restrict__ rowof,
                             const int* __restrict__ col, const double* __restrict__ Fc,
                             const double* __restrict__ F0, const double* __restrict__ shift,
                             double* __restrict__ J) {
    int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= count) return;
    int p = list[q];
    int i = rowof[p], j = col[p];
    J[p] = (Fc[i] - F0[i]) / shift[j];
}

template <class T>
__global__ void __launch_bounds__(128) k_ilu_factor(const int* __restrict__ bstart,
                                                    const int* __restrict__ lu_ptr,
                                                    const int* __restrict__ lu_src,
                                                    const int* __restrict__ lu_diag,
                                                    const unsigned short* __restrict__ lu_col,
                                                    const int* __restrict__ lvl_ptr,
                                                    const int* __restrict__ lvl_rows,
                                                    const int* __restrict__ blk_lvl,
                                                    const double* __restrict__ J, T* lu,
                                                    int* status) {
    int b = blockIdx.x;
    int r0 = bstart[b], r1 = bstart[b + 1];
    for (int p = lu_ptr[r0] + threadIdx.x; p < lu_ptr[r1]; p += blockDim.x) lu[p] = (T)J[lu_src[p]];
    __syncthreads();
    for (int l = blk_lvl[b]; l < blk_lvl[b + 1]; ++l) {
        for (int q = lvl_ptr[l] + threadIdx.x; q < lvl_ptr[l + 1]; q += blockDim.x) {
            int i = lvl_rows[q];
            int s = lu_ptr[i], e = lu_ptr[i + 1], di = lu_diag[i];
            for (int kk = s; kk < di; ++kk) {
                int k = r0 + lu_col[kk];
                T lik = lu[kk] * lu[lu_diag[k]];
                lu[kk] = lik;
                int kpos = lu_diag[k] + 1, kend = lu_ptr[k + 1];
                for (int jj = kk + 1; jj < e && kpos < kend; ++jj) {
                    int j = lu_col[jj];
                    while (kpos < kend && lu_col[kpos] < j) ++kpos;
                    if (kpos < kend && lu_col[kpos] == j) lu[jj] = lu[jj] - lik * lu[kpos];
                }
            }
            T d = lu[di];
            if (d == (T)0 || !isfinite((double)d)) {
                atomicExch(status, 1);
                d = (T)1;
            }
            lu[di] = (T)1 / d;
        }
        __syncthreads();
    }
}

template <class T>
__global__ void __launch_bounds__(128) k_ilu_apply(const int* __restrict__ bstart,
                                                   const int* __restrict__ lu_ptr,
                                                   const int* __restrict__ lu_diag,
                                                   const unsigned short* __restrict__ lu_col,
                                                   const int* __restrict__ lvl_ptr,
                                                   const int* __restrict__ lvl_rows,
                                                   const int* __restrict__ blk_lvl,
                                                   const int* __restrict__ ulvl_ptr,
                                                   const int* __restrict__ ulvl_rows,
                                                   const int* __restrict__ blk_ulvl,
                                                   const T* __restrict__ lu,
                                                   const double* __restrict__ r,
                                                   double* __restrict__ z) {
    extern __shared__ unsigned char smem_raw[];
    T* x = reinterpret_cast<T*>(smem_raw);
    int b = blockIdx.x;
    int r0 = bstart[b], r1 = bstart[b + 1];
    for (int i = r0 + threadIdx.x; i < r1; i += blockDim.x) x[i - r0] = (T)r[i];
    __syncthreads();
    // forward: unit lower triangle
    for (int l = blk_lvl[b] + 1; l < blk_lvl[b + 1]; ++l) {
        for (int q = lvl_ptr[l] + threadIdx.x; q < lvl_ptr[l + 1]; q += blockDim.x) {
            int i = lvl_rows[q];
            T acc = x[i - r0];
            for (int p = lu_ptr[i]; p < lu_diag[i]; ++p) acc -= lu[p] * x[lu_col[p]];
            x[i - r0] = acc;
        }
        __syncthreads();
    }
    // backward: upper triangle with inverted pivots
    for (int l = blk_ulvl[b]; l < blk_ulvl[b + 1]; ++l) {
        for (int q = ulvl_ptr[l] + threadIdx.x; q < ulvl_ptr[l + 1]; q += blockDim.x) {
            int i = ulvl_rows[q];
            int di = lu_diag[i];
            T acc = x[i - r0];
            for (int p = di + 1; p < lu_ptr[i + 1]; ++p) acc -= lu[p] * x[lu_col[p]];
            x[i - r0] = acc * lu[di];
        }
        __syncthreads();
    }
    for (int i = r0 + threadIdx.x; i < r1; i += blockDim.x) z[i] = (double)x[i - r0];
}

// Staged variant: the CTA first copies its block's factor (values, local
// column indices, row pointers, pivot positions) and right-hand side into
// shared memory with coalesced loads, then runs the level loops entirely in
// shared memory, so each level costs a few shared-memory latencies and a
// barrier instead of a dependent chain of L2/HBM loads.
// Shared layout: x[T nrows] | val[T nnz] | col[u16 nnz] | rp[u16 nrows+1] |
// dg[u16 nrows]
template <class T>
__global__ void __launch_bounds__(256) k_ilu_apply_smem(const int* __restrict__ bstart,
                                                        const int* __restrict__ lu_ptr,
                                                        const int* __restrict__ lu_diag,
                                                        const unsigned short* __restrict__ lu_col,
                                                        const int* __restrict__ lvl_ptr,
                                                        const int* __restrict__ lvl_rows,
                                                        const int* __restrict__ blk_lvl,
                                                        const int* __restrict__ ulvl_ptr,
                                                        const int* __restrict__ ulvl_rows,
                                                        const int* __restrict__ blk_ulvl,
                                                        const T* __restrict__ lu,
                                                        const double* __restrict__ r,
                                                        double* __restrict__ z) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int b = blockIdx.x;
    const int r0 = bstart[b], r1 = bstart[b + 1], nr = r1 - r0;
    const int e0 = lu_ptr[r0], nnz = lu_ptr[r1] - e0;
    T* x = reinterpret_cast<T*>(smem_raw);
    T* val = x + nr;
    unsigned short* col = reinterpret_cast<unsigned short*>(val + nnz);
    unsigned short* rp = col + nnz;
    unsigned short* dg = rp + nr + 1;
    for (int q = threadIdx.x; q < nnz; q += blockDim.x) {
        val[q] = lu[e0 + q];
        col[q] = lu_col[e0 + q];
    }
    for (int i = threadIdx.x; i <= nr; i += blockDim.x) rp[i] = (unsigned short)(lu_ptr[r0 + i] - e0);
    for (int i = threadIdx.x; i < nr; i += blockDim.x) {
        dg[i] = (unsigned short)(lu_diag[r0 + i] - e0);
        x[i] = (T)r[r0 + i];
    }
    __syncthreads();
    for (int l = blk_lvl[b] + 1; l < blk_lvl[b + 1]; ++l) {
        for (int q = lvl_ptr[l] + threadIdx.x; q < lvl_ptr[l + 1]; q += blockDim.x) {
            int li = lvl_rows[q] - r0;
            T acc = x[li];
            for (int p = rp[li]; p < dg[li]; ++p) acc -= val[p] * x[col[p]];
            x[li] = acc;
        }
        __syncthreads();
    }
    for (int l = blk_ulvl[b]; l < blk_ulvl[b + 1]; ++l) {
        for (int q = ulvl_ptr[l] + threadIdx.x; q < ulvl_ptr[l + 1]; q += blockDim.x) {
            int li = ulvl_rows[q] - r0;
            int d = dg[li];
            T acc = x[li];
            for (int p = d + 1; p < rp[li + 1]; ++p) acc -= val[p] * x[col[p]];
            x[li] = acc * val[d];
        }
        __syncthreads();
    }
    for (int i = threadIdx.x; i < nr; i += blockDim.x) z[r0 + i] = (double)x[i];
}

// ------------------------------------------------------------------ host set-up
static void build_pattern(fvm_ctx* c, BlockILU* P) {
    const int N = c->N, npe = c->npe, T = c->T;
    // node -> elements (host copy of the incidence lists)
    std::vector<int> inc_ptr(N + 1, 0), inc((size_t)T * npe);
    for (size_t q = 0; q < (size_t)T * npe; ++q) inc_ptr[c->h_elem_nodes[q] + 1]++;
    for (int i = 0; i < N; ++i) inc_ptr[i + 1] += inc_ptr[i];
    {
        std::vector<int> pos(inc_ptr.begin(), inc_ptr.end() - 1);
        for (int e = 0; e < T; ++e)
            for (int k = 0; k < npe; ++k) inc[pos[c->h_elem_nodes[(size_t)e * npe + k]]++] = e;
    }
    // pattern: node i couples to every node of every element containing i
    P->h_rowptr.assign(N + 1, 0);
    P->h_col.clear();
    std::vector<int> mark(N, -1), row;
    for (int i = 0; i < N; ++i) {
        row.clear();
        for (int p = inc_ptr[i]; p < inc_ptr[i + 1]; ++p) {
            int e = inc[p];
            for (int k = 0; k < npe; ++k) {
                int j = c->h_elem_nodes[(size_t)e * npe + k];
                if (mark[j] != i) { mark[j] = i; row.push_back(j); }
            }
        }
        std::sort(row.begin(), row.end());
        P->h_col.insert(P->h_col.end(), row.begin(), row.end());
        P->h_rowptr[i + 1] = (int)P->h_col.size();
    }
    P->nnz = (int)P->h_col.size();
    const std::vector<int>& rp = P->h_rowptr;
    const std::vector<int>& cl = P->h_col;
    // greedy distance-2 colouring in node order (preconditioner_dss.cpp:61-94)
    P->h_colour.assign(N, -1);
    std::vector<int> cmark(N + 1, -1);
    int maxc = 0;
    for (int i = 0; i < N; ++i) {
        for (int p = rp[i]; p < rp[i + 1]; ++p) {
            int nb = cl[p];
            for (int q = rp[nb]; q < rp[nb + 1]; ++q) {
                int cc = P->h_colour[cl[q]];
                if (cc >= 0) cmark[cc] = i;
            }
        }
        int cc = 0;
        while (cc < maxc && cmark[cc] == i) ++cc;
        if (cc == maxc) ++maxc;
        P->h_colour[i] = cc;
    }
    P->ncol = maxc;
    // nnz grouped by the colour of their column
    P->h_cptr.assign(maxc + 1, 0);
    for (int p = 0; p < P->nnz; ++p) P->h_cptr[P->h_colour[cl[p]] + 1]++;
    for (int k = 0; k < maxc; ++k) P->h_cptr[k + 1] += P->h_cptr[k];
    std::vector<int> cnnz(P->nnz), rowof(P->nnz);
    {
        std::vector<int> pos(P->h_cptr.begin(), P->h_cptr.end() - 1);
        for (int i = 0; i < N; ++i)
            for (int p = rp[i]; p < rp[i + 1]; ++p) {
                rowof[p] = i;
                cnnz[pos[P->h_colour[cl[p]]]++] = p;
            }
    }
    // blocks of contiguous nodes; 148 SMs -> block counts in multiples of 148
    int target = 1500;
    int nb;
    if (N >= 148 * 256) nb = 148 * std::max(1, (int)std::lround((double)N / (148.0 * target)));
    else nb = std::max(1, (N + target - 1) / target);
    nb = std::min(nb, N);
    std::vector<int> bstart(nb + 1);
    for (int b = 0; b <= nb; ++b) bstart[b] = (int)(((long)N * b) / nb);
    int maxb = 0;
    for (int b = 0; b < nb; ++b) maxb = std::max(maxb, bstart[b + 1] - bstart[b]);
    if (maxb > 65535) throw Error("block-ILU: block too large");
    std::vector<int> lu_ptr(N + 1, 0), lu_src, lu_diag(N);
    std::vector<unsigned short> lu_col;
    std::vector<int> lvl(N), ulvl(N);
    std::vector<int> lvl_ptr(1, 0), lvl_rows, blk_lvl(1, 0), ulvl_ptr(1, 0), ulvl_rows, blk_ulvl(1, 0);
    int nlmax = 0;
    for (int b = 0; b < nb; ++b) {
        int r0 = bstart[b], r1 = bstart[b + 1];
        for (int i = r0; i < r1; ++i) {
            lu_diag[i] = -1;
            for (int p = rp[i]; p < rp[i + 1]; ++p) {
                int j = cl[p];
                if (j < r0 || j >= r1) continue;
                if (j == i) lu_diag[i] = (int)lu_src.size();
                lu_src.push_back(p);
                lu_col.push_back((unsigned short)(j - r0));
            }
            lu_ptr[i + 1] = (int)lu_src.size();
            if (lu_diag[i] < 0) throw Error("block-ILU: missing diagonal");
        }
        int nl = 0;
        for (int i = r0; i < r1; ++i) {
            int l = 0;
            for (int p = lu_ptr[i]; p < lu_diag[i]; ++p) l = std::max(l, lvl[r0 + lu_col[p]] + 1);
            lvl[i] = l;
            nl = std::max(nl, l + 1);
        }
        int nu = 0;
        for (int i = r1 - 1; i >= r0; --i) {
            int l = 0;
            for (int p = lu_diag[i] + 1; p < lu_ptr[i + 1]; ++p) l = std::max(l, ulvl[r0 + lu_col[p]] + 1);
            ulvl[i] = l;
            nu = std::max(nu, l + 1);
        }
        nlmax = std::max(nlmax, std::max(nl, nu));
        for (int l = 0; l < nl; ++l) {
            for (int i = r0; i < r1; ++i) if (lvl[i] == l) lvl_rows.push_back(i);
            lvl_ptr.push_back((int)lvl_rows.size());
        }
        blk_lvl.push_back((int)lvl_ptr.size() - 1);
        for (int l = 0; l < nu; ++l) {
            for (int i = r0; i < r1; ++i) if (ulvl[i] == l) ulvl_rows.push_back(i);
            ulvl_ptr.push_back((int)ulvl_rows.size());
        }
        blk_ulvl.push_back((int)ulvl_ptr.size() - 1);
    }
    P->nb = nb;
    P->maxb = maxb;
    P->nlevels_max = nlmax;
    {
        size_t need64 = 0, need32 = 0;
        bool fits16 = true;
        for (int b = 0; b < nb; ++b) {
            size_t nr = bstart[b + 1] - bstart[b];
            size_t nz = lu_ptr[bstart[b + 1]] - lu_ptr[bstart[b]];
            if (nz >= 65535 || nr + 1 >= 65535) fits16 = false;
            need64 = std::max(need64, nr * 8 + nz * 8 + nz * 2 + (nr + 1) * 2 + nr * 2);
            need32 = std::max(need32, nr * 4 + nz * 4 + nz * 2 + (nr + 1) * 2 + nr * 2);
        }
        P->smem_stage[0] = (fits16 && need64 <= kMaxDynSmem) ? need64 : 0;
        P->smem_stage[1] = (fits16 && need32 <= kMaxDynSmem) ? need32 : 0;
        if (P->smem_stage[0])
            FVM_CUDA(cudaFuncSetAttribute(k_ilu_apply_smem<double>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                          (int)P->smem_stage[0]));
        if (P->smem_stage[1])
            FVM_CUDA(cudaFuncSetAttribute(k_ilu_apply_smem<float>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                          (int)P->smem_stage[1]));
    }
    cudaStream_t s = c->stream;
    P->col.upload(P->h_col, s);
    P->rowof.upload(rowof, s);
    P->J.alloc(P->nnz);
    P->colour.upload(P->h_colour, s);
    P->cnnz.upload(cnnz, s);
    P->shift.alloc(N);
    P->Fc.alloc(N);
    P->bstart.upload(bstart, s);
    P->lu_ptr.upload(lu_ptr, s);
    P->lu_src.upload(lu_src, s);
    P->lu_diag.upload(lu_diag, s);
    P->lu_col.upload(lu_col, s);
    P->lvl_ptr.upload(lvl_ptr, s);
    P->lvl_rows.upload(lvl_rows, s);
    P->blk_lvl.upload(blk_lvl, s);
    P->ulvl_ptr.upload(ulvl_ptr, s);
    P->ulvl_rows.upload(ulvl_rows, s);
    P->blk_ulvl.upload(blk_ulvl, s);
    P->status.alloc(1);
    P->status.zero(s);
    FVM_CUDA(cudaMallocHost(&P->h_status, sizeof(int)));
    FVM_CUDA(cudaStreamSynchronize(s));
    P->built = true;
}

void psetup_dev(fvm_ctx* c, double cj, double h, const double* y, const double* yp,
                const double* F0, const double* ewt, int precision) {
    if (!c->ilu) c->ilu = new BlockILU();
    BlockILU* P = c->ilu;
    if (!P->built) build_pattern(c, P);
    cudaStream_t s = c->stream;
    const int N = c->N;
    c->tm.begin(TM_FD_JAC, s);
    fvm_launch(c, k_shift, grid_for(N, 256), 256, 0, s, N, y, yp, ewt, h, std::sqrt(DBL_EPSILON), P->shift.p);
    for (int col = 0; col < P->ncol; ++col) {
        Perturb pt;
        pt.mode = 2;
        pt.cj = cj;
        pt.shift = P->shift.p;
        pt.colour = P->colour.p;
        pt.c = col;
        launch_residual(c, y, yp, pt, nullptr, P->Fc.p);
        int cnt = P->h_cptr[col + 1] - P->h_cptr[col];
        if (cnt > 0)
            fvm_launch(c, k_fd_scatter, grid_for(cnt, 256), 256, 0, s, cnt, P->cnnz.p + P->h_cptr[col], P->rowof.p,
                                                            P->col.p, P->Fc.p, F0, P->shift.p, P->J.p);
    }
    c->tm.end(TM_FD_JAC, s);
    FVM_CUDA(cudaMemsetAsync(P->status.p, 0, sizeof(int), s));
    size_t nlu = P->lu_src.n;
    c->tm.begin(TM_ILU_FACTOR, s);
    if (precision) {
        P->lu32.alloc(nlu);
        fvm_launch(c, k_ilu_factor<float>, P->nb, 128, 0, s, P->bstart.p, P->lu_ptr.p, P->lu_src.p, P->lu_diag.p, P->lu_col.p,
                                                  P->lvl_ptr.p, P->lvl_rows.p, P->blk_lvl.p, P->J.p, P->lu32.p,
                                                  P->status.p);
    } else {
        P->lu64.alloc(nlu);
        fvm_launch(c, k_ilu_factor<double>, P->nb, 128, 0, s, P->bstart.p, P->lu_ptr.p, P->lu_src.p, P->lu_diag.p, P->lu_col.p,
                                                   P->lvl_ptr.p, P->lvl_rows.p, P->blk_lvl.p, P->J.p, P->lu64.p,
                                                   P->status.p);
    }
    c->tm.end(TM_ILU_FACTOR, s);
    FVM_CUDA(cudaMemcpyAsync(P->h_status, P->status.p, sizeof(int), cudaMemcpyDeviceToHost, s));
    P->factored = precision;
}

int ilu_status(fvm_ctx* c) {
    if (!c->ilu || !c->ilu->h_status) return 0;
    FVM_CUDA(cudaStreamSynchronize(c->stream));
    return *c->ilu->h_status;
}

bool ilu_ready(fvm_ctx* c) { return c->ilu && c->ilu->factored >= 0; }

void psolve_dev(fvm_ctx* c, const double* r, double* z) {
    BlockILU* P = c->ilu;
    if (!P || P->factored < 0) throw Error("psolve: preconditioner not set up");
    cudaStream_t s = c->stream;
    c->tm.begin(TM_ILU_APPLY, s);
    struct EndTimer {
        fvm_ctx* c;
        ~EndTimer() { c->tm.end(TM_ILU_APPLY, c->stream); }
    } end_timer{c};
    if (P->smem_stage[P->factored]) {
        size_t sm = P->smem_stage[P->factored];
        if (P->factored)
            fvm_launch(c, k_ilu_apply_smem<float>, P->nb, 256, sm, s, P->bstart.p, P->lu_ptr.p, P->lu_diag.p, P->lu_col.p,
                                                          P->lvl_ptr.p, P->lvl_rows.p, P->blk_lvl.p, P->ulvl_ptr.p,
                                                          P->ulvl_rows.p, P->blk_ulvl.p, P->lu32.p, r, z);
        else
            fvm_launch(c, k_ilu_apply_smem<double>, P->nb, 256, sm, s, P->bstart.p, P->lu_ptr.p, P->lu_diag.p, P->lu_col.p,
                                                           P->lvl_ptr.p, P->lvl_rows.p, P->blk_lvl.p, P->ulvl_ptr.p,
                                                           P->ulvl_rows.p, P->blk_ulvl.p, P->lu64.p, r, z);
    } else if (P->factored) {
        size_t sm = sizeof(float) * P->maxb;
        fvm_launch(c, k_ilu_apply<float>, P->nb, 128, sm, s, P->bstart.p, P->lu_ptr.p, P->lu_diag.p, P->lu_col.p, P->lvl_ptr.p,
                                                 P->lvl_rows.p, P->blk_lvl.p, P->ulvl_ptr.p, P->ulvl_rows.p,
                                                 P->blk_ulvl.p, P->lu32.p, r, z);
    } else {
        size_t sm = sizeof(double) * P->maxb;
        fvm_launch(c, k_ilu_apply<double>, P->nb, 128, sm, s, P->bstart.p, P->lu_ptr.p, P->lu_diag.p, P->lu_col.p, P->lvl_ptr.p,
                                                  P->lvl_rows.p, P->blk_lvl.p, P->ulvl_ptr.p, P->ulvl_rows.p,
                                                  P->blk_ulvl.p, P->lu64.p, r, z);
    }
}

} // namespace fvmb

using namespace fvmb;

void fvmb_destroy_ilu(fvmb::BlockILU* p) {
    if (!p) return;
    if (p->h_status) cudaFreeHost(p->h_status);
    delete p;
}

extern "C" int fvm_psetup(fvm_ctx* c, double t, double cj, double h, const double* y,
                          const double* yp, const double* F0, const double* ewt, int precision) {
    try {
        (void)t;
        if (!c || !y || !yp || !F0 || !ewt) throw Error("fvm_psetup: null argument");
        if (precision != 0 && precision != 1) throw Error("fvm_psetup: precision must be 0 or 1");
        psetup_dev(c, cj, h, y, yp, F0, ewt, precision);
        FVM_CUDA(cudaGetLastError());
        return ilu_status(c) ? 1 : 0;
    } catch (const Error& ex) {
        set_error(ex.what());
        return ex.code;
    } catch (const std::exception& ex) {
        set_error(ex.what());
        return -1;
    }
}

extern "C" int fvm_psolve(fvm_ctx* c, const double* r, double* z) {
    try {
        if (!c || !r || !z) throw Error("fvm_psolve: null argument");
        psolve_dev(c, r, z);
        FVM_CUDA(cudaGetLastError());
        FVM_CUDA(cudaStreamSynchronize(c->stream));
        return 0;
    } catch (const Error& ex) {
        set_error(ex.what());
        return ex.code;
    } catch (const std::exception& ex) {
        set_error(ex.what());
        return -1;
    }
}

// pattern / partition introspection for tests and the autotuner
extern "C" int fvm_precond_info(fvm_ctx* c, int* nnz, int* ncolours, int* nblocks, int* max_levels) {
    try {
        if (!c || !c->ilu || !c->ilu->built) throw Error("fvm_precond_info: no preconditioner");
        if (nnz) *nnz = c->ilu->nnz;
        if (ncolours) *ncolours = c->ilu->ncol;
        if (nblocks) *nblocks = c->ilu->nb;
        if (max_levels) *max_levels = c->ilu->nlevels_max;
        return 0;
    } catch (const std::exception& ex) {
        set_error(ex.what());
        return -1;
    }
}

// copies the assembled Jacobian (CSR, host buffers of the sizes reported
// by fvm_precond_info) for inspection against the oracle
extern "C" int fvm_precond_jacobian(fvm_ctx* c, int* rowptr, int* col, double* val) {
    try {
        if (!c || !c->ilu || !c->ilu->built) throw Error("fvm_precond_jacobian: no preconditioner");
        BlockILU* P = c->ilu;
        if (rowptr) std::copy(P->h_rowptr.begin(), P->h_rowptr.end(), rowptr);
        if (col) std::copy(P->h_col.begin(), P->h_col.end(), col);
        if (val) {
            FVM_CUDA(cudaMemcpyAsync(val, P->J.p, sizeof(double) * P->nnz, cudaMemcpyDeviceToHost, c->stream));
            FVM_CUDA(cudaStreamSynchronize(c->stream));
        }
        return 0;
    } catch (const std::exception& ex) {
        set_error(ex.what());
        return -1;
    }
}
