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
#include "cgs.cuh"
#include "ctx.cuh"
#include "ilu.cuh"
#include "krylov.cuh"
#include "tc05.cuh"

#include <algorithm>
#include <type_traits>
#include <cfloat>
#include <cmath>

namespace fvmb {

// ------------------------------------------------------------------ kernels
__global__ void k_shift(int N, const double* __restrict__ y, const double* __restrict__ yp,
                        const double* __restrict__ ewt, double h, double eps,
                        double* __restrict__ shift) {
    int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= N) return;
    double a = fabs(y[j]), b = fabs(h * yp[j]), w = 1.0 / ewt[j];
    shift[j] = eps * fmax(a, fmax(b, w));
}

// ---- finite-difference Jacobian, one element at a time
// Column j of the reference's coloured difference quotient is
// (F(y + d_j e_j, y' + cj d_j e_j) - F(y, y')) / d_j (preconditioner_dss.cpp:
// 284-373): the distance-2 colouring makes every row see at most one
// perturbed node per colour, so the coloured evaluation equals these
// single-column quotients.  With the upwind directions frozen, perturbing
// node m changes only the elements that contain m, and only through h_m and
// krw(h_m): each element forms the change of its corner partials for each of
// its nodes in turn,
//   dflux_f = rho0 (q_f (krw'_f - krw_f) + d_m C_fm krw'_f),
// which is the same quotient written without the cancellation of two full
// residuals.  The changes land in fixed slots (nonzero-major, ascending
// element) and one pass per nonzero sums them, adds the storage term on the
// diagonal and writes the Dirichlet rows: npe + 2 kernels per set-up instead
// of one residual evaluation per colour.

// per node: krw at h and h + d (every zone touching the node) and the change
// of the storage term y' ahh(h) on the diagonal
__global__ void k_fd_node(int N, const double* __restrict__ y, const double* __restrict__ yp, double cj,
                          const double* __restrict__ shift, const ZoneDev* __restrict__ zones, int nz,
                          const int* __restrict__ nz_ptr, const int* __restrict__ nz_zone,
                          const double* __restrict__ nz_w, double rho0, double* __restrict__ krwb,
                          double* __restrict__ krwp, double* __restrict__ dstor, double* __restrict__ ahhp_out) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N) return;
    const double h = y[i], d = shift[i];
    const double hp = h + d;
    double phi = 0.0, dsw = 0.0, dswp = 0.0;
    const int p0 = nz == 1 ? i : nz_ptr[i], p1 = nz == 1 ? i + 1 : nz_ptr[i + 1];
    for (int p = p0; p < p1; ++p) {
        const int z = nz == 1 ? 0 : nz_zone[p];
        const double w = nz_w[p];
        double Sw, ds, k, dsp, kp;
        van_genuchten(h, zones[z], Sw, ds, k);
        van_genuchten(hp, zones[z], Sw, dsp, kp);
        krwb[(size_t)z * N + i] = k;
        krwp[(size_t)z * N + i] = kp;
        phi += zones[z].phi * w;
        dsw += ds * w;
        dswp += dsp * w;
    }
    const double ahh = (phi * dsw) * rho0, ahhp = (phi * dswp) * rho0;
    dstor[i] = (yp[i] + cj * d) * ahhp - yp[i] * ahh;
    ahhp_out[i] = ahhp;
}

// y = J x for the assembled difference-quotient Jacobian of the last
// set-up, shifted to another cj: the cj term of J enters only the diagonal
// of free rows, as -cj ahh(h + d) (the quotient of the storage term
// y' ahh(h), k_fd_node), so J(cj) = J(cj_setup) - (cj - cj_setup) ahh(h + d)
// on those rows.  Four lanes per row, rows in node order.
__global__ void k_jac_apply(int N, const int* __restrict__ rowptr, const int* __restrict__ col,
                            const double* __restrict__ J, const double* __restrict__ ahhp,
                            const unsigned char* __restrict__ ntype, double dcj, const double* __restrict__ x,
                            double* __restrict__ y, const int* __restrict__ skip,
                            const double* __restrict__ dcj_dev) {
    pdl_wait_and_trigger();
    if (skip && *skip) return;
    if (dcj_dev) dcj = *dcj_dev;
    const int g = blockIdx.x * blockDim.x + threadIdx.x;
    const int i = g >> 2, lane = g & 3;
    if (i >= N) return;
    const int p0 = rowptr[i], p1 = rowptr[i + 1];
    double acc = 0.0;
    for (int p = p0 + lane; p < p1; p += 4) acc += J[p] * x[col[p]];
    acc += __shfl_xor_sync(0xffffffffu, acc, 1);
    acc += __shfl_xor_sync(0xffffffffu, acc, 2);
    if (lane == 0) y[i] = ntype[i] ? acc : acc - dcj * ahhp[i] * x[i];
}

// per element: the npe x npe changes of its corner partials, one column
// (perturbed node m) at a time, divided by d_m, into their slots
// Slots are FP64, or FP32 when the factor is FP32 (the factor rounds every
// entry to FP32 anyway; the slots then move half the bytes).
template <int NPE, int NFE, bool RC, bool MZ, class S>
// (two blocks per SM: 128 registers, no spills; the unbounded build took
// 130 and ran one block of 8 warps per SM)
__global__ void __launch_bounds__(256, 2) k_fd_elem(int T, int N, const int4* __restrict__ en,
                                                 const double* __restrict__ coef, const double* __restrict__ xyz,
                                                 const double* __restrict__ eK, int kiso, int estride,
                                                 const int* __restrict__ ezone, const double* __restrict__ y,
                                                 const double* __restrict__ shift, const double* __restrict__ krwb,
                                                 const double* __restrict__ krwp,
                                                 const unsigned char* __restrict__ upw, double rho0,
                                                 const int* __restrict__ epos, S* __restrict__ slots) {
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= T) return;
    const int4 nd = en[e];
    const int g[4] = {nd.x, nd.y, nd.z, nd.w};
    const size_t zo = MZ ? (size_t)ezone[e] * N : 0;
    double hv[NPE], dl[NPE], kr[NPE], kp[NPE];
#pragma unroll
    for (int k = 0; k < NPE; ++k) {
        hv[k] = y[g[k]];
        dl[k] = shift[g[k]];
        kr[k] = krwb[zo + g[k]];
        kp[k] = krwp[zo + g[k]];
    }
    double C[NFE][NPE], G[NFE];
    if (RC) {
        double X[4][3];
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            X[k][0] = xyz[g[k]];
            X[k][1] = xyz[(size_t)N + g[k]];
            X[k][2] = xyz[(size_t)2 * N + g[k]];
        }
        double Kx, Ky, Kz;
        if (kiso) Kx = Ky = Kz = eK[e];
        else { Kx = eK[e]; Ky = eK[(size_t)estride + e]; Kz = eK[(size_t)2 * estride + e]; }
        double CC[6][4], GG[6];
        tet_coefficients_fast(X[0], X[1], X[2], X[3], Kx, Ky, Kz, CC, GG);
#pragma unroll
        for (int f = 0; f < NFE; ++f) {
#pragma unroll
            for (int k = 0; k < NPE; ++k) C[f][k] = CC[f][k];
            G[f] = GG[f];
        }
    } else {
#pragma unroll
        for (int f = 0; f < NFE; ++f) {
#pragma unroll
            for (int k = 0; k < NPE; ++k) C[f][k] = coef[(size_t)(f * (NPE + 1) + k) * T + e];
            G[f] = coef[(size_t)(f * (NPE + 1) + NPE) * T + e];
        }
    }
    const uint2 uw = *reinterpret_cast<const uint2*>(upw + (size_t)8 * e);
    double q[NFE];
    unsigned u[NFE];
#pragma unroll
    for (int f = 0; f < NFE; ++f) {
        double s = C[f][0] * hv[0];
#pragma unroll
        for (int k = 1; k < NPE; ++k) s += C[f][k] * hv[k];
        q[f] = s + G[f];
        u[f] = (f < 4 ? uw.x >> (8 * f) : uw.y >> (8 * (f - 4))) & 0xffu;
    }
#pragma unroll
    for (int m = 0; m < NPE; ++m) {
        double dc[NPE];
#pragma unroll
        for (int k = 0; k < NPE; ++k) dc[k] = 0.0;
#pragma unroll
        for (int f = 0; f < NFE; ++f) {
            const int a = NPE == 4 ? tet_edge_a(f) : tri_edge_a(f);
            const int b = NPE == 4 ? tet_edge_b(f) : tri_edge_b(f);
            const double kf = face_krw(u[f], kr[a], kr[b]);
            const double kfp = face_krw(u[f], a == m ? kp[a] : kr[a], b == m ? kp[b] : kr[b]);
            const double df = rho0 * (q[f] * (kfp - kf) + (dl[m] * C[f][m]) * kfp);
            dc[a] -= df;
            dc[b] += df;
        }
        const double inv = 1.0 / dl[m];
#pragma unroll
        for (int k = 0; k < NPE; ++k) slots[epos[(size_t)e * NPE * NPE + m * NPE + k]] = (S)(dc[k] * inv);
    }
}

// per nonzero (i, j): J_ij = (1/V_i) sum of the slots - [i == j] dstor_i / d_i;
// Dirichlet rows h_D - h differentiate to the quotient of that expression
template <class S>
__global__ void k_fd_gather(int nnz, const int* __restrict__ rowof, const int* __restrict__ col,
                            const int* __restrict__ jptr, const S* __restrict__ slots,
                            const double* __restrict__ invV, const double* __restrict__ dstor,
                            const unsigned char* __restrict__ ntype, const double* __restrict__ hD,
                            const double* __restrict__ y, const double* __restrict__ shift,
                            double* __restrict__ J, const int* __restrict__ lu_dst, double* __restrict__ Jw,
                            const int* __restrict__ op_dst, float* __restrict__ op_val) {
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= nnz) return;
    const int i = rowof[q], j = col[q];
    double v;
    if (ntype[i]) {
        v = i == j ? ((hD[i] - (y[i] + shift[i])) - (hD[i] - y[i])) / shift[i] : 0.0;
    } else {
        double s = 0.0;
        const int p1 = jptr[q + 1];
        for (int p = jptr[q]; p < p1; ++p) s += (double)slots[p];
        v = s * invV[i];
        if (i == j) v = v - dstor[i] / shift[i];
    }
    J[q] = v;
    // the same value where the factorisation reads it (its block's copy
    // window, so that it loads its block contiguously) and, once the fused
    // cycle's operator layout exists, in that layout
    const int pw = lu_dst[q];
    if (pw >= 0) Jw[pw] = v;
    if (op_val) op_val[op_dst[q]] = (float)v;
}

template <class T>
__global__ void __launch_bounds__(128) k_ilu_factor(const int* __restrict__ bstart,
                                                    const int* __restrict__ lu_ptr,
                                                    const double* __restrict__ Jw,
                                                    const int* __restrict__ lu_diag,
                                                    const unsigned short* __restrict__ lu_col,
                                                    const int* __restrict__ lvl_ptr,
                                                    const int* __restrict__ lvl_rows,
                                                    const int* __restrict__ blk_lvl, T* lu,
                                                    int* status) {
    int b = blockIdx.x;
    int r0 = bstart[b], r1 = bstart[b + 1];
    for (int p = lu_ptr[r0] + threadIdx.x; p < lu_ptr[r1]; p += blockDim.x) lu[p] = (T)Jw[p];
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
                                                   const T* __restrict__ lu, const int* __restrict__ lu_row,
                                                   const double* __restrict__ r,
                                                   double* __restrict__ z, const int* __restrict__ skip) {
    extern __shared__ unsigned char smem_raw[];
    pdl_wait_and_trigger();
    if (skip && *skip) return;
    T* x = reinterpret_cast<T*>(smem_raw);
    int b = blockIdx.x;
    int r0 = bstart[b], r1 = bstart[b + 1];
    for (int i = r0 + threadIdx.x; i < r1; i += blockDim.x) x[i - r0] = (T)r[lu_row[i]];
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
    for (int i = r0 + threadIdx.x; i < r1; i += blockDim.x) z[lu_row[i]] = (double)x[i - r0];
}

template <class T, int KM>
__global__ void __launch_bounds__(kIluThreads) k_ilu_apply_smem(const int* __restrict__ bstart,
                                                        const int* __restrict__ lu_ptr,
                                                        const unsigned short* __restrict__ lu_col,
                                                        const unsigned short* __restrict__ meta,
                                                        const int* __restrict__ meta_off,
                                                        const int* __restrict__ blk_lvl,
                                                        const int* __restrict__ blk_ulvl,
                                                        const T* __restrict__ lu,
                                                        const int* __restrict__ lu_row,
                                                        const double* __restrict__ r,
                                                        double* __restrict__ z, int* __restrict__ err,
                                                        const int* __restrict__ skip) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int b = blockIdx.x;
    const int r0 = bstart[b], r1 = bstart[b + 1], nr = r1 - r0;
    const IluWindow w = ilu_window(lu_ptr[r0], lu_ptr[r1]);
    const int la = blk_lvl[b], nl = blk_lvl[b + 1] - la;
    const int ua = blk_ulvl[b], nu = blk_ulvl[b + 1] - ua;
    T* x = reinterpret_cast<T*>(smem_raw);
    T* val = reinterpret_cast<T*>(smem_raw + round16(sizeof(T) * nr));
    unsigned short* col = reinterpret_cast<unsigned short*>(val + w.wn);
    unsigned short* rp = col + w.wn;
    unsigned short* dg = rp + nr + 1;
    unsigned short* lrow = dg + nr;
    unsigned short* urow = lrow + nr;
    unsigned short* lptr = urow + nr;
    unsigned short* uptr = lptr + nl + 1;
    uint64_t* bar = reinterpret_cast<uint64_t*>(smem_raw + ilu_stage_bytes(nr, w.wn, nl + nu + 2, sizeof(T)) - 16);
    if (threadIdx.x == 0) {
        tc05::mbar_init(bar, 1);
        asm volatile("fence.mbarrier_init.release.cluster;");
    }
    __syncthreads();
    // factor window and the block's metadata record (row pointers, pivot
    // positions, level lists) by three bulk copies; the right-hand side by
    // the threads meanwhile.  The copies read only set-up data, so they are
    // issued before the wait for the previous kernel (the factorisation has
    // completed before any kernel that lets this launch start early); the
    // right-hand side and the skip flag are read after it.
    const int mo = meta_off[b];
    ilu_stage_bulk(val, col, lu, lu_col, w, bar, rp, meta + mo, meta_off[b + 1] - mo);
    pdl_wait_and_trigger();
    if (skip && *skip) {
        // a step queued after the stop: let the copies land (bounded), leave
        tc05::mbar_wait(bar, 0);
        return;
    }
    for (int i = threadIdx.x; i < nr; i += blockDim.x) x[i] = (T)r[lu_row[r0 + i]];
    bool ok = tc05::mbar_wait(bar, 0);
    if (!ok) ok = tc05::mbar_wait(bar, 0);   // copies in flight get a second bounded chance
    if (!__syncthreads_and(ok ? 1 : 0)) {
        // the factor never arrived: report it and pass the vector through
        // unpreconditioned instead of reading unfilled shared memory
        if (threadIdx.x == 0) atomicExch(err, 2);
        for (int i = threadIdx.x; i < nr; i += blockDim.x) z[lu_row[r0 + i]] = (double)x[i];
        return;
    }
    // level 0 of the lower sweep has no off-diagonal entries
    ilu_sweep<T, KM, false>(x, val, col, rp, dg, lrow, lptr, 1, nl);
    ilu_sweep<T, KM, true>(x, val, col, rp, dg, urow, uptr, 0, nu);
    for (int i = threadIdx.x; i < nr; i += blockDim.x) z[lu_row[r0 + i]] = (double)x[i];
}

// Block ILU(0) coupled through the Schur complement of the block
// interfaces (decomp/schur.c:1407-1636, precon_schur_apply).  Each block's
// factor is ordered [interior B; interface] so that it reads
//   [L_B 0; F~ L_S] [U_B E~; 0 U_S],
// L_S U_S being the ILU(0) of the block's local Schur complement
// C - F B^-1 E on C's pattern; the interface system of the whole matrix is
// S = L_S U_S + C_o, C_o the couplings to the other blocks' interface rows.
// One cooperative launch, one CTA per block, the factor staged in shared
// memory once for the whole apply:
//   z = L^-1 r (the forward sweep; x_L = M_B f and g - F x_L of the
//     reference), kept in shared memory;
//   x_S = U_S^-1 z_S, then `iters` times: publish x_S, grid barrier,
//     x_S <- U_S^-1 (z_S - L_S^-1 C_o x_S) with the other blocks' published
//     values (block-Jacobi sweeps on S, the reference's level-0 solve);
//   x_B = U_B^-1 (z_B - E~ x_S) (x_L = M_B (f - E y)).
// The published iterates alternate between two node-order buffers, so a
// block still reading sweep i never sees sweep i + 1's values.  Barrier
// waits are bounded (error 3 in serr, every block leaves at its next
// barrier); a factor that never reached shared memory passes r through and
// records error 2, as the staged apply does.
template <class T> struct SchurArgs {
    int N, iters;
    size_t stage_max;          // offset of the forward result in shared memory
    const int* bstart;
    const int* lu_ptr;
    const unsigned short* lu_col;
    const unsigned short* meta;
    const int* meta_off;
    const int* blk_lvl;
    const int* blk_ulvl;
    const T* lu;
    const int* lu_row;
    const int* sch_lv;
    const int* sch_nin;
    const int* o_ptr;
    const int* o_col;
    const int* o_src;
    const double* J;
    double* xg;
    unsigned* bar;
    int* serr;
    const double* r;
    double* z;
    int* err;
    const int* skip;
};

template <class T, int KM>
__global__ void __launch_bounds__(kIluThreads) k_ilu_apply_schur(SchurArgs<T> a) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int b = blockIdx.x;
    const int r0 = a.bstart[b], r1 = a.bstart[b + 1], nr = r1 - r0;
    const IluWindow w = ilu_window(a.lu_ptr[r0], a.lu_ptr[r1]);
    const int la = a.blk_lvl[b], nl = a.blk_lvl[b + 1] - la;
    const int ua = a.blk_ulvl[b], nu = a.blk_ulvl[b + 1] - ua;
    T* x = reinterpret_cast<T*>(smem_raw);
    T* val = reinterpret_cast<T*>(smem_raw + round16(sizeof(T) * nr));
    unsigned short* col = reinterpret_cast<unsigned short*>(val + w.wn);
    unsigned short* rp = col + w.wn;
    unsigned short* dg = rp + nr + 1;
    unsigned short* lrow = dg + nr;
    unsigned short* urow = lrow + nr;
    unsigned short* lptr = urow + nr;
    unsigned short* uptr = lptr + nl + 1;
    uint64_t* mbar = reinterpret_cast<uint64_t*>(smem_raw + ilu_stage_bytes(nr, w.wn, nl + nu + 2, sizeof(T)) - 16);
    T* zs = reinterpret_cast<T*>(smem_raw + a.stage_max);
    if (threadIdx.x == 0) {
        tc05::mbar_init(mbar, 1);
        asm volatile("fence.mbarrier_init.release.cluster;");
    }
    __syncthreads();
    const int mo = a.meta_off[b];
    ilu_stage_bulk(val, col, a.lu, a.lu_col, w, mbar, rp, a.meta + mo, a.meta_off[b + 1] - mo);
    pdl_wait_and_trigger();
    if (a.skip && *a.skip) {
        // a step queued after the stop: every block leaves before any barrier
        tc05::mbar_wait(mbar, 0);
        return;
    }
    for (int i = threadIdx.x; i < nr; i += blockDim.x) x[i] = (T)a.r[a.lu_row[r0 + i]];
    bool ok = tc05::mbar_wait(mbar, 0);
    if (!ok) ok = tc05::mbar_wait(mbar, 0);
    const bool good = __syncthreads_and(ok ? 1 : 0) != 0;
    if (!good && threadIdx.x == 0) atomicExch(a.err, 2);
    const int lvB = a.sch_lv[2 * b], uvS = a.sch_lv[2 * b + 1], nin = a.sch_nin[b];
    if (good) {
        ilu_sweep<T, KM, false>(x, val, col, rp, dg, lrow, lptr, 1, nl);
        for (int i = threadIdx.x; i < nr; i += blockDim.x) zs[i] = x[i];
        __syncthreads();
        ilu_sweep<T, KM, true>(x, val, col, rp, dg, urow, uptr, 0, uvS);
    }
    for (int it = 0; it < a.iters; ++it) {
        double* xo = a.xg + (size_t)(it & 1) * a.N;
        if (good)
            for (int q = nin + threadIdx.x; q < nr; q += blockDim.x) xo[a.lu_row[r0 + q]] = (double)x[q];
        // a block without its factor still takes part in every barrier
        if (!grid_barrier(a.bar, a.bar + 1, a.serr)) return;
        if (!good) continue;
        for (int q = threadIdx.x; q < nin; q += blockDim.x) x[q] = (T)0;
        for (int q = nin + threadIdx.x; q < nr; q += blockDim.x) {
            T acc = (T)0;
            const int e1 = a.o_ptr[r0 + q + 1];
            for (int e = a.o_ptr[r0 + q]; e < e1; ++e) acc += (T)a.J[a.o_src[e]] * (T)__ldcg(xo + a.o_col[e]);
            x[q] = acc;
        }
        __syncthreads();
        ilu_sweep<T, KM, false>(x, val, col, rp, dg, lrow, lptr, lvB, nl);
        for (int q = nin + threadIdx.x; q < nr; q += blockDim.x) x[q] = zs[q] - x[q];
        __syncthreads();
        ilu_sweep<T, KM, true>(x, val, col, rp, dg, urow, uptr, 0, uvS);
    }
    if (!good) {
        for (int i = threadIdx.x; i < nr; i += blockDim.x) a.z[a.lu_row[r0 + i]] = (double)x[i];
        return;
    }
    if (a.iters > 0) {
        for (int q = threadIdx.x; q < nin; q += blockDim.x) x[q] = zs[q];
        __syncthreads();
    }
    ilu_sweep<T, KM, true>(x, val, col, rp, dg, urow, uptr, uvS, nu);
    for (int i = threadIdx.x; i < nr; i += blockDim.x) a.z[a.lu_row[r0 + i]] = (double)x[i];
}

static const void* schur_kernel(int precision, int lanes) {
    if (precision) return lanes == 8 ? (const void*)k_ilu_apply_schur<float, 8> : (const void*)k_ilu_apply_schur<float, 4>;
    return lanes == 8 ? (const void*)k_ilu_apply_schur<double, 8> : (const void*)k_ilu_apply_schur<double, 4>;
}

template <class T>
static void launch_schur_apply(fvm_ctx* c, BlockILU* P, const T* lu, const double* r, double* z, const int* skip) {
    SchurArgs<T> a;
    a.N = c->N;
    a.iters = P->schur_iters;
    a.stage_max = round16(P->smem_stage[P->factored]);
    a.bstart = P->bstart.p;
    a.lu_ptr = P->lu_ptr.p;
    a.lu_col = P->lu_col.p;
    a.meta = P->meta.p;
    a.meta_off = P->meta_off.p;
    a.blk_lvl = P->blk_lvl.p;
    a.blk_ulvl = P->blk_ulvl.p;
    a.lu = lu;
    a.lu_row = P->lu_row.p;
    a.sch_lv = P->sch_lv.p;
    a.sch_nin = P->sch_nin.p;
    a.o_ptr = P->o_ptr.p;
    a.o_col = P->o_col.p;
    a.o_src = P->o_src.p;
    a.J = P->J.p;
    a.xg = P->xg.p;
    a.bar = P->sbar.p;
    a.serr = P->serr.p;
    a.r = r;
    a.z = z;
    a.err = P->status.p;
    a.skip = skip;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(P->nb);
    cfg.blockDim = dim3(P->apply_threads);
    cfg.dynamicSmemBytes = P->schur_smem[P->factored];
    cfg.stream = c->stream;
    cudaLaunchAttribute attr[2];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    attr[1].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[1].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 2;
    if (P->lanes == 8) FVM_CUDA(cudaLaunchKernelEx(&cfg, k_ilu_apply_schur<T, 8>, a));
    else FVM_CUDA(cudaLaunchKernelEx(&cfg, k_ilu_apply_schur<T, 4>, a));
    c->launches++;
}

// Shared-memory factorisation: gather the block's Jacobian entries into the
// same copy window the apply uses, eliminate level by level in shared
// memory (IKJ, pivots inverted after their row), write the block back.
// 1024 threads: one block per SM, so the copies in and out and the
// schedule prefetch keep many loads in flight, while a level's rows (one
// thread each, a few hundred) run on the first warps.  Schedule words of
// the next level each thread holds:
constexpr int kIluFactorThreads = 1024;
constexpr int kIluFactorPre = 8;

template <class T>
__global__ void __launch_bounds__(kIluFactorThreads, 1) k_ilu_factor_smem(const int* __restrict__ bstart,
                                                         const int* __restrict__ lu_ptr,
                                                         const double* __restrict__ Jw,
                                                         const int* __restrict__ lu_diag,
                                                         const unsigned short* __restrict__ lu_col,
                                                         const int* __restrict__ lvl_ptr,
                                                         const int* __restrict__ lvl_rows,
                                                         const int* __restrict__ blk_lvl,
                                                         const int* __restrict__ seg_ptr,
                                                         const unsigned* __restrict__ upd, int scr_off,
                                                         int scr_words, T* __restrict__ lu,
                                                         int* status) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int b = blockIdx.x;
    const int r0 = bstart[b], r1 = bstart[b + 1], nr = r1 - r0;
    const int e0 = lu_ptr[r0], e1 = lu_ptr[r1];
    const IluWindow w = ilu_window(e0, e1);
    T* val = reinterpret_cast<T*>(smem_raw + round16(sizeof(T) * nr));
    unsigned short* col = reinterpret_cast<unsigned short*>(val + w.wn);
    unsigned short* rp = col + w.wn;
    unsigned short* dg = rp + nr + 1;
    unsigned short* lrow = dg + nr;
    unsigned short* lptr = lrow + 2 * nr;
    const int la = blk_lvl[b], nl = blk_lvl[b + 1] - la;
    const int lq0 = lvl_ptr[la];
#pragma unroll 4
    for (int p = e0 + threadIdx.x; p < e1; p += blockDim.x) {
        val[p - w.base] = (T)Jw[p];
        col[p - w.base] = lu_col[p];
    }
    for (int i = threadIdx.x; i <= nr; i += blockDim.x) rp[i] = (unsigned short)(lu_ptr[r0 + i] - w.base);
    for (int i = threadIdx.x; i < nr; i += blockDim.x) {
        dg[i] = (unsigned short)(lu_diag[r0 + i] - w.base);
        lrow[i] = (unsigned short)(lvl_rows[lq0 + i] - r0);
    }
    for (int l = threadIdx.x; l <= nl; l += blockDim.x) lptr[l] = (unsigned short)(lvl_ptr[la + l] - lq0);
    __syncthreads();
    // Each level's schedule segment is in shared memory when its rows run
    // (read in place from global when it is larger than a buffer), so a
    // row's update chain never waits on global loads: two buffers; while a
    // level's rows run, every thread holds its share of the next level's
    // segment in registers (loads issued before the rows, stored after).
    unsigned* const buf0 = reinterpret_cast<unsigned*>(smem_raw + scr_off);
    unsigned* const buf1 = buf0 + scr_words;
    int sgc = seg_ptr[la], lenc = seg_ptr[la + 1] - sgc;
    bool cur_smem = lenc <= scr_words;
    if (cur_smem) {
#pragma unroll 4
        for (int t = threadIdx.x; t < lenc; t += blockDim.x) buf0[t] = upd[sgc + t];
    }
    __syncthreads();
    for (int l = 0; l < nl; ++l) {
        int sgn = 0, lenn = 0;
        bool nxt_smem = false;
        unsigned pre[kIluFactorPre];
        if (l + 1 < nl) {
            sgn = seg_ptr[la + l + 1];
            lenn = seg_ptr[la + l + 2] - sgn;
            nxt_smem = lenn <= scr_words;
            if (nxt_smem) {
#pragma unroll
                for (int i = 0; i < kIluFactorPre; ++i) {
                    const int t = threadIdx.x + i * blockDim.x;
                    pre[i] = t < lenn ? upd[sgn + t] : 0u;
                }
            }
        }
        const unsigned* L = cur_smem ? ((l & 1) ? buf1 : buf0) : upd + sgc;
        const int q0 = lptr[l], nq = lptr[l + 1] - q0;
        for (int qq = threadIdx.x; qq < nq; qq += blockDim.x) {
            int li = lrow[q0 + qq];
            int s0 = rp[li], di = dg[li];
            // IKJ with the precomputed schedule: the updates of the L entry
            // kk, in the order a merge of row li with U(k) would find them
            int t = (int)L[qq];
            for (int kk = s0; kk < di; ++kk) {
                const int cnt = (int)L[t++];
                const int k = col[kk];
                T lik = val[kk] * val[dg[k]];
                val[kk] = lik;
                for (int u = 0; u < cnt; ++u) {
                    const unsigned pr = L[t++];
                    const int jj = (int)(pr & 0xffffu), kp = (int)(pr >> 16);
                    val[jj] = val[jj] - lik * val[kp];
                }
            }
            T d = val[di];
            if (d == (T)0 || !isfinite((double)d)) {
                atomicExch(status, 1);
                d = (T)1;
            }
            val[di] = (T)1 / d;
        }
        if (nxt_smem) {
            unsigned* nb = (l & 1) ? buf0 : buf1;   // the buffer of level l - 1, finished
#pragma unroll
            for (int i = 0; i < kIluFactorPre; ++i) {
                const int t = threadIdx.x + i * blockDim.x;
                if (t < lenn) nb[t] = pre[i];
            }
        }
        __syncthreads();
        sgc = sgn;
        lenc = lenn;
        cur_smem = nxt_smem;
    }
    for (int p = e0 + threadIdx.x; p < e1; p += blockDim.x) lu[p] = val[p - w.base];
}

// ------------------------------------------------------------------ host set-up
// Colour order of the rows [r0, r1) of a block (offsets from r0): greedy
// colouring in natural order over the couplings inside the block, then
// stable by colour.  The CPU oracle restates the same rule.
//
// With interface_last (Schur coupling) the rows coupled to a node outside the
// block (interface rows) follow all interior rows: the sort key is
// (interface, colour); *n_interior gets the number of interior rows.
static std::vector<int> block_colour_order(const std::vector<int>& rp, const std::vector<int>& cl, int r0, int r1,
                                           bool interface_last = false, int* n_interior = nullptr) {
    const int nr = r1 - r0;
    std::vector<int> colour(nr, 0), ord(nr), key(nr);
    int ncol = 1, nin = 0;
    for (int i = r0; i < r1; ++i) {
        unsigned long long used = 0ull;
        std::vector<int> more;
        bool iface = false;
        for (int p = rp[i]; p < rp[i + 1]; ++p) {
            const int j = cl[p];
            if (j < r0 || j >= r1) iface = true;
            if (j < r0 || j >= i) continue;
            const int cj = colour[j - r0];
            if (cj < 64) used |= 1ull << cj;
            else more.push_back(cj);
        }
        int cc = 0;
        while (cc < 64 && ((used >> cc) & 1ull)) ++cc;
        if (cc == 64) {
            std::sort(more.begin(), more.end());
            for (int m : more)
                if (m == cc) ++cc;
        }
        colour[i - r0] = cc;
        key[i - r0] = interface_last && iface ? (1 << 20) + cc : cc;
        if (!iface) ++nin;
        ncol = std::max(ncol, cc + 1);
    }
    if (n_interior) *n_interior = interface_last ? nin : nr;
    for (int ii = 0; ii < nr; ++ii) ord[ii] = ii;
    std::stable_sort(ord.begin(), ord.end(), [&](int a, int b2) { return key[a] < key[b2]; });
    return ord;
}

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
    std::vector<int> rowof(P->nnz);
    for (int i = 0; i < N; ++i)
        for (int p = rp[i]; p < rp[i + 1]; ++p) rowof[p] = i;
    // element-wise difference quotients: slot of (element e, perturbed node
    // m, corner k) -> nonzero (node of k, node of m); slots of one nonzero
    // are contiguous and in ascending element order
    const int npe2 = npe * npe;
    std::vector<int> fd_q((size_t)T * npe2), fd_jptr(P->nnz + 1, 0), fd_epos((size_t)T * npe2);
    for (int e = 0; e < T; ++e) {
        const int* v = &c->h_elem_nodes[(size_t)e * npe];
        for (int m = 0; m < npe; ++m)
            for (int k = 0; k < npe; ++k) {
                const int i = v[k], j = v[m];
                const int* b = &cl[rp[i]];
                const int* f = std::lower_bound(b, &cl[0] + rp[i + 1], j);
                const int q = (int)(f - &cl[0]);
                fd_q[(size_t)e * npe2 + m * npe + k] = q;
                fd_jptr[q + 1]++;
            }
    }
    for (int q = 0; q < P->nnz; ++q) fd_jptr[q + 1] += fd_jptr[q];
    {
        std::vector<int> fill(fd_jptr.begin(), fd_jptr.end() - 1);
        for (size_t t = 0; t < fd_q.size(); ++t) fd_epos[t] = fill[fd_q[t]]++;
    }
    // blocks of contiguous nodes; on a large mesh a multiple of the SM count
    // (c->ilu_per_sm blocks per SM: fewer, larger blocks precondition better,
    // more, smaller ones have shorter level chains and share an SM)
    int nsm = 148;
    FVM_CUDA(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, c->device));
    int target = 1500;
    int nb;
    // per_sm 0 (the default): the fewest blocks per SM that keep a block at
    // most kAutoBlockRows rows, the size whose FP32 factor window still fits
    // the staged apply's shared memory (1 on the 200k-node box, 5 at 1M)
    constexpr double kAutoBlockRows = 1600.0;
    const int per_sm = c->ilu_per_sm > 0 ? c->ilu_per_sm
                                         : std::max(1, (int)std::ceil((double)N / (nsm * kAutoBlockRows)));
    if (N >= nsm * 256) nb = nsm * per_sm;
    else nb = std::max(1, (N + target - 1) / target);
    nb = std::min(nb, N);
    std::vector<int> bstart(nb + 1);
    for (int b = 0; b <= nb; ++b) bstart[b] = (int)(((long)N * b) / nb);
    int maxb = 0;
    for (int b = 0; b < nb; ++b) maxb = std::max(maxb, bstart[b + 1] - bstart[b]);
    if (maxb > 65535) throw Error("block-ILU: block too large");
    // Inside each block the factor works in a colour order: a greedy
    // colouring of the block's rows (natural order, smallest colour unused
    // by an earlier neighbour in the block), rows sorted by (colour, row).
    // No two rows of one colour are coupled, so each triangular sweep has as
    // many levels as colours (8 on the tetrahedral meshes, against about 33
    // in natural order).  Position r0 + ii of the factor is global row
    // lu_row[r0 + ii].
    std::vector<int> lu_ptr(N + 1, 0), lu_src, lu_diag(N), lu_row(N);
    std::vector<unsigned short> lu_col;
    std::vector<int> lvl(N), ulvl(N);
    std::vector<int> lvl_ptr(1, 0), lvl_rows, blk_lvl(1, 0), ulvl_ptr(1, 0), ulvl_rows, blk_ulvl(1, 0);
    int nlmax = 0;
    // Schur coupling: interface rows last, levels split by group, and the
    // off-block entries of each factor position
    P->schur_iters = c->schur_iters;
    const bool schur = P->schur_iters >= 0;
    std::vector<int> sch_lv(2 * (size_t)nb, 0), sch_nin(nb, 0), o_ptr(N + 1, 0), o_col, o_src;
    for (int b = 0; b < nb; ++b) {
        int r0 = bstart[b], r1 = bstart[b + 1];
        int nin = r1 - r0;
        const std::vector<int> ord = block_colour_order(rp, cl, r0, r1, schur, &nin);
        sch_nin[b] = nin;
        std::vector<int> linv(r1 - r0);
        for (int ii = 0; ii < r1 - r0; ++ii) linv[ord[ii]] = ii;
        std::vector<std::pair<int, int>> ent;
        for (int ii = 0; ii < r1 - r0; ++ii) {
            const int i = r0 + ord[ii], q = r0 + ii;
            lu_row[q] = i;
            ent.clear();
            for (int p = rp[i]; p < rp[i + 1]; ++p) {
                int j = cl[p];
                if (j < r0 || j >= r1) {
                    if (schur) { o_col.push_back(j); o_src.push_back(p); }
                    continue;
                }
                ent.emplace_back(linv[j - r0], p);
            }
            o_ptr[q + 1] = (int)o_col.size();
            std::sort(ent.begin(), ent.end());
            lu_diag[q] = -1;
            for (auto& e : ent) {
                if (e.first == ii) lu_diag[q] = (int)lu_src.size();
                lu_src.push_back(e.second);
                lu_col.push_back((unsigned short)e.first);
            }
            lu_ptr[q + 1] = (int)lu_src.size();
            if (lu_diag[q] < 0) throw Error("block-ILU: missing diagonal");
        }
        // with the Schur coupling no level mixes interior and interface
        // rows: forward, every interface row comes after the last interior
        // level; backward, every interior row after the last interface level
        int nl = 0, lvB = 0;
        for (int i = r0; i < r1; ++i) {
            int l = 0;
            for (int p = lu_ptr[i]; p < lu_diag[i]; ++p) l = std::max(l, lvl[r0 + lu_col[p]] + 1);
            if (schur && i - r0 >= nin) l = std::max(l, lvB);
            lvl[i] = l;
            nl = std::max(nl, l + 1);
            if (i - r0 < nin) lvB = nl;
        }
        int nu = 0, uvS = 0;
        for (int i = r1 - 1; i >= r0; --i) {
            int l = 0;
            for (int p = lu_diag[i] + 1; p < lu_ptr[i + 1]; ++p) l = std::max(l, ulvl[r0 + lu_col[p]] + 1);
            if (schur && i - r0 < nin) l = std::max(l, uvS);
            ulvl[i] = l;
            nu = std::max(nu, l + 1);
            if (i - r0 >= nin) uvS = nu;
        }
        sch_lv[2 * (size_t)b] = lvB;
        sch_lv[2 * (size_t)b + 1] = uvS;
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
    // elimination schedule in level order (window positions relative to
    // each block's 8-aligned window base, as the factorisation indexes); the
    // same update set and order as merging row i with U(k) for each L entry
    std::vector<int> seg_ptr(lvl_ptr.size(), 0);
    std::vector<unsigned> upd;
    size_t seg_max = 0;
    for (int b = 0; b < nb; ++b) {
        const int r0 = bstart[b];
        const int base = lu_ptr[r0] & ~7;
        for (int g = blk_lvl[b]; g < blk_lvl[b + 1]; ++g) {
            seg_ptr[g] = (int)upd.size();
            const int q0 = lvl_ptr[g], q1 = lvl_ptr[g + 1];
            const size_t head = upd.size();
            upd.resize(head + (q1 - q0), 0u);
            for (int q = q0; q < q1; ++q) {
                const int i = lvl_rows[q];
                upd[head + (q - q0)] = (unsigned)(upd.size() - head);
                for (int p = lu_ptr[i]; p < lu_diag[i]; ++p) {
                    const size_t cw = upd.size();
                    upd.push_back(0u);
                    const int k = r0 + lu_col[p];
                    int kpos = lu_diag[k] + 1;
                    const int kend = lu_ptr[k + 1];
                    for (int jj = p + 1; jj < lu_ptr[i + 1] && kpos < kend; ++jj) {
                        const int j = lu_col[jj];
                        while (kpos < kend && lu_col[kpos] < j) ++kpos;
                        if (kpos < kend && lu_col[kpos] == j)
                            upd.push_back((unsigned)(jj - base) | ((unsigned)(kpos - base) << 16));
                    }
                    upd[cw] = (unsigned)(upd.size() - cw - 1);
                }
            }
            seg_max = std::max(seg_max, upd.size() - head);
        }
        seg_ptr[blk_lvl[b + 1]] = (int)upd.size();
    }
    if (upd.size() >= (size_t)INT32_MAX) throw Error("block-ILU: elimination schedule too large");
    P->nb = nb;
    P->maxb = maxb;
    P->nlevels_max = nlmax;
    // per-block metadata records of the staged apply (layout of
    // ilu_meta_words), 16-byte aligned
    std::vector<unsigned short> meta;
    std::vector<int> meta_off(1, 0);
    for (int b = 0; b < nb; ++b) {
        const int r0 = bstart[b], r1 = bstart[b + 1], nr = r1 - r0;
        const int base = lu_ptr[r0] & ~7;
        const int la = blk_lvl[b], nl = blk_lvl[b + 1] - la;
        const int ua = blk_ulvl[b], nu = blk_ulvl[b + 1] - ua;
        const size_t start = meta.size();
        for (int i = 0; i <= nr; ++i) meta.push_back((unsigned short)(lu_ptr[r0 + i] - base));
        for (int i = 0; i < nr; ++i) meta.push_back((unsigned short)(lu_diag[r0 + i] - base));
        for (int i = 0; i < nr; ++i) meta.push_back((unsigned short)(lvl_rows[r0 + i] - r0));
        for (int i = 0; i < nr; ++i) meta.push_back((unsigned short)(ulvl_rows[r0 + i] - r0));
        for (int l = 0; l <= nl; ++l) meta.push_back((unsigned short)(lvl_ptr[la + l] - r0));
        for (int l = 0; l <= nu; ++l) meta.push_back((unsigned short)(ulvl_ptr[ua + l] - r0));
        meta.resize(start + ilu_meta_words(nr, (size_t)nl + nu + 2), 0);
        meta_off.push_back((int)meta.size());
    }
    {
        size_t need64 = 0, need32 = 0;
        bool fits16 = true;
        for (int b = 0; b < nb; ++b) {
            size_t nr = bstart[b + 1] - bstart[b];
            // the 16-byte aligned copy window of ilu_window()
            size_t wn = (size_t)(((lu_ptr[bstart[b + 1]] + 7) & ~7) - (lu_ptr[bstart[b]] & ~7));
            if (wn >= 65535 || nr + 1 >= 65535) fits16 = false;
            size_t nlev = (size_t)(blk_lvl[b + 1] - blk_lvl[b]) + (size_t)(blk_ulvl[b + 1] - blk_ulvl[b]) + 2;
            for (size_t sz : {(size_t)8, (size_t)4}) {
                size_t need = ilu_stage_bytes(nr, wn, nlev, sz);
                if (sz == 8) need64 = std::max(need64, need);
                else need32 = std::max(need32, need);
            }
        }
        P->smem_stage[0] = (fits16 && need64 <= kMaxDynSmem) ? need64 : 0;
        P->smem_stage[1] = (fits16 && need32 <= kMaxDynSmem) ? need32 : 0;
        // two schedule buffers of scr_words words (at most what the
        // factorisation's threads hold in kIluFactorPre registers each)
        for (int pr = 0; pr < 2; ++pr) {
            const size_t st = round16(P->smem_stage[pr]);
            const size_t room = P->smem_stage[pr] && st < kMaxDynSmem ? (kMaxDynSmem - st) / 8 : 0;
            P->scr_words[pr] = (int)std::min<size_t>(std::min<size_t>(seg_max, room), (size_t)kIluFactorThreads * kIluFactorPre);
        }
        // entries per row held in registers by the staged triangular sweeps:
        // 8 covers the lower or upper part of a 3D row, 4 of a 2D row
        P->lanes = (double)lu_ptr[N] / N > 9.0 ? 8 : 4;
        // one thread per row of the widest level, in whole warps of 128 or 256
        int widest = 0;
        for (size_t g = 0; g + 1 < lvl_ptr.size(); ++g) widest = std::max(widest, lvl_ptr[g + 1] - lvl_ptr[g]);
        for (size_t g = 0; g + 1 < ulvl_ptr.size(); ++g) widest = std::max(widest, ulvl_ptr[g + 1] - ulvl_ptr[g]);
        P->apply_threads = widest > 128 ? 256 : 128;
        // the global-memory apply keeps the block's vector in shared memory
        if (!P->smem_stage[0]) {
            if (sizeof(double) * (size_t)maxb > kMaxDynSmem)
                throw Error("block-ILU: blocks too large for the FP64 apply (set more blocks per SM)");
            raise_smem_limit(k_ilu_apply<double>, sizeof(double) * (size_t)maxb);
        }
        if (!P->smem_stage[1]) {
            if (sizeof(float) * (size_t)maxb > kMaxDynSmem)
                throw Error("block-ILU: blocks too large for the FP32 apply (set more blocks per SM)");
            raise_smem_limit(k_ilu_apply<float>, sizeof(float) * (size_t)maxb);
        }
        if (P->smem_stage[0]) {
            raise_smem_limit(k_ilu_apply_smem<double, 4>, (size_t)P->smem_stage[0]);
            raise_smem_limit(k_ilu_apply_smem<double, 8>, (size_t)P->smem_stage[0]);
            raise_smem_limit(k_ilu_factor_smem<double>, (size_t)(round16(P->smem_stage[0]) + 8 * (size_t)P->scr_words[0]));
        }
        if (P->smem_stage[1]) {
            raise_smem_limit(k_ilu_apply_smem<float, 4>, (size_t)P->smem_stage[1]);
            raise_smem_limit(k_ilu_apply_smem<float, 8>, (size_t)P->smem_stage[1]);
            raise_smem_limit(k_ilu_factor_smem<float>, (size_t)(round16(P->smem_stage[1]) + 8 * (size_t)P->scr_words[1]));
        }
    }
    if (schur) {
        // the coupled apply keeps each block's staged factor plus the
        // forward result in shared memory through its grid barriers, so it
        // needs both to fit and every block resident at once
        int nsm2 = 148, coop = 0;
        FVM_CUDA(cudaDeviceGetAttribute(&nsm2, cudaDevAttrMultiProcessorCount, c->device));
        FVM_CUDA(cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, c->device));
        for (int pr = 0; pr < 2; ++pr) {
            P->schur_smem[pr] = 0;
            if (!P->smem_stage[pr] || !coop) continue;
            const size_t sz = pr ? sizeof(float) : sizeof(double);
            const size_t need = round16(P->smem_stage[pr]) + round16(sz * (size_t)maxb);
            if (need > kMaxDynSmem) continue;
            const void* kfn = schur_kernel(pr, P->lanes);
            raise_smem_limit(kfn, need);
            int per_sm = 0;
            FVM_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kfn, P->apply_threads, need));
            if ((long)per_sm * nsm2 >= nb) P->schur_smem[pr] = need;
        }
        P->schur_nrmax = maxb;
    }
    cudaStream_t s = c->stream;
    if (schur) {
        P->sch_lv.upload(sch_lv, s);
        P->sch_nin.upload(sch_nin, s);
        P->h_sch_nin = sch_nin;
        P->o_ptr.upload(o_ptr, s);
        if (o_col.empty()) { o_col.push_back(0); o_src.push_back(0); }
        P->o_col.upload(o_col, s);
        P->o_src.upload(o_src, s);
        P->xg.alloc(2 * (size_t)N);
        P->sbar.alloc(2);
        P->sbar.zero(s);
        P->serr.alloc(1);
        P->serr.zero(s);
        FVM_CUDA(cudaMallocHost(&P->h_serr, sizeof(int)));
        *P->h_serr = 0;
    }
    P->col.upload(P->h_col, s);
    P->rowof.upload(rowof, s);
    P->J.alloc(P->nnz);
    P->shift.alloc(N);
    P->fd_epos.upload(fd_epos, s);
    P->fd_jptr.upload(fd_jptr, s);
    P->fd_slots.alloc(fd_epos.size());
    P->krwb.alloc((size_t)c->nz * N);
    P->krwp.alloc((size_t)c->nz * N);
    P->dstor.alloc(N);
    P->ahhp.alloc(N);
    P->rowptr.upload(P->h_rowptr, s);
    P->bstart.upload(bstart, s);
    P->h_bstart = bstart;
    P->h_lu_row = lu_row;
    P->lu_ptr.upload(lu_ptr, s);
    // 8 padding entries so every block's widened copy window stays inside
    {
        // where fd_gather puts each Jacobian entry for the factorisation
        std::vector<int> lu_dst(P->nnz, -1);
        for (size_t p = 0; p < lu_src.size(); ++p) lu_dst[lu_src[p]] = (int)p;
        P->lu_dst.upload(lu_dst, s);
    }
    lu_src.resize(lu_src.size() + 8, 0);
    lu_col.resize(lu_col.size() + 8, 0);
    P->lu_src.upload(lu_src, s);
    P->Jw.alloc(lu_src.size());
    P->Jw.zero(s);
    P->lu_diag.upload(lu_diag, s);
    P->lu_row.upload(lu_row, s);
    P->lu_col.upload(lu_col, s);
    if (upd.empty()) upd.push_back(0u);
    P->seg_ptr.upload(seg_ptr, s);
    P->upd.upload(upd, s);
    P->meta.upload(meta, s);
    P->meta_off.upload(meta_off, s);
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
    (void)F0;   // the element-wise quotients difference each element's own partials
    fvm_launch(c, k_shift, grid_for(N, 256), 256, 0, s, N, y, yp, ewt, h, std::sqrt(DBL_EPSILON), P->shift.p);
    fvm_launch(c, k_fd_node, grid_for(N, 256), 256, 0, s, N, y, yp, cj, P->shift.p, c->zones.p, c->nz, c->nz_ptr.p,
               c->nz_zone.p, c->nz_w.p, c->rho0, P->krwb.p, P->krwp.p, P->dstor.p, P->ahhp.p);
    P->cj_setup = cj;
    P->setup_id++;
    {
        const int gb = grid_for(c->T, 256);
        const bool mz = c->nz > 1;
        auto run = [&](auto* slots) {
            using S = std::remove_pointer_t<decltype(slots)>;
            auto go = [&](auto kern) {
                fvm_launch(c, kern, gb, 256, 0, s, c->T, N, c->enodes.p, c->coef.p, c->xyz.p, c->eK.p,
                           c->kiso ? 1 : 0, c->estride, c->ezone.p, y, P->shift.p, P->krwb.p, P->krwp.p, c->upw.p,
                           c->rho0, P->fd_epos.p, slots);
            };
            if (c->dim == 3) {
                if (c->recompute) mz ? go(k_fd_elem<4, 6, true, true, S>) : go(k_fd_elem<4, 6, true, false, S>);
                else mz ? go(k_fd_elem<4, 6, false, true, S>) : go(k_fd_elem<4, 6, false, false, S>);
            } else {
                mz ? go(k_fd_elem<3, 3, false, true, S>) : go(k_fd_elem<3, 3, false, false, S>);
            }
            // the fused cycle's operator values too, once its layout exists
            float* opv = P->op_built && P->fused_ok ? P->op_val.p : nullptr;
            fvm_launch(c, k_fd_gather<S>, grid_for(P->nnz, 256), 256, 0, s, P->nnz, P->rowof.p, P->col.p,
                       P->fd_jptr.p, slots, c->invV.p, P->dstor.p, c->ntype.p, c->hD.p, y, P->shift.p, P->J.p,
                       P->lu_dst.p, P->Jw.p, opv ? P->op_dst.p : nullptr, opv);
            P->op_vals_setup = opv ? P->setup_id : -1;
        };
        // the FP64 slot buffer holds the FP32 slots in its first half
        if (precision) run(reinterpret_cast<float*>(P->fd_slots.p));
        else run(P->fd_slots.p);
    }
    c->tm.end(TM_FD_JAC, s);
    FVM_CUDA(cudaMemsetAsync(P->status.p, 0, sizeof(int), s));
    size_t nlu = P->lu_src.n;
    c->tm.begin(TM_ILU_FACTOR, s);
    if (P->smem_stage[precision]) {
        const int so = (int)round16(P->smem_stage[precision]);
        const int sw = P->scr_words[precision];
        size_t sm = (size_t)so + 8 * (size_t)sw;
        if (precision) {
            P->lu32.alloc(nlu);
            fvm_launch(c, k_ilu_factor_smem<float>, P->nb, kIluFactorThreads, sm, s, P->bstart.p, P->lu_ptr.p, P->Jw.p,
                       P->lu_diag.p, P->lu_col.p, P->lvl_ptr.p, P->lvl_rows.p, P->blk_lvl.p, P->seg_ptr.p, P->upd.p,
                       so, sw, P->lu32.p, P->status.p);
        } else {
            P->lu64.alloc(nlu);
            fvm_launch(c, k_ilu_factor_smem<double>, P->nb, kIluFactorThreads, sm, s, P->bstart.p, P->lu_ptr.p, P->Jw.p,
                       P->lu_diag.p, P->lu_col.p, P->lvl_ptr.p, P->lvl_rows.p, P->blk_lvl.p, P->seg_ptr.p, P->upd.p,
                       so, sw, P->lu64.p, P->status.p);
        }
    } else if (precision) {
        P->lu32.alloc(nlu);
        fvm_launch(c, k_ilu_factor<float>, P->nb, 128, 0, s, P->bstart.p, P->lu_ptr.p, P->Jw.p, P->lu_diag.p, P->lu_col.p,
                                                  P->lvl_ptr.p, P->lvl_rows.p, P->blk_lvl.p, P->lu32.p,
                                                  P->status.p);
    } else {
        P->lu64.alloc(nlu);
        fvm_launch(c, k_ilu_factor<double>, P->nb, 128, 0, s, P->bstart.p, P->lu_ptr.p, P->Jw.p, P->lu_diag.p, P->lu_col.p,
                                                   P->lvl_ptr.p, P->lvl_rows.p, P->blk_lvl.p, P->lu64.p,
                                                   P->status.p);
    }
    c->tm.end(TM_ILU_FACTOR, s);
    FVM_CUDA(cudaMemcpyAsync(P->h_status, P->status.p, sizeof(int), cudaMemcpyDeviceToHost, s));
    P->factored = precision;
}

void jacobian_apply(fvm_ctx* c, double cj, const double* x, double* y, const int* skip, const double* dcj_dev) {
    BlockILU* P = c->ilu;
    if (!P || P->factored < 0) throw Error("jacobian_apply: preconditioner not set up");
    fvm_launch_pdl(c, k_jac_apply, grid_for(4L * c->N, 256), 256, 0, c->stream, c->N, P->rowptr.p, P->col.p,
                   P->J.p, P->ahhp.p, c->ntype.p, cj - P->cj_setup, x, y, skip, dcj_dev);
}

double jacobian_cj_setup(fvm_ctx* c) { return c->ilu ? c->ilu->cj_setup : 0.0; }
int ilu_factored(fvm_ctx* c) { return c->ilu ? c->ilu->factored : -1; }
bool schur_active(fvm_ctx* c) { return c->ilu && c->ilu->schur_iters >= 0; }

int ilu_status(fvm_ctx* c) {
    if (!c->ilu || !c->ilu->h_status) return 0;
    ctx_sync(c);
    return *c->ilu->h_status;
}

int ilu_status_seen(fvm_ctx* c) { return c->ilu && c->ilu->h_status ? *c->ilu->h_status : 0; }

bool ilu_ready(fvm_ctx* c) { return c->ilu && c->ilu->factored >= 0; }

int schur_status(fvm_ctx* c) {
    BlockILU* P = c->ilu;
    if (!P || P->schur_iters < 0 || !P->h_serr) return 0;
    FVM_CUDA(cudaMemcpyAsync(P->h_serr, P->serr.p, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
    ctx_sync(c);
    const int e = *P->h_serr;
    if (e) FVM_CUDA(cudaMemsetAsync(P->serr.p, 0, sizeof(int), c->stream));
    return e;
}

void psolve_dev(fvm_ctx* c, const double* r, double* z, const int* skip) {
    BlockILU* P = c->ilu;
    if (!P || P->factored < 0) throw Error("psolve: preconditioner not set up");
    cudaStream_t s = c->stream;
    c->tm.begin(TM_ILU_APPLY, s);
    struct EndTimer {
        fvm_ctx* c;
        ~EndTimer() { c->tm.end(TM_ILU_APPLY, c->stream); }
    } end_timer{c};
    if (P->schur_iters >= 0) {
        if (!P->schur_smem[P->factored])
            throw Error("psolve: the Schur coupling needs every block's staged factor and forward result in shared "
                        "memory with all blocks resident at once (use the FP32 factor on large blocks)");
        if (P->factored) launch_schur_apply(c, P, P->lu32.p, r, z, skip);
        else launch_schur_apply(c, P, P->lu64.p, r, z, skip);
        return;
    }
    if (P->smem_stage[P->factored]) {
        size_t sm = P->smem_stage[P->factored];
        auto go = [&](auto kern, const auto* lu) {
            fvm_launch_pdl(c, kern, P->nb, P->apply_threads, sm, s, P->bstart.p, P->lu_ptr.p, P->lu_col.p, P->meta.p,
                       P->meta_off.p, P->blk_lvl.p, P->blk_ulvl.p, lu, P->lu_row.p, r, z, P->status.p, skip);
        };
        if (P->factored) {
            if (P->lanes == 8) go(k_ilu_apply_smem<float, 8>, P->lu32.p);
            else go(k_ilu_apply_smem<float, 4>, P->lu32.p);
        } else {
            if (P->lanes == 8) go(k_ilu_apply_smem<double, 8>, P->lu64.p);
            else go(k_ilu_apply_smem<double, 4>, P->lu64.p);
        }
    } else if (P->factored) {
        size_t sm = sizeof(float) * P->maxb;
        fvm_launch_pdl(c, k_ilu_apply<float>, P->nb, 128, sm, s, P->bstart.p, P->lu_ptr.p, P->lu_diag.p, P->lu_col.p, P->lvl_ptr.p,
                                                 P->lvl_rows.p, P->blk_lvl.p, P->ulvl_ptr.p, P->ulvl_rows.p,
                                                 P->blk_ulvl.p, P->lu32.p, P->lu_row.p, r, z, skip);
    } else {
        size_t sm = sizeof(double) * P->maxb;
        fvm_launch_pdl(c, k_ilu_apply<double>, P->nb, 128, sm, s, P->bstart.p, P->lu_ptr.p, P->lu_diag.p, P->lu_col.p, P->lvl_ptr.p,
                                                  P->lvl_rows.p, P->blk_lvl.p, P->ulvl_ptr.p, P->ulvl_rows.p,
                                                  P->blk_ulvl.p, P->lu64.p, P->lu_row.p, r, z, skip);
    }
}

} // namespace fvmb

using namespace fvmb;

void fvmb_destroy_ilu(fvmb::BlockILU* p) {
    if (!p) return;
    if (p->h_status) cudaFreeHost(p->h_status);
    if (p->h_serr) cudaFreeHost(p->h_serr);
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
        if (schur_status(c)) throw Error("fvm_psolve: a grid barrier of the Schur-coupled apply timed out");
        return 0;
    } catch (const Error& ex) {
        set_error(ex.what());
        return ex.code;
    } catch (const std::exception& ex) {
        set_error(ex.what());
        return -1;
    }
}

extern "C" int fvm_set_precond_blocks(fvm_ctx* c, int per_sm) {
    try {
        if (!c) throw Error("fvm_set_precond_blocks: null context");
        if (per_sm < 0 || per_sm > 16)
            throw Error("fvm_set_precond_blocks: blocks per SM must be in [1, 16], or 0 for automatic");
        FVM_CUDA(cudaStreamSynchronize(c->stream));
        c->ilu_per_sm = per_sm;
        if (c->ilu) {
            fvmb_destroy_ilu(c->ilu);
            c->ilu = nullptr;
        }
        return 0;
    } catch (const Error& ex) {
        set_error(ex.what());
        return ex.code;
    } catch (const std::exception& ex) {
        set_error(ex.what());
        return -1;
    }
}

extern "C" int fvm_set_precond_schur(fvm_ctx* c, int iters) {
    try {
        if (!c) throw Error("fvm_set_precond_schur: null context");
        if (iters < -1 || iters > 64) throw Error("fvm_set_precond_schur: iterations must be in [-1, 64]");
        FVM_CUDA(cudaStreamSynchronize(c->stream));
        c->schur_iters = iters;
        if (c->ilu) {
            fvmb_destroy_ilu(c->ilu);
            c->ilu = nullptr;
        }
        return 0;
    } catch (const Error& ex) {
        set_error(ex.what());
        return ex.code;
    } catch (const std::exception& ex) {
        set_error(ex.what());
        return -1;
    }
}

extern "C" int fvm_precond_schur_info(fvm_ctx* c, int* iters, int* interface_rows, int* supported) {
    try {
        if (!c || !c->ilu || !c->ilu->built) throw Error("fvm_precond_schur_info: no preconditioner");
        BlockILU* P = c->ilu;
        if (iters) *iters = P->schur_iters;
        if (interface_rows) {
            long n = 0;
            if (P->schur_iters >= 0)
                for (int b = 0; b < P->nb; ++b) n += P->h_bstart[b + 1] - P->h_bstart[b] - P->h_sch_nin[b];
            *interface_rows = (int)n;
        }
        if (supported) *supported = (P->schur_smem[0] ? 1 : 0) | (P->schur_smem[1] ? 2 : 0);
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
