// Block-ILU(0) preconditioner state and the device helpers of its
// shared-memory ("staged") triangular solves, shared by the preconditioner
// kernels (precond.cu) and the fused Arnoldi kernel (arnoldi_fused.cu).
#pragma once

#include "ctx.cuh"
#include "tc05.cuh"

#include <cstdint>
#include <vector>

namespace fvmb {

struct BlockILU {
    bool built = false;
    int nnz = 0, ncol = 0;
    std::vector<int> h_rowptr, h_col, h_colour;
    DevBuf<int> rowof, col;
    DevBuf<double> J;
    DevBuf<double> shift;
    // element-wise finite-difference Jacobian
    DevBuf<int> fd_epos;      // [T*npe*npe] slot of (element, perturbed node, corner)
    DevBuf<int> fd_jptr;      // [nnz+1] slots of each nonzero
    DevBuf<double> fd_slots;  // [T*npe*npe]
    DevBuf<double> krwb, krwp, dstor;
    // assembled-operator Krylov products (fvm_opts.krylov_operator = 1):
    // device row pointers of J, the storage coefficient ahh(h + d) behind
    // the cj term of J's diagonal, and the cj of the current set-up
    DevBuf<int> rowptr;
    DevBuf<double> ahhp;
    double cj_setup = 0.0;
    long setup_id = 0;             // set-ups done (the fused operator refreshes after each)
    std::vector<int> h_lu_row, h_bstart;
    // the same operator for the fused Arnoldi kernel: J's rows in factor
    // order, 32 rows per slice (one warp), each slice stored entry-major
    // (entry k of the slice's lane l at slice start + 32 k + l, rows shorter
    // than the slice's longest padded with zero entries of their own column)
    bool op_built = false, fused_ok = false;
    long op_setup_id = -1;
    DevBuf<int> op_slptr, op_blksl, op_src;
    DevBuf<int> op_dst;                        // [nnz] slice position of each Jacobian entry
    long op_vals_setup = -1;                   // set-up whose values fd_gather wrote into op_val
    DevBuf<unsigned short> op_lcol, op_self;   // 16-bit columns into each block's node list
    DevBuf<int> halo_ptr, halo_node;           // each block's node list: its rows and halo
    DevBuf<int> nbr_ptr, nbr;                  // blocks whose rows a block's operator reads
    DevBuf<unsigned> flags;                    // per block: last step published
    DevBuf<float> op_val, op_dg;
    size_t fused_smem = 0, fused_smem_d = 0, fused_stage = 0;
    bool fused_var_ok[2] = {false, false};   // CGS2 / delayed variant can run
    int fused_threads = 0, fused_nrmax = 0, fused_nhmax = 0, fused_nqp = 0;
    int nb = 0, maxb = 0;
    DevBuf<int> bstart, lu_ptr, lu_src, lu_diag;
    DevBuf<int> lu_dst;       // [nnz] factor position of each Jacobian entry, -1 off the blocks
    DevBuf<double> Jw;        // the set-up's Jacobian in factor order (written by fd_gather)
    DevBuf<int> lu_row;       // global row of each factor position (colour order inside the blocks)
    // ILU(0) elimination schedule of the shared-memory factorisation, one
    // contiguous segment per level (upd[seg_ptr[g] .. seg_ptr[g+1]) for the
    // global level g): the offset of each row's list in the segment, then
    // per row and per L entry in column order a count word followed by that
    // many (target | source << 16) window positions
    DevBuf<int> seg_ptr;
    DevBuf<unsigned> upd;
    int scr_words[2] = {0, 0};   // shared-memory schedule scratch of the factorisation (words), by precision
    DevBuf<unsigned short> lu_col;
    DevBuf<int> lvl_ptr, lvl_rows, blk_lvl, ulvl_ptr, ulvl_rows, blk_ulvl;
    DevBuf<unsigned short> meta;   // per-block metadata records of the staged apply
    DevBuf<int> meta_off;
    DevBuf<double> lu64;
    DevBuf<float> lu32;
    int factored = -1;        // precision of the current factor, -1 none
    DevBuf<int> status;
    int* h_status = nullptr;  // pinned
    int nlevels_max = 0;
    size_t smem_stage[2] = {0, 0};   // staged apply: shared bytes for FP64 / FP32, 0 = not possible
    int lanes = 4;                   // row entries prefetched per thread in the staged sweeps
    int apply_threads = 128;         // CTA of the staged apply: 128, or 256 when a level is wider
    // Schur interface coupling (fvm_set_precond_schur; decomp/schur.c):
    // each block's interface rows (coupled to another block) follow its
    // interior rows in the factor; the forward levels [0, lvB) of a block
    // hold only interior rows and the rest only interface rows, the
    // backward levels [0, uvS) only interface rows and the rest only
    // interior rows (sch_lv[2b] = lvB, sch_lv[2b+1] = uvS, sch_nin[b] =
    // interior rows).  o_ptr/o_col/o_src: the off-block entries of each
    // factor position (global column, index into J), ascending column.
    int schur_iters = -1;
    DevBuf<int> sch_lv, sch_nin, o_ptr, o_col, o_src;
    std::vector<int> h_sch_nin;
    DevBuf<double> xg;               // 2 N: published interface iterates (node order), by parity
    DevBuf<unsigned> sbar;           // grid barrier of the coupled apply
    DevBuf<int> serr;                // 3: a grid barrier of the coupled apply timed out
    int* h_serr = nullptr;           // pinned
    size_t schur_smem[2] = {0, 0};   // dynamic shared bytes of the coupled apply, 0 = not possible
    int schur_nrmax = 0;
};

// largest dynamic shared-memory carve-out a CTA may request on sm_100
constexpr size_t kMaxDynSmem = 227 * 1024;
// threads of a staged triangular-solve CTA: levels hold a few dozen rows,
// so a small CTA keeps the per-level barrier cheap
constexpr int kIluThreads = 256;   // largest CTA of the staged apply

// Staged variant: the CTA first brings its block's factor into shared
// memory, then runs the level loops entirely there, so each level costs a
// few shared-memory latencies and a barrier instead of a dependent chain of
// L2/HBM loads.  The block's entries are one contiguous range of the factor
// arrays; the copy window is that range widened to 8-entry (16-byte)
// boundaries and moved by two 1D TMA bulk copies (cp.async.bulk, completion
// counted on an mbarrier, bounded wait), while the threads fill the row
// pointers, pivot positions, level lists and right-hand side alongside.
// Shared layout: x[T nrows, 16-B padded] | val[T window] | col[u16 window] |
// rp[u16 nrows+1] | dg[u16 nrows] | lrow[u16 nrows] | urow[u16 nrows] |
// lptr[u16 nl+1] | uptr[u16 nu+1] | mbarrier (8-B aligned)
struct IluWindow {
    int base, wn;   // first entry of the copy window (multiple of 8), window length
};
__device__ __forceinline__ IluWindow ilu_window(int e0, int e1) {
    IluWindow w;
    w.base = e0 & ~7;
    w.wn = ((e1 + 7) & ~7) - w.base;
    return w;
}
__host__ __device__ __forceinline__ size_t round16(size_t b) { return (b + 15) & ~(size_t)15; }

// u16 words of a block's metadata record: rp (nr+1) | dg (nr) | lrow (nr) |
// urow (nr) | lptr (nl+1) | uptr (nu+1), padded to 16 bytes
__host__ __device__ __forceinline__ size_t ilu_meta_words(size_t nr, size_t nlev) {
    return (4 * nr + 1 + nlev + 7) & ~(size_t)7;
}

// shared bytes of the staged kernels for one block (host and device agree);
// nlev = nl + 1 + nu + 1 level offsets of the two sweeps
__host__ __device__ __forceinline__ size_t ilu_stage_bytes(size_t nr, size_t wn, size_t nlev, size_t sz) {
    return round16(round16(nr * sz) + wn * (sz + 2) + ilu_meta_words(nr, nlev) * 2) + 16;
}

template <class T>
__device__ __forceinline__ void ilu_stage_bulk(T* val, unsigned short* col, const T* lu,
                                               const unsigned short* lu_col, IluWindow w, uint64_t* bar,
                                               unsigned short* meta_dst = nullptr,
                                               const unsigned short* meta_src = nullptr, int meta_words = 0) {
    if (threadIdx.x == 0) {
        uint32_t b = tc05::smem_u32(bar);
        uint32_t bytes = (uint32_t)(w.wn * (sizeof(T) + sizeof(unsigned short)) + meta_words * 2);
        asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(b), "r"(bytes));
        asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                         tc05::smem_u32(val)),
                     "l"(lu + w.base), "r"((uint32_t)(w.wn * sizeof(T))), "r"(b)
                     : "memory");
        asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                         tc05::smem_u32(col)),
                     "l"(lu_col + w.base), "r"((uint32_t)(w.wn * sizeof(unsigned short))), "r"(b)
                     : "memory");
        if (meta_words)
            asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                             tc05::smem_u32(meta_dst)),
                         "l"(meta_src), "r"((uint32_t)(meta_words * 2)), "r"(b)
                         : "memory");
    }
}

// One triangular sweep over the levels [l0, nlv): rows of a level are
// independent, one thread per row.  UPPER: x_i = (x_i - sum_{p>diag}) *
// inverse pivot; else x_i = x_i - sum_{p<diag} (unit lower triangle).  A
// thread's row of level l+1 -- its index, range, first KM entries and pivot,
// none of which depend on x -- is fetched while level l is computed, so after
// each barrier only the x loads (independent of each other) and the
// accumulation remain on the critical path.
template <class T, int KM, bool UPPER> struct IluRow {
    int li, p0, p1;
    T v[KM];
    unsigned short c[KM];
    T piv;
};

template <class T, int KM, bool UPPER>
__device__ __forceinline__ void ilu_fetch(IluRow<T, KM, UPPER>& R, int l, int nlv, const T* val,
                                          const unsigned short* col, const unsigned short* rp,
                                          const unsigned short* dg, const unsigned short* rows,
                                          const unsigned short* lptr) {
    R.li = -1;
#pragma unroll
    for (int k = 0; k < KM; ++k) R.c[k] = 0;
    if (l >= nlv) return;
    const int q = lptr[l] + threadIdx.x;
    if (q >= lptr[l + 1]) return;
    R.li = rows[q];
    const int d = dg[R.li];
    R.p0 = UPPER ? d + 1 : rp[R.li];
    R.p1 = UPPER ? rp[R.li + 1] : d;
#pragma unroll
    for (int k = 0; k < KM; ++k) {
        const int p = R.p0 + k < R.p1 ? R.p0 + k : 0;   // unused slots read entry 0
        R.v[k] = val[p];
        R.c[k] = col[p];
    }
    R.piv = UPPER ? val[d] : (T)1;
}

template <class T, int KM, bool UPPER>
__device__ __forceinline__ void ilu_sweep(T* x, const T* val, const unsigned short* col, const unsigned short* rp,
                                          const unsigned short* dg, const unsigned short* rows,
                                          const unsigned short* lptr, int l0, int nlv) {
    IluRow<T, KM, UPPER> cur, nxt;
    ilu_fetch(cur, l0, nlv, val, col, rp, dg, rows, lptr);
    const int wbase = threadIdx.x & ~31;
    for (int l = l0; l < nlv; ++l) {
        // a warp with no row in this level or the next goes straight to the
        // level barrier
        const int nq_cur = lptr[l + 1] - lptr[l];
        const int nq_nxt = l + 1 < nlv ? lptr[l + 2] - lptr[l + 1] : 0;
        if (wbase >= nq_cur && wbase >= nq_nxt) {
            nxt.li = -1;
#pragma unroll
            for (int k = 0; k < KM; ++k) nxt.c[k] = 0;
            __syncthreads();
            cur = nxt;
            continue;
        }
        // issue this level's x loads first (threads without a row read entry
        // 0 and store nothing), then fetch the next level's row while they
        // are in flight, then accumulate
        const bool act = cur.li >= 0;
        const int li = act ? cur.li : 0;
        T xv[KM];
#pragma unroll
        for (int k = 0; k < KM; ++k) xv[k] = x[cur.c[k]];
        const T xi = x[li];
        const int q0 = lptr[l], q1 = lptr[l + 1];
        ilu_fetch(nxt, l + 1, nlv, val, col, rp, dg, rows, lptr);
        if (act) {
            T acc = (T)0;
#pragma unroll
            for (int k = 0; k < KM; ++k)
                if (cur.p0 + k < cur.p1) acc += cur.v[k] * xv[k];
            // entries past the first KM: loads four at a time, then the
            // accumulation in entry order
            for (int p = cur.p0 + KM; p < cur.p1; p += 4) {
                T tv[4], tx[4];
#pragma unroll
                for (int k = 0; k < 4; ++k) {
                    const bool in = p + k < cur.p1;
                    const int cc = in ? col[p + k] : 0;
                    tv[k] = in ? val[p + k] : (T)0;
                    tx[k] = x[cc];
                }
#pragma unroll
                for (int k = 0; k < 4; ++k)
                    if (p + k < cur.p1) acc += tv[k] * tx[k];
            }
            x[li] = UPPER ? (xi - acc) * cur.piv : xi - acc;
        }
        // rows of a level wider than the CTA
        for (int q = q0 + threadIdx.x + blockDim.x; q < q1; q += blockDim.x) {
            const int lj = rows[q];
            const int d = dg[lj];
            const int p0 = UPPER ? d + 1 : rp[lj], p1 = UPPER ? rp[lj + 1] : d;
            T acc = (T)0;
            for (int p = p0; p < p1; ++p) acc += val[p] * x[col[p]];
            x[lj] = UPPER ? (x[lj] - acc) * val[d] : x[lj] - acc;
        }
        __syncthreads();
        cur = nxt;
    }
}

} // namespace fvmb
