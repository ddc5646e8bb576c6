// fvm_create / fvm_destroy and the residual kernel chain.
//
// One residual evaluation F(t, y, y') is three launches:
//   1. node pass    van Genuchten at every (node, zone) pair -> krw, and the
//                   storage term ahh * y' (process_volumes_psk +
//                   process_derivative_coefficients, fvmpor.h:875-945);
//   2. element pass for each element the CV-face fluxes
//                   rho0 * krw_up * (sum_k C_fk h_k + G_f) of its dim+1
//                   choose 2 faces, summed into one partial per element node
//                   (shape-gradient SpMVs + process_fluxes, fvmpor.h:682-759,
//                   fvmpor_ODE_impl.cpp:75-80);
//   3. node gather  res_i = (1/V_i) sum over the node's incident elements, in
//                   ascending element order, of those partials, plus the
//                   boundary-flux term, minus ahh_i y'_i; Dirichlet rows
//                   h_D - h (residual_evaluation, fvmpor_ODE_impl.cpp:99-116).
// The gather reads a fixed node-ordered incidence list, so the result is
// bitwise reproducible run to run and independent of the launch shape; no
// floating-point atomics are used anywhere.
#include "ctx.cuh"
#include "tc05.cuh"

#include <algorithm>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <numeric>

namespace fvmb {

static thread_local std::string g_last_error;
void set_error(const std::string& msg) { g_last_error = msg; }

void raise_smem_limit(const void* func, size_t bytes) {
    static std::mutex mu;
    static std::map<std::pair<int, const void*>, size_t> limit;
    int dev = 0;
    FVM_CUDA(cudaGetDevice(&dev));
    std::lock_guard<std::mutex> lock(mu);
    size_t& cur = limit[{dev, func}];
    if (bytes <= cur) return;
    FVM_CUDA(cudaFuncSetAttribute(func, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes));
    cur = bytes;
}

constexpr int kBlock = 256;
constexpr int kDefaultChunk = 512;   // elements per chunk of the element pass

// ------------------------------------------------------------------ kernels
// Besides the node arrays, the node pass writes the head and (single zone)
// krw of every node into each element chunk that holds the node, at the
// chunk-major copy positions cpos[part_ptr[i] .. part_ptr[i+1]), so the
// element pass streams its chunk's node data contiguously.
struct NodeCopies {
    const int* part_ptr = nullptr;   // [N+1]
    const int* cpos = nullptr;       // [P] chunk-major position of each copy
    double* ch_h = nullptr;          // [P] (several zones)
    double* ch_hk = nullptr;         // [P][2] (head, krw) pairs (one zone): one 16-byte store per copy
};

__global__ void k_node(int N, const double* __restrict__ y, const double* __restrict__ yp,
                       Perturb pt, const ZoneDev* __restrict__ zones, int nz,
                       const int* __restrict__ nz_ptr, const int* __restrict__ nz_zone,
                       const double* __restrict__ nz_w, double rho0, double* __restrict__ krw,
                       double* __restrict__ hstar, double* __restrict__ stor, NodeCopies cp) {
    pdl_wait_and_trigger();
    if (pt.skip && *pt.skip) return;
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N) return;
    double h = y[i], hp = yp[i];
    if (pt.mode == 1) {
        double sg = pt.sigma_dev ? *pt.sigma_dev : pt.sigma;
        double p = sg * pt.v[i];
        h = h + p;
        hp = hp + (pt.cj_dev ? *pt.cj_dev : pt.cj) * p;
        hstar[i] = h;
    } else if (pt.mode == 2) {
        if (pt.colour[i] == pt.c) {
            double p = pt.shift[i];
            h = h + p;
            hp = hp + pt.cj * p;
        }
        hstar[i] = h;
    }
    double phi = 0.0, dsw = 0.0;
    const int c0 = cp.part_ptr[i], c1 = cp.part_ptr[i + 1];
    if (nz == 1) {
        double Sw, d, k;
        van_genuchten(h, zones[0], Sw, d, k);
        krw[i] = k;
        phi = zones[0].phi * nz_w[i];
        dsw = d * nz_w[i];
        for (int q = c0; q < c1; ++q) {
            const int cm = cp.cpos[q];
            reinterpret_cast<double2*>(cp.ch_hk)[cm] = make_double2(h, k);
        }
    } else {
        for (int q = c0; q < c1; ++q) cp.ch_h[cp.cpos[q]] = h;
        for (int p = nz_ptr[i]; p < nz_ptr[i + 1]; ++p) {
            int z = nz_zone[p];
            double w = nz_w[p];
            double Sw, d, k;
            van_genuchten(h, zones[z], Sw, d, k);
            krw[(size_t)z * N + i] = k;
            phi += zones[z].phi * w;
            dsw += d * w;
        }
    }
    double ahh = phi * dsw;
    ahh = ahh * rho0;
    stor[i] = hp * ahh;
}


// Element pass: persistent CTAs walk the element chunks (CE consecutive
// elements each, chunk c = blockIdx.x, blockIdx.x + gridDim.x, ...) through
// a two-stage TMA pipeline.  While the CTA computes chunk i from one shared
// stage, one thread has already issued the 1D bulk copies (cp.async.bulk,
// completion counted on that stage's mbarrier) that bring chunk i+1 into the
// other stage: the chunk's distinct nodes -- head, krw and, for the
// rebuilt-geometry variant, coordinates, from the chunk-major copies the
// node pass wrote -- and its element records (local corner ids, upwind
// flags, conductivity) and node-ordered corner lists.  Every array is padded
// per chunk to 16-byte multiples, so each copy is one aligned transfer.
// Each element then reads its corners from shared memory through 16-bit
// local ids and leaves its dim+1 corner partials
//   sum over its faces of -/+ rho0 krw_up (sum_k C_fk h_k + G_f)
// (shape-gradient SpMVs + process_fluxes, fvmpor.h:682-759,
// fvmpor_ODE_impl.cpp:75-80) in shared memory (corner-major, so the writes
// of a warp hit distinct banks).  Every chunk node sums its corners in
// ascending element order and writes ONE partial, chunk-major; the gather
// adds a node's partials in ascending chunk order, so the residual is
// bitwise reproducible and independent of the launch shape, without
// floating-point atomics.
//   VAR 0: stored coefficients C_fk, G_f (any simplex), streamed from global
//   VAR 1: tetrahedra, fluxes rebuilt from the vertices (tet_face_fluxes)
struct ElemArgs {
    int T, N, CE, nch, kiso, estride;
    int nnmax;                    // largest padded node segment of a chunk
    const int2* ch_seg;           // [nchunk] (padded start, node count) of each chunk
    const int* ch_node;           // [P] global node ids, ascending per chunk (several zones)
    const ushort4* elocal;        // [estride] chunk-local corner ids
    const unsigned short* ch_lptr;// [P] corner-list offsets, at the chunk's node segment
    const unsigned short* ch_lc;  // [estride*npe] corner lists (k*CE + el), per chunk
    const double* coef;           // VAR 0
    const double* ch_xyz;         // VAR 1: [3][P] chunk-major coordinates
    const double* eK;             // VAR 1: [estride] (kiso) or [3][estride]
    const int* ezone;
    const double* krw;            // [nz][N] (several zones)
    const double* ch_h;           // [P] chunk-major head (written by the node pass; several zones)
    const double* ch_hk;          // [P][2] chunk-major (head, krw) pairs (one zone)
    const unsigned char* upw;     // [8*estride]
    double rho0;
    double* part;                 // [P] chunk-major partials
    int* err;                     // 5 = a pipeline wait gave up
    size_t P;
    const int* skip;              // skip the launch when *skip != 0
};

constexpr int kElemThreads = 256;

__host__ __device__ __forceinline__ int pad8(int n) { return (n + 7) & ~7; }

// byte offsets inside one pipeline stage (host and device agree)
struct StageLayout {
    size_t h, krw, xyz, eloc, upw, ek, lc, lp, bytes;
    __host__ __device__ StageLayout(int CE, int npe, int nnmax, bool mz, bool rc, bool kiso) {
        const size_t nd = (size_t)nnmax * 8;
        // one zone: (head, krw) pairs in [h, h + 2 nd); several zones: head
        // only (krw is read per zone from the node-major array)
        h = 0;
        krw = h + nd;
        xyz = krw + (mz ? 0 : nd);
        eloc = xyz + (rc ? 3 * nd : 0);
        upw = eloc + (size_t)CE * 8;
        ek = upw + (size_t)CE * 8;
        lc = ek + (rc ? (size_t)CE * 8 * (kiso ? 1 : 3) : 0);
        lp = lc + (size_t)CE * npe * 2;
        bytes = (lp + (size_t)nnmax * 2 + 127) & ~(size_t)127;
    }
};

__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     tc05::smem_u32(dst)),
                 "l"(src), "r"(bytes), "r"(tc05::smem_u32(bar))
                 : "memory");
}

template <int NPE, bool VAR1, bool MZ>
__device__ __forceinline__ void elem_issue(const ElemArgs& a, const StageLayout& L, unsigned char* st,
                                           int4* meta, uint64_t* bar, int c) {
    const int2 sg = a.ch_seg[c];
    const int e0 = c * a.CE;
    const int ne = min(a.CE, a.T - e0);
    const int nnp = pad8(sg.y + 1), nep = pad8(ne);
    *meta = make_int4(sg.x, sg.y, e0, ne);
    uint32_t bytes = (uint32_t)nnp * 8 * (1 + (MZ ? 0 : 1) + (VAR1 ? 3 : 0)) + (uint32_t)nep * 16 +
                     (VAR1 ? (uint32_t)nep * 8 * (a.kiso ? 1 : 3) : 0) + (uint32_t)nep * NPE * 2 + (uint32_t)nnp * 2;
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(tc05::smem_u32(bar)), "r"(bytes)
                 : "memory");
    if (MZ) bulk_g2s(st + L.h, a.ch_h + sg.x, nnp * 8, bar);
    else bulk_g2s(st + L.h, a.ch_hk + 2 * (size_t)sg.x, nnp * 16, bar);
    if (VAR1)
        for (int d = 0; d < 3; ++d) bulk_g2s(st + L.xyz + (size_t)d * a.nnmax * 8, a.ch_xyz + d * a.P + sg.x, nnp * 8, bar);
    bulk_g2s(st + L.eloc, a.elocal + e0, nep * 8, bar);
    bulk_g2s(st + L.upw, a.upw + (size_t)8 * e0, nep * 8, bar);
    if (VAR1) {
        const int nk = a.kiso ? 1 : 3;
        for (int d = 0; d < nk; ++d)
            bulk_g2s(st + L.ek + (size_t)d * a.CE * 8, a.eK + (size_t)d * a.estride + e0, nep * 8, bar);
    }
    bulk_g2s(st + L.lc, a.ch_lc + (size_t)e0 * NPE, nep * NPE * 2, bar);
    bulk_g2s(st + L.lp, a.ch_lptr + sg.x, nnp * 2, bar);
}

template <int NPE, int NFE, int VAR, bool MZ, int EPT>
__global__ void __launch_bounds__(kElemThreads) k_elem_chunk(ElemArgs a) {
    extern __shared__ __align__(128) unsigned char smem_e[];
    const StageLayout L(a.CE, NPE, a.nnmax, MZ, VAR == 1, a.kiso != 0);
    double* cc = reinterpret_cast<double*>(smem_e + 2 * L.bytes);               // [NPE][CE]
    int4* meta = reinterpret_cast<int4*>(cc + (size_t)NPE * a.CE);                // [2]
    uint64_t* full = reinterpret_cast<uint64_t*>(meta + 2);                      // [2]
    pdl_wait_and_trigger();
    if ((int)blockIdx.x >= a.nch) return;
    if (a.skip && *a.skip) return;
    if (threadIdx.x == 0) {
        tc05::mbar_init(&full[0], 1);
        tc05::mbar_init(&full[1], 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        elem_issue<NPE, VAR == 1, MZ>(a, L, smem_e, &meta[0], &full[0], blockIdx.x);
    }
    __syncthreads();
    int i = 0;
    for (int c = blockIdx.x; c < a.nch; c += gridDim.x, ++i) {
        const int s = i & 1;
        const int cn = c + gridDim.x;
        if (threadIdx.x == 0 && cn < a.nch) {
            // the other stage was released by the barrier that ended the
            // previous chunk; order those generic reads before the copies
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            elem_issue<NPE, VAR == 1, MZ>(a, L, smem_e + (s ^ 1) * L.bytes, &meta[s ^ 1], &full[s ^ 1], cn);
        }
        const bool ok = tc05::mbar_wait(&full[s], (uint32_t)((i >> 1) & 1));
        if (!__syncthreads_and(ok ? 1 : 0)) {
            // a chunk never arrived: report it, let the copies already issued
            // land (bounded) and leave
            if (threadIdx.x == 0) {
                atomicExch(a.err, 5);
                tc05::mbar_wait(&full[s], (uint32_t)((i >> 1) & 1));
                if (cn < a.nch) tc05::mbar_wait(&full[s ^ 1], (uint32_t)(((i + 1) >> 1) & 1));
            }
            __syncthreads();
            return;
        }
        const int4 md = meta[s];
        const int j0 = md.x, nn = md.y, e0 = md.z, ne = md.w;
        const unsigned char* st = smem_e + s * L.bytes;
        const double* sh = reinterpret_cast<const double*>(st + L.h);
        const double* sx = reinterpret_cast<const double*>(st + L.xyz);
        const ushort4* sel = reinterpret_cast<const ushort4*>(st + L.eloc);
        const uint2* sup = reinterpret_cast<const uint2*>(st + L.upw);
        const double* sk = reinterpret_cast<const double*>(st + L.ek);
        const unsigned short* slc = reinterpret_cast<const unsigned short*>(st + L.lc);
        const unsigned short* slp = reinterpret_cast<const unsigned short*>(st + L.lp);
#pragma unroll
        for (int t = 0; t < EPT; ++t) {
            const int el = threadIdx.x + t * kElemThreads;
            if (el >= ne) continue;
            const int e = e0 + el;
            const ushort4 lq = sel[el];
            const int li[4] = {lq.x, lq.y, lq.z, lq.w};
            double hv[NPE], kr[NPE];
            const size_t zo = MZ ? (size_t)a.ezone[e] * a.N : 0;
#pragma unroll
            for (int k = 0; k < NPE; ++k) {
                if (MZ) {
                    hv[k] = sh[li[k]];
                    kr[k] = a.krw[zo + a.ch_node[j0 + li[k]]];
                } else {
                    const double2 hk = reinterpret_cast<const double2*>(sh)[li[k]];
                    hv[k] = hk.x;
                    kr[k] = hk.y;
                }
            }
            double q[NFE];
            if (VAR == 0) {
#pragma unroll
                for (int f = 0; f < NFE; ++f) {
                    const double* cf = a.coef + (size_t)(f * (NPE + 1)) * a.T + e;
                    double sacc = cf[0] * hv[0];
#pragma unroll
                    for (int k = 1; k < NPE; ++k) sacc += cf[(size_t)k * a.T] * hv[k];
                    q[f] = sacc + cf[(size_t)NPE * a.T];
                }
            } else {
                double X[4][3];
#pragma unroll
                for (int k = 0; k < 4; ++k) {
                    X[k][0] = sx[li[k]];
                    X[k][1] = sx[a.nnmax + li[k]];
                    X[k][2] = sx[2 * a.nnmax + li[k]];
                }
                const double K0 = sk[el];
                const double K1 = a.kiso ? K0 : sk[a.CE + el];
                const double K2 = a.kiso ? K0 : sk[2 * a.CE + el];
                double qq[6];
                tet_face_fluxes(X[0], X[1], X[2], X[3], K0, K1, K2, hv[0], hv[1], hv[2], hv[3 % NPE], qq);
#pragma unroll
                for (int f = 0; f < NFE; ++f) q[f] = qq[f];
            }
            const uint2 uw = sup[el];
            double cacc[NPE];
#pragma unroll
            for (int k = 0; k < NPE; ++k) cacc[k] = 0.0;
#pragma unroll
            for (int f = 0; f < NFE; ++f) {
                const int fa = NPE == 4 ? tet_edge_a(f) : tri_edge_a(f);
                const int fb = NPE == 4 ? tet_edge_b(f) : tri_edge_b(f);
                const unsigned u = (f < 4 ? uw.x >> (8 * f) : uw.y >> (8 * (f - 4))) & 0xffu;
                const double flux = a.rho0 * (q[f] * face_krw(u, kr[fa], kr[fb]));
                cacc[fa] -= flux;
                cacc[fb] += flux;
            }
#pragma unroll
            for (int k = 0; k < NPE; ++k) cc[k * a.CE + el] = cacc[k];
        }
        __syncthreads();
        // one partial per chunk node, corners in ascending element order
        for (int j = threadIdx.x; j < nn; j += kElemThreads) {
            const int p0 = slp[j], p1 = slp[j + 1];
            double sacc = 0.0;
            for (int p = p0; p < p1; ++p) sacc += cc[slc[p]];
            a.part[j0 + j] = sacc;
        }
        __syncthreads();
    }
}

// node gather: the element pass left node i's partials, one per chunk that
// touches the node, at the chunk-major positions cpos[part_ptr[i] ..
// part_ptr[i+1]) in ascending chunk order; sum them in that order.
// F0 != nullptr turns the result into (F - F0) * inv_sigma.
__global__ void k_gather(int N, GatherSrc g, double* __restrict__ out, const int* __restrict__ skip) {
    pdl_wait_and_trigger();
    if (skip && *skip) return;
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N) return;
    out[i] = gather_row(g, i);
}

// begin-step element pass: averaged-weight face fluxes in the global edge
// orientation (back -> front), the qdotn_faces that process_spatial_weights
// sums per edge (fvmpor.h:765)
template <int NPE, int NFE, bool MULTIZONE>
__global__ void k_faceq(int T, int N, const int4* __restrict__ en, const double* __restrict__ coef,
                        const int* __restrict__ ezone, const double* __restrict__ krw,
                        const double* __restrict__ h, const unsigned char* __restrict__ flip,
                        double* __restrict__ faceq) {
    int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= T) return;
    int4 nd = en[e];
    int ids[4] = {nd.x, nd.y, nd.z, nd.w};
    size_t zo = MULTIZONE ? (size_t)ezone[e] * N : 0;
    double hv[NPE], kr[NPE];
#pragma unroll
    for (int k = 0; k < NPE; ++k) { hv[k] = h[ids[k]]; kr[k] = krw[zo + ids[k]]; }
    unsigned fl = flip[e];
#pragma unroll
    for (int f = 0; f < NFE; ++f) {
        const double* cf = coef + (size_t)(f * (NPE + 1)) * T + e;
        double q = cf[0] * hv[0];
#pragma unroll
        for (int k = 1; k < NPE; ++k) q += cf[(size_t)k * T] * hv[k];
        q += cf[(size_t)NPE * T];
        int a = NPE == 4 ? tet_edge_a(f) : tri_edge_a(f);
        int b = NPE == 4 ? tet_edge_b(f) : tri_edge_b(f);
        double kf = kr[a] * 0.5 + kr[b] * 0.5;
        double qn = q * kf;
        faceq[(size_t)NFE * e + f] = ((fl >> f) & 1u) ? qn : -qn;
    }
}

// The same face fluxes for the rebuilt-geometry 3D variant: the face
// geometry from the element's vertices (tet_face_fluxes, the quantity
// sum_k C[f][k] h_k + G[f] with the head gradient formed once), so that the
// step's upwinding reads the vertices and one K instead of 30 stored
// coefficients per element (the element pass of this variant does the same)
template <bool MULTIZONE>
__global__ void k_faceq_rc(int T, int N, const int4* __restrict__ en, const double* __restrict__ xyz,
                           const double* __restrict__ eK, int kiso, int estride, const int* __restrict__ ezone,
                           const double* __restrict__ krw, const double* __restrict__ h,
                           const unsigned char* __restrict__ flip, double* __restrict__ faceq) {
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= T) return;
    const int4 nd = en[e];
    const int ids[4] = {nd.x, nd.y, nd.z, nd.w};
    const size_t zo = MULTIZONE ? (size_t)ezone[e] * N : 0;
    double X[4][3], hv[4], kr[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        X[k][0] = xyz[ids[k]];
        X[k][1] = xyz[(size_t)N + ids[k]];
        X[k][2] = xyz[(size_t)2 * N + ids[k]];
        hv[k] = h[ids[k]];
        kr[k] = krw[zo + ids[k]];
    }
    double Kx, Ky, Kz;
    if (kiso) Kx = Ky = Kz = eK[e];
    else { Kx = eK[e]; Ky = eK[(size_t)estride + e]; Kz = eK[(size_t)2 * estride + e]; }
    double q[6];
    tet_face_fluxes(X[0], X[1], X[2], X[3], Kx, Ky, Kz, hv[0], hv[1], hv[2], hv[3], q);
    const unsigned fl = flip[e];
#pragma unroll
    for (int f = 0; f < 6; ++f) {
        const double kf = kr[tet_edge_a(f)] * 0.5 + kr[tet_edge_b(f)] * 0.5;
        const double qn = q[f] * kf;
        faceq[(size_t)6 * e + f] = ((fl >> f) & 1u) ? qn : -qn;
    }
}

// per edge: edge_flux = sum_j (1/A_edge) qdotn_j; upwind = front when the
// edge flux is negative, back otherwise (process_spatial_weights,
// fvmpor.h:765, 784-793).  Writes the per-face flag in element-local terms.
__global__ void k_edge_upwind(int E, int nfe, const int* __restrict__ edge_ptr,
                              const int* __restrict__ edge_face, const double* __restrict__ edge_w,
                              const double* __restrict__ faceq,
                              const unsigned char* __restrict__ flip,
                              unsigned char* __restrict__ upw) {
    int ed = blockIdx.x * blockDim.x + threadIdx.x;
    if (ed >= E) return;
    double w = edge_w[ed];
    double s = 0.0;
    int p0 = edge_ptr[ed], p1 = edge_ptr[ed + 1];
    for (int p = p0; p < p1; ++p) s += w * faceq[edge_face[p]];
    bool up_front = s < 0.0;
    for (int p = p0; p < p1; ++p) {
        int fid = edge_face[p];
        int e = fid / nfe, f = fid - e * nfe;
        bool front_is_b = (flip[e] >> f) & 1u;
        upw[(size_t)8 * e + f] = (unsigned char)(up_front ? front_is_b : !front_is_b);
    }
}

// ------------------------------------------------------------------ drivers
static NodeCopies node_copies(fvm_ctx* c) {
    NodeCopies cp;
    cp.part_ptr = c->part_ptr.p;
    cp.cpos = c->ch_cpos.p;
    cp.ch_h = c->ch_h.p;
    cp.ch_hk = c->ch_hk.p;
    return cp;
}

// elements per thread of a chunk CTA (powers of two up to 8)
static int chunk_ept(int CE) {
    int t = (CE + kElemThreads - 1) / kElemThreads;
    return t <= 1 ? 1 : t <= 2 ? 2 : t <= 4 ? 4 : 8;
}

// dispatch on the run-time shape: f is called with the kernel instance
template <class F> static void with_elem_kernel(const fvm_ctx* c, F&& f) {
    const bool mz = c->nz > 1;
    const int ept = chunk_ept(c->chunk_e);
    auto by_ept = [&](auto k1, auto k2, auto k4, auto k8) {
        if (ept == 1) f(k1);
        else if (ept == 2) f(k2);
        else if (ept == 4) f(k4);
        else f(k8);
    };
#define FVM_EPT(NPE, NFE, V, M) k_elem_chunk<NPE, NFE, V, M, 1>, k_elem_chunk<NPE, NFE, V, M, 2>, \
                                k_elem_chunk<NPE, NFE, V, M, 4>, k_elem_chunk<NPE, NFE, V, M, 8>
    if (c->dim == 3) {
        if (c->recompute) mz ? by_ept(FVM_EPT(4, 6, 1, true)) : by_ept(FVM_EPT(4, 6, 1, false));
        else mz ? by_ept(FVM_EPT(4, 6, 0, true)) : by_ept(FVM_EPT(4, 6, 0, false));
    } else {
        mz ? by_ept(FVM_EPT(3, 3, 0, true)) : by_ept(FVM_EPT(3, 3, 0, false));
    }
#undef FVM_EPT
}

// shared bytes of one element-pass CTA: two pipeline stages, the corner
// partials, the stage descriptors and the two mbarriers
static size_t chunk_smem_bytes(const fvm_ctx* c, int CE, int nnmax) {
    const StageLayout L(CE, c->npe, nnmax, c->nz > 1, c->recompute, c->kiso);
    return 2 * L.bytes + sizeof(double) * (size_t)CE * c->npe + 2 * sizeof(int4) + 2 * sizeof(uint64_t);
}

static void set_chunk_attrs(fvm_ctx* c) {
    with_elem_kernel(c, [&](auto k) {
        raise_smem_limit(k, c->chunk_smem);
    });
}

static void launch_elem(fvm_ctx* c, const double* h, const int* skip = nullptr) {
    ElemArgs a;
    a.skip = skip;
    (void)h;   // the node pass left the head in the chunk-major copies
    a.T = c->T; a.N = c->N; a.CE = c->chunk_e; a.nch = c->nchunk; a.kiso = c->kiso ? 1 : 0;
    a.estride = c->estride; a.nnmax = c->chunk_maxnn;
    a.ch_seg = c->ch_seg.p; a.ch_node = c->ch_node.p;
    a.elocal = c->elocal.p; a.ch_lptr = c->ch_lptr.p; a.ch_lc = c->ch_lc.p;
    a.coef = c->coef.p; a.ch_xyz = c->ch_xyz.p; a.eK = c->eK.p; a.ezone = c->ezone.p;
    a.krw = c->krw.p; a.ch_h = c->ch_h.p; a.ch_hk = c->ch_hk.p; a.upw = c->upw.p; a.rho0 = c->rho0;
    a.part = c->part.p; a.err = c->elem_err.p; a.P = c->ch_node.n;
    with_elem_kernel(c, [&](auto k) { fvm_launch_pdl(c, k, c->chunk_grid, kElemThreads, c->chunk_smem, c->stream, a); });
}

// Chunk the elements (consecutive ids, CE per chunk) and build the tables
// of the chunked element pass: the distinct nodes of every chunk, the
// 16-bit local corner ids, the node-ordered corner lists, and the node-major
// layout of the per-(node, chunk) partials that the gather sums.
static void build_chunks(fvm_ctx* c, int CE) {
    const int T = c->T, N = c->N, npe = c->npe;
    if (CE < 32 || CE > 8 * kElemThreads) throw Error("chunk size out of range (32..2048 elements)");
    if (CE % 8) throw Error("chunk size must be a multiple of 8");
    const int nch = (T + CE - 1) / CE;
    const size_t ES = (size_t)c->estride;
    const std::vector<int>& en = c->h_elem_nodes;
    // chunk c's nodes occupy the padded segment [seg.x, seg.x + pad8(nn + 1))
    std::vector<int2> seg(nch);
    std::vector<int> ch_node;
    ch_node.reserve((size_t)T);
    std::vector<ushort4> elocal(ES, make_ushort4(0, 0, 0, 0));
    std::vector<unsigned short> lptr, lc(ES * npe, 0);
    lptr.reserve((size_t)T + 8 * nch);
    std::vector<int> stamp(N, -1), lid(N, 0), pcount(N, 0), nodes, cnt;
    int maxnn = 0;
    for (int ch = 0; ch < nch; ++ch) {
        const int e0 = ch * CE, e1 = std::min(T, e0 + CE);
        nodes.clear();
        for (int e = e0; e < e1; ++e)
            for (int k = 0; k < npe; ++k) {
                int g = en[(size_t)e * npe + k];
                if (stamp[g] != ch) { stamp[g] = ch; nodes.push_back(g); }
            }
        std::sort(nodes.begin(), nodes.end());
        const int nn = (int)nodes.size();
        const int nnp = pad8(nn + 1);
        maxnn = std::max(maxnn, nnp);
        seg[ch] = make_int2((int)ch_node.size(), nn);
        for (int j = 0; j < nn; ++j) { lid[nodes[j]] = j; pcount[nodes[j]]++; }
        cnt.assign(nn + 1, 0);
        for (int e = e0; e < e1; ++e) {
            unsigned short l[4] = {0, 0, 0, 0};
            for (int k = 0; k < npe; ++k) {
                l[k] = (unsigned short)lid[en[(size_t)e * npe + k]];
                cnt[l[k] + 1]++;
            }
            elocal[e] = make_ushort4(l[0], l[1], l[2], l[3]);
        }
        for (int j = 0; j < nn; ++j) cnt[j + 1] += cnt[j];
        for (int j = 0; j <= nn; ++j) lptr.push_back((unsigned short)cnt[j]);
        lptr.resize(lptr.size() + (nnp - nn - 1), 0);
        for (int e = e0; e < e1; ++e)
            for (int k = 0; k < npe; ++k) {
                int j = lid[en[(size_t)e * npe + k]];
                lc[(size_t)e0 * npe + cnt[j]++] = (unsigned short)(k * CE + (e - e0));
            }
        ch_node.insert(ch_node.end(), nodes.begin(), nodes.end());
        ch_node.resize(ch_node.size() + (nnp - nn), nodes.empty() ? 0 : nodes.back());
    }
    std::vector<int> part_ptr(N + 1, 0);
    for (int i = 0; i < N; ++i) part_ptr[i + 1] = part_ptr[i] + pcount[i];
    // node-major copy slot q -> chunk-major position (ascending chunk per node)
    std::vector<int> cpos(part_ptr[N]), seen(N, 0);
    for (int ch = 0; ch < nch; ++ch)
        for (int j = 0; j < seg[ch].y; ++j) {
            const int p = seg[ch].x + j;
            const int g = ch_node[p];
            cpos[part_ptr[g] + seen[g]++] = p;
        }
    cudaStream_t s = c->stream;
    c->chunk_e = CE;
    c->nchunk = nch;
    c->chunk_maxnn = maxnn;
    c->ch_seg.upload(seg, s);
    c->ch_node.upload(ch_node, s);
    c->ch_cpos.upload(cpos, s);
    const size_t P = ch_node.size();
    if (c->dim == 3) {
        std::vector<double> cx(3 * P);
        for (size_t p = 0; p < P; ++p)
            for (int d = 0; d < 3; ++d) cx[(size_t)d * P + p] = c->h_xyz[(size_t)d * N + ch_node[p]];
        c->ch_xyz.upload(cx, s);
    }
    c->ch_h.alloc(P);
    c->ch_hk.alloc(2 * P);
    c->elocal.upload(elocal, s);
    c->ch_lptr.upload(lptr, s);
    c->ch_lc.upload(lc, s);
    c->part_ptr.upload(part_ptr, s);
    c->part.alloc(ch_node.size());
    c->chunk_smem = chunk_smem_bytes(c, CE, maxnn);
    if (c->chunk_smem > 227 * 1024) throw Error("chunk does not fit in shared memory");
    set_chunk_attrs(c);
    // persistent grid: as many CTAs as fit on the device at once
    int per_sm = 0, nsm = 0;
    with_elem_kernel(c, [&](auto k) {
        FVM_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k, kElemThreads, c->chunk_smem));
    });
    FVM_CUDA(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, c->device));
    if (per_sm < 1) throw Error("element pass: chunk does not fit on an SM");
    c->chunk_grid = std::min(nch, per_sm * nsm);
    FVM_CUDA(cudaStreamSynchronize(s));
}

GatherSrc launch_residual_partials(fvm_ctx* c, const double* y, const double* yp, const Perturb& pt,
                                   const double* F0) {
    cudaStream_t s = c->stream;
    const double* h = pt.mode ? c->hstar.p : y;
    c->tm.begin(TM_NODE, s);
    fvm_launch_pdl(c, k_node, grid_for(c->N, kBlock), kBlock, 0, s, c->N, y, yp, pt, c->zones.p, c->nz, c->nz_ptr.p,
                   c->nz_zone.p, c->nz_w.p, c->rho0, c->krw.p, c->hstar.p, c->stor.p, node_copies(c));
    c->tm.end(TM_NODE, s);
    c->tm.begin(TM_ELEM, s);
    launch_elem(c, h, pt.skip);
    c->tm.end(TM_ELEM, s);
    c->n_residuals++;
    GatherSrc g;
    g.part_ptr = c->part_ptr.p;
    g.cpos = c->ch_cpos.p;
    g.part = c->part.p;
    g.invV = c->invV.p;
    g.bterm = c->bterm.p;
    g.hD = c->hD.p;
    g.ntype = c->ntype.p;
    g.h = h;
    g.stor = c->stor.p;
    g.F0 = F0;
    g.inv_sigma = (F0 && !pt.sigma_dev) ? 1.0 / pt.sigma : 0.0;
    g.sigma_dev = F0 ? pt.sigma_dev : nullptr;
    return g;
}

void gather_into(fvm_ctx* c, const GatherSrc& g, double* out, const int* skip) {
    c->tm.begin(TM_GATHER, c->stream);
    fvm_launch_pdl(c, k_gather, grid_for(c->N, kBlock), kBlock, 0, c->stream, c->N, g, out, skip);
    c->tm.end(TM_GATHER, c->stream);
}

void launch_residual(fvm_ctx* c, const double* y, const double* yp, const Perturb& pt,
                     const double* F0, double* out) {
    const GatherSrc g = launch_residual_partials(c, y, yp, pt, F0);
    gather_into(c, g, out, pt.skip);
}

void launch_begin_step(fvm_ctx* c, const double* y, const double* yp) {
    cudaStream_t s = c->stream;
    Perturb none;
    fvm_launch(c, k_node, grid_for(c->N, kBlock), kBlock, 0, s, c->N, y, yp, none, c->zones.p, c->nz, c->nz_ptr.p,
                                                      c->nz_zone.p, c->nz_w.p, c->rho0, c->krw.p,
                                                      c->hstar.p, c->stor.p, node_copies(c));
    int gb = grid_for(c->T, kBlock);
    if (c->dim == 3 && c->recompute) {
        if (c->nz > 1)
            fvm_launch(c, k_faceq_rc<true>, gb, kBlock, 0, s, c->T, c->N, c->enodes.p, c->xyz.p, c->eK.p,
                       c->kiso ? 1 : 0, c->estride, c->ezone.p, c->krw.p, y, c->flip.p, c->faceq.p);
        else
            fvm_launch(c, k_faceq_rc<false>, gb, kBlock, 0, s, c->T, c->N, c->enodes.p, c->xyz.p, c->eK.p,
                       c->kiso ? 1 : 0, c->estride, c->ezone.p, c->krw.p, y, c->flip.p, c->faceq.p);
    } else if (c->dim == 3) {
        if (c->nz > 1) fvm_launch(c, k_faceq<4, 6, true>, gb, kBlock, 0, s, c->T, c->N, c->enodes.p, c->coef.p, c->ezone.p, c->krw.p, y, c->flip.p, c->faceq.p);
        else fvm_launch(c, k_faceq<4, 6, false>, gb, kBlock, 0, s, c->T, c->N, c->enodes.p, c->coef.p, c->ezone.p, c->krw.p, y, c->flip.p, c->faceq.p);
    } else {
        if (c->nz > 1) fvm_launch(c, k_faceq<3, 3, true>, gb, kBlock, 0, s, c->T, c->N, c->enodes.p, c->coef.p, c->ezone.p, c->krw.p, y, c->flip.p, c->faceq.p);
        else fvm_launch(c, k_faceq<3, 3, false>, gb, kBlock, 0, s, c->T, c->N, c->enodes.p, c->coef.p, c->ezone.p, c->krw.p, y, c->flip.p, c->faceq.p);
    }
    fvm_launch(c, k_edge_upwind, grid_for(c->E, kBlock), kBlock, 0, s, c->E, c->nfe, c->edge_ptr.p, c->edge_face.p,
                                                              c->edge_w.p, c->faceq.p, c->flip.p, c->upw.p);
}

void reset_upwind(fvm_ctx* c) {
    FVM_CUDA(cudaMemsetAsync(c->upw.p, 2, c->upw.n, c->stream));
}

// head from the hydrostatic/Dirichlet rules of set_initial_conditions
// (vs.h:8-32)
static std::vector<double> initial_head_host(const fvm_ctx* c, double water_table) {
    std::vector<double> h(c->N);
    for (int i = 0; i < c->N; ++i) h[i] = c->h_node_type[i] ? c->h_hD[i] : water_table - c->h_vert[i];
    return h;
}

// ------------------------------------------------------------------ autotuner
// Times the element pass for every (variant, chunk size) candidate on the
// context's own mesh and keeps the fastest.  Each candidate runs on the
// hydrostatic initial head; every timed launch follows a write of a buffer
// larger than the L2 cache, so no candidate profits from data left there by
// the previous launch.  CUDA events on the context stream, median of the
// timed launches.
static void autotune(fvm_ctx* c, fvm_tune_result* out) {
    const int chunks[] = {256, 512, 1024, 2048};
    const int nvar = c->dim == 3 ? 2 : 1;
    cudaStream_t s = c->stream;
    std::vector<double> y0 = initial_head_host(c, 0.0);
    DevBuf<double> y, yp, flush;
    y.alloc(c->N);
    yp.alloc(c->N);
    yp.zero(s);
    FVM_CUDA(cudaMemcpyAsync(y.p, y0.data(), sizeof(double) * c->N, cudaMemcpyHostToDevice, s));
    const size_t flush_n = (size_t)192 << 20;   // 192 MiB > 126 MB L2
    flush.alloc(flush_n / sizeof(double));
    Perturb none;
    cudaEvent_t e0, e1;
    FVM_CUDA(cudaEventCreate(&e0));
    FVM_CUDA(cudaEventCreate(&e1));
    const bool rc0 = c->recompute;
    const int ce0 = c->chunk_e;
    double best = 1e300;
    int best_var = rc0 ? 1 : 0, best_ce = ce0, n = 0, best_i = -1;
    for (int v = 0; v < nvar; ++v)
        for (int ce : chunks) {
            c->recompute = v == 1;
            try {
                build_chunks(c, ce);
            } catch (const Error&) {
                continue;   // does not fit in shared memory
            }
            // chunk-major node copies of this partition
            fvm_launch(c, k_node, grid_for(c->N, kBlock), kBlock, 0, s, c->N, y.p, yp.p, none, c->zones.p, c->nz,
                       c->nz_ptr.p, c->nz_zone.p, c->nz_w.p, c->rho0, c->krw.p, c->hstar.p, c->stor.p,
                       node_copies(c));
            for (int w = 0; w < 2; ++w) launch_elem(c, y.p);
            std::vector<float> t;
            for (int k = 0; k < 7; ++k) {
                FVM_CUDA(cudaMemsetAsync(flush.p, k, flush_n, s));
                FVM_CUDA(cudaEventRecord(e0, s));
                launch_elem(c, y.p);
                FVM_CUDA(cudaEventRecord(e1, s));
                FVM_CUDA(cudaEventSynchronize(e1));
                float ms = 0.0f;
                FVM_CUDA(cudaEventElapsedTime(&ms, e0, e1));
                t.push_back(ms);
            }
            std::sort(t.begin(), t.end());
            double us = 1e3 * t[t.size() / 2];
            if (out && n < FVM_TUNE_MAX) {
                out->variant[n] = v;
                out->chunk[n] = ce;
                out->us[n] = us;
            }
            if (us < best) { best = us; best_var = v; best_ce = ce; best_i = n; }
            ++n;
        }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    c->recompute = best_var == 1;
    build_chunks(c, best_ce);
    if (out) {
        out->n = std::min(n, FVM_TUNE_MAX);
        out->best = best_i;
    }
}

// ------------------------------------------------------------------ set-up
static void build(fvm_ctx* c, const fvm_mesh* m, const fvm_physics* ph, int flags) {
    if (!m || !ph) throw Error("fvm_create: null argument");
    if (m->dim != 2 && m->dim != 3) throw Error("fvm_create: dim must be 2 or 3");
    if (m->n_nodes <= 0 || m->n_elements <= 0) throw Error("fvm_create: empty mesh");
    if (!m->coords || !m->elem_nodes || !m->elem_zone || !m->node_tag) throw Error("fvm_create: missing mesh array");
    if (m->n_bfaces > 0 && (!m->bface_nodes || !m->bface_elem || !m->bface_tag)) throw Error("fvm_create: missing boundary arrays");
    if (ph->n_zones <= 0 || !ph->zones) throw Error("fvm_create: no soil zones");
    const int dim = m->dim, N = m->n_nodes, T = m->n_elements;
    const int npe = dim + 1, nfe = dim == 2 ? 3 : 6;
    if ((long)T * nfe >= (1l << 31) - 1) throw Error("fvm_create: mesh too large");
    c->dim = dim; c->N = N; c->T = T; c->npe = npe; c->nfe = nfe;
    c->estride = pad8(T) + 8;   // per-element arrays padded for whole 16-byte chunk copies
    c->nz = ph->n_zones; c->rho0 = ph->rho0;
    // 3D default: rebuild the face geometry from the vertices (FP64 ALU
    // instead of 240 B of streamed coefficients per element)
    c->recompute = dim == 3 && !(flags & FVM_FLAG_STORED_GEOMETRY);
    if (flags & FVM_FLAG_RECOMPUTE_GEOMETRY) c->recompute = dim == 3;
    FVM_CUDA(cudaGetDevice(&c->device));
    FVM_CUDA(cudaStreamCreate(&c->stream));   // blocking: orders after the legacy default stream
    cudaStream_t s = c->stream;

    auto bc_of = [&](int tag) -> const fvm_bc* {
        for (int i = 0; i < ph->n_bcs; ++i) if (ph->bcs[i].tag == tag) return &ph->bcs[i];
        return nullptr;
    };

    // ---- element geometry
    c->h_elem_nodes.assign(m->elem_nodes, m->elem_nodes + (size_t)T * npe);
    std::vector<int4> en(T);
    std::vector<double> coef((size_t)nfe * (npe + 1) * T), area((size_t)nfe * T), vol(T);
    std::vector<double> eK3((size_t)3 * T);
    for (int e = 0; e < T; ++e) {
        const int* v = m->elem_nodes + (size_t)e * npe;
        for (int k = 0; k < npe; ++k)
            if (v[k] < 0 || v[k] >= N) throw Error("fvm_create: element node id out of range");
        int z = m->elem_zone[e];
        if (z < 0 || z >= ph->n_zones) throw Error("fvm_create: element zone out of range");
        const fvm_zone& Z = ph->zones[z];
        double Kx = Z.Kxx, Ky = Z.Kyy, Kz = Z.Kzz;
        if (m->elem_K) Kx = Ky = Kz = m->elem_K[e];
        eK3[e] = Kx; eK3[(size_t)T + e] = Ky; eK3[(size_t)2 * T + e] = Kz;
        en[e] = make_int4(v[0], v[1], v[2], dim == 3 ? v[3] : -1);
        if (dim == 3) {
            double C[6][4], G[6], A[6];
            if (!tet_coefficients(m->coords + 3 * (size_t)v[0], m->coords + 3 * (size_t)v[1], m->coords + 3 * (size_t)v[2],
                                  m->coords + 3 * (size_t)v[3], Kx, Ky, Kz, C, G, A, &vol[e]))
                throw Error("fvm_create: degenerate tetrahedron " + std::to_string(e));
            for (int f = 0; f < 6; ++f) {
                for (int k = 0; k < 4; ++k) coef[(size_t)(f * 5 + k) * T + e] = C[f][k];
                coef[(size_t)(f * 5 + 4) * T + e] = G[f];
                area[(size_t)6 * e + f] = A[f];
            }
        } else {
            double C[3][3], G[3], A[3];
            if (!tri_coefficients(m->coords + 3 * (size_t)v[0], m->coords + 3 * (size_t)v[1], m->coords + 3 * (size_t)v[2],
                                  Kx, Ky, C, G, A, &vol[e]))
                throw Error("fvm_create: degenerate triangle " + std::to_string(e));
            for (int f = 0; f < 3; ++f) {
                for (int k = 0; k < 3; ++k) coef[(size_t)(f * 4 + k) * T + e] = C[f][k];
                coef[(size_t)(f * 4 + 3) * T + e] = G[f];
                area[(size_t)3 * e + f] = A[f];
            }
        }
    }

    // ---- control volumes and zone weights (fvmpor.h:471-498)
    std::vector<double> V(N, 0.0);
    for (int e = 0; e < T; ++e)
        for (int k = 0; k < npe; ++k) V[m->elem_nodes[(size_t)e * npe + k]] += vol[e] / npe;
    for (int i = 0; i < N; ++i)
        if (!(V[i] > 0.0)) throw Error("fvm_create: node " + std::to_string(i) + " belongs to no element");
    // incidence lists (ascending element id)
    std::vector<int> inc_ptr(N + 1, 0), inc((size_t)T * npe);
    for (size_t q = 0; q < (size_t)T * npe; ++q) inc_ptr[m->elem_nodes[q] + 1]++;
    for (int i = 0; i < N; ++i) inc_ptr[i + 1] += inc_ptr[i];
    {
        std::vector<int> pos(inc_ptr.begin(), inc_ptr.end() - 1);
        for (int e = 0; e < T; ++e)
            for (int k = 0; k < npe; ++k) inc[pos[m->elem_nodes[(size_t)e * npe + k]]++] = e * npe + k;
    }
    std::vector<int> nz_ptr(N + 1, 0), nz_zone;
    std::vector<double> nz_w;
    {
        std::vector<double> wz(ph->n_zones);
        std::vector<int> cnt(ph->n_zones);
        for (int i = 0; i < N; ++i) {
            std::fill(wz.begin(), wz.end(), 0.0);
            std::fill(cnt.begin(), cnt.end(), 0);
            for (int p = inc_ptr[i]; p < inc_ptr[i + 1]; ++p) {
                int e = inc[p] / npe;
                int z = m->elem_zone[e];
                wz[z] += (vol[e] / npe) / V[i];
                cnt[z]++;
            }
            for (int z = 0; z < ph->n_zones; ++z)
                if (cnt[z]) { nz_zone.push_back(z); nz_w.push_back(wz[z]); }
            nz_ptr[i + 1] = (int)nz_zone.size();
        }
    }
    if (ph->n_zones == 1) {
        // single zone: node i's weight sits at index i
        if ((int)nz_w.size() != N) throw Error("fvm_create: zone bookkeeping");
    }

    // ---- global edges: sort (min,max) keys; first encounter fixes the
    // orientation (Edge(front = node a, back = node b), mesh.cpp:383-441)
    // The faces in (key, face id) order, built as a counting sort on the
    // smaller node (faces enter their bucket in ascending face id) followed
    // by a stable insertion sort on the larger node inside each bucket
    // (about 35 faces per bucket on a tetrahedral mesh): linear in the
    // faces, where one global sort of the 36 M keys of the 1M-node mesh took
    // seconds.
    std::vector<std::pair<uint64_t, int>> keys((size_t)T * nfe);
    {
        auto ends = [&](int e, int f, int& a, int& b) {
            const int* v = m->elem_nodes + (size_t)e * npe;
            a = v[dim == 3 ? tet_edge_a(f) : tri_edge_a(f)];
            b = v[dim == 3 ? tet_edge_b(f) : tri_edge_b(f)];
        };
        std::vector<size_t> bptr((size_t)N + 1, 0);
        for (int e = 0; e < T; ++e)
            for (int f = 0; f < nfe; ++f) {
                int a, b;
                ends(e, f, a, b);
                bptr[(size_t)std::min(a, b) + 1]++;
            }
        for (int i = 0; i < N; ++i) bptr[i + 1] += bptr[i];
        std::vector<size_t> fill(bptr.begin(), bptr.end() - 1);
        for (int e = 0; e < T; ++e)
            for (int f = 0; f < nfe; ++f) {
                int a, b;
                ends(e, f, a, b);
                const uint64_t key = ((uint64_t)(uint32_t)std::min(a, b) << 32) | (uint32_t)std::max(a, b);
                keys[fill[std::min(a, b)]++] = {key, e * nfe + f};
            }
        for (int i = 0; i < N; ++i)
            for (size_t r = bptr[i] + 1; r < bptr[i + 1]; ++r) {
                const auto kv = keys[r];
                size_t q = r;
                while (q > bptr[i] && keys[q - 1].first > kv.first) {
                    keys[q] = keys[q - 1];
                    --q;
                }
                keys[q] = kv;
            }
    }
    std::vector<int> edge_ptr(1, 0), edge_face;
    std::vector<double> edge_w;
    std::vector<unsigned char> flip(T, 0);
    edge_face.reserve(keys.size());
    for (size_t p = 0; p < keys.size();) {
        size_t q = p;
        while (q < keys.size() && keys[q].first == keys[p].first) ++q;
        int fid0 = keys[p].second;
        int e0 = fid0 / nfe, f0 = fid0 % nfe;
        int back = m->elem_nodes[(size_t)e0 * npe + (dim == 3 ? tet_edge_b(f0) : tri_edge_b(f0))];
        double atot = 0.0;
        for (size_t r = p; r < q; ++r) {
            int fid = keys[r].second;
            int e = fid / nfe, f = fid % nfe;
            int a = m->elem_nodes[(size_t)e * npe + (dim == 3 ? tet_edge_a(f) : tri_edge_a(f))];
            if (a == back) flip[e] |= (unsigned char)(1u << f);
            atot += area[fid];
            edge_face.push_back(fid);
        }
        edge_w.push_back(1.0 / atot);
        edge_ptr.push_back((int)edge_face.size());
        p = q;
    }
    c->E = (int)edge_w.size();

    // ---- boundary-flux term and Dirichlet rows (process_fluxes :721-758,
    // residual_evaluation :113-114, initialise_vectors :405-451)
    std::vector<double> bterm(N, 0.0), hD(N, 0.0), invV(N);
    std::vector<unsigned char> ntype(N, 0);
    c->h_vert.resize(N);
    for (int i = 0; i < N; ++i) {
        invV[i] = 1.0 / V[i];
        c->h_vert[i] = m->coords[3 * (size_t)i + (dim == 2 ? 1 : 2)];
        int tag = m->node_tag[i];
        if (tag) {
            const fvm_bc* bc = bc_of(tag);
            if (!bc) throw Error("fvm_create: node tag without boundary condition: " + std::to_string(tag));
            if (bc->type == 1) { ntype[i] = 1; hD[i] = bc->value; }
            else if (bc->type == 4) { ntype[i] = 1; hD[i] = (1.0 + bc->eta) * (bc->b - c->h_vert[i]); }
        }
    }
    for (int b = 0; b < m->n_bfaces; ++b) {
        const fvm_bc* bc = bc_of(m->bface_tag[b]);
        if (!bc) throw Error("fvm_create: boundary tag without condition: " + std::to_string(m->bface_tag[b]));
        if (bc->type != 3) continue;
        const int* v = m->bface_nodes + (size_t)b * dim;
        double meas;
        const double* p0 = m->coords + 3 * (size_t)v[0];
        const double* p1 = m->coords + 3 * (size_t)v[1];
        if (dim == 2) {
            meas = std::sqrt((p1[0] - p0[0]) * (p1[0] - p0[0]) + (p1[1] - p0[1]) * (p1[1] - p0[1]));
        } else {
            const double* p2 = m->coords + 3 * (size_t)v[2];
            double u[3] = {p1[0] - p0[0], p1[1] - p0[1], p1[2] - p0[2]};
            double w[3] = {p2[0] - p0[0], p2[1] - p0[1], p2[2] - p0[2]};
            double cr[3] = {u[1] * w[2] - u[2] * w[1], u[2] * w[0] - u[0] * w[2], u[0] * w[1] - u[1] * w[0]};
            meas = 0.5 * std::sqrt(cr[0] * cr[0] + cr[1] * cr[1] + cr[2] * cr[2]);
        }
        double a = meas / dim;   // boundary CV face per face node
        for (int k = 0; k < dim; ++k) {
            int i = v[k];
            if (i < 0 || i >= N) throw Error("fvm_create: boundary node out of range");
            bterm[i] += -invV[i] * (c->rho0 * (bc->value * a));
        }
    }
    c->h_node_type.assign(ntype.begin(), ntype.end());
    {
        // static learned-predictor inputs: mean ln K of the incident
        // elements, elevation, and the area of the node's CV faces
        std::vector<float> sf((size_t)3 * N, 0.0f);
        std::vector<double> lnk(N, 0.0), asum(N, 0.0);
        std::vector<int> cnt(N, 0);
        for (int e = 0; e < T; ++e) {
            double lk = std::log(std::max(eK3[e], 1e-300));
            for (int k = 0; k < npe; ++k) {
                int i = m->elem_nodes[(size_t)e * npe + k];
                lnk[i] += lk;
                cnt[i]++;
            }
            for (int f = 0; f < nfe; ++f) {
                int a = m->elem_nodes[(size_t)e * npe + (dim == 3 ? tet_edge_a(f) : tri_edge_a(f))];
                int b = m->elem_nodes[(size_t)e * npe + (dim == 3 ? tet_edge_b(f) : tri_edge_b(f))];
                asum[a] += area[(size_t)nfe * e + f];
                asum[b] += area[(size_t)nfe * e + f];
            }
        }
        for (int i = 0; i < N; ++i) {
            sf[i] = (float)(lnk[i] / std::max(cnt[i], 1));
            sf[(size_t)N + i] = (float)c->h_vert[i];
            sf[(size_t)2 * N + i] = (float)asum[i];
        }
        c->statf.upload(sf, s);
    }
    c->h_hD = hD;

    // ---- upload
    c->enodes.upload(en, s);
    if (dim == 3) {
        // vertices and conductivities for the rebuilt-geometry element pass;
        // one K per element when every element is isotropic
        std::vector<double> xyz((size_t)3 * N);
        for (int i = 0; i < N; ++i)
            for (int d = 0; d < 3; ++d) xyz[(size_t)d * N + i] = m->coords[3 * (size_t)i + d];
        c->xyz.upload(xyz, s);
        c->h_xyz = xyz;
        c->kiso = true;
        for (int e = 0; e < T && c->kiso; ++e)
            c->kiso = eK3[e] == eK3[(size_t)T + e] && eK3[e] == eK3[(size_t)2 * T + e];
        const size_t ES = (size_t)c->estride;
        std::vector<double> ek((c->kiso ? 1 : 3) * ES, 0.0);
        for (int d = 0; d < (c->kiso ? 1 : 3); ++d)
            for (int e = 0; e < T; ++e) ek[(size_t)d * ES + e] = eK3[(size_t)d * T + e];
        c->eK.upload(ek, s);
    }
    c->coef.upload(coef, s);
    if (c->nz > 1) c->ezone.upload(std::vector<int>(m->elem_zone, m->elem_zone + T), s);
    c->invV.upload(invV, s);
    c->bterm.upload(bterm, s);
    c->hD.upload(hD, s);
    c->ntype.upload(ntype, s);
    c->nz_ptr.upload(nz_ptr, s);
    c->nz_zone.upload(nz_zone, s);
    c->nz_w.upload(nz_w, s);
    std::vector<ZoneDev> zd(ph->n_zones);
    for (int z = 0; z < ph->n_zones; ++z) {
        const fvm_zone& Z = ph->zones[z];
        if (!(Z.nVG > 1.0) || !(Z.alphaVG > 0.0) || !(Z.phi > 0.0)) throw Error("fvm_create: invalid soil zone");
        zd[z] = ZoneDev{Z.phi, Z.alphaVG, Z.nVG, 1.0 - 1.0 / Z.nVG, Z.S_r};
    }
    c->zones.upload(zd, s);
    c->edge_ptr.upload(edge_ptr, s);
    c->edge_face.upload(edge_face, s);
    c->edge_w.upload(edge_w, s);
    c->flip.upload(flip, s);
    // averaged weights until the first begin_step (fvmpor.h:594-595)
    c->upw.upload(std::vector<unsigned char>((size_t)8 * c->estride, 2), s);
    c->krw.alloc((size_t)c->nz * N);
    c->krw.zero(s);
    c->hstar.alloc(N);
    c->stor.alloc(N);
    c->faceq.alloc((size_t)T * nfe);
    for (auto& b : c->tmpN) b.alloc(N);
    c->elem_err.alloc(1);
    c->elem_err.zero(s);
    build_chunks(c, kDefaultChunk);
    if (flags & FVM_FLAG_AUTOTUNE) autotune(c, nullptr);
}

} // namespace fvmb

using namespace fvmb;

void fvmb_destroy_ilu(fvmb::BlockILU* p);
void fvmb_destroy_krylov(fvmb::Krylov* p);
void fvmb_destroy_integ_work(fvmb::IntegWork* w);
void fvmb_destroy_predictor(fvmb::Predictor* p);

extern "C" const char* fvm_last_error(void) { return g_last_error.c_str(); }

extern "C" fvm_ctx* fvm_create(const fvm_mesh* m, const fvm_physics* ph, int flags) {
    std::unique_ptr<fvm_ctx> c(new fvm_ctx());
    try {
        build(c.get(), m, ph, flags);
        return c.release();
    } catch (const std::exception& ex) {
        set_error(ex.what());
        if (c->stream) cudaStreamDestroy(c->stream);
        c->stream = nullptr;
        return nullptr;
    }
}

extern "C" void fvm_destroy(fvm_ctx* c) {
    if (!c) return;
    cudaStreamSynchronize(c->stream);
    fvmb_destroy_ilu(c->ilu);
    fvmb_destroy_krylov(c->kry[0]);
    fvmb_destroy_krylov(c->kry[1]);
    fvmb_destroy_integ_work(c->work);
    fvmb_destroy_predictor(c->pred);
    if (c->stream2) {
        cudaStreamSynchronize(c->stream2);
        cudaStreamDestroy(c->stream2);
    }
    if (c->ev_fork) cudaEventDestroy(c->ev_fork);
    if (c->ev_join) cudaEventDestroy(c->ev_join);
    cudaStream_t s = c->stream;
    delete c;
    if (s) cudaStreamDestroy(s);
}

extern "C" int fvm_n_nodes(const fvm_ctx* c) { return c ? c->N : 0; }

#define FVM_API_BEGIN try {
#define FVM_API_END                                              \
    }                                                            \
    catch (const Error& ex) {                                    \
        set_error(ex.what());                                    \
        return ex.code;                                          \
    }                                                            \
    catch (const std::exception& ex) {                           \
        set_error(ex.what());                                    \
        return -1;                                               \
    }

extern "C" int fvm_initial_head(fvm_ctx* c, double water_table, double* y) {
    FVM_API_BEGIN
    if (!c || !y) throw Error("fvm_initial_head: null argument");
    std::vector<double> h = initial_head_host(c, water_table);
    FVM_CUDA(cudaMemcpyAsync(y, h.data(), sizeof(double) * c->N, cudaMemcpyHostToDevice, c->stream));
    FVM_CUDA(cudaStreamSynchronize(c->stream));
    return 0;
    FVM_API_END
}

extern "C" int fvm_residual(fvm_ctx* c, double t, const double* y, const double* yp, double* res) {
    FVM_API_BEGIN
    (void)t;
    if (!c || !y || !yp || !res) throw Error("fvm_residual: null argument");
    Perturb none;
    launch_residual(c, y, yp, none, nullptr, res);
    FVM_CUDA(cudaGetLastError());
    FVM_CUDA(cudaStreamSynchronize(c->stream));
    return 0;
    FVM_API_END
}

extern "C" int fvm_begin_step(fvm_ctx* c, double t, const double* y, const double* yp) {
    FVM_API_BEGIN
    (void)t;
    if (!c || !y || !yp) throw Error("fvm_begin_step: null argument");
    launch_begin_step(c, y, yp);
    FVM_CUDA(cudaGetLastError());
    FVM_CUDA(cudaStreamSynchronize(c->stream));
    return 0;
    FVM_API_END
}

extern "C" int fvm_jv(fvm_ctx* c, double t, double cj, const double* y, const double* yp,
                      const double* F0, const double* v, double sigma, double* Jv) {
    FVM_API_BEGIN
    (void)t;
    if (!c || !y || !yp || !F0 || !v || !Jv) throw Error("fvm_jv: null argument");
    if (!(sigma != 0.0)) throw Error("fvm_jv: sigma must be non-zero");
    Perturb pt;
    pt.mode = 1;
    pt.sigma = sigma;
    pt.cj = cj;
    pt.v = v;
    launch_residual(c, y, yp, pt, F0, Jv);
    FVM_CUDA(cudaGetLastError());
    FVM_CUDA(cudaStreamSynchronize(c->stream));
    return 0;
    FVM_API_END
}

extern "C" int fvm_set_members(fvm_ctx* c, int n_members, const int* member_ptr) {
    FVM_API_BEGIN
    if (!c || !member_ptr || n_members < 1) throw Error("fvm_set_members: bad argument");
    if (member_ptr[0] != 0 || member_ptr[n_members] != c->N) throw Error("fvm_set_members: ranges must cover the mesh");
    for (int m = 0; m < n_members; ++m)
        if (member_ptr[m + 1] <= member_ptr[m]) throw Error("fvm_set_members: empty or decreasing range");
    c->n_members = n_members;
    c->h_member_ptr.assign(member_ptr, member_ptr + n_members + 1);
    c->member_ptr.upload(c->h_member_ptr, c->stream);
    FVM_CUDA(cudaStreamSynchronize(c->stream));
    return 0;
    FVM_API_END
}

extern "C" int fvm_autotune(fvm_ctx* c, fvm_tune_result* out) {
    FVM_API_BEGIN
    if (!c) throw Error("fvm_autotune: null context");
    if (out) std::memset(out, 0, sizeof(*out));
    autotune(c, out);
    FVM_CUDA(cudaStreamSynchronize(c->stream));
    return 0;
    FVM_API_END
}

extern "C" int fvm_set_element_pass(fvm_ctx* c, int variant, int chunk) {
    FVM_API_BEGIN
    if (!c) throw Error("fvm_set_element_pass: null context");
    if (variant != 0 && variant != 1) throw Error("fvm_set_element_pass: variant must be 0 or 1");
    if (variant == 1 && c->dim != 3) throw Error("fvm_set_element_pass: rebuilt geometry is a 3D variant");
    const bool old_rc = c->recompute;
    const int old_ce = c->chunk_e;
    c->recompute = variant == 1;
    try {
        build_chunks(c, chunk);
    } catch (...) {
        c->recompute = old_rc;
        build_chunks(c, old_ce);
        throw;
    }
    return 0;
    FVM_API_END
}

extern "C" int fvm_element_pass(const fvm_ctx* c, int* variant, int* chunk) {
    FVM_API_BEGIN
    if (!c) throw Error("fvm_element_pass: null context");
    if (variant) *variant = c->recompute ? 1 : 0;
    if (chunk) *chunk = c->chunk_e;
    return 0;
    FVM_API_END
}

extern "C" int fvm_profile(fvm_ctx* c, int enable) {
    FVM_API_BEGIN
    if (!c) throw Error("fvm_profile: null context");
    c->tm.reset();
    c->tm.on = enable != 0;
    return 0;
    FVM_API_END
}

extern "C" int fvm_profile_read(fvm_ctx* c, double* ms, long* counts) {
    FVM_API_BEGIN
    if (!c) throw Error("fvm_profile_read: null context");
    FVM_CUDA(cudaStreamSynchronize(c->stream));
    c->tm.flush();
    for (int k = 0; k < TM_NCAT; ++k) {
        if (ms) ms[k] = c->tm.ms[k];
        if (counts) counts[k] = c->tm.count[k];
    }
    return 0;
    FVM_API_END
}

extern "C" int fvm_set_krylov_variant(fvm_ctx* c, int variant) {
    if (!c) return -1;
    if (variant != 0 && variant != 1) {
        set_error("fvm_set_krylov_variant: variant must be 0 or 1");
        return -1;
    }
    c->krylov_variant = variant;
    return 0;
}

extern "C" int fvm_graph_counters(fvm_ctx* c, long* captures, long* replays) {
    if (!c) return -1;
    if (captures) *captures = c->graph_captures;
    if (replays) *replays = c->graph_replays;
    return 0;
}

extern "C" int fvm_counters(fvm_ctx* c, long* launches, long* residuals) {
    FVM_API_BEGIN
    if (!c) throw Error("fvm_counters: null context");
    if (launches) *launches = c->launches;
    if (residuals) *residuals = c->n_residuals;
    return 0;
    FVM_API_END
}
