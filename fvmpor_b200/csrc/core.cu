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

#include <algorithm>
#include <cstring>
#include <memory>
#include <mutex>
#include <numeric>

namespace fvmb {

static thread_local std::string g_last_error;
void set_error(const std::string& msg) { g_last_error = msg; }

constexpr int kBlock = 256;

// ------------------------------------------------------------------ kernels
__global__ void k_node(int N, const double* __restrict__ y, const double* __restrict__ yp,
                       Perturb pt, const ZoneDev* __restrict__ zones, int nz,
                       const int* __restrict__ nz_ptr, const int* __restrict__ nz_zone,
                       const double* __restrict__ nz_w, double rho0, double* __restrict__ krw,
                       double* __restrict__ hstar, double* __restrict__ stor) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N) return;
    double h = y[i], hp = yp[i];
    if (pt.mode == 1) {
        double sg = pt.sigma_dev ? *pt.sigma_dev : pt.sigma;
        double p = sg * pt.v[i];
        h = h + p;
        hp = hp + pt.cj * p;
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
    if (nz == 1) {
        double Sw, d, k;
        van_genuchten(h, zones[0], Sw, d, k);
        krw[i] = k;
        phi = zones[0].phi * nz_w[i];
        dsw = d * nz_w[i];
    } else {
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

// krw at a face: upwind node (0/1) or the averaged weights 0.5/0.5 the
// reference uses before the first step (fvmpor.h:594-595, 919-924)
__device__ __forceinline__ double face_krw(unsigned u, double ka, double kb) {
    return u == 0 ? ka : (u == 1 ? kb : ka * 0.5 + kb * 0.5);
}

// stored-coefficient element pass, tetrahedra
template <bool MULTIZONE>
__global__ void __launch_bounds__(256) k_elem_tet(int T, int N, const int4* __restrict__ en,
                                                   const double* __restrict__ coef,
                                                   const int* __restrict__ ezone,
                                                   const double* __restrict__ krw,
                                                   const double* __restrict__ h,
                                                   const unsigned char* __restrict__ upw,
                                                   double rho0, const int4* __restrict__ epos,
                                                   double* __restrict__ slots) {
    int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= T) return;
    int4 nd = en[e];
    double hv[4] = {h[nd.x], h[nd.y], h[nd.z], h[nd.w]};
    size_t zo = MULTIZONE ? (size_t)ezone[e] * N : 0;
    double kr[4] = {krw[zo + nd.x], krw[zo + nd.y], krw[zo + nd.z], krw[zo + nd.w]};
    uint2 uw = *reinterpret_cast<const uint2*>(upw + (size_t)8 * e);
    double c[4] = {0.0, 0.0, 0.0, 0.0};
#pragma unroll
    for (int f = 0; f < 6; ++f) {
        const double* cf = coef + (size_t)(f * 5) * T + e;
        double q = cf[0] * hv[0];
        q += cf[(size_t)T] * hv[1];
        q += cf[(size_t)2 * T] * hv[2];
        q += cf[(size_t)3 * T] * hv[3];
        q += cf[(size_t)4 * T];
        int a = tet_edge_a(f), b = tet_edge_b(f);
        unsigned u = ((f < 4 ? uw.x >> (8 * f) : uw.y >> (8 * (f - 4)))) & 0xffu;
        double flux = rho0 * (q * face_krw(u, kr[a], kr[b]));
        c[a] -= flux;
        c[b] += flux;
    }
    int4 ps = epos[e];
    slots[ps.x] = c[0];
    slots[ps.y] = c[1];
    slots[ps.z] = c[2];
    slots[ps.w] = c[3];
}

// recompute-geometry element pass, tetrahedra: the face coefficients are
// rebuilt from the (L2-resident) node coordinates instead of streamed
template <bool MULTIZONE>
__global__ void __launch_bounds__(256) k_elem_tet_rc(int T, int N, const int4* __restrict__ en,
                                                      const double* __restrict__ xyz,
                                                      const double* __restrict__ eK,
                                                      const int* __restrict__ ezone,
                                                      const double* __restrict__ krw,
                                                      const double* __restrict__ h,
                                                      const unsigned char* __restrict__ upw,
                                                      double rho0, const int4* __restrict__ epos,
                                                      double* __restrict__ slots) {
    int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= T) return;
    int4 nd = en[e];
    int ids[4] = {nd.x, nd.y, nd.z, nd.w};
    double X[4][3];
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        X[k][0] = xyz[ids[k]];
        X[k][1] = xyz[(size_t)N + ids[k]];
        X[k][2] = xyz[(size_t)2 * N + ids[k]];
    }
    double C[6][4], G[6], A[6], vol;
    tet_coefficients(X[0], X[1], X[2], X[3], eK[e], eK[(size_t)T + e], eK[(size_t)2 * T + e], C, G, A, &vol);
    double hv[4] = {h[nd.x], h[nd.y], h[nd.z], h[nd.w]};
    size_t zo = MULTIZONE ? (size_t)ezone[e] * N : 0;
    double kr[4] = {krw[zo + nd.x], krw[zo + nd.y], krw[zo + nd.z], krw[zo + nd.w]};
    uint2 uw = *reinterpret_cast<const uint2*>(upw + (size_t)8 * e);
    double c[4] = {0.0, 0.0, 0.0, 0.0};
#pragma unroll
    for (int f = 0; f < 6; ++f) {
        double q = C[f][0] * hv[0];
        q += C[f][1] * hv[1];
        q += C[f][2] * hv[2];
        q += C[f][3] * hv[3];
        q += G[f];
        int a = tet_edge_a(f), b = tet_edge_b(f);
        unsigned u = ((f < 4 ? uw.x >> (8 * f) : uw.y >> (8 * (f - 4)))) & 0xffu;
        double flux = rho0 * (q * face_krw(u, kr[a], kr[b]));
        c[a] -= flux;
        c[b] += flux;
    }
    int4 ps = epos[e];
    slots[ps.x] = c[0];
    slots[ps.y] = c[1];
    slots[ps.z] = c[2];
    slots[ps.w] = c[3];
}

template <bool MULTIZONE>
__global__ void __launch_bounds__(256) k_elem_tri(int T, int N, const int4* __restrict__ en,
                                                   const double* __restrict__ coef,
                                                   const int* __restrict__ ezone,
                                                   const double* __restrict__ krw,
                                                   const double* __restrict__ h,
                                                   const unsigned char* __restrict__ upw,
                                                   double rho0, const int4* __restrict__ epos,
                                                   double* __restrict__ slots) {
    int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= T) return;
    int4 nd = en[e];
    double hv[3] = {h[nd.x], h[nd.y], h[nd.z]};
    size_t zo = MULTIZONE ? (size_t)ezone[e] * N : 0;
    double kr[3] = {krw[zo + nd.x], krw[zo + nd.y], krw[zo + nd.z]};
    unsigned uw = *reinterpret_cast<const unsigned*>(upw + (size_t)8 * e);
    double c[3] = {0.0, 0.0, 0.0};
#pragma unroll
    for (int f = 0; f < 3; ++f) {
        const double* cf = coef + (size_t)(f * 4) * T + e;
        double q = cf[0] * hv[0];
        q += cf[(size_t)T] * hv[1];
        q += cf[(size_t)2 * T] * hv[2];
        q += cf[(size_t)3 * T];
        int a = tri_edge_a(f), b = tri_edge_b(f);
        unsigned u = (uw >> (8 * f)) & 0xffu;
        double flux = rho0 * (q * face_krw(u, kr[a], kr[b]));
        c[a] -= flux;
        c[b] += flux;
    }
    int4 ps = epos[e];
    slots[ps.x] = c[0];
    slots[ps.y] = c[1];
    slots[ps.z] = c[2];
}

// node gather: the element pass left node i's partials in the contiguous
// slot range [inc_ptr[i], inc_ptr[i+1]) in ascending element order; sum
// them in that order.  F0 != nullptr turns the result into
// (F - F0) * inv_sigma.
__global__ void k_gather(int N, const int* __restrict__ inc_ptr,
                         const double* __restrict__ slots, const double* __restrict__ invV,
                         const double* __restrict__ bterm, const double* __restrict__ hD,
                         const unsigned char* __restrict__ ntype, const double* __restrict__ h,
                         const double* __restrict__ stor, const double* __restrict__ F0,
                         double inv_sigma, const double* __restrict__ sigma_dev,
                         double* __restrict__ out) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N) return;
    double r;
    if (ntype[i]) {
        r = hD[i] - h[i];
    } else {
        double s = 0.0;
        int p1 = inc_ptr[i + 1];
        for (int p = inc_ptr[i]; p < p1; ++p) s += slots[p];
        r = s * invV[i];
        r = r + bterm[i];
        r = r - stor[i];
    }
    if (F0) r = (r - F0[i]) * (sigma_dev ? 1.0 / *sigma_dev : inv_sigma);
    out[i] = r;
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
void launch_residual(fvm_ctx* c, const double* y, const double* yp, const Perturb& pt,
                     const double* F0, double* out) {
    cudaStream_t s = c->stream;
    const double* h = pt.mode ? c->hstar.p : y;
    c->tm.begin(TM_NODE, s);
    fvm_launch(c, k_node, grid_for(c->N, kBlock), kBlock, 0, s, c->N, y, yp, pt, c->zones.p, c->nz, c->nz_ptr.p,
                                                      c->nz_zone.p, c->nz_w.p, c->rho0, c->krw.p,
                                                      c->hstar.p, c->stor.p);
    c->tm.end(TM_NODE, s);
    int gb = grid_for(c->T, kBlock);
    c->tm.begin(TM_ELEM, s);
    if (c->dim == 3) {
        if (c->recompute) {
            if (c->nz > 1)
                fvm_launch(c, k_elem_tet_rc<true>, gb, kBlock, 0, s, c->T, c->N, c->enodes.p, c->xyz.p, c->eK.p, c->ezone.p, c->krw.p, h, c->upw.p, c->rho0, c->epos.p, c->slots.p);
            else
                fvm_launch(c, k_elem_tet_rc<false>, gb, kBlock, 0, s, c->T, c->N, c->enodes.p, c->xyz.p, c->eK.p, c->ezone.p, c->krw.p, h, c->upw.p, c->rho0, c->epos.p, c->slots.p);
        } else {
            if (c->nz > 1)
                fvm_launch(c, k_elem_tet<true>, gb, kBlock, 0, s, c->T, c->N, c->enodes.p, c->coef.p, c->ezone.p, c->krw.p, h, c->upw.p, c->rho0, c->epos.p, c->slots.p);
            else
                fvm_launch(c, k_elem_tet<false>, gb, kBlock, 0, s, c->T, c->N, c->enodes.p, c->coef.p, c->ezone.p, c->krw.p, h, c->upw.p, c->rho0, c->epos.p, c->slots.p);
        }
    } else {
        if (c->nz > 1)
            fvm_launch(c, k_elem_tri<true>, gb, kBlock, 0, s, c->T, c->N, c->enodes.p, c->coef.p, c->ezone.p, c->krw.p, h, c->upw.p, c->rho0, c->epos.p, c->slots.p);
        else
            fvm_launch(c, k_elem_tri<false>, gb, kBlock, 0, s, c->T, c->N, c->enodes.p, c->coef.p, c->ezone.p, c->krw.p, h, c->upw.p, c->rho0, c->epos.p, c->slots.p);
    }
    c->tm.end(TM_ELEM, s);
    double inv_sigma = 0.0;
    if (F0 && !pt.sigma_dev) inv_sigma = 1.0 / pt.sigma;
    c->tm.begin(TM_GATHER, s);
    fvm_launch(c, k_gather, grid_for(c->N, kBlock), kBlock, 0, s, c->N, c->inc_ptr.p, c->slots.p,
                                                        c->invV.p, c->bterm.p, c->hD.p, c->ntype.p,
                                                        h, c->stor.p, F0, inv_sigma,
                                                        F0 ? pt.sigma_dev : nullptr, out);
    c->tm.end(TM_GATHER, s);
    c->n_residuals++;
}

void launch_begin_step(fvm_ctx* c, const double* y, const double* yp) {
    cudaStream_t s = c->stream;
    Perturb none;
    fvm_launch(c, k_node, grid_for(c->N, kBlock), kBlock, 0, s, c->N, y, yp, none, c->zones.p, c->nz, c->nz_ptr.p,
                                                      c->nz_zone.p, c->nz_w.p, c->rho0, c->krw.p,
                                                      c->hstar.p, c->stor.p);
    int gb = grid_for(c->T, kBlock);
    if (c->dim == 3) {
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
    c->nz = ph->n_zones; c->rho0 = ph->rho0;
    c->recompute = (flags & FVM_FLAG_RECOMPUTE_GEOMETRY) && dim == 3;
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
    std::vector<std::pair<uint64_t, int>> keys((size_t)T * nfe);
    for (int e = 0; e < T; ++e)
        for (int f = 0; f < nfe; ++f) {
            const int* v = m->elem_nodes + (size_t)e * npe;
            int a = v[dim == 3 ? tet_edge_a(f) : tri_edge_a(f)];
            int b = v[dim == 3 ? tet_edge_b(f) : tri_edge_b(f)];
            uint64_t key = ((uint64_t)(uint32_t)std::min(a, b) << 32) | (uint32_t)std::max(a, b);
            keys[(size_t)e * nfe + f] = {key, e * nfe + f};
        }
    std::sort(keys.begin(), keys.end());
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
    if (c->recompute) {
        std::vector<double> xyz((size_t)3 * N);
        for (int i = 0; i < N; ++i)
            for (int d = 0; d < 3; ++d) xyz[(size_t)d * N + i] = m->coords[3 * (size_t)i + d];
        c->xyz.upload(xyz, s);
        c->eK.upload(eK3, s);
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
    c->inc_ptr.upload(inc_ptr, s);
    c->inc.upload(inc, s);
    {
        // slot of (e, k) in the node-ordered partial array: the inverse of inc
        std::vector<int4> epos(T, make_int4(0, 0, 0, 0));
        for (size_t p = 0; p < inc.size(); ++p) {
            int e = inc[p] / npe, k = inc[p] % npe;
            int* q = reinterpret_cast<int*>(&epos[e]);
            q[k] = (int)p;
        }
        c->epos.upload(epos, s);
    }
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
    c->upw.upload(std::vector<unsigned char>((size_t)8 * T, 2), s);
    c->krw.alloc((size_t)c->nz * N);
    c->krw.zero(s);
    c->hstar.alloc(N);
    c->stor.alloc(N);
    c->slots.alloc((size_t)T * npe);
    c->faceq.alloc((size_t)T * nfe);
    for (auto& b : c->tmpN) b.alloc(N);
    FVM_CUDA(cudaStreamSynchronize(s));
}

} // namespace fvmb

using namespace fvmb;

void fvmb_destroy_ilu(fvmb::BlockILU* p);
void fvmb_destroy_krylov(fvmb::Krylov* p);
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
    fvmb_destroy_krylov(c->kry);
    fvmb_destroy_predictor(c->pred);
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
    std::vector<double> h(c->N);
    for (int i = 0; i < c->N; ++i) h[i] = c->h_node_type[i] ? c->h_hD[i] : water_table - c->h_vert[i];
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

extern "C" int fvm_counters(fvm_ctx* c, long* launches, long* residuals) {
    FVM_API_BEGIN
    if (!c) throw Error("fvm_counters: null context");
    if (launches) *launches = c->launches;
    if (residuals) *residuals = c->n_residuals;
    return 0;
    FVM_API_END
}
