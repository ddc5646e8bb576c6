// Device-resident state of one Richards problem (the fvm_ctx behind the C
// ABI) and the small device helpers shared by the kernel files.
#pragma once

#include "common.hpp"
#include "cvfe_geom.cuh"
#include "ktimer.hpp"

#include <cuda_runtime.h>

#include <cmath>
#include <string>
#include <utility>
#include <vector>

namespace fvmb {

#define FVM_CUDA(call)                                                                 \
    do {                                                                               \
        cudaError_t e_ = (call);                                                       \
        if (e_ != cudaSuccess)                                                         \
            throw ::fvmb::Error(std::string(#call) + ": " + cudaGetErrorString(e_), -2); \
    } while (0)

template <class T> struct DevBuf {
    T* p = nullptr;
    size_t n = 0;
    DevBuf() = default;
    DevBuf(const DevBuf&) = delete;
    DevBuf& operator=(const DevBuf&) = delete;
    ~DevBuf() { release(); }
    void release() {
        if (p) cudaFree(p);
        p = nullptr;
        n = 0;
    }
    void alloc(size_t count) {
        if (count == n && p) return;
        release();
        if (count == 0) return;
        FVM_CUDA(cudaMalloc((void**)&p, count * sizeof(T)));
        n = count;
    }
    void upload(const std::vector<T>& v, cudaStream_t s) {
        alloc(v.size());
        if (!v.empty()) FVM_CUDA(cudaMemcpyAsync(p, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice, s));
    }
    void zero(cudaStream_t s) {
        if (n) FVM_CUDA(cudaMemsetAsync(p, 0, n * sizeof(T), s));
    }
};

// van Genuchten parameters of one soil zone on the device
struct ZoneDev {
    double phi, alpha, n, m, Sr;
};

// Van Genuchten-Mualem relations of VarSatPhysicsImpl::saturation
// (examples/fvmporMinlin/fvmpor.h:302-343):
//   a = (-alpha h)^n, b = 1 + a, Se = b^-m, Sw = S_r + (1 - S_r) Se,
//   dSw/dh = -(1 - S_r)(n - 1) (a / b) Se / h,
//   krw = sqrt(Se) ((a / b)^m - 1)^2,
// overridden by Sw = 1, dSw = 0, krw = 1 for h >= 0.
// The reference evaluates three pow() calls; here the powers share their
// logarithms: with L = ln(-alpha h) and lb = ln(1 + a),
//   a = exp(n L), Se = exp(-m lb), (a/b)^m = exp(m (n L - lb)),
// one log, one log1p, two exp and one expm1 instead of three pow (each a
// log and an exp in extended precision); expm1 also removes the
// cancellation in (a/b)^m - 1 that the pow form suffers for dry nodes.  The
// FP64 node pass is bound by these transcendentals; values agree with the
// pow() form to a few ulp (more where pow() cancels).
FVM_HD void van_genuchten(double h, const ZoneDev& z, double& Sw, double& dSw, double& krw) {
    if (h >= 0.0) {
        Sw = 1.0;
        dSw = 0.0;
        krw = 1.0;
        return;
    }
    double L = log(-z.alpha * h);
    double nL = z.n * L;
    double a = exp(nL);
    double lb = log1p(a);
    double Se = exp(-z.m * lb);
    double d = a / (1.0 + a);
    d = d * Se;
    d = d / h;
    d = d * (-(1.0 - z.Sr) * (z.n - 1.0));
    double k = expm1(z.m * (nL - lb));   // (a / b)^m - 1 without cancellation
    k = k * k;
    k = k * sqrt(Se);
    Sw = Se * (1.0 - z.Sr) + z.Sr;
    dSw = d;
    krw = k;
}

// krw at a face: upwind node (0/1) or the averaged weights 0.5/0.5 the
// reference uses before the first step (fvmpor.h:594-595, 919-924)
FVM_HD double face_krw(unsigned u, double ka, double kb) {
    return u == 0 ? ka : (u == 1 ? kb : ka * 0.5 + kb * 0.5);
}

// ---------------------------------------------------------------------------
// Perturbation applied by the node pass before the residual:
//   mode 0: none (plain residual)
//   mode 1: y + sigma v, y' + cj sigma v           (Jacobian-vector product)
//   mode 2: y + d_j, y' + cj d_j on colour c only   (finite-difference Jacobian)
struct Perturb {
    int mode = 0;
    double sigma = 0.0, cj = 0.0;
    const double* sigma_dev = nullptr; // mode 1: device-resident sigma (overrides sigma)
    const double* v = nullptr;       // mode 1
    const double* shift = nullptr;   // mode 2: shift vector d
    const int* colour = nullptr;     // mode 2: colour of every node
    int c = 0;                       // mode 2: active colour
    const int* skip = nullptr;       // when set and *skip != 0 the evaluation is skipped
                                     // (a device-driven loop that has already finished)
    const double* cj_dev = nullptr;  // mode 1: device-resident cj (overrides cj; graph replays)
};

// Node gather of the residual chain: the sum of a node's per-chunk element
// partials (chunk-major positions cpos[part_ptr[i] .. part_ptr[i+1]), in
// ascending chunk order), times 1/V, plus the boundary-flux term, minus the
// storage term; Dirichlet rows h_D - h (residual_evaluation,
// fvmpor_ODE_impl.cpp:99-116).  With F0 set the result becomes the
// difference quotient (F - F0) / sigma.
struct GatherSrc {
    const int* part_ptr;
    const int* cpos;
    const double* part;
    const double* invV;
    const double* bterm;
    const double* hD;
    const unsigned char* ntype;
    const double* h;
    const double* stor;
    const double* F0;
    double inv_sigma;
    const double* sigma_dev;
};

#ifdef __CUDACC__
__device__ __forceinline__ double gather_row(const GatherSrc& g, int i) {
    double r;
    if (g.ntype[i]) {
        r = g.hD[i] - g.h[i];
    } else {
        double s = 0.0;
        const int p1 = g.part_ptr[i + 1];
        for (int p = g.part_ptr[i]; p < p1; ++p) s += g.part[g.cpos[p]];
        r = s * g.invV[i];
        r = r + g.bterm[i];
        r = r - g.stor[i];
    }
    if (g.F0) r = (r - g.F0[i]) * (g.sigma_dev ? 1.0 / *g.sigma_dev : g.inv_sigma);
    return r;
}
#endif

struct BlockILU;   // precond.cu
struct Krylov;     // linalg.cu
struct Predictor;  // predictor.cu
struct IntegWork;  // bdf.cu

} // namespace fvmb

struct fvm_ctx {
    int dim = 0, N = 0, T = 0, nz = 0;
    int npe = 0;   // nodes per element (3 / 4)
    int nfe = 0;   // CV faces per element (3 / 6)
    int E = 0;     // edges
    double rho0 = 1000.0;
    bool recompute = false;
    cudaStream_t stream = nullptr;
    // the integrator's preconditioner set-up runs on stream2 beside the
    // residual evaluation it does not depend on (fork at ev_fork, joined by
    // ev_join before the Krylov solve); made on first use
    cudaStream_t stream2 = nullptr;
    cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
    int device = 0;

    // host copies needed by the preconditioner set-up and the integrator
    std::vector<int> h_elem_nodes;   // [T][npe]
    std::vector<fvm_step_record> last_trace;   // steps of the last integration
    std::vector<int> h_node_type;    // 0 free, 1 Dirichlet
    std::vector<double> h_vert;      // elevation of each node
    std::vector<double> h_hD;        // Dirichlet head (valid where type 1)
    std::vector<double> h_xyz;       // [3][N] coordinates (3D)

    // element data
    fvmb::DevBuf<int4> enodes;        // [T] node ids (4th = -1 for triangles)
    fvmb::DevBuf<double> coef;        // [(f*(npe+1)+k)*T + e]
    fvmb::DevBuf<int> ezone;          // [T], only when nz > 1
    fvmb::DevBuf<double> eK;          // [T] (kiso) or [3][T] conductivities (3D)
    fvmb::DevBuf<double> xyz;         // [3][N] coordinates (3D)
    fvmb::DevBuf<unsigned char> upw;  // [T*8] upwind flag per face: 1 = node b
    fvmb::DevBuf<unsigned char> flip; // [T] bit f set when node a of face f is
                                      // the global back node of its edge

    // node data
    fvmb::DevBuf<double> invV;        // 1 / control-volume measure
    fvmb::DevBuf<double> bterm;       // constant boundary-flux term / V
    fvmb::DevBuf<double> hD;          // Dirichlet head (type 1 nodes)
    fvmb::DevBuf<unsigned char> ntype;
    fvmb::DevBuf<int> nz_ptr, nz_zone;  // zones touching each node (CSR)
    fvmb::DevBuf<double> nz_w;          // SCV volume fraction per node-zone
    fvmb::DevBuf<fvmb::ZoneDev> zones;

    // edges (for the frozen upwind directions)
    fvmb::DevBuf<int> edge_ptr, edge_face;  // edge -> e*nfe + f, ascending e
    fvmb::DevBuf<double> edge_w;            // 1 / sum of the edge's face areas

    // workspace
    fvmb::DevBuf<double> krw;        // [nz][N]
    fvmb::DevBuf<double> hstar;      // perturbed head
    fvmb::DevBuf<double> stor;       // ahh * y'
    // chunked element pass: CE consecutive elements per CTA
    int chunk_e = 0, nchunk = 0, chunk_maxnn = 0;
    size_t chunk_smem = 0;
    bool kiso = false;                    // eK holds one K per element
    int chunk_grid = 0;                   // persistent CTAs of the element pass
    int estride = 0;                      // padded element count of the per-element arrays
    fvmb::DevBuf<int2> ch_seg;            // [nchunk] (padded start, count) of each chunk's nodes
    fvmb::DevBuf<int> elem_err;           // element-pass pipeline status
    fvmb::DevBuf<int> ch_node;            // [P] distinct nodes per chunk, ascending
    fvmb::DevBuf<int> ch_cpos;            // [P] node-major copy slot -> chunk-major position
    fvmb::DevBuf<double> ch_xyz;          // [3][P] chunk-major coordinates (3D)
    fvmb::DevBuf<double> ch_h;            // [P] chunk-major head (several zones)
    fvmb::DevBuf<double> ch_hk;           // [P][2] chunk-major (head, krw) pairs (one zone)
    fvmb::DevBuf<ushort4> elocal;         // [T] chunk-local corner ids
    fvmb::DevBuf<unsigned short> ch_lptr; // [P + nchunk] corner-list offsets
    fvmb::DevBuf<unsigned short> ch_lc;   // [T*npe] node-ordered corner lists
    fvmb::DevBuf<int> part_ptr;           // [N+1] node -> its chunk copies (node-major slots)
    fvmb::DevBuf<double> part;            // [P] per-(chunk, node) partials, chunk-major
    fvmb::DevBuf<double> faceq;      // [T*nfe] averaged-weight face fluxes
    fvmb::DevBuf<double> tmpN[4];    // scratch vectors
    fvmb::DevBuf<float> statf;       // [3][N] static node features: mean ln K, elevation,
                                     // CV surface area (learned predictor inputs)

    int ilu_per_sm = 0;              // block-ILU blocks per SM on large meshes, 0 = automatic
    int schur_iters = -1;            // Schur interface coupling: < 0 off, else sweeps per apply
    // ensemble of independent members (disjoint node ranges): the integrator's
    // error and Newton tests take the largest per-member WRMS norm
    int n_members = 1;
    std::vector<int> h_member_ptr;
    fvmb::DevBuf<int> member_ptr;
    fvmb::BlockILU* ilu = nullptr;
    fvmb::Krylov* kry[2] = {nullptr, nullptr};   // Krylov workspaces by precision (0 FP64, 1 FP32)
    fvmb::Krylov* kry_last = nullptr;            // the one used last (scratch for reductions)
    fvmb::IntegWork* work = nullptr;             // the integrator's vectors (bdf.cu)
    fvmb::Predictor* pred = nullptr;

    long n_residuals = 0;
    long launches = 0;               // kernels launched on this context
    long n_syncs = 0;                // host waits on the context's stream (ctx_sync)
    bool graph_ok = true;            // cleared when a batch capture failed: launch directly
    bool use_graph = false;          // the running integration asked for CUDA-graph batches
    int krylov_variant = 1;          // fused cycle's Gram-Schmidt: 0 CGS2, 1 delayed (fvm_set_krylov_variant)
    long graph_captures = 0, graph_replays = 0;   // CUDA-graph batches of the Arnoldi loop
    fvmb::KernelTimer tm;
    std::string err;
};

namespace fvmb {

// every kernel of the library is launched through this, so the context
// can report how many of its kernels ran
template <typename... KArgs, typename... Args>
inline void fvm_launch(fvm_ctx* c, void (*k)(KArgs...), dim3 grid, dim3 block, size_t smem,
                       cudaStream_t s, Args&&... args) {
    k<<<grid, block, smem, s>>>(std::forward<Args>(args)...);
    c->launches++;
}

// Programmatic dependent launch for the short kernels of the Krylov step
// (node pass, element pass, gather, preconditioner apply): the launch may
// be processed, and the kernel's blocks made resident, while the previous
// kernel on the stream finishes.  Every kernel launched this way calls
// pdl_wait_and_trigger() first, so it reads nothing before its predecessor
// has completed and its writes are visible.
template <typename... KArgs, typename... Args>
inline void fvm_launch_pdl(fvm_ctx* c, void (*k)(KArgs...), dim3 grid, dim3 block, size_t smem,
                           cudaStream_t s, Args&&... args) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = smem;
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    FVM_CUDA(cudaLaunchKernelEx(&cfg, k, std::forward<Args>(args)...));
    c->launches++;
}

// first statement of a kernel launched by fvm_launch_pdl: wait for the
// previous kernel's completion (a no-op after an ordinary launch), then let
// the next programmatic launch begin
// the host waits for the context's stream (counted: fvm_stats.nsync)
inline void ctx_sync(fvm_ctx* c) {
    c->n_syncs++;
    FVM_CUDA(cudaStreamSynchronize(c->stream));
}

__device__ __forceinline__ void pdl_wait_and_trigger() {
    asm volatile("griddepcontrol.wait;" ::: "memory");
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}

// residual driver shared by fvm_residual / fvm_jv / the FD Jacobian
// out = F(t, y~, y'~) (or (F - F0) / sigma when F0 != nullptr)
void launch_residual(fvm_ctx* c, const double* y, const double* yp, const Perturb& pt,
                     const double* F0, double* out);
void launch_begin_step(fvm_ctx* c, const double* y, const double* yp);
// the node and element passes of launch_residual without the gather; the
// returned source describes the gather a consumer performs per row
GatherSrc launch_residual_partials(fvm_ctx* c, const double* y, const double* yp, const Perturb& pt,
                                   const double* F0);
void gather_into(fvm_ctx* c, const GatherSrc& g, double* out, const int* skip);
// back to the averaged 0.5/0.5 face weights used before the first step
void reset_upwind(fvm_ctx* c);

inline int grid_for(long n, int block) { return (int)((n + block - 1) / block); }

// Raises a kernel's dynamic shared-memory limit on the current device to at
// least `bytes`.  The limit belongs to the kernel function for the whole
// process, not to a context, so it is only ever raised: a context built for
// a smaller mesh must not lower the limit that another live context's
// launches need.
void raise_smem_limit(const void* func, size_t bytes);
template <typename... KArgs> inline void raise_smem_limit(void (*k)(KArgs...), size_t bytes) {
    raise_smem_limit(reinterpret_cast<const void*>(k), bytes);
}

} // namespace fvmb
