// Krylov workspace and the internal (device-pointer, no host sync unless
// stated) entry points shared between the ABI, the preconditioner and the
// integrator.
#pragma once

#include "ctx.cuh"

namespace fvmb {

// state of a device-driven Arnoldi cycle (k_arnoldi_givens)
struct ArnState {
    int j;          // completed Arnoldi steps
    int done;       // 0 running, 1 converged, 2 basis full, 3 breakdown
    int m;
    int pad;
    double tol;     // stop when |g_j| / sqrt(N) <= tol
    double sqrtN;
    double rnorm;   // |g_j| / sqrt(N) after the last step
};

struct Krylov {
    int m = 0;
    int precision = 0;        // 0: FP64 basis, 1: FP32 basis
    size_t ld = 0;            // leading dimension of the basis
    void* U = nullptr;        // (m+1) x ld basis, float or double
    DevBuf<double> scale;     // s_i, V_i = s_i U_i
    DevBuf<double> W, t, z, Jv;
    DevBuf<double> partial;
    DevBuf<unsigned> counter;
    DevBuf<double> res;       // reduction results
    DevBuf<double> sigma;
    DevBuf<unsigned> bar;     // grid barrier of the fused orthogonalisation
    DevBuf<int> err;          // 3 = a grid barrier timed out
    int coop_grid = 0;        // blocks of the cooperative launch, 0 = three-pass path
    size_t coop_smem = 0;     // dynamic shared memory of the fused kernel
    int coop_threads = 0;     // its block size: one thread per row quad of a block, 128..512
    DevBuf<ArnState> st;      // device-driven Arnoldi state
    DevBuf<float> tdir;       // FP32 direction of the fused cycle (arnoldi_fused.cu)
    DevBuf<double> ls;        // H [(m+1) x m], cs [m], sn [m], g [m+1]
    double* host = nullptr;   // pinned
    double* host_ls = nullptr;   // pinned: H and g of a fused cycle
    // CUDA graph of one full batch (8 steps) of the device-driven Arnoldi
    // loop (fvm_opts.graph): captured for one key (operator, precision,
    // vectors, preconditioner state), replayed for every full batch; cj and
    // the operator's cj shift come from cjd, written before each batch
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t gexec = nullptr;
    size_t gkey = 0;
    long g_launches = 0, g_residuals = 0;   // launches and residuals one replay runs
    DevBuf<double> cjd;       // [0] cj, [1] cj - cj of the set-up
};

struct GmresCounters {
    long njv = 0;
    long nps = 0;
};

Krylov* krylov_get(fvm_ctx* c, int m, int precision);
// the workspace used last (created small if none): reduction scratch for
// the controller and the learned iterate
inline Krylov* krylov_scratch(fvm_ctx* c) { return c->kry_last ? c->kry_last : krylov_get(c, 1, 0); }
void fvmb_destroy_krylov_impl(Krylov* K);
double reduce_sumsq(fvm_ctx* c, const double* x, const double* w);
double reduce_dot(fvm_ctx* c, const double* x, const double* y);

// op 0: J v by the residual's difference quotient; 1: by the assembled
// Jacobian of the last set-up (jacobian_apply).  sync_end false: a converged
// solve returns with the update of x still queued on the context's stream
int gmres_dev(fvm_ctx* c, double cj, const double* y, const double* yp, const double* F0,
              const double* ewt, const double* b, double* x, int m, int max_restarts,
              int precision, double tol, int* iters, double* res_norm, GmresCounters* cnt, int op = 0,
              bool sync_end = true);

// preconditioner (precond.cu)
void psetup_dev(fvm_ctx* c, double cj, double h, const double* y, const double* yp,
                const double* F0, const double* ewt, int precision);
void psolve_dev(fvm_ctx* c, const double* r, double* z, const int* skip = nullptr);
// y = J(cj) x with the assembled difference-quotient Jacobian of the last
// set-up (the Krylov operator of fvm_opts.krylov_operator = 1)
void jacobian_apply(fvm_ctx* c, double cj, const double* x, double* y, const int* skip = nullptr,
                    const double* dcj_dev = nullptr);
double jacobian_cj_setup(fvm_ctx* c);   // cj of the last set-up
int ilu_factored(fvm_ctx* c);           // precision of the current factor, -1 none
bool schur_active(fvm_ctx* c);          // the Schur-coupled apply is on
// fused Arnoldi cycle of the assembled operator (arnoldi_fused.cu):
// fused_prepare refreshes the operator after a set-up and tells whether the
// cycle can run (FP32 factor staged in shared memory, every block resident);
// fused_cycle runs one cycle from the state gmres has put in place
bool fused_prepare(fvm_ctx* c, int m);
void fused_cycle(fvm_ctx* c, Krylov* K, double cj, const double* ewt, double* H_d, double* cs_d, double* sn_d,
                 double* g_d);
bool ilu_ready(fvm_ctx* c);
int ilu_status(fvm_ctx* c);   // 0 ok, 1 zero pivot in the last factorisation
// the same status as the last host wait saw it (no wait of its own: valid
// once any ctx_sync has followed the set-up)
int ilu_status_seen(fvm_ctx* c);
int schur_status(fvm_ctx* c); // 0 ok, 3 a barrier of the Schur-coupled apply timed out (then cleared)

} // namespace fvmb
