/*
 * fvmpor_b200 — C ABI of the B200 Richards-equation hot path.
 *
 * The reference (FVMPor) exposes its hot path as three C++ template concepts
 * and no C ABI:
 *   Physics         include/fvm/physics_base.h:18-131,
 *                   examples/fvmporMinlin/fvmpor.h:221-231
 *   Callback        include/fvm/fvm.h:347-359
 *   Preconditioner  examples/fvmporMinlin/preconditioner_dss.h:27-39
 * bridged to SUNDIALS IDAS by include/fvm/integrators/ida_integrator.h:479-587.
 * Each entry point below names the reference interface it replaces.
 *
 * Conventions (all entry points):
 *   - Vectors passed to fvm_* compute calls are DEVICE pointers (cudaMalloc'd,
 *     CUDA-visible), length n_nodes, owned by the caller, unless the name ends
 *     in _host.
 *   - Return status follows the IDA callback convention the reference keeps
 *     (ida_integrator.h:498,549,576): 0 ok, >0 recoverable (NaN/Inf in a
 *     result, Krylov non-convergence, zero pivot), <0 fatal (bad argument,
 *     CUDA error, missing setup).  No C++ exception crosses this boundary.
 *   - One CUDA stream per context; calls on one context are single-threaded.
 *     Inside fvm_integrate* the preconditioner set-up runs on a second,
 *     internal stream of the context beside the residual evaluation it does
 *     not depend on, joined back before the Krylov solve; every call still
 *     returns with its work ordered on the context's stream.
 *   - Every device-side wait is bounded and reports a status; nothing spins
 *     forever.
 */
#ifndef FVMPOR_B200_H
#define FVMPOR_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ------------------------------------------------------------------ */
/* Problem description (host memory, read once by fvm_create)          */
/* ------------------------------------------------------------------ */

/* Unstructured simplex mesh.  Replaces the .pmesh reader state of
 * mesh::Mesh (src/fvm/mesh.cpp:82-366): node coordinates, element
 * connectivity with a physical-zone tag per element (mesh.cpp:294-296),
 * boundary faces with boundary tags (mesh.cpp:333-341) and the per-node
 * boundary tag list the reader attaches to nodes (mesh.cpp:246-262),
 * reduced here to the tag that decides Dirichlet rows
 * (fvmpor.h:405-417). */
typedef struct {
    int dim;                 /* 2 (triangles) or 3 (tetrahedra)            */
    int n_nodes;
    int n_elements;
    int n_bfaces;            /* boundary segments (2D) / triangles (3D)    */
    const double* coords;    /* [n_nodes][3]; z = 0 in 2D                  */
    const int* elem_nodes;   /* [n_elements][dim+1]                        */
    const int* elem_zone;    /* [n_elements] index into fvm_physics.zones  */
    const double* elem_K;    /* [n_elements] isotropic K override, or NULL */
    const int* bface_nodes;  /* [n_bfaces][dim]                            */
    const int* bface_elem;   /* [n_bfaces] element owning the face         */
    const int* bface_tag;    /* [n_bfaces] boundary tag (>0)               */
    const int* node_tag;     /* [n_nodes] boundary tag of a Dirichlet-type
                                condition touching the node, 0 = none      */
} fvm_mesh;

/* Soil zone.  PhysicalZone (examples/fvmporMinlin/definitions.h:267-299);
 * mVG = 1 - 1/nVG as set in vs.h:53.  Soil and fluid compressibility are
 * zero in every configuration (vs.h:43,71), so porosity is constant. */
typedef struct {
    double Kxx, Kyy, Kzz;    /* saturated conductivity [m/s]               */
    double phi;              /* porosity (theta_s)                         */
    double alphaVG, nVG;     /* van Genuchten parameters                   */
    double S_r;              /* residual saturation (theta_r / theta_s)    */
} fvm_zone;

/* Boundary condition.  BoundaryCondition (definitions.h:105-265); the
 * hot path supports type 1 (Dirichlet value), 3 (prescribed normal flux
 * value, positive outwards) and 4 (hydrostatic head (1+eta)(b - z)). */
typedef struct {
    int tag;
    int type;
    double value;
    double b;
    double eta;
} fvm_bc;

typedef struct {
    int n_zones;
    const fvm_zone* zones;
    int n_bcs;
    const fvm_bc* bcs;
    double rho0;             /* Constants::rho_0 (definitions.h:301-326)   */
} fvm_physics;

/* flags for fvm_create.  The element pass of the residual has two
 * variants: stored face coefficients streamed from HBM (240 B per
 * tetrahedron) or the face geometry rebuilt from the vertices on every
 * launch (3D only, the 3D default). */
#define FVM_FLAG_RECOMPUTE_GEOMETRY 1  /* rebuilt geometry (3D)            */
#define FVM_FLAG_AUTOTUNE           2  /* time every element-pass variant
                                          and chunk size on this mesh at
                                          creation and keep the fastest    */
#define FVM_FLAG_STORED_GEOMETRY    4  /* stored coefficients in 3D too    */

/* Autotuner report: candidate i ran `variant[i]` (0 stored, 1 rebuilt
 * geometry) with `chunk[i]` elements per CTA in `us[i]` microseconds (median
 * element-pass time, L2 flushed before every launch); `best` indexes the
 * candidate kept. */
#define FVM_TUNE_MAX 16
typedef struct {
    int n, best;
    int variant[FVM_TUNE_MAX];
    int chunk[FVM_TUNE_MAX];
    double us[FVM_TUNE_MAX];
} fvm_tune_result;

typedef struct fvm_ctx fvm_ctx;

/* Builds the device-resident CVFE data for one mesh on the current CUDA
 * device.  Replaces VarSatPhysicsImpl::initialise_vectors and
 * initialise_shape_functions (fvmpor.h:347-644, 948-1124) and the CV
 * construction of mesh::Mesh (src/fvm/mesh.cpp:786-1156).  Returns NULL on
 * error; fvm_last_error() tells why. */
fvm_ctx* fvm_create(const fvm_mesh* mesh, const fvm_physics* phys, int flags);
void fvm_destroy(fvm_ctx* ctx);
const char* fvm_last_error(void);
int fvm_n_nodes(const fvm_ctx* ctx);

/* Initial state: head from the hydrostatic/Dirichlet rules of
 * set_initial_conditions (vs.h:8-32) with the given water-table elevation
 * for the non-Dirichlet nodes (h = wt - elevation), written to y (device). */
int fvm_initial_head(fvm_ctx* ctx, double water_table, double* y);

/* F(t, y, y') -> res.  Replaces Physics::preprocess_evaluation +
 * residual_evaluation (fvmpor_ODE_impl.cpp:62-116) behind the Callback
 * (solver.h:123-133) that IDAIntegrator::f calls (ida_integrator.h:479-498). */
int fvm_residual(fvm_ctx* ctx, double t, const double* y, const double* yp,
                 double* res);

/* Freezes the upwind direction of every edge for the coming step.
 * Replaces Physics::preprocess_timestep + process_spatial_weights
 * (fvmpor_ODE_impl.cpp:118-141, fvmpor.h:762-795). */
int fvm_begin_step(fvm_ctx* ctx, double t, const double* y, const double* yp);

/* Difference-quotient Jacobian action
 *   Jv = [F(t, y + sigma v, y' + cj sigma v) - F0] / sigma,
 * the J*v IDAS SPGMR forms internally (selected at ida_integrator.h:252). */
int fvm_jv(fvm_ctx* ctx, double t, double cj, const double* y,
           const double* yp, const double* F0, const double* v,
           double sigma, double* Jv);

/* Preconditioner setup: coloured finite-difference Jacobian
 * J = dF/dy + cj dF/dy' (Preconditioner::setup, preconditioner_dss.cpp:
 * 284-373, shift rule :322-329) followed by a block-ILU(0) factorisation
 * (decomp/ILU.c:12-115) in place of the MKL DSS factorisation (:368).
 * ewt are the inverse error weights 1/(rtol|y|+atol).
 * precision: 0 = FP64 factor, 1 = FP32 factor. */
int fvm_psetup(fvm_ctx* ctx, double t, double cj, double h, const double* y,
               const double* yp, const double* F0, const double* ewt,
               int precision);

/* z = P^{-1} r.  Replaces Preconditioner::apply (preconditioner_dss.cpp:
 * 375-405); forward/backward substitution of decomp/ILU.c:133-223. */
int fvm_psolve(fvm_ctx* ctx, const double* r, double* z);

/* Pattern statistics of the last set-up (Preconditioner::initialise,
 * preconditioner_dss.cpp:144-282): non-zeros of J, colours, ILU blocks and
 * the largest number of dependency levels in a block.  Any pointer may be
 * NULL. */
int fvm_precond_info(fvm_ctx* ctx, int* nnz, int* ncolours, int* nblocks,
                     int* max_levels);

/* Copies the assembled J (CSR, rows ascending, columns ascending) into HOST
 * buffers of n_nodes+1 / nnz / nnz entries (the values the reference
 * gathers into values_ at preconditioner_dss.cpp:362, with the sign
 * convention +J).  Any pointer may be NULL. */
int fvm_precond_jacobian(fvm_ctx* ctx, int* rowptr, int* col, double* val);

/* Preconditioned restarted GMRES(m) on J x = b, zero initial guess, left
 * preconditioned and scaled by D = diag(ewt) as IDAS SPGMR runs it inside
 * Newton (ida_integrator.h:248-254): stops when ||D P^-1 (b - J x)||_wrms
 * <= tol.  Arnoldi, Givens least squares and restarts follow
 * decomp/gmres.c:26-201, :412-511 and decomp/linalg_dense.c:128-173.
 * J*v is the difference quotient (fvm_jv) with sigma = 1/||v||_wrms.
 * precision 1 keeps the Krylov basis in FP32; the Hessenberg, Givens and
 * stopping test stay FP64.  Needs fvm_psetup first.  Returns 0 on
 * convergence, 1 (recoverable) otherwise; *iters gets the Arnoldi steps. */
int fvm_gmres(fvm_ctx* ctx, double t, double cj, const double* y,
              const double* yp, const double* F0, const double* ewt,
              const double* b, double* x, int m, int max_restarts,
              int precision, double tol, int* iters, double* res_norm);

/* WRMS norm sqrt(mean((x*ewt)^2)) and dot product (N_Vector ops of the
 * reference's nvector_parallel_cuda, examples/fvmporMinlin/makefile:30). */
double fvm_wrms(fvm_ctx* ctx, const double* x, const double* ewt);
double fvm_dot(fvm_ctx* ctx, const double* x, const double* y);

/* Live per-kernel timing with CUDA events on the context stream (the
 * reference's util::TimerCuda, include/util/timer_cuda.h:11-57, and the
 * preconditioner time_J/time_M/time_apply accumulators, preconditioner_dss.
 * cpp:297-373).  fvm_profile(ctx, 1) resets and starts, (ctx, 0) stops;
 * fvm_profile_read fills FVM_PROF_NCAT milliseconds / launch counts in
 * the order node pass, element pass, node gather, ILU apply, Gram-Schmidt
 * (with the Givens update), ILU factor, FD Jacobian, learned-iterate
 * network (features + forward), learned-iterate attempt (all of it). */
#define FVM_PROF_NCAT 9
int fvm_profile(fvm_ctx* ctx, int enable);
int fvm_profile_read(fvm_ctx* ctx, double* ms, long* counts);

/* WRMS norm sqrt(mean((x*ewt)^2)) of n values, like fvm_wrms, but without
 * any device allocation and without a context: for callers that cannot
 * call cudaMalloc (a host integrator that owns all device memory through its
 * own pool and calls the norm inside its step loop, where an allocation
 * would stall the device or is forbidden).  No counterpart in the
 * reference.  The reduction scratch is a static __device__ array of 4,128
 * doubles (33,024 bytes: partial sums for 4,096 blocks plus a 256-byte
 * counter and result tail) that every GPU loading the library keeps until
 * exit, which bounds n to fvm_wrms_noalloc_max_n() = 8,388,608; larger n is
 * rejected (status < 0, message in fvm_last_error()).  The first call on a
 * device looks the array's address up with cudaGetSymbolAddress and keeps
 * it for the life of the process, so make that first call before any
 * stream capture, and do not call this entry point again after a
 * cudaDeviceReset of that device (the module, and with it the array, may
 * then be loaded at another address).  x, ewt (may be NULL = 1) and result are
 * device pointers; the work is queued on `stream` (a cudaStream_t, NULL for
 * the legacy default stream) and *result is valid once that stream reaches
 * it.  All calls share the one scratch array: calls that overlap on the GPU
 * (on different streams) race and must be serialised by the caller. */
long fvm_wrms_noalloc_max_n(void);
int fvm_wrms_noalloc(const double* x, const double* ewt, long n,
                     double* result, void* stream);

/* Element-pass tuning.  The residual's element pass runs over chunks of
 * consecutive elements, one CTA per chunk, with the chunk's nodes staged in
 * shared memory; the chunk size and the geometry variant (see the flags
 * above) set its speed, not its result beyond rounding.  fvm_autotune times
 * every candidate on this context's mesh and keeps the fastest (out may be
 * NULL); fvm_set_element_pass selects one explicitly (chunk: 32..2048
 * elements, bounded by shared memory); fvm_element_pass reports the
 * current choice.  No counterpart in the reference, whose residual is a
 * fixed sequence of cuSPARSE SpMVs (fvmpor.h:948-1124). */
int fvm_autotune(fvm_ctx* ctx, fvm_tune_result* out);
/* Ensemble of independent problems in one context: member m owns nodes
 * [member_ptr[m], member_ptr[m+1]) (host array of n_members + 1 entries,
 * 0 .. n_nodes, no coupling between members).  The integrator's Newton
 * and error tests then use the largest per-member WRMS norm, so every
 * member meets the tolerances on its own; the residual, preconditioner
 * and Krylov kernels run over all members in the same launches.  No
 * counterpart in the reference (one mesh per run). */
int fvm_set_members(fvm_ctx* ctx, int n_members, const int* member_ptr);
/* Block-ILU partition on large meshes: per_sm (1..16) blocks per SM, or 0
 * (the default) for the fewest blocks per SM that keep every block at most
 * 1,600 rows, the size whose FP32 factor fits the shared-memory apply.  Fewer,
 * larger blocks couple more nodes inside the factor (fewer Krylov
 * iterations); more, smaller ones shorten the level chains of the
 * triangular solves and let several blocks share an SM.  Drops the current
 * factor; the next fvm_psetup rebuilds the pattern.  The reference's
 * preconditioner is one direct factorisation (preconditioner_dss.cpp:284-405). */
int fvm_set_precond_blocks(fvm_ctx* ctx, int per_sm);
/* Schur interface coupling of the block ILU(0) (decomp/schur.c:887-987
 * S = C - F B^-1 E, :1407-1636 precon_schur_apply).  iters < 0: off (plain
 * block-Jacobi ILU(0), the default).  iters >= 0: every block orders its
 * interface rows (those coupled to another block) after its interior rows,
 * so its ILU(0) holds the ILU(0) of its local Schur complement, and each
 * apply runs `iters` block-Jacobi sweeps of the global interface system
 * (local Schur factors plus the couplings between blocks) before the
 * interior back substitution.  Needs every block's staged factor in shared
 * memory (the FP32 factor on the 3D meshes); fvm_psolve reports an error
 * otherwise.  Drops the current factor; the next fvm_psetup rebuilds the
 * pattern.  The Krylov paths then use separate kernels per Arnoldi step
 * (no fused cycle). */
int fvm_set_precond_schur(fvm_ctx* ctx, int iters);
/* The Schur option of the current pattern: its iterations, the number of
 * interface rows, and which factor precisions can run it (bit 0 FP64,
 * bit 1 FP32).  Any pointer may be NULL. */
int fvm_precond_schur_info(fvm_ctx* ctx, int* iters, int* interface_rows, int* supported);
int fvm_set_element_pass(fvm_ctx* ctx, int variant, int chunk);
int fvm_element_pass(const fvm_ctx* ctx, int* variant, int* chunk);

/* Running totals since fvm_create: kernels launched by the library on this
 * context and residual evaluations (the Physics::calls() counter,
 * fvmpor.h:206).  Either pointer may be NULL. */
int fvm_counters(fvm_ctx* ctx, long* launches, long* residuals);

/* ------------------------------------------------------------------ */
/* Integrator: variable-order BDF + Newton-Krylov driving the above.     */
/* Replaces IDAIntegrator (ida_integrator.h:39-340) and the time loop of */
/* examples/fvmporMinlin/fvmpor_ODE.cpp:202-232.                         */
/* ------------------------------------------------------------------ */
typedef struct {
    double rtol, atol;       /* scalar tolerances (IDASStolerances :243)   */
    int max_order;           /* <= 5 (set_max_order :467)                  */
    int krylov_dim;          /* GMRES(m)                                   */
    int max_restarts;
    int precision;           /* 0 = FP64, 1 = FP32 factor/apply + basis    */
    int use_predictor;       /* learned Newton initial iterate (fvm_mlp_*):
                                0 off, 1 on the retry after a failed
                                corrector, 2 on every step             */
    double h0;               /* first step, 0 = automatic                  */
    double hmax;             /* 0 = unbounded                              */
    long max_steps;
    double eps_lin;          /* Krylov tolerance factor: GMRES stops at
                                eps_lin * 0.33 weighted units (IDA's
                                epslin); default and 0: 3e-5, tighter
                                than IDA's 0.05 because block-ILU(0) is
                                far weaker than the reference's direct
                                factorisation                            */
    double cj_refresh;       /* new preconditioner when cj moved by more
                                than this factor since the last set-up
                                (0 = 1.05)                               */
    int psetup_age;          /* ... or after this many steps (0 = 1:
                                every step)                              */
    int krylov_operator;     /* 0: J v as the difference quotient of the
                                residual (Jacobian-free, IDAS SPGMR's
                                product); 1: J v as the product with the
                                preconditioner set-up's assembled
                                difference-quotient Jacobian, shifted
                                exactly to the current cj (the residual,
                                Newton update and tests stay FP64)        */
    int graph;               /* 1: the device-driven Arnoldi loop runs its
                                full batches (8 steps of the separate
                                kernels: J v, apply, orthogonalisation)
                                from one CUDA graph per operator and
                                vector set, instead of 40 launches; no
                                effect on the fused cycle (one launch per
                                GMRES cycle already)                     */
} fvm_opts;

typedef struct {
    long nst;     /* steps                          */
    long nre;     /* residual evaluations (any)     */
    long nni;     /* Newton iterations              */
    long nli;     /* Krylov (Arnoldi) iterations    */
    long npe;     /* preconditioner setups          */
    long nps;     /* preconditioner solves          */
    long ncfn;    /* Newton convergence failures    */
    long ncfl;    /* linear convergence failures    */
    long netf;    /* error test failures            */
    long npred;   /* steps that used the learned iterate */
    int  last_order;
    double last_h;
    double t;
    long nsync;   /* host waits on the device during the call      */
} fvm_stats;

void fvm_opts_default(fvm_opts* o);

/* One accepted BDF step of the last integration on a context: its end
 * time, step size, order, local error test value (<= 1 accepts), the host
 * wall-clock seconds since the integration started when the step was
 * accepted, the attempts it took (error-test or corrector failures + 1)
 * and the Newton iterations, Krylov iterations and preconditioner set-ups
 * spent on it, and whether the corrector started from the learned iterate.
 * The reference prints the same counters in aggregate
 * (fvmpor_ODE.cpp:35-61). */
typedef struct {
    double t, h, err, wall;
    int order, attempts, nni, nli, npe, learned;
} fvm_step_record;

/* Copies up to cap records of the last fvm_integrate* call into out and
 * returns how many that call produced. */
long fvm_step_trace(const fvm_ctx* ctx, fvm_step_record* out, long cap);

/* Integrate from (t0, y0) to t_end.  y0 / y_end are HOST buffers; the
 * solve itself runs on the device.  Returns 0 on success. */
int fvm_integrate_host(fvm_ctx* ctx, const fvm_opts* opts, double t0,
                       double t_end, const double* y0_host,
                       double* y_end_host, fvm_stats* stats);

/* Same, with y0/y_end device pointers. */
int fvm_integrate(fvm_ctx* ctx, const fvm_opts* opts, double t0,
                  double t_end, const double* y0, double* y_end,
                  fvm_stats* stats);

/* Integrate from (t0, y0) through the n_out output times t_out_host
 * (ascending, all after t0) as IDAIntegrator::advance(next_time) does
 * (ida_integrator.h:325-340): whole BDF steps with no stop time, none
 * shortened to land on an output time, then the head and its time
 * derivative at each output time from the interpolating polynomial of the
 * step that reached it (IDAGetDky orders 0 and 1).  y_out and yp_out are
 * device buffers of n_out * N doubles, output i at offset i * N; yp_out may
 * be NULL.  The run ends with the step that passes the last output time
 * (stats->t).  Returns 0 on success, 1 when opts->max_steps ended the run
 * first (outputs after stats->t are then not written), < 0 on failure. */
int fvm_integrate_outputs(fvm_ctx* ctx, const fvm_opts* opts, double t0,
                          const double* y0, int n_out,
                          const double* t_out_host, double* y_out,
                          double* yp_out, fvm_stats* stats);

/* Replays a given sequence of accepted steps: step i has size steps[i].h
 * and order steps[i].order (the other fields are ignored), from (t0, y0),
 * with the history started as the adaptive integrator starts it (phi_1 =
 * h0 y'0, y'0 from the initial residual).  No error test and no step-size or
 * order choice: each corrector is solved until ||delta||_wrms <= newton_tol
 * (error weights from opts->rtol, opts->atol), at most max_newton updates,
 * with GMRES(opts->krylov_dim) at 0.05 newton_tol in opts->precision.  Run
 * on the trace of an adaptive integration (fvm_step_trace), it removes the
 * step-size decisions from a comparison of two implementations, so that
 * their states agree to the corrector tolerance rather than to rtol.  With
 * opts->use_predictor set, every replayed step first tries the learned
 * Newton iterate (kept when its residual test passes; stats->npred counts
 * the kept ones, the trace marks them), so that replays with and without it
 * measure the work it saves at one corrector tolerance.  The
 * orders may rise by at most one per step.  y0, y_end are device pointers.
 * Returns 0, 1 when some corrector stopped at max_newton (the run still
 * completes), < 0 on failure.  No counterpart in the reference: IDAS has no
 * replay mode (the step loop it replaces is ida_integrator.h:296-321). */
/* Gram-Schmidt of the fused GMRES cycle (fvm_opts.krylov_operator = 1):
 * 1 (the default) delayed reorthogonalisation, one reduction and two passes
 * over the basis per Arnoldi step; 0 classical Gram-Schmidt with
 * reorthogonalisation, two reductions and four passes.  The same Krylov
 * space; decomp/gmres.c:412-511 orthogonalises by modified Gram-Schmidt. */
int fvm_set_krylov_variant(fvm_ctx* ctx, int variant);

/* CUDA-graph batches of the Arnoldi loop run on this context so far
 * (fvm_opts.graph): graphs captured and batches replayed from them.  Either
 * pointer may be NULL. */
int fvm_graph_counters(fvm_ctx* ctx, long* captures, long* replays);

/* Independent problems, one context each (for example the members of an
 * ensemble, each with its own mesh and Ks field), integrated from t0 to
 * t_end with one step-size and order sequence per member: n_threads host
 * threads take the contexts in turn, and the members' kernels overlap on
 * the device through their own streams.  y0[i], y_end[i] are device
 * vectors of context i; stats (may be NULL) and status have n entries;
 * status[i] is what fvm_integrate would return for member i, and a member
 * that fails stops alone.  Returns 0 when every member reached t_end, 1
 * when some did not (the first failure in fvm_last_error()), < 0 on a bad
 * call.  The reference runs one mesh per process
 * (examples/fvmporMinlin/fvmpor_ODE.cpp:75-266). */
int fvm_integrate_batch(fvm_ctx* const* ctxs, int n, const fvm_opts* opts,
                        double t0, double t_end, const double* const* y0,
                        double* const* y_end, fvm_stats* stats, int* status,
                        int n_threads);

int fvm_integrate_replay(fvm_ctx* ctx, const fvm_opts* opts, double t0,
                         const double* y0, double h0, long n_steps,
                         const fvm_step_record* steps, double newton_tol,
                         int max_newton, double* y_end, fvm_stats* stats);

/* ------------------------------------------------------------------ */
/* Learned Newton initial iterate (no counterpart in the reference:     */
/* IDAS always starts Newton from its BDF predictor).  A per-node MLP    */
/* 8 -> 64 -> 64 -> 64 -> 1 (GELU), BF16 weights, FP32 accumulation on   */
/* tcgen05 tensor cores, proposes y_pred + (rtol|h|+atol) * MLP(x) with  */
/* x = (h_n, h_n - h_{n-1}, y_pred - h_n, log10 dt, ln K, z, CV area, 0);*/
/* the integrator keeps it only when its residual norm is below the BDF  */
/* predictor's (opts.use_predictor = 1).                                 */
/* ------------------------------------------------------------------ */
int fvm_mlp_nparams(void);   /* packed FP32 parameters: W1 b1 W2 b2 W3 b3
                                w4 b4, then 8 feature means, 8 scales */
int fvm_mlp_set_params(fvm_ctx* ctx, const float* params_host);
int fvm_mlp_get_params(fvm_ctx* ctx, float* params_host);
/* out[i] = MLP(X[i]) for n rows of raw features X[n][8] (device).      */
int fvm_mlp_forward(fvm_ctx* ctx, const float* X, int n, float* out);
/* Full-batch gradient of mean((MLP(X) - Y)^2) over the trainable
 * parameters (host buffer of fvm_mlp_nparams() - 16) and the loss.      */
int fvm_mlp_grad(fvm_ctx* ctx, const float* X, const float* Y, int n,
                 float* grad_host, float* loss);
/* Adam on (X, Y) in consecutive mini-batches of `batch` rows (0 = 148 x
 * 256); loss_history_host gets the mean loss of each epoch.             */
int fvm_mlp_train(fvm_ctx* ctx, const float* X, const float* Y, int n,
                  int epochs, int batch, float lr, float* loss_history_host);
/* fvm_integrate that also records training pairs: the features of every
 * stride-th node (offset rotating per step) at the BDF predictor and the
 * target (y_{n+1} - y_pred) / (rtol |h_n| + atol) of each accepted step,
 * into device buffers X[capacity][8], Y[capacity]; *count gets the rows
 * written. */
int fvm_integrate_record(fvm_ctx* ctx, const fvm_opts* opts, double t0,
                         double t_end, const double* y0, double* y_end,
                         fvm_stats* stats, float* X, float* Y, long capacity,
                         int stride, long* count);

/* ------------------------------------------------------------------ */
/* Synthetic problem generators (host).  The reference reads gmsh-made   */
/* .pmesh files (meshing/genMesh.sh, decomp/split.c:459-500); these      */
/* build the benchmark meshes directly.  Arrays are malloc'd by the      */
/* library and released with fvm_problem_free.                           */
/* ------------------------------------------------------------------ */
typedef struct {
    fvm_mesh mesh;
    fvm_physics phys;
    double water_table;      /* initial hydrostatic level                  */
    double t_end;            /* simulated horizon [s]                      */
    /* owned storage */
    double* coords; int* elem_nodes; int* elem_zone; double* elem_K;
    int* bface_nodes; int* bface_elem; int* bface_tag; int* node_tag;
    fvm_zone* zones; fvm_bc* bcs;
    int* grid_dims;          /* [3] structured node grid extents           */
} fvm_problem;

/* 2D Richards infiltration: nx*ny node grid over Lx*Ly, Delaunay of the
 * jittered grid, two soil layers, Dirichlet strip on top. */
int fvm_problem_richards2d(int nx, int ny, double Lx, double Ly,
                           double jitter, uint64_t seed,
                           double ln_var, double corr_len,
                           fvm_problem* out);
/* 3D Richards: nx*ny*nz hex cells split into 6 tets, lognormal Ks. */
int fvm_problem_richards3d(int nx, int ny, int nz, double Lx, double Ly,
                           double Lz, double jitter, uint64_t seed,
                           double ln_var, double cx, double cy, double cz,
                           double Kg, fvm_problem* out);
/* Ensemble: n_members independent 2D problems (node counts uniform in
 * [nmin, nmax], each with its own jitter and lognormal Ks field: ln-variance
 * uniform in [0.5, 2], correlation length uniform in [0.5, 3] m) as one
 * disjoint mesh; member m owns nodes [member_ptr[m], member_ptr[m+1])
 * (member_ptr has n_members + 1 entries, caller-allocated). */
int fvm_problem_ensemble2d(int n_members, int nmin, int nmax, uint64_t seed,
                           fvm_problem* out, int* member_ptr);
void fvm_problem_free(fvm_problem* p);

/* ------------------------------------------------------------------ */
/* Mesh files and output.                                               */
/* ------------------------------------------------------------------ */
/* A .pmesh mesh (the text format Mesh::read_mesh_data parses,
 * src/fvm/mesh.cpp:102-366) of triangles or tetrahedra, single domain.
 * elem_tag is the file's physical tag minus 100 (mesh.cpp:288), the index
 * of the element's zone.  Boundary faces are the element faces with a
 * non-zero boundary id, in element order.  Node boundary tags are kept as
 * CSR (node_bc_ptr[n_nodes + 1], node_bc).  With FVM_PMESH_RCM the nodes
 * are renumbered by reverse Cuthill-McKee as Mesh::reorder_nodes_edges does
 * (mesh.cpp:116-148); perm[new] = the node's index in the file.  Arrays
 * are malloc'd by the library and released with fvm_pmesh_free. */
#define FVM_PMESH_RCM 1
typedef struct {
    int n_dom, dom_id;       /* header: domain count and this domain's id  */
    int dim;                 /* 2 triangles, 3 tetrahedra                  */
    int n_nodes, n_elements, n_bfaces;
    double* coords;          /* [n_nodes][3]                               */
    int* elem_nodes;         /* [n_elements][dim+1]                        */
    int* elem_tag;           /* [n_elements]                               */
    int* bface_nodes;        /* [n_bfaces][dim]                            */
    int* bface_elem;         /* [n_bfaces]                                 */
    int* bface_tag;          /* [n_bfaces], > 0                            */
    int* node_bc_ptr;        /* [n_nodes + 1]                              */
    int* node_bc;            /* node boundary tags                         */
    int* perm;               /* [n_nodes] new -> file node index           */
    int bandwidth_file;      /* node-graph bandwidth in file order         */
    int bandwidth;           /* ... in the returned order                  */
} fvm_pmesh;

/* 0 ok; -1 I/O, -2 malformed file (fvm_last_error gives file:line),
 * -3 halo nodes (multi-domain file), -4 element type other than triangle
 * or tetrahedron.  Replaces Mesh::Mesh's file reading (mesh.cpp:70-80). */
int fvm_pmesh_read(const char* path, int flags, fvm_pmesh* out);
/* writes m as a one-domain .pmesh (node_bc_ptr may be NULL: no tags) */
int fvm_pmesh_write(const char* path, const fvm_pmesh* m);
void fvm_pmesh_free(fvm_pmesh* m);
/* A problem on a .pmesh mesh: element zone = elem_tag (0 <= tag < n_zones,
 * as physical_zone() asserts, fvmpor.h:1128-1132); node_tag = the node's
 * last boundary tag whose condition is Dirichlet (types 1, 4), as
 * VarSatPhysicsImpl::initialise_vectors sets is_dirichlet_h_vec_
 * (fvmpor.h:405-417).  Every boundary-face tag must have a condition.
 * Release with fvm_problem_free. */
int fvm_problem_from_pmesh(const fvm_pmesh* m, int n_zones, const fvm_zone* zones,
                           int n_bcs, const fvm_bc* bcs, double rho0,
                           fvm_problem* out);

/* VTK XML output of a head field (host array, n_nodes values) as
 * <stem>_dom<rank>_<step>.vtu and, from rank 0, the header
 * <stem>_head_<step>.pvtu naming n_ranks pieces: the files
 * util::Solution::write_timestep_VTK_XML writes (include/util/solution.h:
 * 175-357). */
int fvm_write_vtu(const char* stem, int step, int rank, int n_ranks,
                  const fvm_mesh* mesh, const double* head);

#ifdef __cplusplus
}
#endif
#endif /* FVMPOR_B200_H */
