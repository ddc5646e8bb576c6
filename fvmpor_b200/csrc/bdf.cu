// Device operations for the BDF controller (bdf_controller.hpp) and the
// fvm_integrate entry points: the time loop of examples/fvmporMinlin/
// fvmpor_ODE.cpp:202-232 and IDAIntegrator::advance(t)
// (include/fvm/integrators/ida_integrator.h:325-340) with the solver state
// resident in HBM.  Initial y' = F(t0, y0, 0) / ahh on free rows
// (Physics::initialise, examples/fvmporMinlin/fvmpor_ODE_impl.cpp:34-58).
#include "bdf_controller.hpp"
#include "ctx.cuh"
#include "krylov.cuh"
#include "predictor.cuh"
#include "reduce.cuh"

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstring>
#include <limits>
#include <thread>
#include <vector>

namespace fvmb {

constexpr int kNPhi = 7;

struct PhiPtrs {
    double* p[kNPhi];
};
struct Coef7 {
    double v[kNPhi];
};

__global__ void k_ewt(int N, const double* __restrict__ y, double rtol, double atol,
                      double* __restrict__ ewt) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < N) ewt[i] = 1.0 / (rtol * fabs(y[i]) + atol);
}

// y = sum_{j<=k} phi_j ; yp = sum_{1<=j<=k} gamma_j phi_j ; e = 0
__global__ void k_predict(int N, int k, PhiPtrs ph, Coef7 gamma, double* __restrict__ y,
                          double* __restrict__ yp, double* __restrict__ e) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N) return;
    double s = ph.p[0][i], sp = 0.0;
    for (int j = 1; j <= k; ++j) {
        double v = ph.p[j][i];
        s += v;
        sp += gamma.v[j] * v;
    }
    y[i] = s;
    yp[i] = sp;
    e[i] = 0.0;
}

// dense output: y = sum_{j<=k} c_j phi_j ; yp = sum_{1<=j<=k} d_j phi_j
// (yp may be null)
__global__ void k_interp(int N, int k, PhiPtrs ph, Coef7 c, Coef7 d, double* __restrict__ y,
                         double* __restrict__ yp) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N) return;
    double s = ph.p[0][i], sp = 0.0;
    for (int j = 1; j <= k; ++j) {
        const double v = ph.p[j][i];
        s += c.v[j] * v;
        sp += d.v[j] * v;
    }
    y[i] = s;
    if (yp) yp[i] = sp;
}

__global__ void k_phi_scale(int N, int j0, int j1, PhiPtrs ph, Coef7 f) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N) return;
    for (int j = j0; j <= j1; ++j) ph.p[j][i] *= f.v[j];
}

// y -= x, y' -= cj x, e -= x ; out = sum (x ewt)^2
__global__ void k_newton_update(int N, const double* __restrict__ x, double cj,
                                const double* __restrict__ ewt, double* __restrict__ y,
                                double* __restrict__ yp, double* __restrict__ e, double* partial,
                                unsigned* counter, double* out) {
    double s = 0.0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < N; i += gridDim.x * blockDim.x) {
        double d = x[i];
        y[i] -= d;
        yp[i] -= cj * d;
        e[i] -= d;
        double w = d * ewt[i];
        s += w * w;
    }
    double t = block_sum(s);
    if (threadIdx.x == 0) partial[blockIdx.x] = t;
    last_block_reduce(partial, 1, counter, out);
}

// out = sum (y ewt)^2: the predictor's squared WRMS norm times N
__global__ void k_pred_sumsq(int N, const double* __restrict__ y, const double* __restrict__ ewt, double* partial,
                             unsigned* counter, double* out) {
    double s = 0.0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < N; i += gridDim.x * blockDim.x) {
        const double w = y[i] * ewt[i];
        s += w * w;
    }
    double t = block_sum(s);
    if (threadIdx.x == 0) partial[blockIdx.x] = t;
    last_block_reduce(partial, 1, counter, out);
}

// squared error-test norms times N:
//  0: e  1: phi_k + e  2: phi_{k-1} + phi_k + e  3: e - phi_{k+1}
__global__ void k_err_norms(int N, int k, PhiPtrs ph, const double* __restrict__ e,
                            const double* __restrict__ ewt, double* partial, unsigned* counter,
                            double* out) {
    double s0 = 0, s1 = 0, s2 = 0, s3 = 0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < N; i += gridDim.x * blockDim.x) {
        double w = ewt[i], ei = e[i];
        double a = ei * w;
        s0 += a * a;
        double d1 = ph.p[k][i] + ei;
        double b = d1 * w;
        s1 += b * b;
        if (k >= 2) {
            double d2 = ph.p[k - 1][i] + d1;
            double c2 = d2 * w;
            s2 += c2 * c2;
        }
        if (k + 1 < kNPhi) {
            double d3 = ei - ph.p[k + 1][i];
            double c3 = d3 * w;
            s3 += c3 * c3;
        }
    }
    double t0 = block_sum(s0);
    double t1 = block_sum(s1);
    double t2 = block_sum(s2);
    double t3 = block_sum(s3);
    if (threadIdx.x == 0) {
        partial[4 * blockIdx.x + 0] = t0;
        partial[4 * blockIdx.x + 1] = t1;
        partial[4 * blockIdx.x + 2] = t2;
        partial[4 * blockIdx.x + 3] = t3;
    }
    last_block_reduce(partial, 4, counter, out);
}

// Ensemble versions (one block per member, member m = nodes [mp[m],
// mp[m+1])): the same updates, with the squared norms summed per member in a
// fixed order into out[m * nq + q].
__global__ void k_newton_update_seg(const int* __restrict__ mp, const double* __restrict__ x, double cj,
                                    const double* __restrict__ ewt, double* __restrict__ y,
                                    double* __restrict__ yp, double* __restrict__ e, double* out) {
    const int m = blockIdx.x;
    double s = 0.0;
    for (int i = mp[m] + threadIdx.x; i < mp[m + 1]; i += blockDim.x) {
        double d = x[i];
        y[i] -= d;
        yp[i] -= cj * d;
        e[i] -= d;
        double w = d * ewt[i];
        s += w * w;
    }
    double t = block_sum(s);
    if (threadIdx.x == 0) out[m] = t;
}

__global__ void k_err_norms_seg(const int* __restrict__ mp, int k, PhiPtrs ph, const double* __restrict__ e,
                                const double* __restrict__ ewt, double* out) {
    const int m = blockIdx.x;
    double s0 = 0, s1 = 0, s2 = 0, s3 = 0;
    for (int i = mp[m] + threadIdx.x; i < mp[m + 1]; i += blockDim.x) {
        double w = ewt[i], ei = e[i];
        double a = ei * w;
        s0 += a * a;
        double d1 = ph.p[k][i] + ei;
        double b = d1 * w;
        s1 += b * b;
        if (k >= 2) {
            double d2 = ph.p[k - 1][i] + d1;
            double c2 = d2 * w;
            s2 += c2 * c2;
        }
        if (k + 1 < kNPhi) {
            double d3 = ei - ph.p[k + 1][i];
            double c3 = d3 * w;
            s3 += c3 * c3;
        }
    }
    double t0 = block_sum(s0);
    double t1 = block_sum(s1);
    double t2 = block_sum(s2);
    double t3 = block_sum(s3);
    if (threadIdx.x == 0) {
        out[4 * m + 0] = t0;
        out[4 * m + 1] = t1;
        out[4 * m + 2] = t2;
        out[4 * m + 3] = t3;
    }
}

__global__ void k_sumsq_seg(const int* __restrict__ mp, const double* __restrict__ x,
                            const double* __restrict__ w, double* out) {
    const int m = blockIdx.x;
    double s = 0.0;
    for (int i = mp[m] + threadIdx.x; i < mp[m + 1]; i += blockDim.x) {
        double v = x[i] * w[i];
        s += v * v;
    }
    double t = block_sum(s);
    if (threadIdx.x == 0) out[m] = t;
}

// phi_{k+1} = e (set_kp2), phi_k += e, phi_j += phi_{j+1} for j = k-1..0
__global__ void k_phi_update(int N, int k, int set_kp2, PhiPtrs ph, const double* __restrict__ e) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N) return;
    double ei = e[i];
    if (set_kp2) ph.p[k + 1][i] = ei;
    double v = ph.p[k][i] + ei;
    ph.p[k][i] = v;
    for (int j = k - 1; j >= 0; --j) {
        v = ph.p[j][i] + v;
        ph.p[j][i] = v;
    }
}

// y'0 = F / ahh on free rows with ahh != 0, else 0
__global__ void k_initial_yp(int N, const double* __restrict__ F, const double* __restrict__ ahh,
                             const unsigned char* __restrict__ ntype, double* __restrict__ yp) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N) return;
    double a = ahh[i];
    yp[i] = (!ntype[i] && a != 0.0) ? F[i] / a : 0.0;
}

__global__ void k_fill(int N, double v, double* __restrict__ x) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < N) x[i] = v;
}

__global__ void k_scale_vec(int N, double a, const double* __restrict__ x, double* __restrict__ y) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < N) y[i] = a * x[i];
}

} // namespace fvmb

// The integrator's vectors, kept by the context from its first integration
// on, so that an integration allocates and frees nothing (cudaFree and
// cudaFreeHost synchronise the device and occasionally stall for a
// fraction of a second on a busy host).
struct fvmb::IntegWork {
    DevBuf<double> phi[kNPhi];
    DevBuf<double> y, yp, e, ewt, F, x, tmp;
    DevBuf<double> partial, res;
    DevBuf<unsigned> counter;
    DevBuf<double> ypred, yppred, hprev;
    DevBuf<float> feat;
    DevBuf<double> host_in, host_out;   // device copies for fvm_integrate_host
    double* host = nullptr;             // pinned
    size_t host_n = 0;
    ~IntegWork() {
        if (host) cudaFreeHost(host);
    }
};

void fvmb_destroy_integ_work(fvmb::IntegWork* w) { delete w; }

namespace fvmb {

static IntegWork& integ_work(fvm_ctx* c) {
    if (!c->work) c->work = new IntegWork();
    IntegWork& w = *c->work;
    const int N = c->N;
    for (int j = 0; j < kNPhi; ++j) w.phi[j].alloc(N);
    w.y.alloc(N); w.yp.alloc(N); w.e.alloc(N); w.ewt.alloc(N); w.F.alloc(N); w.x.alloc(N); w.tmp.alloc(N);
    w.partial.alloc((size_t)kRedBlocks * 4);
    // reduction results: Newton norms [0, nm), error norms [nm, 5 nm), the
    // predictor's norm at 5 nm (fetched together, one host wait)
    const size_t nh = (size_t)(5 * std::max(1, c->n_members) + 8);
    w.res.alloc(nh);
    w.counter.alloc(1);
    if (w.host_n < nh) {
        if (w.host) FVM_CUDA(cudaFreeHost(w.host));
        w.host = nullptr;
        FVM_CUDA(cudaMallocHost(&w.host, sizeof(double) * nh));
        w.host_n = nh;
    }
    return w;
}

struct DeviceOps {
    fvm_ctx* c;
    const fvm_opts& o;
    int N;
    IntegWork& w;
    DevBuf<double> (&phi)[kNPhi];
    DevBuf<double> &y, &yp, &e, &ewt, &F, &x, &tmp;
    DevBuf<double> &partial, &res;
    DevBuf<unsigned>& counter;
    double* host;
    double tcur = 0.0, hcur = 0.0;
    Predictor* pred = nullptr;     // learned Newton iterate (optional)
    Recorder* rec = nullptr;       // training-set recorder (optional)
    DevBuf<double> &ypred, &yppred, &hprev;
    DevBuf<float>& feat;
    bool f_fresh = false;          // F already holds F(t, y, y')
    bool forked = false;           // residual() recorded the set-up's fork point

    int nm = 1;                    // ensemble members (per-member norms when > 1)
    // Krylov tolerance factor of an ensemble: GMRES stops on the RMS over
    // all nodes, so it runs to tol * sqrt(N_min / N), which bounds every
    // member's own RMS by tol (N_m rms_m^2 <= N rms^2); with the plain
    // global tolerance the smallest members' Newton updates were up to
    // sqrt(N / N_min) times less accurate than their own Newton test
    // needs, and their correctors failed until the step size collapsed
    double tol_scale = 1.0;
    // One host wait per Newton iteration: predict() queues the predictor's
    // norm, newton_update() queues its own norm and, speculatively, the
    // error norms the step's test needs if this update converges; one fetch
    // brings all three.  psetup() does not wait for the pivot status either:
    // gmres() reads it after its own wait.
    int korder = 1;                // order of the step being solved (set_order)
    double pn = 0.0;               // WRMS norm of this attempt's predictor
    bool err_ready = false;        // err_cache holds the norms for (korder, e)
    double err_cache[4] = {};

    DeviceOps(fvm_ctx* ctx, const fvm_opts& opts)
        : c(ctx), o(opts), N(ctx->N), w(integ_work(ctx)), phi(w.phi), y(w.y), yp(w.yp), e(w.e), ewt(w.ewt),
          F(w.F), x(w.x), tmp(w.tmp), partial(w.partial), res(w.res), counter(w.counter), host(w.host),
          ypred(w.ypred), yppred(w.yppred), hprev(w.hprev), feat(w.feat) {
        for (int j = 0; j < kNPhi; ++j) phi[j].zero(c->stream);
        nm = c->n_members;
        if (nm > 1) {
            int nmin = N;
            for (int m = 0; m < nm; ++m) nmin = std::min(nmin, c->h_member_ptr[m + 1] - c->h_member_ptr[m]);
            tol_scale = std::sqrt((double)std::max(nmin, 1) / N);
        }
        counter.zero(c->stream);
        c->use_graph = o.graph != 0;
    }
    ~DeviceOps() { c->use_graph = false; }
    DeviceOps(const DeviceOps&) = delete;
    DeviceOps& operator=(const DeviceOps&) = delete;
    // largest per-member WRMS norm from per-member squared sums
    // host[off + m*nq + q]
    double member_max_at(size_t off, int nq, int q) const {
        double best = 0.0;
        for (int m = 0; m < nm; ++m) {
            const int nmem = c->h_member_ptr[m + 1] - c->h_member_ptr[m];
            if (nmem > 0) best = std::max(best, std::sqrt(host[off + (size_t)m * nq + q] / nmem));
        }
        return best;
    }
    double member_max(int nq, int q) const { return member_max_at(0, nq, q); }
    int g() const { return grid_for(N, 256); }
    PhiPtrs ptrs() const {
        PhiPtrs p;
        for (int j = 0; j < kNPhi; ++j) p.p[j] = phi[j].p;
        return p;
    }
    double fetch(int n) {
        FVM_CUDA(cudaMemcpyAsync(host, res.p, sizeof(double) * n, cudaMemcpyDeviceToHost, c->stream));
        ctx_sync(c);
        return host[0];
    }
    size_t pn_slot() const { return 5 * (size_t)std::max(1, nm); }

    // ---- controller interface
    void set_time(double t) { tcur = t; }
    void ewt_from_phi0(double rtol, double atol) {
        fvm_launch(c, k_ewt, g(), 256, 0, c->stream, N, phi[0].p, rtol, atol, ewt.p);
    }
    void begin_step() { launch_begin_step(c, phi[0].p, yp.p); }
    void phi_scale(int j0, int j1, const double* f) {
        Coef7 cf;
        for (int j = 0; j < kNPhi; ++j) cf.v[j] = f[j];
        fvm_launch(c, k_phi_scale, g(), 256, 0, c->stream, N, j0, j1, ptrs(), cf);
    }
    void predict(int k, const double* gamma, double h) {
        Coef7 gm;
        for (int j = 0; j < kNPhi; ++j) gm.v[j] = gamma[j];
        fvm_launch(c, k_predict, g(), 256, 0, c->stream, N, k, ptrs(), gm, y.p, yp.p, e.p);
        fvm_launch(c, k_pred_sumsq, kRedBlocks, kRedThreads, 0, c->stream, N, y.p, ewt.p, partial.p, counter.p,
                   res.p + pn_slot());
        err_ready = false;
        f_fresh = false;
        hcur = h;
        if (pred || rec) {
            // keep the BDF predictor and the learned-iterate features
            FVM_CUDA(cudaMemcpyAsync(ypred.p, y.p, sizeof(double) * N, cudaMemcpyDeviceToDevice, c->stream));
            FVM_CUDA(cudaMemcpyAsync(yppred.p, yp.p, sizeof(double) * N, cudaMemcpyDeviceToDevice, c->stream));
            predictor_features(c, phi[0].p, hprev.p, ypred.p, h, feat.p);
        }
    }
    // the predictor's WRMS norm, as fetched by the attempt's first
    // newton_update (the only place the controller reads it)
    double pred_norm() const { return pn; }
    void set_order(int k) { korder = k; err_ready = false; }
    void residual() {
        // a set-up that follows reads only what is queued up to here (y, y',
        // ewt, the begin-step flags; not F): it may start from this point
        if (!c->ev_fork) {
            FVM_CUDA(cudaStreamCreate(&c->stream2));   // blocking, as the context's stream
            FVM_CUDA(cudaEventCreateWithFlags(&c->ev_fork, cudaEventDisableTiming));
            FVM_CUDA(cudaEventCreateWithFlags(&c->ev_join, cudaEventDisableTiming));
        }
        FVM_CUDA(cudaEventRecord(c->ev_fork, c->stream));
        forked = true;
        if (f_fresh) {   // the learned-iterate check already evaluated it
            f_fresh = false;
            return;
        }
        Perturb none;
        launch_residual(c, y.p, yp.p, none, nullptr, F.p);
    }
    void enable_learning(Predictor* p, Recorder* r) {
        pred = p;
        rec = r;
        if (pred || rec) {
            ypred.alloc(N);
            yppred.alloc(N);
            hprev.alloc(N);
            feat.alloc((size_t)N * 8);
        }
    }
    // the pivot status is copied behind the factorisation and read by
    // gmres() after its wait (status 3 there)
    int psetup(double cj, double h) {
        // (with the per-category timers on, everything stays on one stream so
        // that each category's events bracket its own kernels only)
        if (!forked || c->tm.on) {
            forked = false;
            psetup_dev(c, cj, h, y.p, yp.p, F.p, ewt.p, o.precision);
            return 0;
        }
        // the set-up (difference quotients and factorisation) runs on the
        // second stream beside the residual evaluation queued since the fork;
        // the context's stream waits for it before the Krylov solve
        forked = false;
        FVM_CUDA(cudaStreamWaitEvent(c->stream2, c->ev_fork, 0));
        cudaStream_t s0 = c->stream;
        c->stream = c->stream2;
        try {
            psetup_dev(c, cj, h, y.p, yp.p, F.p, ewt.p, o.precision);
        } catch (...) {
            c->stream = s0;
            throw;
        }
        c->stream = s0;
        FVM_CUDA(cudaEventRecord(c->ev_join, c->stream2));
        FVM_CUDA(cudaStreamWaitEvent(c->stream, c->ev_join, 0));
        return 0;
    }
    int gmres(double cj, double tol, int* its, double* rn, long* nps, long* njv) {
        GmresCounters gc;
        // the Newton update reads x next on the same stream: no wait here
        int r = gmres_dev(c, cj, y.p, yp.p, F.p, ewt.p, F.p, x.p, o.krylov_dim, o.max_restarts,
                          o.precision, tol * tol_scale, its, rn, &gc, o.krylov_operator, false);
        *nps = gc.nps;
        *njv = gc.njv;
        if (ilu_status_seen(c)) return 3;   // zero pivot in the factor this solve used
        return r;
    }
    double newton_update(double cj) {
        const size_t ps = pn_slot();
        if (nm > 1) {
            fvm_launch(c, k_newton_update_seg, nm, 256, 0, c->stream, c->member_ptr.p, x.p, cj, ewt.p, y.p, yp.p,
                       e.p, res.p);
            fvm_launch(c, k_err_norms_seg, nm, 256, 0, c->stream, c->member_ptr.p, korder, ptrs(), e.p, ewt.p,
                       res.p + nm);
            fetch((int)ps + 1);
            for (int q = 0; q < 4; ++q) err_cache[q] = member_max_at(nm, 4, q);
            err_ready = true;
            pn = std::sqrt(host[ps] / N);
            return member_max(1, 0);
        }
        fvm_launch(c, k_newton_update, kRedBlocks, kRedThreads, 0, c->stream, N, x.p, cj, ewt.p, y.p, yp.p, e.p,
                                                                   partial.p, counter.p, res.p);
        fvm_launch(c, k_err_norms, kRedBlocks, kRedThreads, 0, c->stream, N, korder, ptrs(), e.p, ewt.p, partial.p,
                                                               counter.p, res.p + 1);
        const double d = fetch((int)ps + 1);
        for (int q = 0; q < 4; ++q) err_cache[q] = std::sqrt(host[1 + q] / N);
        err_ready = true;
        pn = std::sqrt(host[ps] / N);
        return std::sqrt(d / N);
    }
    void err_norms(int k, double out[4]) {
        if (err_ready && k == korder) {
            for (int q = 0; q < 4; ++q) out[q] = err_cache[q];
            return;
        }
        if (nm > 1) {
            fvm_launch(c, k_err_norms_seg, nm, 256, 0, c->stream, c->member_ptr.p, k, ptrs(), e.p, ewt.p, res.p);
            fetch(4 * nm);
            for (int q = 0; q < 4; ++q) out[q] = member_max(4, q);
            return;
        }
        fvm_launch(c, k_err_norms, kRedBlocks, kRedThreads, 0, c->stream, N, k, ptrs(), e.p, ewt.p, partial.p,
                                                               counter.p, res.p);
        fetch(4);
        for (int q = 0; q < 4; ++q) out[q] = std::sqrt(host[q] / N);
    }
    // head and time derivative at tq from the last accepted step's
    // interpolating polynomial (coefficients from the controller)
    void interpolate(int k, const double* cf, const double* df, double* yo, double* ypo) {
        Coef7 cc, dd;
        for (int j = 0; j < kNPhi; ++j) { cc.v[j] = cf[j]; dd.v[j] = df[j]; }
        fvm_launch(c, k_interp, g(), 256, 0, c->stream, N, k, ptrs(), cc, dd, yo, ypo);
    }
    void phi_update(int k, int set_kp2) {
        if (pred || rec) {
            // the accepted corrector y against the predictor (training
            // target), then h_{n-1} <- h_n before phi_0 advances
            if (rec) recorder_push(c, rec, feat.p, y.p, ypred.p, phi[0].p, o.rtol, o.atol);
            FVM_CUDA(cudaMemcpyAsync(hprev.p, phi[0].p, sizeof(double) * N, cudaMemcpyDeviceToDevice, c->stream));
        }
        fvm_launch(c, k_phi_update, g(), 256, 0, c->stream, N, k, set_kp2, ptrs(), e.p);
    }
    // The learned iterate costs a network evaluation and one or two residual
    // evaluations per attempt.  After a run of attempts that the residual
    // test rejected, the next 2, 4, ... 32 steps use the BDF predictor
    // without trying, so an unhelpful network costs little; one accepted
    // attempt resets the back-off.
    int guess_fails = 0, guess_skip = 0;
    bool newton_guess(double tnew, double h, double cj) {
        (void)tnew;
        if (!pred) return false;
        if (guess_skip > 0) {
            --guess_skip;
            return false;
        }
        bool kept = predictor_apply(c, pred, o.rtol, o.atol, h, cj, phi[0].p, hprev.p, ypred.p, yppred.p, y.p,
                                    yp.p, e.p, F.p);
        f_fresh = true;   // F holds the residual of whichever iterate was kept
        if (kept) {
            guess_fails = 0;
        } else {
            guess_fails = std::min(guess_fails + 1, 5);
            guess_skip = (1 << guess_fails) - 1;
        }
        return kept;
    }

    // y0 -> phi_0, y'0 from the initial residual, phi_1 = h y'0
    double start(double t0, const double* y0, double tout) {
        cudaStream_t s = c->stream;
        FVM_CUDA(cudaMemcpyAsync(y.p, y0, sizeof(double) * N, cudaMemcpyDeviceToDevice, s));
        reset_upwind(c);   // averaged weights for the initial residual
        fvm_launch(c, k_fill, g(), 256, 0, s, N, 0.0, yp.p);
        Perturb none;
        launch_residual(c, y.p, yp.p, none, nullptr, F.p);
        fvm_launch(c, k_fill, g(), 256, 0, s, N, 1.0, tmp.p);
        launch_residual(c, y.p, tmp.p, none, nullptr, x.p);   // leaves ahh * 1 in c->stor
        fvm_launch(c, k_initial_yp, g(), 256, 0, s, N, F.p, c->stor.p, c->ntype.p, yp.p);
        fvm_launch(c, k_ewt, g(), 256, 0, s, N, y.p, o.rtol, o.atol, ewt.p);
        double ypn;
        if (nm > 1) {
            fvm_launch(c, k_sumsq_seg, nm, 256, 0, s, c->member_ptr.p, yp.p, ewt.p, res.p);
            fetch(nm);
            ypn = member_max(1, 0);
        } else {
            ypn = std::sqrt(reduce_sumsq(c, yp.p, ewt.p) / N);
        }
        double h = bdf_first_step(t0, tout, ypn, o.h0, o.hmax);
        FVM_CUDA(cudaMemcpyAsync(phi[0].p, y.p, sizeof(double) * N, cudaMemcpyDeviceToDevice, s));
        fvm_launch(c, k_scale_vec, g(), 256, 0, s, N, h, yp.p, phi[1].p);
        if (hprev.p) FVM_CUDA(cudaMemcpyAsync(hprev.p, y.p, sizeof(double) * N, cudaMemcpyDeviceToDevice, s));
        return h;
    }
};

// requested output times of fvm_integrate_outputs and where their heads go
struct OutputTimes {
    int n = 0;
    const double* t = nullptr;
    double* y = nullptr;
    double* yp = nullptr;
    int done = 0;
};

// t_end is the last output time when out is given: the steps then run
// without a stop time and each output is interpolated from the step that
// reached it
int integrate_dev(fvm_ctx* c, const fvm_opts* opts, double t0, double t_end, const double* y0,
                  double* y_end, fvm_stats* stats, Recorder* rec = nullptr, OutputTimes* out = nullptr) {
    const fvm_opts& o = *opts;
    if (o.max_order < 1 || o.max_order > 5) throw Error("integrate: max_order must be 1..5");
    if (!(o.rtol > 0) || !(o.atol > 0)) throw Error("integrate: tolerances must be positive");
    if (!(t_end > t0)) throw Error("integrate: t_end must exceed t0");
    const long nsync0 = c->n_syncs;
    c->last_trace.clear();
    DeviceOps ops(c, o);
    Predictor* pred = nullptr;
    if (o.use_predictor) {
        pred = predictor_of(c);
        if (!pred) throw Error("integrate: use_predictor set but no trained predictor loaded");
    }
    ops.enable_learning(pred, rec);
    BdfOptions bo;
    bo.rtol = o.rtol;
    bo.atol = o.atol;
    bo.max_order = o.max_order;
    bo.hmax = o.hmax;
    bo.use_guess = o.use_predictor != 0;
    bo.guess_every_step = o.use_predictor == 2;
    if (o.eps_lin > 0.0) bo.eps_lin = o.eps_lin;
    if (o.cj_refresh > 1.0) bo.cj_refresh = o.cj_refresh;
    if (o.psetup_age > 0) bo.psetup_age = o.psetup_age;
    BdfController<DeviceOps> ctl(ops, bo);
    long nre0 = c->n_residuals;
    double h0 = ops.start(t0, y0, t_end);
    ctl.start(t0, h0);
    int rc = 0;
    const double tstop = out ? std::numeric_limits<double>::infinity() : t_end;
    while (out ? out->done < out->n : ctl.t < t_end) {
        if (o.max_steps > 0 && ctl.st.nst >= o.max_steps) { rc = 1; break; }
        rc = ctl.step(tstop);
        if (rc != 0) break;
        if (out) {
            while (out->done < out->n && out->t[out->done] <= ctl.t) {
                double cf[kNPhi], df[kNPhi];
                const int k = ctl.interp_coefs(out->t[out->done], cf, df);
                const size_t off = (size_t)out->done * c->N;
                ops.interpolate(k, cf, df, out->y + off, out->yp ? out->yp + off : nullptr);
                ++out->done;
            }
        } else if (t_end - ctl.t <= 1e-12 * std::max(1.0, std::fabs(t_end))) {
            ctl.t = t_end;
        }
    }
    if (y_end)
        FVM_CUDA(cudaMemcpyAsync(y_end, ops.phi[0].p, sizeof(double) * c->N, cudaMemcpyDeviceToDevice, c->stream));
    ctx_sync(c);
    c->last_trace.swap(ctl.trace);
    if (stats) {
        std::memset(stats, 0, sizeof(*stats));
        stats->nst = ctl.st.nst;
        stats->nre = c->n_residuals - nre0;
        stats->nni = ctl.st.nni;
        stats->nli = ctl.st.nli;
        stats->npe = ctl.st.npe;
        stats->nps = ctl.st.nps;
        stats->ncfn = ctl.st.ncfn;
        stats->ncfl = ctl.st.ncfl;
        stats->netf = ctl.st.netf;
        stats->npred = ctl.st.npred;
        stats->last_order = ctl.st.last_order;
        stats->last_h = ctl.st.last_h;
        stats->t = ctl.t;
        stats->nsync = c->n_syncs - nsync0;
    }
    return rc;
}

// Replay of a given sequence of accepted steps with tight correctors
// (fvm_integrate_replay): the controller's own coefficients and predictor,
// the step sizes and orders forced, no error test
int replay_dev(fvm_ctx* c, const fvm_opts* opts, double t0, const double* y0, double h0, long n,
               const fvm_step_record* steps, double newton_tol, int max_newton, double* y_end, fvm_stats* stats) {
    fvm_opts o = *opts;
    if (o.max_order < 1 || o.max_order > 5) throw Error("replay: max_order must be 1..5");
    if (!(o.rtol > 0) || !(o.atol > 0)) throw Error("replay: tolerances must be positive");
    if (!(h0 > 0) || !std::isfinite(h0)) throw Error("replay: h0 must be positive");
    if (!(newton_tol > 0) || max_newton < 1) throw Error("replay: newton_tol must be positive, max_newton >= 1");
    for (long i = 0; i < n; ++i) {
        const int kk = steps[i].order;
        // the order rises by at most one per step, so history exists for it
        if (!(steps[i].h > 0) || !std::isfinite(steps[i].h) || kk < 1 || kk > o.max_order ||
            kk > (i ? steps[i - 1].order + 1 : 1))
            throw Error("replay: step " + std::to_string(i) + " has a bad size or order");
    }
    o.h0 = h0;      // the first-step rule returns the given h0
    o.hmax = 0.0;
    const long nsync0 = c->n_syncs;
    c->last_trace.clear();
    DeviceOps ops(c, o);
    // with use_predictor every replayed step first tries the learned iterate
    // (kept when its residual test passes), so that two replays of one step
    // sequence, with and without it, measure the Newton and Krylov work it
    // saves at the same corrector tolerance
    Predictor* pred = nullptr;
    if (o.use_predictor) {
        pred = predictor_of(c);
        if (!pred) throw Error("replay: use_predictor set but no trained predictor loaded");
    }
    ops.enable_learning(pred, nullptr);
    BdfOptions bo;
    bo.rtol = o.rtol;
    bo.atol = o.atol;
    bo.max_order = o.max_order;
    bo.use_guess = pred != nullptr;
    BdfController<DeviceOps> ctl(ops, bo);
    const long nre0 = c->n_residuals;
    const double hs = ops.start(t0, y0, t0 + h0);
    ctl.start(t0, hs);
    int rc = 0;
    for (long i = 0; i < n; ++i) {
        const int r = bdf_replay_step(ctl, steps[i].h, steps[i].order, newton_tol, max_newton);
        if (r < 0) { rc = r; break; }
        if (r == 1) rc = 1;
    }
    if (y_end)
        FVM_CUDA(cudaMemcpyAsync(y_end, ops.phi[0].p, sizeof(double) * c->N, cudaMemcpyDeviceToDevice, c->stream));
    ctx_sync(c);
    c->last_trace.swap(ctl.trace);
    if (stats) {
        std::memset(stats, 0, sizeof(*stats));
        stats->nst = ctl.st.nst;
        stats->nre = c->n_residuals - nre0;
        stats->nni = ctl.st.nni;
        stats->nli = ctl.st.nli;
        stats->npe = ctl.st.npe;
        stats->nps = ctl.st.nps;
        stats->npred = ctl.st.npred;
        stats->last_order = ctl.st.last_order;
        stats->last_h = ctl.st.last_h;
        stats->t = ctl.t;
        stats->nsync = c->n_syncs - nsync0;
    }
    return rc;
}

} // namespace fvmb

using namespace fvmb;

extern "C" void fvm_opts_default(fvm_opts* o) {
    if (!o) return;
    std::memset(o, 0, sizeof(*o));
    o->rtol = 1e-6;
    o->atol = 1e-6;
    o->max_order = 5;
    o->krylov_dim = 30;
    o->max_restarts = 5;
    o->eps_lin = 3e-5;
    o->cj_refresh = 1.05;
    o->psetup_age = 1;
}

extern "C" int fvm_integrate(fvm_ctx* c, const fvm_opts* opts, double t0, double t_end,
                             const double* y0, double* y_end, fvm_stats* stats) {
    try {
        if (!c || !opts || !y0 || !y_end) throw Error("fvm_integrate: null argument");
        int rc = integrate_dev(c, opts, t0, t_end, y0, y_end, stats);
        FVM_CUDA(cudaGetLastError());
        if (rc < 0) set_error("fvm_integrate: step failure code " + std::to_string(rc));
        return rc;
    } catch (const Error& ex) {
        set_error(ex.what());
        return ex.code;
    } catch (const std::exception& ex) {
        set_error(ex.what());
        return -1;
    }
}

// Independent problems (ensemble members), each in its own context, each
// with its own step-size and order sequence: n_threads host threads take
// the contexts in turn (largest first when the caller sorts them), so the
// members' kernels overlap on the device through their own streams.  A
// member that fails stops alone; status[i] is its fvm_integrate code.
extern "C" int fvm_integrate_batch(fvm_ctx* const* ctxs, int n, const fvm_opts* opts, double t0, double t_end,
                                   const double* const* y0, double* const* y_end, fvm_stats* stats, int* status,
                                   int n_threads) {
    try {
        if (!ctxs || !opts || !y0 || !y_end || !status || n < 1) throw Error("fvm_integrate_batch: bad argument");
        for (int i = 0; i < n; ++i)
            if (!ctxs[i] || !y0[i] || !y_end[i]) throw Error("fvm_integrate_batch: null context or vector");
        const int nt = std::max(1, std::min(n_threads, n));
        std::atomic<int> next{0};
        std::vector<std::string> errs(n);
        auto work = [&]() {
            for (;;) {
                const int i = next.fetch_add(1);
                if (i >= n) return;
                fvm_ctx* c = ctxs[i];
                try {
                    FVM_CUDA(cudaSetDevice(c->device));
                    status[i] = integrate_dev(c, opts, t0, t_end, y0[i], y_end[i], stats ? stats + i : nullptr);
                    FVM_CUDA(cudaGetLastError());
                } catch (const Error& ex) {
                    status[i] = ex.code;
                    errs[i] = ex.what();
                } catch (const std::exception& ex) {
                    status[i] = -1;
                    errs[i] = ex.what();
                }
            }
        };
        std::vector<std::thread> pool;
        for (int k = 1; k < nt; ++k) pool.emplace_back(work);
        work();
        for (auto& th : pool) th.join();
        int worst = 0, first_bad = -1;
        for (int i = 0; i < n; ++i)
            if (status[i] < 0 && first_bad < 0) { first_bad = i; worst = status[i]; }
        if (first_bad >= 0)
            set_error("fvm_integrate_batch: member " + std::to_string(first_bad) + " failed with code " +
                      std::to_string(worst) + (errs[first_bad].empty() ? "" : ": " + errs[first_bad]));
        return first_bad >= 0 ? 1 : 0;
    } catch (const Error& ex) {
        set_error(ex.what());
        return ex.code;
    } catch (const std::exception& ex) {
        set_error(ex.what());
        return -1;
    }
}

extern "C" int fvm_integrate_outputs(fvm_ctx* c, const fvm_opts* opts, double t0, const double* y0, int n_out,
                                     const double* t_out_host, double* y_out, double* yp_out, fvm_stats* stats) {
    try {
        if (!c || !opts || !y0 || !t_out_host || !y_out) throw Error("fvm_integrate_outputs: null argument");
        if (n_out < 1) throw Error("fvm_integrate_outputs: n_out must be positive");
        for (int i = 0; i < n_out; ++i) {
            const double prev = i ? t_out_host[i - 1] : t0;
            if (!std::isfinite(t_out_host[i]) || !(t_out_host[i] > prev))
                throw Error("fvm_integrate_outputs: output times must be finite, ascending and after t0");
        }
        OutputTimes out;
        out.n = n_out;
        out.t = t_out_host;
        out.y = y_out;
        out.yp = yp_out;
        int rc = integrate_dev(c, opts, t0, t_out_host[n_out - 1], y0, nullptr, stats, nullptr, &out);
        FVM_CUDA(cudaGetLastError());
        if (rc < 0) set_error("fvm_integrate_outputs: step failure code " + std::to_string(rc));
        return rc;
    } catch (const Error& ex) {
        set_error(ex.what());
        return ex.code;
    } catch (const std::exception& ex) {
        set_error(ex.what());
        return -1;
    }
}

extern "C" int fvm_integrate_record(fvm_ctx* c, const fvm_opts* opts, double t0, double t_end,
                                    const double* y0, double* y_end, fvm_stats* stats, float* X, float* Y,
                                    long capacity, int stride, long* count) {
    try {
        if (!c || !opts || !y0 || !y_end || !X || !Y || !count || capacity <= 0 || stride <= 0)
            throw Error("fvm_integrate_record: bad argument");
        Recorder r;
        r.X = X;
        r.Y = Y;
        r.cap = capacity;
        r.stride = stride;
        int rc = integrate_dev(c, opts, t0, t_end, y0, y_end, stats, &r);
        *count = r.count;
        FVM_CUDA(cudaGetLastError());
        if (rc < 0) set_error("fvm_integrate_record: step failure code " + std::to_string(rc));
        return rc;
    } catch (const Error& ex) {
        set_error(ex.what());
        return ex.code;
    } catch (const std::exception& ex) {
        set_error(ex.what());
        return -1;
    }
}

extern "C" int fvm_integrate_host(fvm_ctx* c, const fvm_opts* opts, double t0, double t_end,
                                  const double* y0_host, double* y_end_host, fvm_stats* stats) {
    try {
        if (!c || !opts || !y0_host || !y_end_host) throw Error("fvm_integrate_host: null argument");
        IntegWork& w = integ_work(c);
        DevBuf<double>& a = w.host_in;
        DevBuf<double>& b = w.host_out;
        a.alloc(c->N);
        b.alloc(c->N);
        FVM_CUDA(cudaMemcpyAsync(a.p, y0_host, sizeof(double) * c->N, cudaMemcpyHostToDevice, c->stream));
        int rc = integrate_dev(c, opts, t0, t_end, a.p, b.p, stats);
        FVM_CUDA(cudaMemcpyAsync(y_end_host, b.p, sizeof(double) * c->N, cudaMemcpyDeviceToHost, c->stream));
        ctx_sync(c);
        if (rc < 0) set_error("fvm_integrate_host: step failure code " + std::to_string(rc));
        return rc;
    } catch (const Error& ex) {
        set_error(ex.what());
        return ex.code;
    } catch (const std::exception& ex) {
        set_error(ex.what());
        return -1;
    }
}

extern "C" int fvm_integrate_replay(fvm_ctx* c, const fvm_opts* opts, double t0, const double* y0, double h0,
                                    long n_steps, const fvm_step_record* steps, double newton_tol, int max_newton,
                                    double* y_end, fvm_stats* stats) {
    try {
        if (!c || !opts || !y0 || !steps || !y_end) throw Error("fvm_integrate_replay: null argument");
        if (n_steps < 1) throw Error("fvm_integrate_replay: n_steps must be positive");
        int rc = replay_dev(c, opts, t0, y0, h0, n_steps, steps, newton_tol, max_newton, y_end, stats);
        FVM_CUDA(cudaGetLastError());
        if (rc < 0) set_error("fvm_integrate_replay: step failure code " + std::to_string(rc));
        return rc;
    } catch (const Error& ex) {
        set_error(ex.what());
        return ex.code;
    } catch (const std::exception& ex) {
        set_error(ex.what());
        return -1;
    }
}

extern "C" long fvm_step_trace(const fvm_ctx* c, fvm_step_record* out, long cap) {
    if (!c) return -1;
    const long n = (long)c->last_trace.size();
    if (out && cap > 0) std::memcpy(out, c->last_trace.data(), sizeof(fvm_step_record) * (size_t)std::min(n, cap));
    return n;
}
