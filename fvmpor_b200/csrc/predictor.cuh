// Learned Newton initial iterate: a per-node MLP (BF16 weights, FP32
// accumulation on tcgen05 tensor cores).  See predictor.cu.
#pragma once

#include "ctx.cuh"

namespace fvmb {

constexpr int kMlpIn = 8;        // raw features per node
constexpr int kMlpK0 = 16;       // first-layer K padded to one MMA K-slice
constexpr int kMlpH = 64;        // hidden width
// packed FP32 parameter vector
constexpr int kOffW1 = 0;                         // [64][8]
constexpr int kOffB1 = kOffW1 + kMlpH * kMlpIn;   // [64]
constexpr int kOffW2 = kOffB1 + kMlpH;            // [64][64]
constexpr int kOffB2 = kOffW2 + kMlpH * kMlpH;
constexpr int kOffW3 = kOffB2 + kMlpH;            // [64][64]
constexpr int kOffB3 = kOffW3 + kMlpH * kMlpH;
constexpr int kOffW4 = kOffB3 + kMlpH;            // [64]
constexpr int kOffB4 = kOffW4 + kMlpH;            // [1]
constexpr int kNTrain = kOffB4 + 1;               // trainable parameters
constexpr int kOffMu = kNTrain;                   // feature means [8]
constexpr int kOffSd = kOffMu + kMlpIn;           // feature scales [8]
constexpr int kNParam = kOffSd + kMlpIn;

struct Predictor;

// the predictor attached to a context (created on first use)
Predictor* predictor_get(fvm_ctx* c);
// the trained predictor attached to a context, or nullptr
Predictor* predictor_of(fvm_ctx* c);
bool predictor_ready(Predictor* p);

// raw features of every node for the step t_n -> t_n + dt:
// h_n, h_n - h_{n-1}, y_pred - h_n, log10 dt, ln K, z, CV surface area, 0
void predictor_features(fvm_ctx* c, const double* h_n, const double* h_prev, const double* ypred,
                        double dt, float* X);
// out[i] = MLP(X[i]) in normalised units (tensor-core forward)
void predictor_forward(fvm_ctx* c, Predictor* p, const float* X, int n, float* out);

// Replaces the Newton starting point (y, y', e) with the network's guess
// y_pred + a w MLP, a in (0, 1] the minimiser of the residual norm along
// the learned direction (linearised from the residuals at both ends), when
// that at least halves the BDF predictor's residual norm.  ypred/yppred hold the BDF
// predictor; F receives the residual of the kept iterate.  Returns true when
// the learned iterate was kept.
bool predictor_apply(fvm_ctx* c, Predictor* p, double rtol, double atol, double dt, double cj,
                     const double* h_n, const double* h_prev, const double* ypred,
                     const double* yppred, double* y, double* yp, double* e, double* F);

// training-set recorder: features of a node subset at the predictor and
// the target (y_{n+1} - y_pred) / (rtol |h_n| + atol) after acceptance
struct Recorder {
    float* X = nullptr;   // [cap][8] device
    float* Y = nullptr;   // [cap] device
    long cap = 0;
    long count = 0;
    int stride = 64;      // record every stride-th node, offset rotating per step
    long step = 0;
};
void recorder_push(fvm_ctx* c, Recorder* r, const float* Xall, const double* y_new,
                   const double* ypred, const double* h_n, double rtol, double atol);

} // namespace fvmb
