// Learned Newton initial iterate (per-node MLP); see predictor.cu.
#pragma once

#include "ctx.cuh"

namespace fvmb {

struct Predictor;

// the trained predictor attached to a context, or nullptr
Predictor* predictor_of(fvm_ctx* c);

// Replaces the Newton starting point (y, y', e) with the network's guess
// when its residual is smaller than the BDF predictor's; returns true when
// the learned iterate was kept.
bool predictor_apply(fvm_ctx* c, Predictor* p, double tnew, double cj, const double* h_n,
                     const double* dphi1, double* y, double* yp, double* e, const double* ewt,
                     double* F);

} // namespace fvmb
