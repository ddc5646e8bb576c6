// Learned Newton initial iterate: placeholder until the MLP kernels land.
#include "predictor.cuh"

namespace fvmb {

Predictor* predictor_of(fvm_ctx*) { return nullptr; }

bool predictor_apply(fvm_ctx*, Predictor*, double, double, const double*, const double*, double*,
                     double*, double*, const double*, double*) {
    return false;
}

} // namespace fvmb
