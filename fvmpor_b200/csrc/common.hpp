// Shared host-side helpers of the fvmpor_b200 library.
#pragma once

#include "../../include/fvmpor_b200.h"

#include <cstdint>
#include <cstdlib>
#include <stdexcept>
#include <string>
#include <vector>

namespace fvmb {

struct Error : std::runtime_error {
    int code;
    explicit Error(const std::string& m, int c = -1) : std::runtime_error(m), code(c) {}
};

void set_error(const std::string& msg);

struct Rng {
    uint64_t s;
    bool has_spare = false;
    double spare = 0.0;
    explicit Rng(uint64_t seed);
    uint64_t next();
    double uniform();
    double normal();
};

std::vector<double> gaussian_field(int nx, int ny, int nz, double hx, double hy, double hz,
                                   double var, double Lx, double Ly, double Lz, uint64_t seed);

} // namespace fvmb
