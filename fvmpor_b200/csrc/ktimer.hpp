// Live per-kernel timing with CUDA events on the launching stream.
//
// Each category keeps a ring of (start, stop) event pairs; a pair is folded
// into the running total when its slot is reused or when the totals are
// read, so timing adds no host synchronisation to the hot loop.
#pragma once

#include <cuda_runtime.h>

#include <array>
#include <vector>

namespace fvmb {

enum TimerCat {
    TM_NODE = 0,      // van Genuchten node pass
    TM_ELEM = 1,      // element flux pass
    TM_GATHER = 2,    // node gather
    TM_ILU_APPLY = 3, // block-ILU(0) forward/backward
    TM_CGS = 4,       // Gram-Schmidt passes
    TM_ILU_FACTOR = 5,
    TM_FD_JAC = 6,    // finite-difference Jacobian (whole set-up)
    TM_MLP = 7,       // learned iterate: features + network forward
    TM_PRED = 8,      // learned iterate: the whole attempt (residuals, test, blend)
    TM_NCAT = 9
};

struct KernelTimer {
    static constexpr int kRing = 64;
    bool on = false;
    struct Slot {
        cudaEvent_t a = nullptr, b = nullptr;
        bool pending = false;
    };
    std::array<std::vector<Slot>, TM_NCAT> slots;
    std::array<int, TM_NCAT> next{};
    std::array<int, TM_NCAT> open{};
    std::array<double, TM_NCAT> ms{};
    std::array<long, TM_NCAT> count{};

    ~KernelTimer() {
        for (auto& v : slots)
            for (auto& s : v) {
                if (s.a) cudaEventDestroy(s.a);
                if (s.b) cudaEventDestroy(s.b);
            }
    }
    void fold(Slot& s, int c) {
        if (!s.pending) return;
        cudaEventSynchronize(s.b);
        float t = 0.f;
        if (cudaEventElapsedTime(&t, s.a, s.b) == cudaSuccess) {
            ms[c] += t;
            count[c]++;
        }
        s.pending = false;
    }
    void begin(int c, cudaStream_t st) {
        if (!on) return;
        auto& v = slots[c];
        if (v.empty()) {
            v.resize(kRing);
            for (auto& s : v) {
                cudaEventCreate(&s.a);
                cudaEventCreate(&s.b);
            }
        }
        Slot& s = v[next[c]];
        fold(s, c);
        open[c] = next[c];
        next[c] = (next[c] + 1) % kRing;
        cudaEventRecord(s.a, st);
    }
    void end(int c, cudaStream_t st) {
        if (!on) return;
        Slot& s = slots[c][open[c]];
        cudaEventRecord(s.b, st);
        s.pending = true;
    }
    void flush() {
        for (int c = 0; c < TM_NCAT; ++c)
            for (auto& s : slots[c]) fold(s, c);
    }
    void reset() {
        flush();
        ms.fill(0.0);
        count.fill(0);
    }
};

} // namespace fvmb
