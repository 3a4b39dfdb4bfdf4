// chns_tuned.h -- threads per CTA of the step and transform kernels for each
// grid size and precision (index log2(n) - 5, n = 32 .. 4096).  Chosen by
// ternary-chns_b200/autotune.py from forward-step timings of the binary and
// ternary models on a B200: the candidate with the highest summed steps/s.
// Each CTA runs threads / (n/16) transforms of n points side by side; small
// grids want few threads per CTA so that the rows spread over all 148 SMs.
#pragma once

namespace chns {

constexpr int kCtaThreadsF64[8] = {32, 32, 32, 32, 32, 64, 128, 256};
constexpr int kCtaThreadsF32[8] = {32, 32, 32, 32, 64, 64, 256, 256};

}  // namespace chns
