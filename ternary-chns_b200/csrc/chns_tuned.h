// chns_tuned.h -- launch shapes of the step and transform kernels for each grid
// size and precision (index log2(n) - 5, n = 32 .. 4096): threads per CTA, TMA box
// rows, the P1 split, the source of P4's grad c and programmatic dependent
// launches of the stage kernels.  Chosen by ternary-chns_b200/autotune.py from
// forward-step timings of the binary and ternary models on a B200: the candidate
// with the highest summed steps/s.  Each CTA runs threads / (n/16) transforms of
// n points side by side; small grids want few threads per CTA so that the rows
// spread over all 148 SMs.
#pragma once

namespace chns {

constexpr int kCtaThreadsF64[8] = {32, 32, 32, 32, 32, 64, 128, 256};
constexpr int kCtaThreadsF32[8] = {32, 32, 32, 32, 32, 64, 128, 256};

// Rows per TMA box of the row kernels' tiles (a tile is whole boxes, so smaller
// boxes over-fetch fewer zero rows beyond the cut at the price of more copies).
constexpr int kTmaBoxRowsF64[8] = {256, 256, 256, 256, 256, 256, 256, 256};
constexpr int kTmaBoxRowsF32[8] = {256, 256, 256, 256, 256, 256, 256, 256};

// P1 with two CTAs per row (each half of the outputs): 1 = on.
constexpr int kSpecInvSplitF64[8] = {1, 1, 1, 1, 1, 1, 1, 0};
constexpr int kSpecInvSplitF32[8] = {1, 1, 1, 1, 1, 1, 0, 0};

// grad c_i kept in real space from P2 for P4 (1), or transformed again by P4 (0).
constexpr int kP4GradF64[8] = {0, 0, 0, 1, 1, 1, 0, 1};
constexpr int kP4GradF32[8] = {0, 0, 0, 1, 1, 0, 0, 0};

// stage kernels launched as programmatic dependent launches (1), or plainly (0).
constexpr int kPdlF64[8] = {0, 0, 0, 1, 0, 0, 0, 0};
constexpr int kPdlF32[8] = {0, 0, 0, 0, 1, 0, 0, 0};

}  // namespace chns
