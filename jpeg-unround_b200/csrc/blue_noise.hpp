// The blue-noise matrix of the ordered dither of 8- and 16-bit output (docs/math.md 10;
// rust/unround/src/output.rs:51-65, blue_noise.rs): 64 x 64 ranks, each of 0 .. 4095 once,
// made by Ulichney's void-and-cluster method in integers as the reference's
// scripts/blue_noise.py describes it (its docstring, lines 7-24), so that the same ranks come
// out: the energy of a place is the sum over a pattern's points of a Gaussian of their
// distance on the 64 x 64 torus, each value round(2^40 exp(-d^2 / (2 sigma^2))), sigma = 3/2;
// every least or greatest energy is taken at its first place in row order.
#pragma once

#include <array>
#include <cstdint>

namespace urb {

constexpr int kBlueNoiseSide = 64;

// The ranks, row by row (rank 64 i + j of row i, column j); made once per process.
const std::array<std::uint16_t, kBlueNoiseSide * kBlueNoiseSide>& blue_noise_ranks();

}  // namespace urb
