// 8- and 16-bit levels of a binary64 picture on the device (docs/math.md 10;
// rust/unround/src/output.rs:66-209): each sample times the scale (1, or 257 so that 255 is
// 65535), as its rounding y and that rounding's exact error, to a level clamped to 0 .. top --
// by the ordered dither of the blue-noise matrix (the level below, or the one above where the
// fraction of y reaches 1 - (2 rank + 1) / 8192, the error deciding where it is exactly that),
// or rounded to the nearest level, halves away from 0 (the error deciding at a half). The
// channels of a pixel take the matrix shifted apart ((0, 0), (0, 32), (32, 0), (32, 32) rows
// and columns) or all the same place. A thread per sample; every operation exact or rounded
// as the reference's, so the levels are the reference's bit for bit.
#include <atomic>

#include "blue_noise.hpp"
#include "kernels.hpp"

namespace urb {

namespace {

__constant__ std::uint16_t ranks_on_device[kBlueNoiseSide * kBlueNoiseSide];

__global__ void __launch_bounds__(256) levels_kernel(const LevelsParams P) {
  const std::size_t k = static_cast<std::size_t>(blockIdx.x) * 256 + threadIdx.x;
  if (k >= P.count) return;
  const double sample = P.samples[k];
  if (!isfinite(sample)) {
    atomicExch(P.not_finite, 1);
    return;
  }
  const double y = __dmul_rn(sample, P.scale);
  const double error = fma(sample, P.scale, -y);  // exact: sample x scale = y + error
  const double whole = floor(y);
  double level;
  if (P.dither == 0) {
    level = (__dsub_rn(y, whole) == 0.5 && error < 0.0) ? whole : round(y);
  } else {
    const std::size_t pixel = k / static_cast<std::size_t>(P.channels);
    const int channel = static_cast<int>(k - pixel * P.channels);
    const std::size_t row = pixel / static_cast<std::size_t>(P.width);
    const std::size_t column = pixel - row * P.width;
    const int down = P.dither == 1 && (channel & 2) ? 32 : 0;
    const int across = P.dither == 1 && (channel & 1) ? 32 : 0;
    const int rank = ranks_on_device[((row + down) % kBlueNoiseSide) * kBlueNoiseSide + (column + across) % kBlueNoiseSide];
    const double threshold = (2.0 * rank + 1.0) / 8192.0;  // 13 bits: exact
    const double fraction = __dsub_rn(y, whole), limit = __dsub_rn(1.0, threshold);
    const bool above = fraction > limit || (fraction == limit && error >= 0.0);
    level = above ? __dadd_rn(whole, 1.0) : whole;
  }
  level = fmin(fmax(level, 0.0), P.top);
  if (P.sixteen) {
    const unsigned value = static_cast<unsigned>(level);
    P.out[2 * k] = static_cast<std::uint8_t>(value >> 8);  // most significant byte first
    P.out[2 * k + 1] = static_cast<std::uint8_t>(value & 0xffu);
  } else {
    P.out[k] = static_cast<std::uint8_t>(level);
  }
}

}  // namespace

bool prepare_levels() {
  static std::atomic<unsigned long long> loaded{0};
  int device = 0;
  if (cudaGetDevice(&device) != cudaSuccess) return false;
  const unsigned long long bit = 1ull << (device & 63);
  if ((loaded.load() & bit) != 0) return true;
  const auto& ranks = blue_noise_ranks();
  if (cudaMemcpyToSymbol(ranks_on_device, ranks.data(), sizeof(ranks_on_device)) != cudaSuccess) return false;
  loaded.fetch_or(bit);
  return true;
}

cudaError_t launch_levels(const LevelsParams& p, cudaStream_t stream) {
  if (p.count == 0) return cudaSuccess;
  levels_kernel<<<static_cast<unsigned>((p.count + 255) / 256), 256, 0, stream>>>(p);
  return cudaGetLastError();
}

}  // namespace urb
