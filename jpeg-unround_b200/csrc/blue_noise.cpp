// The void-and-cluster ranks (blue_noise.hpp). The energies are 64-bit integers, so every
// comparison is exact and the order of the additions does not matter.
//
// 1. The initial pattern: 410 points, each put at the least energy of those before it (the
//    first at (0, 0)); then, until the point taken out is the place put back, the point of
//    greatest energy is taken out and a point put at the least energy.
// 2. Ranks 409 down to 0: from the initial pattern, the point of greatest energy is taken out.
// 3. Ranks 410 up to 4095: from the initial pattern, a point is put at the least energy.
#include "blue_noise.hpp"

#include <algorithm>
#include <cmath>
#include <limits>
#include <mutex>
#include <stdexcept>
#include <vector>

namespace urb {

namespace {

constexpr int kSide = kBlueNoiseSide;
constexpr int kPlaces = kSide * kSide;
constexpr int kInitial = 410;

// round(2^40 exp(-d^2 / 4.5)) of the torus distance from (0, 0): exp in the x87 extended
// format, whose error (about 1e-18 relative) is far below the half that the rounding needs.
std::vector<std::int64_t> gaussian() {
  std::vector<std::int64_t> values(kPlaces);
  for (int row = 0; row < kSide; ++row) {
    for (int column = 0; column < kSide; ++column) {
      const int down = std::min(row, kSide - row), across = std::min(column, kSide - column);
      const long double exponent = -static_cast<long double>(down * down + across * across) / 4.5L;
      const long double value = std::ldexp(std::exp(exponent), 40);
      values[row * kSide + column] = static_cast<std::int64_t>(std::floor(value + 0.5L));
    }
  }
  return values;
}

struct Pattern {
  const std::vector<std::int64_t>* kernel = nullptr;
  std::vector<bool> points = std::vector<bool>(kPlaces, false);
  std::vector<std::int64_t> energy = std::vector<std::int64_t>(kPlaces, 0);

  // The kernel centred on `place`, added (sign 1) or taken away (sign -1).
  void add(int place, std::int64_t sign) {
    const int row = place / kSide, column = place % kSide;
    for (int r = 0; r < kSide; ++r) {
      const int to_row = ((r + row) % kSide) * kSide;
      const std::int64_t* from = kernel->data() + r * kSide;
      for (int c = 0; c < kSide; ++c) energy[to_row + (c + column) % kSide] += sign * from[c];
    }
  }
  void put(int place) {
    points[place] = true;
    add(place, 1);
  }
  void take(int place) {
    points[place] = false;
    add(place, -1);
  }
  // The first point of greatest energy.
  int tightest() const {
    int best = -1;
    for (int p = 0; p < kPlaces; ++p) {
      if (points[p] && (best < 0 || energy[p] > energy[best])) best = p;
    }
    return best;
  }
  // The first place without a point of least energy.
  int emptiest() const {
    int best = -1;
    for (int p = 0; p < kPlaces; ++p) {
      if (!points[p] && (best < 0 || energy[p] < energy[best])) best = p;
    }
    return best;
  }
};

std::array<std::uint16_t, kPlaces> make_ranks() {
  const std::vector<std::int64_t> kernel = gaussian();
  Pattern initial;
  initial.kernel = &kernel;
  for (int n = 0; n < kInitial; ++n) initial.put(initial.emptiest());
  bool settled = false;
  for (int n = 0; n < kPlaces * 16; ++n) {
    const int out = initial.tightest();
    initial.take(out);
    const int into = initial.emptiest();
    initial.put(into);
    if (into == out) {
      settled = true;
      break;
    }
  }
  if (!settled) throw std::runtime_error("the blue-noise matrix's initial pattern did not settle");
  std::array<int, kPlaces> ranks;
  ranks.fill(-1);
  Pattern pattern = initial;
  for (int rank = kInitial - 1; rank >= 0; --rank) {
    const int place = pattern.tightest();
    pattern.take(place);
    ranks[place] = rank;
  }
  pattern = initial;
  for (int rank = kInitial; rank < kPlaces; ++rank) {
    const int place = pattern.emptiest();
    pattern.put(place);
    ranks[place] = rank;
  }
  std::array<std::uint16_t, kPlaces> out{};
  std::vector<bool> seen(kPlaces, false);
  for (int p = 0; p < kPlaces; ++p) {
    if (ranks[p] < 0 || seen[ranks[p]]) throw std::runtime_error("the blue-noise ranks are not each rank once");
    seen[ranks[p]] = true;
    out[p] = static_cast<std::uint16_t>(ranks[p]);
  }
  return out;
}

}  // namespace

const std::array<std::uint16_t, kBlueNoiseSide * kBlueNoiseSide>& blue_noise_ranks() {
  static const std::array<std::uint16_t, kPlaces> ranks = make_ranks();
  return ranks;
}

}  // namespace urb
