// The host model of rounded samples (samples_model.hpp). The rational ends n / d are rounded
// to doubles exactly, in integers: n 2^p / d is divided with p chosen so that the quotient has
// 53 bits, and the remainder tells whether anything was cut off.
#include "samples_model.hpp"

#include <bit>
#include <cmath>
#include <string>

namespace urb {

namespace {

using u128 = unsigned __int128;

// n / d (n > 0) as q 2^-p with 2^52 <= q < 2^53, and the remainder of the division.
struct Scaled {
  std::uint64_t q = 0;
  int p = 0;
  std::uint64_t remainder = 0;
  std::uint64_t denominator = 1;
};

Scaled scaled(std::uint64_t n, std::uint64_t d) {
  int p = 52 + std::bit_width(d) - std::bit_width(n);
  for (;;) {
    const u128 numerator = p >= 0 ? static_cast<u128>(n) << p : static_cast<u128>(n) >> (-p);
    const u128 q = numerator / d;
    if (q >= (u128{1} << 53)) {
      --p;
    } else if (q < (u128{1} << 52)) {
      ++p;
    } else {
      return Scaled{static_cast<std::uint64_t>(q), p, static_cast<std::uint64_t>(numerator % d), d};
    }
  }
}

// The least double at or above n / d.
double at_or_above(std::uint64_t n, std::uint64_t d) {
  if (n == 0) return 0.0;
  const Scaled s = scaled(n, d);
  return std::ldexp(static_cast<double>(s.q + (s.remainder != 0 ? 1 : 0)), -s.p);
}

// The greatest double below n / d.
double under(std::uint64_t n, std::uint64_t d) {
  const Scaled s = scaled(n, d);
  const double down = std::ldexp(static_cast<double>(s.q), -s.p);
  return s.remainder != 0 ? down : std::nextafter(down, 0.0);
}

// The double nearest to n / d, ties to even.
double nearest(std::uint64_t n, std::uint64_t d) {
  if (n == 0) return 0.0;
  const Scaled s = scaled(n, d);
  const u128 twice = static_cast<u128>(s.remainder) * 2;
  std::uint64_t q = s.q;
  if (twice > s.denominator || (twice == s.denominator && (q & 1) != 0)) ++q;
  return std::ldexp(static_cast<double>(q), -s.p);
}

}  // namespace

SampleInterval sample_interval(std::uint32_t level, int bits, double slack) {
  const std::uint64_t top = (std::uint64_t{1} << bits) - 1;
  const std::uint64_t v = level;
  SampleInterval out;
  out.centre = nearest(255 * v, top);
  if (slack == 0.0) {
    out.lower = v == 0 ? 0.0 : at_or_above(255 * (2 * v - 1), 2 * top);
    out.upper = v == top ? 255.0 : under(255 * (2 * v + 1), 2 * top);
    return out;
  }
  const double step = nearest(255, top);
  const double own = static_cast<double>(v);
  const double lower = ((own - 0.5) - slack) * step;
  const double upper = ((own + 0.5) + slack) * step;
  out.lower = lower > 0.0 ? lower : 0.0;
  out.upper = upper < 255.0 ? upper : 255.0;
  return out;
}

std::optional<SamplesModel> make_samples_model(const std::uint16_t* levels, std::size_t rows, std::size_t columns,
                                               std::size_t channels, int bits, std::size_t first, std::size_t count,
                                               double slack, double mu, Failure& failure) {
  if (bits < 1 || bits > 16) {
    failure = {kUnsupported, "samples of " + std::to_string(bits) + " bits are not taken"};
    return std::nullopt;
  }
  if (!(slack >= 0.0 && std::isfinite(slack)) || !(mu >= 0.0 && std::isfinite(mu))) {
    failure = {kOptions, "the slack and mu are at least 0 and finite, not " + shortest(slack) + " and " + shortest(mu)};
    return std::nullopt;
  }
  if (first + count > channels || rows == 0 || columns == 0 || levels == nullptr) {
    failure = {kOptions, "the channels are not the picture's"};
    return std::nullopt;
  }
  const std::size_t level_count = std::size_t{1} << bits;
  const std::size_t plane = rows * columns;
  std::uint16_t highest = 0;
  for (std::size_t k = 0; k < plane; ++k) {
    const std::uint16_t* sample = levels + k * channels + first;
    for (std::size_t c = 0; c < count; ++c) highest = sample[c] > highest ? sample[c] : highest;
  }
  if (highest >= level_count) {
    failure = {kOptions, "a level of " + std::to_string(bits) + " bits is below 2^" + std::to_string(bits)};
    return std::nullopt;
  }
  SamplesModel model;
  model.rows = rows;
  model.columns = columns;
  model.channels = count;
  model.bits = bits;
  model.mu = mu;
  model.levels = levels;
  model.stride = channels;
  model.first = first;
  model.intervals.resize(level_count);
  for (std::size_t v = 0; v < level_count; ++v) {
    model.intervals[v] = sample_interval(static_cast<std::uint32_t>(v), bits, slack);
  }
  return model;
}

bool check_samples_settings(const Settings& settings, Failure& failure) {
  std::vector<std::string> errors;
  const DataTerm defaults;
  if (!settings.data.empty()) {
    const DataTerm& term = settings.data.front();
    const std::pair<const char*, bool> others[] = {
        {"mu-scale", term.mu_scale != defaults.mu_scale},        {"mu-power", term.mu_power != defaults.mu_power},
        {"mu-chroma", term.mu_chroma != defaults.mu_chroma},     {"weight-power", term.power != defaults.power},
        {"dc-weight", term.dc_weight != defaults.dc_weight},     {"centres", term.centres != defaults.centres},
        {"slack-cost", term.slack_cost != defaults.slack_cost},  {"flat-weight", term.flat_weight != defaults.flat_weight},
        {"flat-levels", term.flat_levels != defaults.flat_levels}, {"flat-dc", term.flat_dc != defaults.flat_dc}};
    for (const auto& [name, given] : others) {
      if (given) errors.push_back(std::string("--") + name + " is not for a PNG file");
    }
  }
  if (settings.method != Method::tv && settings.method != Method::tgv) {
    errors.emplace_back("a PNG file is reconstructed by tv or tgv");
  }
  if (settings.data.size() != 1) errors.emplace_back("the data term of a PNG file is one for every channel");
  if (errors.empty()) return true;
  failure.status = kOptions;
  failure.message.clear();
  for (const std::string& e : errors) failure.message += (failure.message.empty() ? "" : "; ") + e;
  return false;
}

PlanDefaults samples_plan_defaults() {
  PlanDefaults d;
  d.tgv_ratio = 0.3;
  d.tv_tolerance = 1e-4;
  d.tgv_tolerance = 1e-4;
  d.tv_iterations = 10000;
  d.tgv_iterations = 10000;
  return d;
}

}  // namespace urb
