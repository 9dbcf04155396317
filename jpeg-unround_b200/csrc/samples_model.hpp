// The host model of a picture of rounded samples (docs/math.md 11; cpp/include/unround/samples.hpp,
// rust/unround/src/samples.rs): each level v of a file of b bits (1 to 16) stands for the
// values that round to v s, s = 255 / (2^b - 1): without slack the doubles of
// max(0, (v - 1/2) s) <= x < (v + 1/2) s (x <= 255 at the last level), the rational ends
// rounded inward -- the lower one up to the least double at or above it, the upper one down to
// the greatest double below it; with a slack in levels, max(0, ((v - 1/2) - slack) s) and
// min(255, ((v + 1/2) + slack) s) in floating point with s the nearest double. The centre is
// the double nearest to v s. The model is the levels themselves and a table of the 2^b
// intervals: the device expands neither, each kernel looks a sample's ends up by its level.
#pragma once

#include <cstddef>
#include <cstdint>
#include <optional>
#include <vector>

#include "model.hpp"
#include "settings.hpp"

namespace urb {

struct SampleInterval {
  double lower = 0.0;
  double upper = 0.0;
  double centre = 0.0;
};

// The interval and centre of level `level` of `bits` bits (cpp/src/samples.cpp:86-105).
SampleInterval sample_interval(std::uint32_t level, int bits, double slack);

struct SamplesModel {
  std::size_t rows = 0, columns = 0, channels = 0;
  int bits = 8;
  double mu = 0.0;
  // Borrowed: rows x columns x stride levels interleaved, of which channels first ..
  // first + channels - 1 are the model's. They outlive the model's use.
  const std::uint16_t* levels = nullptr;
  std::size_t stride = 1, first = 0;
  std::vector<SampleInterval> intervals;  // one per level, 2^bits
};

// The model of channels first .. first + count - 1 of levels (rows x columns x `channels`
// interleaved) of `bits` bits, with a slack and mu at least 0 (cpp/src/samples.cpp:107-151):
// every level of those channels below 2^bits, the table of their intervals.
std::optional<SamplesModel> make_samples_model(const std::uint16_t* levels, std::size_t rows, std::size_t columns,
                                               std::size_t channels, int bits, std::size_t first, std::size_t count,
                                               double slack, double mu, Failure& failure);

// What a picture of rounded samples takes of the settings, as the reference reconstructs a PNG
// file's (cpp/src/samples.cpp:344-367): tv or tgv, one data term whose mu is a number (0
// unless given) and slack; the data term's other options are refused where they differ from
// their defaults.
bool check_samples_settings(const Settings& settings, Failure& failure);

// The defaults of the plan of pictures of rounded samples (cpp/include/unround/samples.hpp:29-34):
// TGV's ratio of the steps 0.3, a gap per sample of 1e-4, 10000 iterations.
PlanDefaults samples_plan_defaults();

}  // namespace urb
