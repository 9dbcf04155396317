// The settings of a reconstruction under the option names of the reference's command
// line (docs/cli.md:182-243 of JPEG-Unround), as unround_settings_new takes them
// (rust/capi/include/unround.h:63-69): the method, the regularizer, the data term of
// every component or of each, the primal-dual method, the subgradient method and the
// limits of reading. The names, ranges and defaults are the reference's, so that the same
// option strings give the same settings (cpp/include/unround/settings.hpp:34-47).
#pragma once

#include <cstdint>
#include <optional>
#include <string>
#include <vector>

namespace urb {

enum class Method : std::int32_t { mmse = 0, tv = 1, tgv = 2, subgradient = 3 };
enum class Centres : std::int32_t { mmse = 0, midpoint = 1 };

// The options of G of one component (docs/math.md 4.1; cpp/include/unround/model.hpp:41-66).
struct DataTerm {
  std::optional<double> mu;
  double mu_scale = 9.0;
  double mu_power = 0.9;
  double mu_chroma = 0.3;
  double slack = 0.0;
  double dc_weight = 1.0;
  Centres centres = Centres::midpoint;
  double power = 2.0;
  double slack_cost = 0.0;
  double flat_weight = 0.1;
  std::uint32_t flat_levels = 0;
  std::optional<std::uint32_t> flat_dc = 1u;

  // Cb and Cr of a file in YCbCr: a rule's scale times mu_chroma (model.cpp:117-122).
  [[nodiscard]] DataTerm of_chroma() const {
    if (mu) return *this;
    DataTerm chroma = *this;
    chroma.mu_scale = mu_scale * mu_chroma;
    return chroma;
  }
  bool operator==(const DataTerm&) const = default;
};

struct Regularizer {
  double alpha = 1.0;
  double alpha1 = 1.0;
  double alpha0 = 2.0;
  std::vector<double> channel_weights;
  bool coupled = true;
};

struct PdhgOptions {
  std::optional<std::uint64_t> iterations;
  std::optional<double> tolerance;
  double relative_tolerance = 0.0;
  double partial_tolerance = 0.0;
  std::optional<double> partial_radius;
  std::optional<double> step_ratio;
  double relaxation = 1.9;
  double step_product = 0.99;
  std::optional<double> norm_squared;
  bool weight_scaling = true;
  std::uint64_t record_every = 10;
  double free_radius = 255.0;
  std::uint64_t threads = 0;
};

struct SubgradientOptions {
  std::uint64_t iterations = 50;
  double step = 0.5;
  double decay = 0.5;
  bool momentum = true;
  std::uint64_t record_every = 1;
};

struct Reading {
  std::uint64_t max_pixels = 268435456;
  std::int32_t max_scans = 500;
  bool warnings_are_errors = false;
};

struct Settings {
  Method method = Method::tgv;
  Regularizer regularizer;
  std::vector<DataTerm> data = {DataTerm{}};
  PdhgOptions pdhg;
  SubgradientOptions subgradient;
  Reading reading;
};

// Parses option strings as the command line takes them ("--mu", "0.01", "--mu=0.01").
// Returns false with every refusal joined by "; " in `errors`.
bool parse_settings(const std::vector<std::string>& arguments, Settings& out, std::string& errors);

// The options that give the settings back: "--name=value" or "--flag", each number the
// shortest decimal that reads back as the same double (cpp/src/settings.cpp:455-503).
std::vector<std::string> options_of(const Settings& settings);

// The shortest decimal that reads back as the same double.
std::string shortest(double value);

}  // namespace urb

// The opaque settings handle of the C interface (unround.h's unround_settings), shared by every
// source that takes one.
struct unround_settings {
  urb::Settings settings;
};
