// Host model and plan, binary64 throughout. Compiled with -ffp-contract=off so that the
// interval ends, weights and steps round exactly as the reference's statements do
// (docs/math.md, Arithmetic; cpp/src/model.cpp:41-46 keeps the product and the sum of an
// interval end apart for the same reason).
#include "model.hpp"

#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <limits>
#include <map>
#include <mutex>
#include <thread>

namespace urb {

namespace {

// The reused blocks: each starts with a header of its size; idle ones are kept up to kKeep bytes
// in all, a request taking the smallest idle block that holds it and is at most twice its size.
constexpr std::size_t kHeader = 64;
constexpr std::size_t kKeep = std::size_t{1} << 30;

struct Blocks {
  std::mutex lock;
  std::multimap<std::size_t, void*> idle;  // bytes -> block
  std::size_t idle_bytes = 0;
};

Blocks& blocks() {
  static Blocks* made = new Blocks;  // never destroyed: blocks may be returned during exit
  return *made;
}

}  // namespace

void* reused_block(std::size_t bytes) {
  Blocks& b = blocks();
  {
    std::lock_guard<std::mutex> hold(b.lock);
    auto it = b.idle.lower_bound(bytes + kHeader);
    if (it != b.idle.end() && it->first <= 2 * (bytes + kHeader)) {
      void* block = it->second;
      b.idle_bytes -= it->first;
      b.idle.erase(it);
      return static_cast<char*>(block) + kHeader;
    }
  }
  const std::size_t size = bytes + kHeader;
  void* block = std::malloc(size);
  if (block == nullptr) throw std::bad_alloc();
  *static_cast<std::size_t*>(block) = size;
  return static_cast<char*>(block) + kHeader;
}

void return_block(void* at) {
  if (at == nullptr) return;
  void* block = static_cast<char*>(at) - kHeader;
  const std::size_t size = *static_cast<std::size_t*>(block);
  Blocks& b = blocks();
  {
    std::lock_guard<std::mutex> hold(b.lock);
    if (b.idle_bytes + size <= kKeep) {
      b.idle.emplace(size, block);
      b.idle_bytes += size;
      return;
    }
  }
  std::free(block);
}

namespace {

// body(first, end) over block rows [0, rows), shared out among the host's threads in contiguous
// ranges (one thread for small pictures); returns once every range is done.
template <typename Body>
void in_parallel(std::uint32_t rows, const Body& body) {
  const unsigned threads = std::max(1u, std::min(16u, std::thread::hardware_concurrency()));
  const auto parts = static_cast<std::uint32_t>(std::min<std::uint32_t>(threads, std::max<std::uint32_t>(rows / 32, 1)));
  std::vector<std::thread> workers;
  for (std::uint32_t t = 1; t < parts; ++t) {
    workers.emplace_back([&body, rows, t, parts] { body(rows * t / parts, rows * (t + 1) / parts); });
  }
  body(0, rows / parts);
  for (std::thread& worker : workers) worker.join();
}

constexpr double kLevelShiftDc = 1024.0;  // 8 x 128 on DC (docs/math.md 1.1)
constexpr std::uint32_t kBlock = 8;

// B_2k / (2k)! for k = 1..11, each the double nearest to the exact rational (docs/math.md
// 2.2: the Taylor series of delta / Q below rho = 1). Computed from the Bernoulli numbers
// 1/6, -1/30, 1/42, -1/30, 5/66, -691/2730, 7/6, -3617/510, 43867/798, -174611/330,
// 854513/138 with exact fractions and rounded once.
constexpr double kSeries[11] = {
    0x1.5555555555555p-4,  -0x1.6c16c16c16c17p-10, 0x1.1566abc011567p-15, -0x1.bbd779334ef0bp-21,
    0x1.66a8f2bf70ebep-26, -0x1.22805d644267fp-31, 0x1.d6db2c4e09162p-37, -0x1.7da4e1f79955cp-42,
    0x1.355871d652e9ep-47, -0x1.f57d968caacf1p-53, 0x1.967e1f09c376fp-58,
};

bool nonnegative(double x) { return x >= 0.0 && std::isfinite(x); }
bool positive(double x) { return x > 0.0 && std::isfinite(x); }

std::uint32_t ceiling(std::uint64_t n, std::uint64_t d) { return static_cast<std::uint32_t>((n + d - 1) / d); }

// Q^p: exact for the powers 1 and 2 (cpp/src/model.cpp:35-39).
double power_of(double step, double power) {
  if (power == 2.0) return step * step;
  if (power == 1.0) return step;
  return std::pow(step, power);
}

// ((q + half) + widen) Q + shift, each operation rounded apart.
double interval_end(double level, double half, double widen, double step, double shift) {
  const double widened = (level + half) + widen;
  const double scaled = widened * step;
  return scaled + shift;
}

// The rule of mu: the mean of the 64 steps (exact) to the power, times the scale
// (cpp/src/model.cpp:124-132).
double rule_mu(const DataTerm& data, const std::array<std::uint16_t, 64>& table) {
  if (data.mu) return *data.mu;
  std::uint32_t sum = 0;
  for (std::uint16_t step : table) sum += step;
  const double mean = static_cast<double>(sum) / 64.0;
  if (data.mu_power == 1.0) return data.mu_scale * mean;
  return data.mu_scale * std::pow(mean, data.mu_power);
}

double nearest(unsigned __int128 value) { return static_cast<double>(value); }

}  // namespace

double Component::lower(std::int16_t q, int k) const {
  return interval_end(static_cast<double>(q), -0.5, -slack, steps[k], k == 0 ? kLevelShiftDc : 0.0);
}

double Component::upper(std::int16_t q, int k) const {
  return interval_end(static_cast<double>(q), 0.5, slack, steps[k], k == 0 ? kLevelShiftDc : 0.0);
}

double Component::centre(std::int16_t q, int k) const {
  const double level = static_cast<double>(q);
  if (k == 0 || !mmse) return level * steps[k] + (k == 0 ? kLevelShiftDc : 0.0);
  // sign(q) (|q| - delta / Q) Q, 0 for q = 0 (cpp/include/unround/laplace.hpp:51-56).
  const double size = (std::fabs(level) - shrink[k]) * steps[k];
  const double signed_size = level < 0.0 ? -size : size;
  return level == 0.0 ? 0.0 : signed_size;
}

std::uint32_t Frame::mcu_rows() const {
  std::uint32_t most = 1;
  for (const Component& c : components) most = std::max(most, c.cell_rows);
  return kBlock * most;
}

std::uint32_t Frame::mcu_columns() const {
  std::uint32_t most = 1;
  for (const Component& c : components) most = std::max(most, c.cell_columns);
  return kBlock * most;
}

double laplace_scale(std::uint64_t zeros, std::uint64_t others, std::uint64_t sum, double step) {
  if (sum == 0) return 0.0;
  using u128 = unsigned __int128;
  const u128 n0 = zeros, n1 = others, s = sum;
  const u128 a = n0 + s + 2u * n1;
  const u128 discriminant = n0 * n0 + 4u * a * s;
  const double root = std::sqrt(nearest(discriminant));
  const double n0d = nearest(n0);
  // t* = 2S / (n0 + sqrt D): nothing cancels.
  const double t = nearest(2u * s) / (n0d + root);
  double log_inverse;
  if (t >= 0.5) {
    // 1 - t* = 8 S (n0 + n1) / ((sqrt D + 2S - n0)(n0 + sqrt D)), every term positive.
    const double top = nearest(8u * s * (n0 + n1));
    const double first = root + nearest(2u * s - n0);
    const double second = n0d + root;
    log_inverse = -std::log1p(-(top / (first * second)));
  } else {
    log_inverse = -std::log(t);
  }
  return step / (2.0 * log_inverse);
}

double laplace_shrinkage(double rho) {
  if (!(rho > 0.0)) return 0.0;
  if (std::isinf(rho)) return 0.5;
  if (rho < 1.0) {
    const double square = rho * rho;
    double sum = kSeries[10];
    for (int k = 9; k >= 0; --k) sum = sum * square + kSeries[k];
    return sum * rho;
  }
  const double decay = std::exp(-rho);
  return (0.5 - 1.0 / rho) + decay / -std::expm1(-rho);
}

namespace {

// One component's problem (rust/unround/src/model.rs Problem::new; cpp/src/model.cpp:134-256).
bool make_component(const ComponentInput& input, std::uint32_t block_rows, std::uint32_t block_columns,
                    const DataTerm& data, Component& out, Failure& failure) {
  std::vector<std::string> errors;
  if (!(nonnegative(data.mu_scale) && nonnegative(data.mu_chroma) && std::isfinite(data.mu_power))) {
    errors.push_back("the scale of mu and its factor in the chroma are at least 0 and finite, and its power finite");
  }
  const double mu = rule_mu(data, input.table);
  if (!(nonnegative(mu) && nonnegative(data.slack) && nonnegative(data.dc_weight))) {
    errors.push_back("mu, slack and the weight of DC are at least 0 and finite");
  }
  if (!nonnegative(data.power)) errors.push_back("the power of the steps in the weights is at least 0 and finite");
  if (!nonnegative(data.slack_cost)) errors.push_back("the cost of the slack is at least 0 and finite");
  if (!nonnegative(data.flat_weight) || data.flat_levels > 63) {
    errors.push_back("the weight of flat blocks is at least 0 and finite, and their AC levels not 0 at most 63");
  }
  if (std::find(input.table.begin(), input.table.end(), std::uint16_t{0}) != input.table.end()) {
    errors.push_back("a quantization step is at least 1");
  }
  if (!errors.empty()) {
    failure.status = kOptions;
    failure.message.clear();
    for (const auto& e : errors) failure.message += (failure.message.empty() ? "" : "; ") + e;
    return false;
  }
  out.block_rows = block_rows;
  out.block_columns = block_columns;
  out.mu = mu;
  out.slack = data.slack;
  out.mmse = data.centres == Centres::mmse;
  out.costed = data.slack > 0.0 && data.slack_cost > 0.0;
  // The kept blocks: the top-left block_rows x block_columns of the given ones.
  const std::size_t count = static_cast<std::size_t>(block_rows) * block_columns;
  out.levels.resize(count * 64);
  in_parallel(block_rows, [&](std::uint32_t first, std::uint32_t end) {
    for (std::uint32_t by = first; by < end; ++by) {
      const std::int16_t* from = input.levels + (static_cast<std::size_t>(by) * input.columns) * 64;
      std::copy(from, from + static_cast<std::size_t>(block_columns) * 64,
                out.levels.begin() + static_cast<std::ptrdiff_t>(by) * block_columns * 64);
    }
  });
  for (int k = 0; k < 64; ++k) {
    out.steps[k] = static_cast<double>(input.table[k]);
    out.weights[k] = mu / power_of(out.steps[k], data.power);
  }
  out.weights[0] *= data.dc_weight;
  for (int k = 0; k < 64; ++k) out.flat_weights[k] = out.weights[k] * data.flat_weight;
  if (out.costed) {
    for (int k = 0; k < 64; ++k) out.costs[k] = data.slack_cost / out.steps[k];
  }
  // Flat blocks (docs/math.md 4.1): at most flat_levels AC levels not 0 and, with a bound,
  // a DC level within it of the blocks above, below, left and right.
  out.flat.resize(count);  // every entry written below
  auto dc = [&](std::uint32_t by, std::uint32_t bx) {
    return static_cast<std::int32_t>(out.levels[(static_cast<std::size_t>(by) * block_columns + bx) * 64]);
  };
  in_parallel(block_rows, [&](std::uint32_t first, std::uint32_t end) {
  for (std::uint32_t by = first; by < end; ++by) {
    for (std::uint32_t bx = 0; bx < block_columns; ++bx) {
      const std::int16_t* q = &out.levels[(static_cast<std::size_t>(by) * block_columns + bx) * 64];
      std::uint32_t nonzero = 0;
      for (int k = 1; k < 64; ++k) nonzero += q[k] != 0 ? 1u : 0u;
      bool flat = nonzero <= data.flat_levels;
      if (flat && data.flat_dc) {
        const std::int32_t own = dc(by, bx);
        auto near = [&](std::uint32_t y, std::uint32_t x) {
          const std::int32_t other = dc(y, x);
          return static_cast<std::uint32_t>(own > other ? own - other : other - own) <= *data.flat_dc;
        };
        flat = (by == 0 || near(by - 1, bx)) && (by + 1 == block_rows || near(by + 1, bx)) &&
               (bx == 0 || near(by, bx - 1)) && (bx + 1 == block_columns || near(by, bx + 1));
      }
      out.flat[static_cast<std::size_t>(by) * block_columns + bx] = flat ? 1 : 0;
    }
  }
  });
  // MMSE centres: the Laplace scale of each AC frequency from the component's levels
  // (cpp/src/laplace.cpp:109-130), and delta / Q at rho = Q / beta.
  if (out.mmse) {
    std::array<std::uint64_t, 64> zeros{}, others{}, sums{};
    for (std::size_t b = 0; b < count; ++b) {
      const std::int16_t* q = &out.levels[b * 64];
      for (int k = 0; k < 64; ++k) {
        const std::int64_t level = q[k];
        if (level == 0) {
          ++zeros[k];
        } else {
          ++others[k];
          sums[k] += static_cast<std::uint64_t>(2 * (level < 0 ? -level : level) - 1);
        }
      }
    }
    for (int k = 1; k < 64; ++k) {
      const double scale = laplace_scale(zeros[k], others[k], sums[k], out.steps[k]);
      const double rho = scale > 0.0 ? out.steps[k] / scale : std::numeric_limits<double>::infinity();
      out.shrink[k] = laplace_shrinkage(rho);
    }
  }
  return true;
}

}  // namespace

std::optional<Frame> make_frame(std::uint32_t height, std::uint32_t width, std::int32_t color_space,
                                const std::vector<ComponentInput>& inputs, const Settings& settings,
                                Failure& failure) {
  const std::size_t count = inputs.size();
  if (color_space < 1 || color_space > 3) {
    failure = {kArgument, "a color space of 1, 2 or 3, not " + std::to_string(color_space)};
    return std::nullopt;
  }
  if (count == 0) {
    failure = {kArgument, "components are given"};
    return std::nullopt;
  }
  const std::size_t expected = color_space == 1 ? 1 : 3;
  if (count != expected) {
    failure = {kUnsupported, "a file of this color space has " + std::to_string(expected) + " components, not " +
                                 std::to_string(count)};
    return std::nullopt;
  }
  if (settings.data.size() != 1 && settings.data.size() != count) {
    failure = {kOptions, "options of G for each of the " + std::to_string(count) + " components, or one for all, not " +
                             std::to_string(settings.data.size())};
    return std::nullopt;
  }
  if (height == 0 || width == 0) {
    failure = {kUnsupported, "a picture without samples is refused"};
    return std::nullopt;
  }
  for (const ComponentInput& in : inputs) {
    if (in.levels == nullptr) {
      failure = {kArgument, "a component's levels are a null pointer"};
      return std::nullopt;
    }
    if (in.h < 0 || in.v < 0) {
      failure = {kArgument, "a sampling factor below 0"};
      return std::nullopt;
    }
  }
  Frame frame;
  frame.height = height;
  frame.width = width;
  frame.color_space = color_space;
  std::int32_t h_max = 1, v_max = 1;
  for (const ComponentInput& in : inputs) {
    h_max = std::max(h_max, in.h);
    v_max = std::max(v_max, in.v);
  }
  for (std::size_t c = 0; c < count; ++c) {
    const ComponentInput& in = inputs[c];
    std::uint32_t cell_rows = 1, cell_columns = 1, block_rows = in.rows, block_columns = in.columns;
    if (count == 1) {
      if (static_cast<std::uint64_t>(kBlock) * in.rows < height ||
          static_cast<std::uint64_t>(kBlock) * in.columns < width) {
        failure = {kUnsupported, "the blocks, " + std::to_string(in.rows) + " by " + std::to_string(in.columns) +
                                     ", do not cover the picture, " + std::to_string(height) + " by " +
                                     std::to_string(width)};
        return std::nullopt;
      }
    } else {
      if (in.h < 1 || in.v < 1 || in.h > 4 || in.v > 4 || h_max % in.h != 0 || v_max % in.v != 0) {
        failure = {kUnsupported, "the sampling factors " + std::to_string(in.h) + " x " + std::to_string(in.v) +
                                     " do not divide " + std::to_string(h_max) + " x " + std::to_string(v_max) +
                                     ": only whole cells are taken"};
        return std::nullopt;
      }
      cell_rows = static_cast<std::uint32_t>(v_max / in.v);
      cell_columns = static_cast<std::uint32_t>(h_max / in.h);
      block_rows = ceiling(height, static_cast<std::uint64_t>(kBlock) * cell_rows);
      block_columns = ceiling(width, static_cast<std::uint64_t>(kBlock) * cell_columns);
      if (in.rows != block_rows || in.columns != block_columns) {
        failure = {kUnsupported, "a component of " + std::to_string(in.rows) + " x " + std::to_string(in.columns) +
                                     " blocks, where a picture of " + std::to_string(height) + " x " +
                                     std::to_string(width) + " has " + std::to_string(block_rows) + " x " +
                                     std::to_string(block_columns)};
        return std::nullopt;
      }
    }
    DataTerm term = settings.data.size() == 1 ? settings.data[0] : settings.data[c];
    if (settings.method == Method::mmse) term.centres = Centres::mmse;
    if (color_space == 2 && c > 0) term = term.of_chroma();
    Component component;
    component.cell_rows = cell_rows;
    component.cell_columns = cell_columns;
    if (!make_component(in, block_rows, block_columns, term, component, failure)) {
      failure.message = "component " + std::to_string(c) + ": " + failure.message;
      return std::nullopt;
    }
    frame.components.push_back(std::move(component));
  }
  if (count == 1) {
    frame.rows = kBlock * inputs[0].rows;
    frame.columns = kBlock * inputs[0].columns;
  } else {
    frame.rows = kBlock * v_max * ceiling(height, static_cast<std::uint64_t>(kBlock) * v_max);
    frame.columns = kBlock * h_max * ceiling(width, static_cast<std::uint64_t>(kBlock) * h_max);
  }
  for (Component& c : frame.components) {
    c.free = c.cells() > 1 || kBlock * c.block_rows * c.cell_rows < frame.rows ||
             kBlock * c.block_columns * c.cell_columns < frame.columns;
  }
  return frame;
}

std::optional<Plan> make_plan(const Settings& settings, std::size_t channels, Failure& failure,
                              const PlanDefaults& defaults) {
  const Regularizer& reg = settings.regularizer;
  const PdhgOptions& o = settings.pdhg;
  const bool tv = settings.method == Method::tv;
  std::vector<std::string> errors;
  if (!positive(reg.alpha) || !positive(reg.alpha1) || !positive(reg.alpha0)) {
    errors.push_back("the weights alpha, alpha1 and alpha0 are above 0 and finite");
  }
  if (!reg.channel_weights.empty() && reg.channel_weights.size() != channels) {
    errors.push_back("the channel weights are one for each of the " + std::to_string(channels) + " channels, not " +
                     std::to_string(reg.channel_weights.size()));
  }
  if (!errors.empty()) {
    failure.status = kOptions;
    failure.message.clear();
    for (const auto& e : errors) failure.message += (failure.message.empty() ? "" : "; ") + e;
    return std::nullopt;
  }
  Plan plan;
  plan.tgv = !tv;
  plan.channel_weights = reg.channel_weights.empty() ? std::vector<double>(channels, 1.0) : reg.channel_weights;
  plan.coupled = reg.coupled && channels > 1;
  plan.alpha = reg.alpha;
  plan.alpha1 = reg.alpha1;
  plan.alpha0 = reg.alpha0;
  double largest = 0.0;
  for (double w : plan.channel_weights) largest = std::fmax(largest, w);
  const double bound = tv ? 8.0 : (17.0 + std::sqrt(33.0)) / 2.0;
  const double norm_squared = o.norm_squared ? *o.norm_squared : bound * (largest * largest);
  const double weight = tv ? reg.alpha : reg.alpha1;
  const double default_ratio = tv ? defaults.tv_ratio : defaults.tgv_ratio;
  const double default_tolerance = tv ? defaults.tv_tolerance : defaults.tgv_tolerance;
  const double ratio = o.step_ratio ? *o.step_ratio : o.weight_scaling ? default_ratio / (weight * weight)
                                                                        : default_ratio;
  plan.tolerance = o.tolerance ? *o.tolerance : o.weight_scaling ? default_tolerance * weight : default_tolerance;
  plan.iterations = o.iterations ? *o.iterations : tv ? defaults.tv_iterations : defaults.tgv_iterations;
  const double product = o.step_product;
  plan.tau = std::sqrt((ratio * product) / norm_squared);
  plan.sigma = std::sqrt(product / (ratio * norm_squared));
  plan.relative_tolerance = o.relative_tolerance;
  plan.partial_tolerance = o.partial_tolerance;
  plan.partial_radius = o.partial_radius;
  plan.relaxation = o.relaxation;
  plan.record_every = o.record_every;
  plan.free_radius = o.free_radius;
  return plan;
}

}  // namespace urb
