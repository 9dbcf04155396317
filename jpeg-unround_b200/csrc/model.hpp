// The host side of the model: each component's problem (docs/math.md 1.2, 1.3, 2, 4.1) and
// the canvas they share, and the plan of the primal-dual method (5, 6.5). Every value here
// is computed in binary64 exactly as the reference computes it, so that the rational
// quantities (steps, weights, interval ends, tau and sigma) agree to the last bit
// (docs/math.md 9.2); the device reads them, rounded once to binary32 where its iterations
// compute in binary32.
#pragma once

#include <array>
#include <cstdint>
#include <memory>
#include <new>
#include <optional>
#include <string>
#include <utility>
#include <vector>

#include "settings.hpp"

namespace urb {

// A status of the C interface (rust/capi/include/unround.h:44-52).
enum Status : std::int32_t {
  kOk = 0,
  kArgument = 1,
  kRead = 2,
  kUnsupported = 3,
  kOptions = 4,
  kIo = 5,
  kInternal = 6,
};

struct Failure {
  Status status = kInternal;
  std::string message;
};

// A component as the caller gives it (unround_component, unround.h:101-108).
struct ComponentInput {
  const std::int16_t* levels = nullptr;
  std::uint32_t rows = 0;
  std::uint32_t columns = 0;
  std::int32_t h = 1;
  std::int32_t v = 1;
  std::array<std::uint16_t, 64> table{};
};

// Host blocks of the model's large arrays, kept for the next solve when freed (up to a limit),
// so that a solve writes into memory whose pages the process already holds instead of faulting in
// fresh pages (model.cpp).
void* reused_block(std::size_t bytes);
void return_block(void* block);

// An allocator whose resize leaves new elements uninitialised (the threads that fill a large array
// touch it first, not one thread zeroing it), from the reused host blocks.
template <typename T>
struct Uninitialised : std::allocator<T> {
  using is_always_equal = std::true_type;
  template <typename U>
  struct rebind {
    using other = Uninitialised<U>;
  };
  Uninitialised() = default;
  template <typename U>
  Uninitialised(const Uninitialised<U>&) noexcept {}
  T* allocate(std::size_t n) { return static_cast<T*>(reused_block(n * sizeof(T))); }
  void deallocate(T* at, std::size_t) noexcept { return_block(at); }
  template <typename U>
  void construct(U* at) noexcept {
    ::new (static_cast<void*>(at)) U;
  }
  template <typename U, typename... Args>
  void construct(U* at, Args&&... args) {
    ::new (static_cast<void*>(at)) U(std::forward<Args>(args)...);
  }
};

// One component's problem on the canvas (cpp/src/model.cpp:124-256 and
// rust/unround/src/model.rs Problem::new): the kept levels, the steps, the weights of
// the data term in a block that is not flat and in one that is, which blocks are flat,
// the MMSE shrinkage of each frequency where the centres are MMSE, and the slack's cost.
struct Component {
  std::uint32_t block_rows = 0;
  std::uint32_t block_columns = 0;
  std::uint32_t cell_rows = 1;     // canvas samples down per sample of the component
  std::uint32_t cell_columns = 1;  // and across
  bool free = false;               // some canvas samples are free (docs/math.md 1.3)
  std::vector<std::int16_t, Uninitialised<std::int16_t>> levels;  // [by][bx][64], natural order
  std::vector<std::uint8_t, Uninitialised<std::uint8_t>> flat;    // [by][bx]
  std::array<double, 64> steps{};
  std::array<double, 64> weights{};
  std::array<double, 64> flat_weights{};
  std::array<double, 64> shrink{};  // delta / Q of the MMSE centres; 0 for the middles
  std::array<double, 64> costs{};   // beta / Q where the slack has a cost
  double mu = 0.0;
  double slack = 0.0;
  bool mmse = false;
  bool costed = false;

  [[nodiscard]] std::uint32_t cells() const { return cell_rows * cell_columns; }
  [[nodiscard]] std::size_t coefficient_count() const {
    return static_cast<std::size_t>(block_rows) * block_columns * 64u;
  }
  // The ends of the interval and the centre of coefficient k (0..63) of level q
  // (cpp/src/model.cpp:41-46, 237-247; laplace.hpp:51-56 for the MMSE centres).
  [[nodiscard]] double lower(std::int16_t q, int k) const;
  [[nodiscard]] double upper(std::int16_t q, int k) const;
  [[nodiscard]] double centre(std::int16_t q, int k) const;
};

// The components on one canvas (docs/math.md 1.3): the picture's size, the canvas's
// rows and columns, and every component with its cells.
struct Frame {
  std::uint32_t height = 0;  // picture
  std::uint32_t width = 0;
  std::int32_t color_space = 1;  // 1 grey, 2 YCbCr, 3 RGB
  std::uint32_t rows = 0;        // canvas
  std::uint32_t columns = 0;
  std::vector<Component> components;

  [[nodiscard]] std::size_t channels() const { return components.size(); }
  [[nodiscard]] std::size_t plane() const { return static_cast<std::size_t>(rows) * columns; }
  // The canvas rows and columns of an MCU: every component's blocks tile it.
  [[nodiscard]] std::uint32_t mcu_rows() const;
  [[nodiscard]] std::uint32_t mcu_columns() const;
};

// The frame of the caller's components with the settings' data terms, or why not: the
// reference's frame_of (rust/unround/src/decode.rs:233-262) with Frame::of_file
// (rust/unround/src/frames.rs:207-250) and Problem::new (rust/unround/src/model.rs:333-425).
std::optional<Frame> make_frame(std::uint32_t height, std::uint32_t width, std::int32_t color_space,
                                const std::vector<ComponentInput>& inputs, const Settings& settings,
                                Failure& failure);

// The plan of the primal-dual method for a frame (cpp/src/pdhg.cpp:147-233,
// rust/unround/src/pdhg.rs:186-353): the steps tau = sqrt(kappa theta / L^2) and
// sigma = sqrt(theta / (kappa L^2)), the most iterations, the tolerances, the relaxation,
// the records and the channel weights.
struct Plan {
  bool tgv = true;
  double tau = 0.0;
  double sigma = 0.0;
  std::uint64_t iterations = 0;
  double tolerance = 0.0;
  double relative_tolerance = 0.0;
  double partial_tolerance = 0.0;
  std::optional<double> partial_radius;
  double relaxation = 1.9;
  std::uint64_t record_every = 10;
  double free_radius = 255.0;
  std::vector<double> channel_weights;
  bool coupled = true;
  double alpha = 1.0;   // TV's
  double alpha1 = 1.0;  // TGV's
  double alpha0 = 2.0;
};

// The defaults of a plan where the options give none: JPEG files' (cpp/include/unround/pdhg.hpp)
// unless a caller gives others (pictures of rounded samples).
struct PlanDefaults {
  double tv_ratio = 10.0;
  double tgv_ratio = 3.0;
  double tv_tolerance = 2e-4;
  double tgv_tolerance = 2e-3;
  std::uint64_t tv_iterations = 5000;
  std::uint64_t tgv_iterations = 10000;
};

std::optional<Plan> make_plan(const Settings& settings, std::size_t channels, Failure& failure,
                              const PlanDefaults& defaults = PlanDefaults{});

// The Laplace scale of a frequency from its counts (docs/math.md 2.1,
// cpp/src/laplace.cpp:81-107), and delta / Q of a bin's mean (2.2, laplace.cpp:132-146).
double laplace_scale(std::uint64_t zeros, std::uint64_t others, std::uint64_t sum, double step);
double laplace_shrinkage(double rho);

}  // namespace urb
