// The C interface (include/unround.h, include/unround_b200.h): the reference's unround_capi
// entry points (rust/capi/src/lib.rs) over the device solver. Inputs are copied for the call
// (rust/capi/src/lib.rs:617-660), results are owned by the library until unround_result_free,
// and no exception crosses the interface: each entry point catches everything and returns a
// status with its message (rust/capi/src/lib.rs:99-115, `guarded`).
#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <limits>
#include <memory>
#include <mutex>
#include <new>
#include <string>
#include <thread>
#include <vector>

#include <cuda_runtime.h>
#include <dlfcn.h>
#include <nccl.h>
#include <zlib.h>

#include "batch.hpp"
#include "blue_noise.hpp"
#include "jpeg_reader.hpp"
#include "colour.hpp"
#include "dct.cuh"
#include "model.hpp"
#include "png_io.hpp"
#include "samples_model.hpp"
#include "settings.hpp"
#include "solver.hpp"
#include "unround.h"
#include "unround_b200.h"

struct unround_result {
  urb::Frame frame;
  urb::Outcome outcome;  // the canvas, the planes and the picture (made on the device)
  std::uint64_t height = 0, width = 0, channels = 0;
  // The planes cut to the picture: the canvas itself where it is no larger; and the picture:
  // the planes themselves where there is one channel.
  [[nodiscard]] const double* planes() const {
    return outcome.planes.empty() ? outcome.canvas.data() : outcome.planes.data();
  }
  [[nodiscard]] const double* picture() const {
    return outcome.picture.empty() ? planes() : outcome.picture.data();
  }
  std::vector<std::uint64_t> record_iterations;
  std::vector<double> record_values[5];
  // What the model holds, made when first asked for (rust/capi/src/lib.rs:888-930): each
  // component's lower ends, upper ends and centres, coefficient by coefficient.
  mutable std::once_flag problem_once;
  mutable std::vector<std::unique_ptr<double[]>> problem[3];
  mutable std::vector<std::size_t> problem_sizes;
  std::vector<std::vector<double>> steps, weights;
  // What the file held besides its picture (unround_result_format and the rest).
  std::int32_t format = UNROUND_FORMAT_JPEG;
  std::int32_t bits = 8;
  std::int32_t exif_orientation = 0;
  std::vector<std::uint8_t> icc;
  std::string warning;
  std::vector<std::vector<double>> excess;  // of a projection: each component's, in steps
};

namespace {

const char kVersion[] = "unround 0.1.0 (B200: CUDA sm_100a, C interface)";

// Writes text into the caller's buffer, NUL-terminated, cut at a UTF-8 character's boundary.
void say(char* buffer, std::size_t size, const std::string& text) {
  if (buffer == nullptr || size == 0) return;
  std::size_t end = std::min(text.size(), size - 1);
  while (end > 0 && end < text.size() && (static_cast<unsigned char>(text[end]) & 0xC0u) == 0x80u) --end;
  std::memcpy(buffer, text.data(), end);
  buffer[end] = 0;
}

template <typename Body>
std::int32_t guarded(char* message, std::size_t size, Body&& body) {
  try {
    urb::Failure failure;
    if (body(failure)) return urb::kOk;
    say(message, size, failure.message);
    return failure.status;
  } catch (const std::bad_alloc&) {
    say(message, size, "an internal error of JPEG-Unround: out of host memory");
    return urb::kInternal;
  } catch (const std::exception& error) {
    say(message, size, std::string("an internal error of JPEG-Unround: ") + error.what());
    return urb::kInternal;
  } catch (...) {
    say(message, size, "an internal error of JPEG-Unround");
    return urb::kInternal;
  }
}

bool have_device(urb::Failure& failure) {
  int count = 0;
  cudaError_t error = cudaGetDeviceCount(&count);
  if (error != cudaSuccess || count == 0) {
    failure = {urb::kInternal, std::string("no CUDA device for the solver: ") +
                                   (error != cudaSuccess ? cudaGetErrorString(error) : "none found")};
    return false;
  }
  // The solves' buffers come from the device's stream-ordered pool; keep what a solve frees
  // for the next one instead of returning it to the driver at every synchronization.
  int device = 0;
  error = cudaGetDevice(&device);
  static std::once_flag pooled[64];
  if (error == cudaSuccess && device >= 0 && device < 64) {
    std::call_once(pooled[device], [device] {
      cudaMemPool_t pool = nullptr;
      if (cudaDeviceGetDefaultMemPool(&pool, device) == cudaSuccess) {
        std::uint64_t keep = UINT64_MAX;
        cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
      }
    });
  }
  return true;
}

// A CUDA stream of the call's own.
struct Stream {
  cudaStream_t stream = nullptr;
  cudaError_t error = cudaSuccess;
  Stream() { error = cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking); }
  ~Stream() {
    if (stream != nullptr) cudaStreamDestroy(stream);
  }
};

bool inputs_of(const unround_input* input, std::vector<urb::ComponentInput>& out, urb::Failure& failure) {
  if (input->components == nullptr || input->count == 0) {
    failure = {urb::kArgument, "components are given"};
    return false;
  }
  for (std::uint32_t c = 0; c < input->count; ++c) {
    const unround_component& given = input->components[c];
    if (given.levels == nullptr) {
      failure = {urb::kArgument, "a component's levels are a null pointer"};
      return false;
    }
    urb::ComponentInput in;
    in.levels = given.levels;
    in.rows = given.rows;
    in.columns = given.columns;
    in.h = given.h_samp_factor;
    in.v = given.v_samp_factor;
    for (int k = 0; k < 64; ++k) in.table[k] = given.quant_table[k];
    out.push_back(in);
  }
  return true;
}

using urb::kB;
using urb::kCb;
using urb::kCr;
using urb::kG;
using urb::kGb;
using urb::kGr;
using urb::kR;
using urb::kToCb;
using urb::kToCr;

void to_rgb(const double* planes, std::size_t size, double* picture) {
  for (std::size_t k = 0; k < size; ++k) {
    const double y = planes[k], cb = planes[size + k] - 128.0, cr = planes[2 * size + k] - 128.0;
    picture[3 * k] = y + kCr * cr;
    picture[3 * k + 1] = (y - kGb * cb) - kGr * cr;
    picture[3 * k + 2] = y + kCb * cb;
  }
}

void to_ycbcr(const double* picture, std::size_t size, double* planes) {
  for (std::size_t k = 0; k < size; ++k) {
    const double r = picture[3 * k], g = picture[3 * k + 1], b = picture[3 * k + 2];
    const double y = (kR * r + kG * g) + kB * b;
    planes[k] = y;
    planes[size + k] = 128.0 + kToCb * (b - y);
    planes[2 * size + k] = 128.0 + kToCr * (r - y);
  }
}

// The projection of a picture made elsewhere onto a frame's intervals (docs/math.md 12;
// cpp/src/picture.cpp:70-148, rust/unround/src/picture.rs:130), on the host in binary64. The
// canvas is made as an encoder makes the file's: of a file in YCbCr JFIF's YCbCr of the picture's
// RGB, of a grey or RGB file its own channels, each extended over the canvas's whole MCUs by
// repeating its last column and then its last row. Then channel by channel and block by block:
// the cell means (each cell's samples summed down its columns, those sums across, divided by the
// cell's samples), their DCT e (rows, then columns), each coefficient's excess
// max(0, a - e, e - b) / Q, zeta = clip(e, a, b), and the canvas moved: with cells of one sample
// the inverse DCT of zeta, else each cell's samples by the change of its mean; the samples beyond
// the blocks as they are. Into `out` (the projected canvas, zeta, the planes and the picture)
// and `excess` (component by component, 64 a block).
bool project_picture(const urb::Frame& frame, const double* picture, urb::Outcome& out,
                     std::vector<std::vector<double>>& excess, urb::Failure& failure) {
  const std::size_t height = frame.height, width = frame.width, rows = frame.rows, columns = frame.columns;
  const std::size_t channels = frame.channels(), count = height * width, plane = frame.plane();
  const std::size_t given = frame.color_space == 1 ? 1 : 3;
  for (std::size_t k = 0; k < count * given; ++k) {
    if (!std::isfinite(picture[k])) {
      failure = {urb::kOptions, "a picture's samples are finite"};
      return false;
    }
  }
  std::vector<double> planes(channels * count);
  if (frame.color_space == 2) {
    to_ycbcr(picture, count, planes.data());
  } else {
    for (std::size_t k = 0; k < count; ++k) {
      for (std::size_t c = 0; c < channels; ++c) planes[c * count + k] = picture[k * given + c];
    }
  }
  out.canvas.resize(channels * plane);
  double* canvas = out.canvas.data();
  for (std::size_t c = 0; c < channels; ++c) {
    double* grid = canvas + c * plane;
    for (std::size_t i = 0; i < rows; ++i) {
      const double* from = planes.data() + c * count + std::min(i, height - 1) * width;
      double* to = grid + i * columns;
      std::copy(from, from + width, to);
      std::fill(to + width, to + columns, from[width - 1]);
    }
  }
  double basis[8][8];
  for (int k = 0; k < 8; ++k) {
    for (int n = 0; n < 8; ++n) basis[k][n] = urb::basis(k, n);
  }
  excess.assign(channels, {});
  out.coefficients.clear();
  for (std::size_t c = 0; c < channels; ++c) {
    const urb::Component& comp = frame.components[c];
    const std::size_t down = comp.cell_rows, across = comp.cell_columns;
    const double cells = static_cast<double>(down * across);
    double* grid = canvas + c * plane;
    std::vector<double>& beyond = excess[c];
    beyond.assign(comp.coefficient_count(), 0.0);
    urb::HostBuffer kept;
    kept.resize(comp.coefficient_count());
    for (std::size_t by = 0; by < comp.block_rows; ++by) {
      for (std::size_t bx = 0; bx < comp.block_columns; ++bx) {
        // The block's samples of the component: the cell means.
        double m[8][8];
        for (std::size_t y = 0; y < 8; ++y) {
          for (std::size_t x = 0; x < 8; ++x) {
            const std::size_t i0 = (8 * by + y) * down, j0 = (8 * bx + x) * across;
            double total = 0.0;
            for (std::size_t b = 0; b < across; ++b) {
              double column = grid[i0 * columns + j0 + b];
              for (std::size_t a = 1; a < down; ++a) column += grid[(i0 + a) * columns + j0 + b];
              total = b == 0 ? column : total + column;
            }
            m[y][x] = cells == 1.0 ? total : total / cells;
          }
        }
        double t[8][8], e[8][8];
        for (int y = 0; y < 8; ++y) {
          for (int u = 0; u < 8; ++u) {
            double sum = 0.0;
            for (int x = 0; x < 8; ++x) sum += basis[u][x] * m[y][x];
            t[y][u] = sum;
          }
        }
        for (int v = 0; v < 8; ++v) {
          for (int u = 0; u < 8; ++u) {
            double sum = 0.0;
            for (int y = 0; y < 8; ++y) sum += basis[v][y] * t[y][u];
            e[v][u] = sum;
          }
        }
        const std::size_t block = by * comp.block_columns + bx;
        const std::int16_t* levels = comp.levels.data() + block * 64;
        double z[8][8];
        for (int k = 0; k < 64; ++k) {
          const double value = e[k / 8][k % 8];
          const double low = comp.lower(levels[k], k), high = comp.upper(levels[k], k);
          beyond[block * 64 + k] = std::max(std::max(low - value, value - high), 0.0) / comp.steps[k];
          z[k / 8][k % 8] = std::min(std::max(value, low), high);
          kept.data()[block * 64 + k] = z[k / 8][k % 8];
        }
        for (int y = 0; y < 8; ++y) {
          for (int u = 0; u < 8; ++u) {
            double sum = 0.0;
            for (int v = 0; v < 8; ++v) sum += basis[v][y] * z[v][u];
            t[y][u] = sum;
          }
        }
        for (std::size_t y = 0; y < 8; ++y) {
          for (std::size_t x = 0; x < 8; ++x) {
            double back = 0.0;
            for (int u = 0; u < 8; ++u) back += basis[u][x] * t[y][u];
            const std::size_t i0 = (8 * by + y) * down, j0 = (8 * bx + x) * across;
            if (cells == 1.0) {
              grid[i0 * columns + j0] = back;
            } else {
              const double change = back - m[y][x];
              for (std::size_t a = 0; a < down; ++a) {
                for (std::size_t b = 0; b < across; ++b) grid[(i0 + a) * columns + j0 + b] += change;
              }
            }
          }
        }
      }
    }
    out.coefficients.push_back(std::move(kept));
  }
  // The planes cut to the picture, and of colour the picture interleaved (of YCbCr, its RGB).
  if (height != rows || width != columns) {
    out.planes.resize(channels * count);
    for (std::size_t c = 0; c < channels; ++c) {
      for (std::size_t i = 0; i < height; ++i) {
        std::copy(canvas + c * plane + i * columns, canvas + c * plane + i * columns + width,
                  out.planes.data() + c * count + i * width);
      }
    }
  }
  if (channels == 3) {
    const double* cut = out.planes.empty() ? canvas : out.planes.data();
    out.picture.resize(3 * count);
    if (frame.color_space == 2) {
      to_rgb(cut, count, out.picture.data());
    } else {
      for (std::size_t k = 0; k < count; ++k) {
        for (std::size_t c = 0; c < 3; ++c) out.picture.data()[3 * k + c] = cut[c * count + k];
      }
    }
  }
  out.iterations = 0;
  out.stop = 0;
  out.solved = false;
  return true;
}

// The result of a solve (rust/unround/src/decode.rs:306-364): the canvas cut to the picture,
// and of YCbCr its JFIF RGB, interleaved.
unround_result* result_of(urb::Frame&& frame, urb::Outcome&& outcome) {
  auto* made = new unround_result;
  made->frame = std::move(frame);
  made->outcome = std::move(outcome);
  const urb::Frame& f = made->frame;
  made->height = f.height;
  made->width = f.width;
  made->channels = f.color_space == 2 ? 3 : f.channels();
  for (const urb::Record& r : made->outcome.records) {
    made->record_iterations.push_back(r.iteration);
    made->record_values[0].push_back(r.seconds);
    made->record_values[1].push_back(r.primal);
    made->record_values[2].push_back(r.dual);
    made->record_values[3].push_back(r.scaling);
    made->record_values[4].push_back(r.partial_gap);
  }
  for (const urb::Component& c : f.components) {
    made->steps.emplace_back(c.steps.begin(), c.steps.end());
    made->weights.emplace_back(c.weights.begin(), c.weights.end());
  }
  return made;
}

// The samples of a picture of height x width pixels of 1 to 4 interleaved channels, counted
// (rust/capi/src/lib.rs:1259-1269; rust/unround/src/output.rs:232-246).
bool picture_count(const double* samples, std::uint64_t height, std::uint64_t width, std::uint64_t channels,
                   std::size_t& count, urb::Failure& failure) {
  const std::uint64_t limit = std::numeric_limits<std::uint64_t>::max();
  if ((width != 0 && height > limit / width) || (channels != 0 && height * width > limit / channels)) {
    failure = {urb::kArgument, "a picture too large"};
    return false;
  }
  if (samples == nullptr) {
    failure = {urb::kArgument, "the samples are a null pointer"};
    return false;
  }
  count = static_cast<std::size_t>(height * width * channels);
  if (channels < 1 || channels > 4 || height == 0 || width == 0 || width > (1u << 30)) {
    failure = {urb::kOptions, "a picture of " + std::to_string(height) + " x " + std::to_string(width) +
                                  " x 1 to 4 samples, not empty, and not of " + std::to_string(count) + " samples in " +
                                  std::to_string(channels) + " channels"};
    return false;
  }
  return true;
}

// The 8- or 16-bit levels of the samples (output.cu), into `out` (count bytes, or 2 count
// most significant byte first): the samples copied to the device, quantized there, and the
// levels copied back; where a sample is not finite, the first such is named and nothing is
// made (rust/unround/src/output.rs:220-230).
bool quantize(const double* samples, std::size_t count, int width, int channels, bool sixteen, int dither,
              std::uint8_t* out, urb::Failure& failure) {
  if (!have_device(failure)) return false;
  if (!urb::prepare_levels()) {
    failure = {urb::kInternal, "the blue-noise matrix could not be loaded onto the device"};
    return false;
  }
  Stream stream;
  cudaError_t error = stream.error;
  const std::size_t out_bytes = count * (sixteen ? 2 : 1);
  void* block = nullptr;
  const std::size_t in_bytes = (count * sizeof(double) + 255) / 256 * 256;
  if (error == cudaSuccess) error = cudaMallocAsync(&block, in_bytes + (out_bytes + 255) / 256 * 256 + 256, stream.stream);
  auto* in = static_cast<double*>(block);
  auto* levels = static_cast<std::uint8_t*>(block) + in_bytes;
  auto* flag = reinterpret_cast<int*>(levels + (out_bytes + 255) / 256 * 256);
  int not_finite = 0;
  if (error == cudaSuccess) error = cudaMemcpyAsync(in, samples, count * sizeof(double), cudaMemcpyHostToDevice, stream.stream);
  if (error == cudaSuccess) error = cudaMemsetAsync(flag, 0, sizeof(int), stream.stream);
  urb::LevelsParams p;
  p.samples = in;
  p.count = count;
  p.width = width;
  p.channels = channels;
  p.scale = sixteen ? 257.0 : 1.0;
  p.top = sixteen ? 65535.0 : 255.0;
  p.dither = dither;
  p.sixteen = sixteen;
  p.out = levels;
  p.not_finite = flag;
  if (error == cudaSuccess) error = urb::launch_levels(p, stream.stream);
  if (error == cudaSuccess) error = cudaMemcpyAsync(&not_finite, flag, sizeof(int), cudaMemcpyDeviceToHost, stream.stream);
  if (error == cudaSuccess) error = cudaMemcpyAsync(out, levels, out_bytes, cudaMemcpyDeviceToHost, stream.stream);
  if (block != nullptr) cudaFreeAsync(block, stream.stream);
  const cudaError_t synced = cudaStreamSynchronize(stream.stream);
  if (error == cudaSuccess) error = synced;
  if (error != cudaSuccess) {
    failure = {urb::kInternal, std::string("the device failed in the levels: ") + cudaGetErrorString(error)};
    return false;
  }
  if (not_finite != 0) {
    double first = std::numeric_limits<double>::quiet_NaN();
    for (std::size_t k = 0; k < count; ++k) {
      if (!std::isfinite(samples[k])) {
        first = samples[k];
        break;
      }
    }
    failure = {urb::kOptions, std::string("a sample to quantize is not finite: ") +
                                  (std::isnan(first) ? "NaN" : (first > 0 ? "inf" : "-inf"))};
    return false;
  }
  return true;
}

bool solve_input(const unround_input* input, const unround_settings* settings, const urb::Start* start,
                 unround_observer observer, void* user, unround_result** result, urb::Failure& failure,
                 const unround_b200_start* given) {
  if (input == nullptr || settings == nullptr || result == nullptr) {
    failure = {urb::kArgument, "the input, the settings and the result are not null pointers"};
    return false;
  }
  std::vector<urb::ComponentInput> inputs;
  if (!inputs_of(input, inputs, failure)) return false;
  const urb::Settings& s = settings->settings;
  auto frame = urb::make_frame(input->height, input->width, input->color_space, inputs, s, failure);
  if (!frame) return false;
  if (s.method == urb::Method::subgradient) {
    failure = {urb::kUnsupported,
               "the subgradient method (docs/math.md 7) is not on this build's path: use mmse, tv or tgv"};
    return false;
  }
  std::optional<urb::Plan> plan;
  if (s.method != urb::Method::mmse) {
    plan = urb::make_plan(s, frame->channels(), failure);
    if (!plan) return false;
  }
  urb::Start owned_start;
  if (given != nullptr) {
    const std::size_t plane = frame->plane(), channels = frame->channels();
    if (given->coefficients != nullptr) {
      std::size_t offset = 0;
      for (const urb::Component& c : frame->components) {
        owned_start.coefficients.emplace_back(given->coefficients + offset,
                                              given->coefficients + offset + c.coefficient_count());
        offset += c.coefficient_count();
      }
    }
    if (given->p != nullptr) owned_start.p.assign(given->p, given->p + 2 * channels * plane);
    if (given->w != nullptr) owned_start.w.assign(given->w, given->w + 2 * channels * plane);
    if (given->r != nullptr) owned_start.r.assign(given->r, given->r + 3 * channels * plane);
    start = &owned_start;
  }
  if (!have_device(failure)) return false;
  Stream stream;
  if (stream.error != cudaSuccess) {
    failure = {urb::kInternal, std::string("a CUDA stream: ") + cudaGetErrorString(stream.error)};
    return false;
  }
  urb::Outcome outcome;
  {
    urb::Solver solver(*frame, stream.stream);
    urb::Observer watch;
    if (observer != nullptr) {
      const std::uint64_t channels = frame->channels(), rows = frame->rows, columns = frame->columns;
      watch = [&](const urb::Record& r, double gap, const double* canvas) {
        unround_record raw{r.iteration, gap, r.primal, r.dual, channels, rows, columns, canvas};
        return observer(user, &raw) != 0;
      };
    }
    if (!solver.solve(s.method, plan ? &*plan : nullptr, start, watch, outcome, failure)) return false;
  }
  *result = result_of(std::move(*frame), std::move(outcome));
  return true;
}

}  // namespace

// The solve of unround_b200_solve_samples, and of a PNG file's levels in unround_decode: the
// result's format is PNG, of the levels' bits.
static bool solve_samples_into(const uint16_t* levels, uint64_t rows, uint64_t columns, uint64_t channels, int32_t bits,
                               const unround_settings* settings, unround_observer observer, void* user,
                               unround_result** result, urb::Failure& failure) {
  if (levels == nullptr || settings == nullptr || result == nullptr) {
    failure = {urb::kArgument, "the levels, the settings and the result are not null pointers"};
    return false;
  }
  if (channels < 1 || channels > 4 || rows == 0 || columns == 0 || rows > (1u << 24) || columns > (1u << 24)) {
    failure = {urb::kOptions, "a picture of " + std::to_string(rows) + " x " + std::to_string(columns) + " x " +
                                  std::to_string(channels) + " samples: 1 to 4 channels, not empty"};
    return false;
  }
  const urb::Settings& s = settings->settings;
  if (!urb::check_samples_settings(s, failure)) return false;
  const urb::DataTerm& term = s.data.front();
  const double mu = term.mu ? *term.mu : 0.0;
  const bool alpha = channels == 2 || channels == 4;
  const std::size_t colours = alpha ? channels - 1 : channels;
  auto colour_model = urb::make_samples_model(levels, rows, columns, channels, bits, 0, colours, term.slack, mu,
                                              failure);
  if (!colour_model) return false;
  std::optional<urb::SamplesModel> alpha_model;
  if (alpha) {
    alpha_model = urb::make_samples_model(levels, rows, columns, channels, bits, colours, 1, term.slack, mu, failure);
    if (!alpha_model) return false;
  }
  auto plan = urb::make_plan(s, colours, failure, urb::samples_plan_defaults());
  if (!plan) return false;
  urb::Settings alone = s;
  alone.regularizer.channel_weights.clear();
  std::optional<urb::Plan> alpha_plan;
  if (alpha) {
    alpha_plan = urb::make_plan(alone, 1, failure, urb::samples_plan_defaults());
    if (!alpha_plan) return false;
  }
  if (!have_device(failure)) return false;
  // The solvers' frame: the picture's size and colours, no components (the samples are the
  // data term); the result's gets a component (with no blocks) per channel.
  urb::Frame frame;
  frame.height = static_cast<std::uint32_t>(rows);
  frame.width = static_cast<std::uint32_t>(columns);
  frame.rows = static_cast<std::uint32_t>(rows);
  frame.columns = static_cast<std::uint32_t>(columns);
  frame.color_space = colours == 3 ? 3 : 1;
  urb::Observer watch;
  if (observer != nullptr) {
    watch = [&](const urb::Record& r, double gap, const double* canvas) {
      unround_record raw{r.iteration, gap, r.primal, r.dual, colours, rows, columns, canvas};
      return observer(user, &raw) != 0;
    };
  }
  Stream stream;
  if (stream.error != cudaSuccess) {
    failure = {urb::kInternal, std::string("a CUDA stream: ") + cudaGetErrorString(stream.error)};
    return false;
  }
  urb::Outcome outcome;
  {
    urb::Solver solver(frame, *colour_model, stream.stream);
    if (!solver.solve(s.method, &*plan, nullptr, watch, outcome, failure)) return false;
  }
  if (!alpha) {
    frame.components.resize(colours);
    *result = result_of(std::move(frame), std::move(outcome));
    (*result)->format = UNROUND_FORMAT_PNG;
    (*result)->bits = bits;
    return true;
  }
  urb::Frame alpha_frame = frame;
  alpha_frame.color_space = 1;
  urb::Outcome alpha_outcome;
  {
    urb::Solver solver(alpha_frame, *alpha_model, stream.stream);
    if (!solver.solve(s.method, &*alpha_plan, nullptr, watch, alpha_outcome, failure)) return false;
  }
  // The colours' planes and the alpha's, and the picture interleaved, in one result.
  const std::size_t plane = static_cast<std::size_t>(rows) * columns;
  urb::Outcome merged;
  merged.canvas.resize(channels * plane);
  std::memcpy(merged.canvas.data(), outcome.canvas.data(), colours * plane * sizeof(double));
  std::memcpy(merged.canvas.data() + colours * plane, alpha_outcome.canvas.data(), plane * sizeof(double));
  merged.picture.resize(channels * plane);
  for (std::size_t k = 0; k < plane; ++k) {
    for (std::size_t c = 0; c < channels; ++c) merged.picture.data()[k * channels + c] = merged.canvas.data()[c * plane + k];
  }
  merged.records = std::move(outcome.records);
  merged.iterations = outcome.iterations;
  merged.stop = outcome.stop;
  merged.solved = outcome.solved;
  merged.tau = outcome.tau;
  merged.sigma = outcome.sigma;
  frame.components.resize(channels);
  frame.color_space = colours == 3 ? 3 : 1;
  *result = result_of(std::move(frame), std::move(merged));
  (*result)->format = UNROUND_FORMAT_PNG;
  (*result)->bits = bits;
  return true;
}

extern "C" {

int32_t unround_abi_version(void) { return UNROUND_ABI_VERSION; }

const char* unround_version(void) { return kVersion; }

unround_settings* unround_settings_new(size_t count, const char* const* options, char* message, size_t message_size) {
  unround_settings* made = nullptr;
  guarded(message, message_size, [&](urb::Failure& failure) {
    std::vector<std::string> arguments;
    if (count > 0 && options == nullptr) {
      failure = {urb::kArgument, "the strings are a null pointer"};
      return false;
    }
    for (std::size_t i = 0; i < count; ++i) {
      if (options[i] == nullptr) {
        failure = {urb::kArgument, "a string is a null pointer"};
        return false;
      }
      arguments.emplace_back(options[i]);
    }
    auto* settings = new unround_settings;
    std::string errors;
    if (!urb::parse_settings(arguments, settings->settings, errors)) {
      delete settings;
      failure = {urb::kOptions, errors};
      return false;
    }
    made = settings;
    return true;
  });
  return made;
}

void unround_settings_free(unround_settings* settings) { delete settings; }

size_t unround_settings_options(const unround_settings* settings, char* buffer, size_t size) {
  if (settings == nullptr) return 0;
  try {
    std::string text;
    for (const std::string& option : urb::options_of(settings->settings)) text += (text.empty() ? "" : " ") + option;
    say(buffer, size, text);
    return text.size();
  } catch (...) {
    return 0;
  }
}

// A file reconstructed (rust/capi/src/lib.rs, unround_decode; rust/unround/src/decode.rs and
// rounded.rs): a PNG file, known by its signature, within the intervals of its rounded samples
// (the levels read on the host, solved as unround_b200_solve_samples does); any other file as a
// JPEG file, its coefficients read on the host (jpeg_reader.hpp) and solved as unround_solve
// does. The reading's refusals map as the reference maps them: UNSUPPORTED stays, a limit is
// OPTIONS, anything else READ.
unround_status unround_decode(const uint8_t* data, size_t size, const unround_settings* settings,
                              unround_observer observer, void* user, unround_result** result, char* message,
                              size_t message_size) {
  return guarded(message, message_size, [&](urb::Failure& failure) {
    if (data == nullptr || settings == nullptr || result == nullptr) {
      failure = {urb::kArgument, "the data, the settings and the result are not null pointers"};
      return false;
    }
    const urb::Settings& s = settings->settings;
    auto read_failure = [&](int status, const std::string& text) {
      const urb::Status mapped = status == urb::kJpegUnsupported ? urb::kUnsupported
                                  : status == urb::kJpegLimit     ? urb::kOptions
                                                                  : urb::kRead;
      failure = {mapped, text};
      return false;
    };
    if (urb::is_png(data, size)) {
      urb::PngPicture picture;
      std::string text;
      const int status = urb::read_png(data, size, s.reading.max_pixels, picture, text);
      if (status != urb::kPngOk) return read_failure(status, text);
      if (!solve_samples_into(picture.samples.data(), picture.height, picture.width,
                              static_cast<std::uint64_t>(picture.channels), picture.bits, settings, observer, user,
                              result, failure)) {
        return false;
      }
      (*result)->icc = std::move(picture.icc);
      (*result)->warning = picture.warning;
      return true;
    }
    urb::JpegLimits limits;
    limits.max_pixels = s.reading.max_pixels;
    limits.max_scans = s.reading.max_scans;
    limits.warnings_are_errors = s.reading.warnings_are_errors;
    urb::JpegFile file;
    std::string text;
    const int status = urb::read_jpeg(data, size, limits, file, text);
    if (status != urb::kJpegOk) return read_failure(status, text);
    std::vector<unround_component> components(file.components.size());
    for (std::size_t c = 0; c < components.size(); ++c) {
      const urb::JpegComponent& from = file.components[c];
      unround_component& to = components[c];
      to.levels = from.coefficients.data();
      to.rows = from.height_in_blocks;
      to.columns = from.width_in_blocks;
      to.h_samp_factor = from.h;
      to.v_samp_factor = from.v;
      std::copy(from.table, from.table + 64, to.quant_table);
    }
    unround_input input{file.height, file.width, file.color_space, static_cast<std::uint32_t>(components.size()),
                        components.data()};
    if (!solve_input(&input, settings, nullptr, observer, user, result, failure, nullptr)) return false;
    (*result)->exif_orientation = file.exif_orientation;
    (*result)->icc = std::move(file.icc);
    (*result)->warning = file.warning;
    return true;
  });
}

unround_status unround_solve(const unround_input* input, const unround_settings* settings, unround_observer observer,
                             void* user, unround_result** result, char* message, size_t message_size) {
  return guarded(message, message_size, [&](urb::Failure& failure) {
    return solve_input(input, settings, nullptr, observer, user, result, failure, nullptr);
  });
}

unround_status unround_b200_solve_from(const unround_input* input, const unround_settings* settings,
                                       const unround_b200_start* start, unround_observer observer, void* user,
                                       unround_result** result, char* message, size_t message_size) {
  return guarded(message, message_size, [&](urb::Failure& failure) {
    return solve_input(input, settings, nullptr, observer, user, result, failure, start);
  });
}

unround_status unround_b200_measure(const unround_input* input, const unround_settings* settings, uint64_t warmup,
                                    uint64_t iterations, unround_b200_timing* timing, unround_result** result,
                                    char* message, size_t message_size) {
  return guarded(message, message_size, [&](urb::Failure& failure) {
    if (input == nullptr || settings == nullptr || timing == nullptr) {
      failure = {urb::kArgument, "the input, the settings and the timing are not null pointers"};
      return false;
    }
    std::vector<urb::ComponentInput> inputs;
    if (!inputs_of(input, inputs, failure)) return false;
    const urb::Settings& s = settings->settings;
    if (s.method != urb::Method::tv && s.method != urb::Method::tgv) {
      failure = {urb::kOptions, "the measurement is of the primal-dual methods, tv or tgv"};
      return false;
    }
    auto frame = urb::make_frame(input->height, input->width, input->color_space, inputs, s, failure);
    if (!frame) return false;
    auto plan = urb::make_plan(s, frame->channels(), failure);
    if (!plan) return false;
    if (!have_device(failure)) return false;
    Stream stream;
    urb::Outcome outcome;
    {
      urb::Solver solver(*frame, stream.stream);
      if (!solver.prepare(*plan, failure)) return false;
      if (warmup > 0 && !solver.iterate(warmup, failure)) return false;
      cudaEvent_t begin, end;
      cudaEventCreate(&begin);
      cudaEventCreate(&end);
      cudaStreamSynchronize(stream.stream);
      cudaEventRecord(begin, stream.stream);
      const bool ok = solver.iterate(iterations, failure);
      cudaEventRecord(end, stream.stream);
      cudaEventSynchronize(end);
      float ms = 0.0f;
      cudaEventElapsedTime(&ms, begin, end);
      cudaEventDestroy(begin);
      cudaEventDestroy(end);
      if (!ok) return false;
      double dual_ms = 0.0, primal_ms = 0.0;
      if (!solver.breakdown(20, dual_ms, primal_ms, failure)) return false;
      timing->milliseconds = ms;
      timing->dual_milliseconds = dual_ms;
      timing->primal_milliseconds = primal_ms;
      timing->iterations = iterations;
      timing->launches_per_iteration = static_cast<std::uint64_t>(solver.launches_per_iteration());
      timing->samples = static_cast<std::uint64_t>(frame->channels()) * frame->rows * frame->columns;
      timing->pixels = static_cast<std::uint64_t>(frame->rows) * frame->columns;
      timing->device_bytes = solver.device_bytes();
      if (result != nullptr) {
        if (!solver.finish(outcome, failure)) return false;
        outcome.solved = true;
        outcome.iterations = warmup + iterations + 20;
        outcome.stop = 2;
        outcome.tau = plan->tau;
        outcome.sigma = plan->sigma;
      }
    }
    if (result != nullptr) *result = result_of(std::move(*frame), std::move(outcome));
    return true;
  });
}

unround_status unround_b200_solve_batch(uint64_t count, const unround_input* inputs,
                                        const unround_settings* const* settings, unround_result** results,
                                        unround_b200_batch_timing* timing, char* message, size_t message_size) {
  return guarded(message, message_size, [&](urb::Failure& failure) {
    if (count == 0 || inputs == nullptr || settings == nullptr || results == nullptr) {
      failure = {urb::kArgument, "a batch has pictures, settings and result slots (not null pointers)"};
      return false;
    }
    for (uint64_t n = 0; n < count; ++n) results[n] = nullptr;
    std::vector<urb::Frame> frames;
    frames.reserve(count);
    std::vector<urb::BatchEntry> entries;
    for (uint64_t n = 0; n < count; ++n) {
      if (settings[n] == nullptr) {
        failure = {urb::kArgument, "picture " + std::to_string(n) + " has no settings"};
        return false;
      }
      const urb::Settings& s = settings[n]->settings;
      if (s.method != urb::Method::tv && s.method != urb::Method::tgv) {
        failure = {urb::kOptions, "picture " + std::to_string(n) + ": a batch solves by tv or tgv"};
        return false;
      }
      std::vector<urb::ComponentInput> components;
      if (!inputs_of(&inputs[n], components, failure)) return false;
      auto frame = urb::make_frame(inputs[n].height, inputs[n].width, inputs[n].color_space, components, s, failure);
      if (!frame) {
        failure.message = "picture " + std::to_string(n) + ": " + failure.message;
        return false;
      }
      frames.push_back(std::move(*frame));
      auto plan = urb::make_plan(s, frames.back().channels(), failure);
      if (!plan) {
        failure.message = "picture " + std::to_string(n) + ": " + failure.message;
        return false;
      }
      entries.push_back({&frames.back(), *plan});
    }
    if (!urb::check_batch(entries, failure)) return false;
    if (!have_device(failure)) return false;
    Stream stream;
    if (stream.error != cudaSuccess) {
      failure = {urb::kInternal, std::string("a CUDA stream: ") + cudaGetErrorString(stream.error)};
      return false;
    }
    std::vector<urb::Outcome> outcomes;
    urb::BatchTiming measured;
    if (!urb::solve_batch(entries, stream.stream, outcomes, measured, failure)) return false;
    if (timing != nullptr) {
      timing->milliseconds = measured.milliseconds;
      timing->iterations = measured.iterations;
      timing->launches_per_iteration = measured.launches_per_iteration;
      timing->samples = measured.samples;
      timing->pixels = measured.pixels;
      timing->tuning_milliseconds = measured.tuning_milliseconds;
    }
    for (uint64_t n = 0; n < count; ++n) results[n] = result_of(std::move(frames[n]), std::move(outcomes[n]));
    return true;
  });
}

unround_status unround_b200_model(const unround_input* input, const unround_settings* settings, uint64_t component,
                                  int32_t which, double* out, uint64_t capacity, uint64_t* count, char* message,
                                  size_t message_size) {
  return guarded(message, message_size, [&](urb::Failure& failure) {
    if (input == nullptr || settings == nullptr) {
      failure = {urb::kArgument, "the input and the settings are not null pointers"};
      return false;
    }
    std::vector<urb::ComponentInput> inputs;
    if (!inputs_of(input, inputs, failure)) return false;
    const urb::Settings& s = settings->settings;
    auto frame = urb::make_frame(input->height, input->width, input->color_space, inputs, s, failure);
    if (!frame) return false;
    if (component >= frame->channels() || which < 0 || which > 7) {
      failure = {urb::kArgument, "no such component or value of the model"};
      return false;
    }
    const urb::Component& c = frame->components[component];
    std::vector<double> values;
    if (which <= 2) {
      values.resize(c.coefficient_count());
      for (std::size_t at = 0; at < values.size(); ++at) {
        const int k = static_cast<int>(at % 64);
        values[at] = which == 0 ? c.lower(c.levels[at], k) : which == 1 ? c.upper(c.levels[at], k)
                                                                          : c.centre(c.levels[at], k);
      }
    } else if (which == 3) {
      values.assign(c.steps.begin(), c.steps.end());
    } else if (which == 4) {
      values.assign(c.weights.begin(), c.weights.end());
    } else if (which == 5) {
      values.assign(c.flat_weights.begin(), c.flat_weights.end());
    } else if (which == 6) {
      values.assign(c.flat.begin(), c.flat.end());
    } else {
      if (s.method != urb::Method::tv && s.method != urb::Method::tgv) {
        failure = {urb::kOptions, "a plan is of the primal-dual methods, tv or tgv"};
        return false;
      }
      auto plan = urb::make_plan(s, frame->channels(), failure);
      if (!plan) return false;
      values = {plan->tau, plan->sigma, static_cast<double>(plan->iterations), plan->tolerance};
    }
    if (count != nullptr) *count = values.size();
    if (out != nullptr) std::copy_n(values.begin(), std::min<std::size_t>(values.size(), capacity), out);
    return true;
  });
}

// A picture made elsewhere measured against a JPEG file's intervals and projected onto them
// (rust/capi/src/lib.rs, unround_project; docs/math.md 12): the file's coefficients read on the
// host as unround_decode reads them, its frame with the settings' slack, and the projection of
// project_picture. The picture is the file's size as it stores it, grey or RGB.
unround_status unround_project(const uint8_t* data, size_t size, const unround_settings* settings,
                               const double* picture, uint64_t height, uint64_t width, uint64_t channels,
                               unround_result** result, char* message, size_t message_size) {
  return guarded(message, message_size, [&](urb::Failure& failure) {
    if (data == nullptr || settings == nullptr || picture == nullptr || result == nullptr) {
      failure = {urb::kArgument, "the data, the settings, the picture and the result are not null pointers"};
      return false;
    }
    const urb::Settings& s = settings->settings;
    urb::JpegLimits limits;
    limits.max_pixels = s.reading.max_pixels;
    limits.max_scans = s.reading.max_scans;
    limits.warnings_are_errors = s.reading.warnings_are_errors;
    urb::JpegFile file;
    std::string text;
    const int status = urb::read_jpeg(data, size, limits, file, text);
    if (status != urb::kJpegOk) {
      failure = {status == urb::kJpegUnsupported ? urb::kUnsupported : status == urb::kJpegLimit ? urb::kOptions
                                                                                                 : urb::kRead,
                 text};
      return false;
    }
    const std::uint64_t expected = file.color_space == 1 ? 1 : 3;
    if (height != file.height || width != file.width || channels != expected) {
      failure = {urb::kOptions, "a picture of the file is " + std::to_string(file.height) + " x " +
                                    std::to_string(file.width) + " x " + std::to_string(expected) + " samples, not " +
                                    std::to_string(height) + " x " + std::to_string(width) + " x " +
                                    std::to_string(channels)};
      return false;
    }
    std::vector<urb::ComponentInput> inputs;
    for (const urb::JpegComponent& c : file.components) {
      urb::ComponentInput in;
      in.levels = c.coefficients.data();
      in.rows = c.height_in_blocks;
      in.columns = c.width_in_blocks;
      in.h = c.h;
      in.v = c.v;
      std::copy(c.table, c.table + 64, in.table.begin());
      inputs.push_back(in);
    }
    auto frame = urb::make_frame(file.height, file.width, file.color_space, inputs, s, failure);
    if (!frame) return false;
    urb::Outcome outcome;
    std::vector<std::vector<double>> excess;
    if (!project_picture(*frame, picture, outcome, excess, failure)) return false;
    *result = result_of(std::move(*frame), std::move(outcome));
    (*result)->excess = std::move(excess);
    (*result)->exif_orientation = file.exif_orientation;
    (*result)->icc = std::move(file.icc);
    (*result)->warning = file.warning;
    return true;
  });
}

void unround_result_free(unround_result* result) { delete result; }

static void put(uint64_t* target, uint64_t value) {
  if (target != nullptr) *target = value;
}

const double* unround_result_picture(const unround_result* result, uint64_t* height, uint64_t* width,
                                     uint64_t* channels) {
  if (result == nullptr) return nullptr;
  put(height, result->height);
  put(width, result->width);
  put(channels, result->channels);
  return result->picture();
}

const double* unround_result_planes(const unround_result* result, uint64_t* count) {
  if (result == nullptr) return nullptr;
  put(count, result->frame.channels() * result->height * result->width);
  return result->planes();
}

int32_t unround_result_color_space(const unround_result* result) {
  return result == nullptr ? 0 : result->frame.color_space;
}

const double* unround_result_canvas(const unround_result* result, uint64_t* channels, uint64_t* height,
                                    uint64_t* width) {
  if (result == nullptr) return nullptr;
  put(channels, result->frame.channels());
  put(height, result->frame.rows);
  put(width, result->frame.columns);
  return result->outcome.canvas.data();
}

uint64_t unround_result_components(const unround_result* result) {
  return result == nullptr ? 0 : result->frame.channels();
}

const double* unround_result_coefficients(const unround_result* result, uint64_t component, uint64_t* count) {
  if (result == nullptr || component >= result->outcome.coefficients.size()) return nullptr;
  put(count, result->outcome.coefficients[component].size());
  return result->outcome.coefficients[component].data();
}

const double* unround_result_problem(const unround_result* result, uint64_t component, int32_t which, uint64_t* count) {
  if (result == nullptr || component >= result->frame.channels() || which < 0 || which > 4) return nullptr;
  if (which == 3) {
    put(count, 64);
    return result->steps[component].data();
  }
  if (which == 4) {
    put(count, 64);
    return result->weights[component].data();
  }
  try {
    std::call_once(result->problem_once, [result] {
      // Blocks of coefficients shared out among the host's threads, each filling (and first
      // touching) its own part of the three arrays.
      const unsigned threads = std::max(1u, std::min(16u, std::thread::hardware_concurrency()));
      for (const urb::Component& c : result->frame.components) {
        const std::size_t n = c.coefficient_count();
        auto lower = std::make_unique_for_overwrite<double[]>(n);
        auto upper = std::make_unique_for_overwrite<double[]>(n);
        auto centres = std::make_unique_for_overwrite<double[]>(n);
        auto fill = [&](std::size_t first, std::size_t end) {
          for (std::size_t at = first; at < end; ++at) {
            const int k = static_cast<int>(at % 64);
            lower[at] = c.lower(c.levels[at], k);
            upper[at] = c.upper(c.levels[at], k);
            centres[at] = c.centre(c.levels[at], k);
          }
        };
        const std::size_t blocks = n / 64;
        // A thread a part of at least 512 blocks (about 0.2 ms of work), so that small pictures
        // are shared out too.
        const unsigned parts = static_cast<unsigned>(std::min<std::size_t>(threads, std::max<std::size_t>(blocks / 512, 1)));
        std::vector<std::thread> workers;
        for (unsigned t = 1; t < parts; ++t) {
          workers.emplace_back(fill, blocks * t / parts * 64, blocks * (t + 1) / parts * 64);
        }
        fill(0, blocks / parts * 64);
        for (std::thread& w : workers) w.join();
        result->problem[0].push_back(std::move(lower));
        result->problem[1].push_back(std::move(upper));
        result->problem[2].push_back(std::move(centres));
        result->problem_sizes.push_back(n);
      }
    });
  } catch (...) {
    return nullptr;
  }
  put(count, result->problem_sizes[component]);
  return result->problem[which][component].get();
}

unround_status unround_result_component(const unround_result* result, uint64_t component, uint64_t* rows,
                                        uint64_t* columns, uint64_t* down, uint64_t* across) {
  if (result == nullptr || component >= result->frame.channels()) return UNROUND_ERROR_ARGUMENT;
  const urb::Component& c = result->frame.components[component];
  put(rows, c.block_rows);
  put(columns, c.block_columns);
  put(down, c.cell_rows);
  put(across, c.cell_columns);
  return UNROUND_OK;
}

int32_t unround_result_solver(const unround_result* result, uint64_t* iterations, int32_t* stop) {
  if (result == nullptr || !result->outcome.solved) return 0;
  put(iterations, result->outcome.iterations);
  if (stop != nullptr) *stop = result->outcome.stop;
  return 1;
}

const uint64_t* unround_result_record_iterations(const unround_result* result, uint64_t* count) {
  if (result == nullptr || !result->outcome.solved) return nullptr;
  put(count, result->record_iterations.size());
  return result->record_iterations.data();
}

const double* unround_result_record_values(const unround_result* result, int32_t which, uint64_t* count) {
  if (result == nullptr || !result->outcome.solved || which < 0 || which > 4) return nullptr;
  put(count, result->record_values[which].size());
  return result->record_values[which].data();
}

int32_t unround_result_alpha_solver(const unround_result*, uint64_t*, int32_t*) { return 0; }
const uint64_t* unround_result_alpha_record_iterations(const unround_result*, uint64_t*) { return nullptr; }
const double* unround_result_alpha_record_values(const unround_result*, int32_t, uint64_t*) { return nullptr; }
const uint8_t* unround_result_icc_profile(const unround_result* result, uint64_t* size) {
  if (result == nullptr || result->icc.empty()) {
    put(size, 0);
    return nullptr;
  }
  put(size, result->icc.size());
  return result->icc.data();
}
int32_t unround_result_exif_orientation(const unround_result* result) {
  return result == nullptr ? 0 : result->exif_orientation;
}
int32_t unround_result_format(const unround_result* result) { return result == nullptr ? 0 : result->format; }
int32_t unround_result_bits(const unround_result* result) { return result == nullptr ? 0 : result->bits; }
const char* unround_result_warning(const unround_result* result) {
  return result == nullptr ? nullptr : result->warning.c_str();
}
const double* unround_result_excess(const unround_result* result, uint64_t component, uint64_t* count) {
  if (result == nullptr || component >= result->excess.size()) {
    put(count, 0);
    return nullptr;
  }
  put(count, result->excess[component].size());
  return result->excess[component].data();
}

// A TIFF of the picture's binary64 samples, bit for bit (rust/capi/src/lib.rs, unround_tiff; the
// TIFF 6.0 specification): little-endian, one uncompressed strip, the samples of a pixel together,
// SampleFormat IEEE floating point of 64 bits; grey (BlackIsZero) or RGB, with an alpha last
// declared unassociated (ExtraSamples 2); with ycbcr, three samples declared as JFIF's Y, Cb and
// Cr (YCbCrCoefficients 0.299, 0.587, 0.114; no subsampling; ReferenceBlackWhite 0-255 and
// 128-centred); the ICC profile (tag 34675) where it goes with the picture's colours (as
// unround_jpeg_check_icc checks it; of YCbCr, its RGB), otherwise left out and the message says why.
unround_status unround_tiff(const double* samples, uint64_t height, uint64_t width, uint64_t channels, int32_t ycbcr,
                            const uint8_t* icc, uint64_t icc_size, uint8_t** bytes, uint64_t* size, char* message,
                            size_t message_size) {
  std::string warning;
  const unround_status status = guarded(message, message_size, [&](urb::Failure& failure) {
    if (bytes == nullptr || size == nullptr) {
      failure = {urb::kArgument, "the bytes and the size are not null pointers"};
      return false;
    }
    std::size_t count = 0;
    if (!picture_count(samples, height, width, channels, count, failure)) return false;
    if (ycbcr != 0 && channels != 3) {
      failure = {urb::kOptions, "YCbCr is three samples a pixel, not " + std::to_string(channels)};
      return false;
    }
    const std::uint64_t data_bytes = static_cast<std::uint64_t>(count) * 8u;
    if (height > 0xFFFFFFFFull || width > 0xFFFFFFFFull || data_bytes > 0xFFFF0000ull) {
      failure = {urb::kOptions, "a TIFF of this build holds at most 4 GB of samples"};
      return false;
    }
    bool with_icc = false;
    if (icc != nullptr) {
      std::string reason;
      with_icc = urb::check_icc(icc, icc_size, static_cast<int>(channels), reason);
      if (!with_icc) warning = "the ICC profile is not written: " + reason;
    }
    // The IFD's entries (tag, type, count, value or offset), in tag order; values of more than
    // 4 bytes go after the IFD.
    struct Entry {
      std::uint16_t tag, type;
      std::uint32_t count;
      std::vector<std::uint8_t> value;
    };
    auto shorts = [](std::initializer_list<std::uint32_t> values) {
      std::vector<std::uint8_t> v;
      for (std::uint32_t x : values) {
        v.push_back(static_cast<std::uint8_t>(x));
        v.push_back(static_cast<std::uint8_t>(x >> 8));
      }
      return v;
    };
    auto longs = [](std::initializer_list<std::uint32_t> values) {
      std::vector<std::uint8_t> v;
      for (std::uint32_t x : values) {
        for (int b = 0; b < 4; ++b) v.push_back(static_cast<std::uint8_t>(x >> (8 * b)));
      }
      return v;
    };
    auto repeated_short = [&](std::uint32_t value, std::size_t n) {
      std::vector<std::uint8_t> v;
      for (std::size_t k = 0; k < n; ++k) {
        const auto one = shorts({value});
        v.insert(v.end(), one.begin(), one.end());
      }
      return v;
    };
    const std::uint32_t spp = static_cast<std::uint32_t>(channels);
    const std::uint32_t photometric = ycbcr != 0 ? 6 : (spp <= 2 ? 1 : 2);
    std::vector<Entry> entries = {
        {256, 4, 1, longs({static_cast<std::uint32_t>(width)})},
        {257, 4, 1, longs({static_cast<std::uint32_t>(height)})},
        {258, 3, spp, repeated_short(64, spp)},
        {259, 3, 1, shorts({1})},
        {262, 3, 1, shorts({photometric})},
        {273, 4, 1, longs({0})},  // the strip's offset, set below
        {277, 3, 1, shorts({spp})},
        {278, 4, 1, longs({static_cast<std::uint32_t>(height)})},
        {279, 4, 1, longs({static_cast<std::uint32_t>(data_bytes)})},
        {284, 3, 1, shorts({1})},
    };
    if (spp == 2 || spp == 4) entries.push_back({338, 3, 1, shorts({2})});
    entries.push_back({339, 3, spp, repeated_short(3, spp)});
    if (ycbcr != 0) {
      entries.push_back({529, 5, 3, longs({299, 1000, 587, 1000, 114, 1000})});
      entries.push_back({530, 3, 2, shorts({1, 1})});
      entries.push_back({532, 5, 6, longs({0, 1, 255, 1, 128, 1, 255, 1, 128, 1, 255, 1})});
    }
    if (with_icc) entries.push_back({34675, 7, static_cast<std::uint32_t>(icc_size), std::vector<std::uint8_t>(icc, icc + icc_size)});
    // Layout: header (8), IFD (2 + 12 n + 4), the values that do not fit, then the samples at an
    // offset that is a multiple of 8.
    const std::uint32_t ifd_bytes = 2 + 12 * static_cast<std::uint32_t>(entries.size()) + 4;
    std::uint32_t extra = 8 + ifd_bytes;
    std::vector<std::uint32_t> offsets(entries.size(), 0);
    for (std::size_t e = 0; e < entries.size(); ++e) {
      if (entries[e].value.size() > 4) {
        offsets[e] = extra;
        extra += static_cast<std::uint32_t>((entries[e].value.size() + 1) / 2 * 2);
      }
    }
    const std::uint32_t data_offset = (extra + 7) / 8 * 8;
    entries[5].value = longs({data_offset});
    const std::size_t total = data_offset + static_cast<std::size_t>(data_bytes);
    std::unique_ptr<std::uint8_t[]> file(new std::uint8_t[total]());
    std::uint8_t* out = file.get();
    const std::uint8_t header[8] = {'I', 'I', 42, 0, 8, 0, 0, 0};
    std::memcpy(out, header, 8);
    std::uint8_t* at = out + 8;
    const std::uint16_t n = static_cast<std::uint16_t>(entries.size());
    std::memcpy(at, &n, 2);
    at += 2;
    for (std::size_t e = 0; e < entries.size(); ++e) {
      const Entry& entry = entries[e];
      std::memcpy(at, &entry.tag, 2);
      std::memcpy(at + 2, &entry.type, 2);
      std::memcpy(at + 4, &entry.count, 4);
      if (entry.value.size() > 4) {
        std::memcpy(at + 8, &offsets[e], 4);
        std::memcpy(out + offsets[e], entry.value.data(), entry.value.size());
      } else {
        std::memcpy(at + 8, entry.value.data(), entry.value.size());
      }
      at += 12;
    }
    std::memset(at, 0, 4);  // no next IFD
    std::memcpy(out + data_offset, samples, static_cast<std::size_t>(data_bytes));  // little-endian host
    *size = total;
    *bytes = file.release();
    return true;
  });
  if (status == UNROUND_OK) say(message, message_size, warning);
  return status;
}

// The bytes of a PNG file (rust/capi/src/lib.rs, unround_png; c/jpegio/src/png.c): the levels
// made on the device as unround_pnm makes them, 8 or 16 bits, 1 to 4 channels, written by
// png_io.hpp with zlib's compression level (-1 its default) and the ICC profile where it goes
// with the picture (the message says why where it does not).
unround_status unround_png(const double* samples, uint64_t height, uint64_t width, uint64_t channels, int32_t sixteen,
                           int32_t dither, int32_t compression, const uint8_t* icc, uint64_t icc_size, uint8_t** bytes,
                           uint64_t* size, char* message, size_t message_size) {
  std::string warning;
  const unround_status status = guarded(message, message_size, [&](urb::Failure& failure) {
    if (bytes == nullptr || size == nullptr) {
      failure = {urb::kArgument, "the bytes and the size are not null pointers"};
      return false;
    }
    if (dither < 0 || dither > 2 || compression < -1 || compression > 9) {
      failure = {urb::kOptions, "the dither is 0, 1 or 2 and the compression -1 to 9"};
      return false;
    }
    std::size_t count = 0;
    if (!picture_count(samples, height, width, channels, count, failure)) return false;
    std::vector<std::uint8_t> levels(count * (sixteen != 0 ? 2 : 1));
    if (!quantize(samples, count, static_cast<int>(width), static_cast<int>(channels), sixteen != 0, dither,
                  levels.data(), failure)) {
      return false;
    }
    std::vector<std::uint16_t> wide;
    if (sixteen != 0) {  // the levels most significant byte first, as PNM holds them
      wide.resize(count);
      for (std::size_t i = 0; i < count; ++i) wide[i] = static_cast<std::uint16_t>((levels[2 * i] << 8) | levels[2 * i + 1]);
    }
    std::vector<std::uint8_t> file;
    std::string text;
    const int written = urb::write_png(sixteen != 0 ? static_cast<const void*>(wide.data()) : levels.data(),
                                       static_cast<std::uint32_t>(width), static_cast<std::uint32_t>(height),
                                       static_cast<int>(channels), sixteen != 0 ? 16 : 8, compression, icc,
                                       static_cast<std::size_t>(icc_size), file, warning, text);
    if (written != urb::kPngOk) {
      failure = {written == urb::kPngArgument ? urb::kOptions : urb::kIo, text};
      return false;
    }
    std::unique_ptr<std::uint8_t[]> out(new std::uint8_t[file.size()]);
    std::memcpy(out.get(), file.data(), file.size());
    *size = file.size();
    *bytes = out.release();
    return true;
  });
  if (status == UNROUND_OK) say(message, message_size, warning);
  return status;
}

// The PNM file (rust/unround/src/output.rs:248-271, rust/capi/src/lib.rs:1460-1488): a P5
// (grey) or P6 (RGB) header and the levels, made on the device (quantize).
unround_status unround_pnm(const double* samples, uint64_t height, uint64_t width, uint64_t channels, int32_t sixteen,
                           int32_t dither, uint8_t** bytes, uint64_t* size, char* message, size_t message_size) {
  return guarded(message, message_size, [&](urb::Failure& failure) {
    if (bytes == nullptr || size == nullptr) {
      failure = {urb::kArgument, "the bytes and the size are not null pointers"};
      return false;
    }
    if (dither < 0 || dither > 2) {
      failure = {urb::kOptions, "the dither is 0, 1 or 2, not " + std::to_string(dither)};
      return false;
    }
    std::size_t count = 0;
    if (!picture_count(samples, height, width, channels, count, failure)) return false;
    if (channels == 2 || channels == 4) {
      failure = {urb::kOptions, "PNM holds no alpha: write PNG or TIFF"};
      return false;
    }
    const std::string header = std::string(channels == 1 ? "P5" : "P6") + "\n" + std::to_string(width) + " " +
                               std::to_string(height) + "\n" + (sixteen != 0 ? "65535" : "255") + "\n";
    const std::size_t body = count * (sixteen != 0 ? 2 : 1);
    std::unique_ptr<std::uint8_t[]> file(new std::uint8_t[header.size() + body]);
    std::memcpy(file.get(), header.data(), header.size());
    if (!quantize(samples, count, static_cast<int>(width), static_cast<int>(channels), sixteen != 0, dither,
                  file.get() + header.size(), failure)) {
      return false;
    }
    *size = header.size() + body;
    *bytes = file.release();
    return true;
  });
}

void unround_bytes_free(uint8_t* bytes, uint64_t) { delete[] bytes; }

unround_status unround_b200_solve_levels(const unround_input* input, const unround_settings* settings, int32_t sixteen,
                                        int32_t dither, uint8_t* levels, uint64_t capacity, uint64_t* sizes,
                                        char* message, size_t message_size) {
  return guarded(message, message_size, [&](urb::Failure& failure) {
    if (input == nullptr || settings == nullptr) {
      failure = {urb::kArgument, "the input and the settings are not null pointers"};
      return false;
    }
    if (dither < 0 || dither > 2) {
      failure = {urb::kOptions, "the dither is 0, 1 or 2, not " + std::to_string(dither)};
      return false;
    }
    std::vector<urb::ComponentInput> inputs;
    if (!inputs_of(input, inputs, failure)) return false;
    const urb::Settings& s = settings->settings;
    auto frame = urb::make_frame(input->height, input->width, input->color_space, inputs, s, failure);
    if (!frame) return false;
    if (s.method == urb::Method::subgradient) {
      failure = {urb::kUnsupported,
                 "the subgradient method (docs/math.md 7) is not on this build's path: use mmse, tv or tgv"};
      return false;
    }
    const std::uint64_t channels = frame->channels();
    const std::uint64_t need = static_cast<std::uint64_t>(frame->height) * frame->width * channels * (sixteen ? 2 : 1);
    if (sizes != nullptr) {
      sizes[0] = frame->height;
      sizes[1] = frame->width;
      sizes[2] = channels;
    }
    if (levels == nullptr) return true;  // the sizes alone
    if (capacity < need) {
      failure = {urb::kArgument, "the levels take " + std::to_string(need) + " bytes, not " + std::to_string(capacity)};
      return false;
    }
    std::optional<urb::Plan> plan;
    if (s.method != urb::Method::mmse) {
      plan = urb::make_plan(s, frame->channels(), failure);
      if (!plan) return false;
    }
    if (!have_device(failure)) return false;
    Stream stream;
    if (stream.error != cudaSuccess) {
      failure = {urb::kInternal, std::string("a CUDA stream: ") + cudaGetErrorString(stream.error)};
      return false;
    }
    urb::Outcome outcome;
    urb::Solver solver(*frame, stream.stream);
    solver.keep_result_on_device();
    if (!solver.solve(s.method, plan ? &*plan : nullptr, nullptr, nullptr, outcome, failure)) return false;
    return solver.levels(sixteen != 0, dither, levels, failure);
  });
}

// A picture of rounded samples reconstructed (rust/unround/src/samples.rs; cpp/src/samples.cpp:
// 344-405, samples::reconstruct without the file): the colours by TV or TGV within their
// samples' intervals, an alpha (2 or 4 channels) apart, one channel, without channel weights.
unround_status unround_b200_solve_samples(const uint16_t* levels, uint64_t rows, uint64_t columns, uint64_t channels,
                                         int32_t bits, const unround_settings* settings, unround_observer observer,
                                         void* user, unround_result** result, char* message, size_t message_size) {
  return guarded(message, message_size, [&](urb::Failure& failure) {
    return solve_samples_into(levels, rows, columns, channels, bits, settings, observer, user, result, failure);
  });
}

unround_status unround_b200_measure_samples(const uint16_t* levels, uint64_t rows, uint64_t columns, uint64_t channels,
                                           int32_t bits, const unround_settings* settings, uint64_t warmup,
                                           uint64_t iterations, unround_b200_timing* timing, char* message,
                                           size_t message_size) {
  return guarded(message, message_size, [&](urb::Failure& failure) {
    if (levels == nullptr || settings == nullptr || timing == nullptr) {
      failure = {urb::kArgument, "the levels, the settings and the timing are not null pointers"};
      return false;
    }
    if (channels != 1 && channels != 3) {
      failure = {urb::kOptions, "the measurement takes grey or RGB levels (1 or 3 channels)"};
      return false;
    }
    const urb::Settings& s = settings->settings;
    if (!urb::check_samples_settings(s, failure)) return false;
    const urb::DataTerm& term = s.data.front();
    auto model = urb::make_samples_model(levels, rows, columns, channels, bits, 0, channels, term.slack,
                                         term.mu ? *term.mu : 0.0, failure);
    if (!model) return false;
    auto plan = urb::make_plan(s, channels, failure, urb::samples_plan_defaults());
    if (!plan) return false;
    if (!have_device(failure)) return false;
    urb::Frame frame;
    frame.height = frame.rows = static_cast<std::uint32_t>(rows);
    frame.width = frame.columns = static_cast<std::uint32_t>(columns);
    frame.color_space = channels == 3 ? 3 : 1;
    Stream stream;
    urb::Solver solver(frame, *model, stream.stream);
    if (!solver.prepare(*plan, failure)) return false;
    if (warmup > 0 && !solver.iterate(warmup, failure)) return false;
    cudaEvent_t begin, end;
    cudaEventCreate(&begin);
    cudaEventCreate(&end);
    cudaStreamSynchronize(stream.stream);
    cudaEventRecord(begin, stream.stream);
    const bool ok = solver.iterate(iterations, failure);
    cudaEventRecord(end, stream.stream);
    cudaEventSynchronize(end);
    float ms = 0.0f;
    cudaEventElapsedTime(&ms, begin, end);
    cudaEventDestroy(begin);
    cudaEventDestroy(end);
    if (!ok) return false;
    double dual_ms = 0.0, primal_ms = 0.0;
    if (!solver.breakdown(20, dual_ms, primal_ms, failure)) return false;
    timing->milliseconds = ms;
    timing->dual_milliseconds = dual_ms;
    timing->primal_milliseconds = primal_ms;
    timing->iterations = iterations;
    timing->launches_per_iteration = static_cast<std::uint64_t>(solver.launches_per_iteration());
    timing->samples = channels * rows * columns;
    timing->pixels = rows * columns;
    timing->device_bytes = solver.device_bytes();
    return true;
  });
}

unround_status unround_b200_sample_interval(uint32_t level, int32_t bits, double slack, double* ends, char* message,
                                           size_t message_size) {
  return guarded(message, message_size, [&](urb::Failure& failure) {
    if (ends == nullptr) {
      failure = {urb::kArgument, "the ends are a null pointer"};
      return false;
    }
    if (bits < 1 || bits > 16 || level >= (1u << bits) || !(slack >= 0.0 && std::isfinite(slack))) {
      failure = {urb::kOptions, "a level below 2^bits, bits 1 to 16, and a slack at least 0"};
      return false;
    }
    const urb::SampleInterval made = urb::sample_interval(level, bits, slack);
    ends[0] = made.lower;
    ends[1] = made.upper;
    ends[2] = made.centre;
    return true;
  });
}

unround_status unround_b200_blue_noise(uint16_t* ranks, char* message, size_t message_size) {
  return guarded(message, message_size, [&](urb::Failure& failure) {
    if (ranks == nullptr) {
      failure = {urb::kArgument, "the ranks are a null pointer"};
      return false;
    }
    const auto& made = urb::blue_noise_ranks();
    std::copy(made.begin(), made.end(), ranks);
    return true;
  });
}

// A picture turned upright by its EXIF orientation (rust/capi/src/lib.rs, unround_orient;
// rust/unround/src/orientation.rs:67-150; EXIF 2.3 tag 0x0112): 0 or 1 as stored, 2 mirrored, 3 turned half round, 4 flipped, 5 transposed,
// 6 turned a quarter clockwise, 7 transversed, 8 turned a quarter anticlockwise; 5 to 8 swap
// the height and the width. turned holds height * width * channels samples.
unround_status unround_orient(const double* samples, uint64_t height, uint64_t width, uint64_t channels,
                              int32_t orientation, double* turned, uint64_t* turned_height, uint64_t* turned_width,
                              char* message, size_t message_size) {
  return guarded(message, message_size, [&](urb::Failure& failure) {
    if (samples == nullptr || turned == nullptr) {
      failure = {urb::kArgument, "the samples and the turned picture are not null pointers"};
      return false;
    }
    if (orientation < 0 || orientation > 8) {
      failure = {urb::kOptions, "an EXIF orientation is 1 to 8, or 0 for none, not " + std::to_string(orientation)};
      return false;
    }
    if (height == 0 || width == 0 || channels == 0) {
      failure = {urb::kArgument, "the picture is empty"};
      return false;
    }
    const bool swap = orientation >= 5;
    const std::uint64_t out_h = swap ? width : height, out_w = swap ? height : width;
    for (std::uint64_t y = 0; y < out_h; ++y) {
      for (std::uint64_t x = 0; x < out_w; ++x) {
        std::uint64_t sy = 0, sx = 0;  // the stored pixel shown at (y, x)
        switch (orientation) {
          case 0:
          case 1: sy = y; sx = x; break;
          case 2: sy = y; sx = width - 1 - x; break;
          case 3: sy = height - 1 - y; sx = width - 1 - x; break;
          case 4: sy = height - 1 - y; sx = x; break;
          case 5: sy = x; sx = y; break;
          case 6: sy = height - 1 - x; sx = y; break;
          case 7: sy = height - 1 - x; sx = width - 1 - y; break;
          default: sy = x; sx = width - 1 - y; break;
        }
        std::memcpy(turned + (y * out_w + x) * channels, samples + (sy * width + sx) * channels,
                    channels * sizeof(double));
      }
    }
    if (turned_height != nullptr) *turned_height = out_h;
    if (turned_width != nullptr) *turned_width = out_w;
    return true;
  });
}

unround_status unround_to_rgb(const double* planes, uint64_t height, uint64_t width, double* picture) {
  if (planes == nullptr || picture == nullptr) return UNROUND_ERROR_ARGUMENT;
  to_rgb(planes, static_cast<std::size_t>(height * width), picture);
  return UNROUND_OK;
}

unround_status unround_to_ycbcr(const double* picture, uint64_t height, uint64_t width, double* planes) {
  if (planes == nullptr || picture == nullptr) return UNROUND_ERROR_ARGUMENT;
  to_ycbcr(picture, static_cast<std::size_t>(height * width), planes);
  return UNROUND_OK;
}

int32_t unround_main(size_t, const char* const*) { return 3; }

int32_t unround_jpeg_abi_version(void) { return UNROUND_JPEGIO_ABI_VERSION; }
const char* unround_jpeg_libjpeg_version(void) { return "unround JPEG reader (ITU-T T.81, Huffman)"; }
const char* unround_jpeg_libpng_version(void) { return "unround PNG reader and writer, zlib " ZLIB_VERSION; }

int32_t unround_jpeg_check_icc(const uint8_t* profile, uint64_t size, int32_t channels, char* reason,
                               size_t reason_size) {
  std::string why;
  const bool taken = urb::check_icc(profile, size, channels, why);
  say(reason, reason_size, why);
  return taken ? 1 : 0;
}

// The C layer's reading of a JPEG file (c/jpegio/include/unround/jpegio.h:188-211): the
// coefficients and the metadata, by this build's own reader (jpeg_reader.hpp). The arrays are
// allocated with malloc and freed by unround_jpeg_image_free, as the reference's are.
unround_jpegio_status unround_jpeg_read(const uint8_t* data, size_t size, const unround_jpegio_options* options,
                                        unround_jpegio_image* image, char* message, size_t message_size) {
  if (image == nullptr || (message == nullptr && message_size > 0)) return urb::kJpegArgument;
  *image = unround_jpegio_image{};
  urb::JpegLimits limits;
  if (options != nullptr) {
    if (options->max_pixels != 0) limits.max_pixels = options->max_pixels;
    if (options->max_scans > 0) limits.max_scans = options->max_scans;
    limits.warnings_are_errors = options->warnings_are_errors != 0;
  }
  urb::JpegFile file;
  std::string text;
  const int status = urb::read_jpeg(data, size, limits, file, text);
  say(message, message_size, text);
  if (status != urb::kJpegOk) return status;
  image->width = file.width;
  image->height = file.height;
  image->color_space = file.color_space;
  image->num_components = static_cast<int32_t>(file.components.size());
  image->max_h_samp_factor = file.hmax;
  image->max_v_samp_factor = file.vmax;
  image->progressive = file.progressive ? 1 : 0;
  image->arithmetic = 0;
  image->exif_orientation = file.exif_orientation;
  image->warnings = file.warnings;
  for (std::size_t c = 0; c < file.components.size(); ++c) {
    const urb::JpegComponent& from = file.components[c];
    unround_jpegio_component& to = image->components[c];
    to.id = from.id;
    to.h_samp_factor = from.h;
    to.v_samp_factor = from.v;
    to.quant_table_slot = from.slot;
    to.width = from.width;
    to.height = from.height;
    to.width_in_blocks = from.width_in_blocks;
    to.height_in_blocks = from.height_in_blocks;
    std::copy(from.table, from.table + 64, to.quant_table);
    const std::size_t bytes = std::max<std::size_t>(from.coefficients.size() * sizeof(int16_t), 1);
    to.coefficients = static_cast<int16_t*>(std::malloc(bytes));
    if (to.coefficients == nullptr) {
      unround_jpeg_image_free(image);
      say(message, message_size, "out of memory");
      return urb::kJpegMemory;
    }
    std::memcpy(to.coefficients, from.coefficients.data(), from.coefficients.size() * sizeof(int16_t));
  }
  if (!file.icc.empty()) {
    image->icc_profile = static_cast<uint8_t*>(std::malloc(file.icc.size()));
    if (image->icc_profile == nullptr) {
      unround_jpeg_image_free(image);
      say(message, message_size, "out of memory");
      return urb::kJpegMemory;
    }
    std::memcpy(image->icc_profile, file.icc.data(), file.icc.size());
    image->icc_profile_size = file.icc.size();
  }
  return urb::kJpegOk;
}

void unround_jpeg_image_free(unround_jpegio_image* image) {
  if (image == nullptr) return;
  for (unround_jpegio_component& c : image->components) std::free(c.coefficients);
  std::free(image->icc_profile);
  *image = unround_jpegio_image{};
}

// Each component's samples (c/jpegio/include/unround/jpegio.h:116-132, 203-211): the inverse DCT
// of its dequantized coefficients, level-shifted and clamped to 0-255, padded to whole blocks, no
// upsampling or colour conversion. The reference's are libjpeg's integer inverse DCT; these are
// the exact transform rounded, within 1 of it.
unround_jpegio_status unround_jpeg_decode_planes(const uint8_t* data, size_t size, const unround_jpegio_options* options,
                                                 unround_jpegio_planes* planes, char* message, size_t message_size) {
  if (planes == nullptr || (message == nullptr && message_size > 0)) return urb::kJpegArgument;
  *planes = unround_jpegio_planes{};
  urb::JpegLimits limits;
  if (options != nullptr) {
    if (options->max_pixels != 0) limits.max_pixels = options->max_pixels;
    if (options->max_scans > 0) limits.max_scans = options->max_scans;
    limits.warnings_are_errors = options->warnings_are_errors != 0;
  }
  urb::JpegFile file;
  std::string text;
  const int status = urb::read_jpeg(data, size, limits, file, text);
  say(message, message_size, text);
  if (status != urb::kJpegOk) return status;
  planes->num_components = static_cast<int32_t>(file.components.size());
  for (std::size_t c = 0; c < file.components.size(); ++c) {
    const std::vector<std::uint8_t> plane = urb::component_plane(file.components[c]);
    unround_jpegio_plane& to = planes->planes[c];
    to.width = file.components[c].width_in_blocks * 8;
    to.height = file.components[c].height_in_blocks * 8;
    to.stride = to.width;
    to.samples = static_cast<uint8_t*>(std::malloc(std::max<std::size_t>(plane.size(), 1)));
    if (to.samples == nullptr) {
      unround_jpeg_planes_free(planes);
      say(message, message_size, "out of memory");
      return urb::kJpegMemory;
    }
    std::memcpy(to.samples, plane.data(), plane.size());
  }
  return urb::kJpegOk;
}

void unround_jpeg_planes_free(unround_jpegio_planes* planes) {
  if (planes == nullptr) return;
  for (unround_jpegio_plane& p : planes->planes) std::free(p.samples);
  *planes = unround_jpegio_planes{};
}

// One strip of a picture solved in row strips across ranks (strips.py): the solver of the
// strip's own canvas (its bands and the halo bands either side), driven iteration by iteration
// so that the caller can exchange the halo rows of the state between the steps.
struct unround_b200_strip {
  urb::Frame frame;
  urb::Plan plan;
  Stream stream;
  std::unique_ptr<urb::Solver> solver;
  std::uint64_t done = 0;
};

unround_status unround_b200_strip_new(const unround_input* input, const unround_settings* settings,
                                      unround_b200_strip** strip, char* message, size_t message_size) {
  return guarded(message, message_size, [&](urb::Failure& failure) {
    if (input == nullptr || settings == nullptr || strip == nullptr) {
      failure = {urb::kArgument, "the input, the settings and the strip are not null pointers"};
      return false;
    }
    *strip = nullptr;
    std::vector<urb::ComponentInput> inputs;
    if (!inputs_of(input, inputs, failure)) return false;
    const urb::Settings& s = settings->settings;
    if (s.method != urb::Method::tv && s.method != urb::Method::tgv) {
      failure = {urb::kOptions, "a picture is solved in strips by tv or tgv"};
      return false;
    }
    auto frame = urb::make_frame(input->height, input->width, input->color_space, inputs, s, failure);
    if (!frame) return false;
    auto plan = urb::make_plan(s, frame->channels(), failure);
    if (!plan) return false;
    if (!have_device(failure)) return false;
    auto made = std::make_unique<unround_b200_strip>();
    if (made->stream.error != cudaSuccess) {
      failure = {urb::kInternal, std::string("a CUDA stream: ") + cudaGetErrorString(made->stream.error)};
      return false;
    }
    made->frame = std::move(*frame);
    made->plan = *plan;
    made->solver = std::make_unique<urb::Solver>(made->frame, made->stream.stream);
    if (!made->solver->begin_batch(made->plan, failure)) return false;
    *strip = made.release();
    return true;
  });
}

unround_status unround_b200_strip_step(unround_b200_strip* strip, uint64_t iterations, char* message,
                                       size_t message_size) {
  return guarded(message, message_size, [&](urb::Failure& failure) {
    if (strip == nullptr) {
      failure = {urb::kArgument, "the strip is a null pointer"};
      return false;
    }
    if (strip->done + iterations >= strip->plan.iterations && iterations > 0) {
      failure = {urb::kArgument, "the strip's last iteration is made by unround_b200_strip_finish"};
      return false;
    }
    if (!strip->solver->step(iterations, failure)) return false;
    strip->done += iterations;
    return true;
  });
}

uint64_t unround_b200_strip_state(const unround_b200_strip* strip, float** planes, uint64_t most, uint64_t* rows,
                                  uint64_t* columns, uint64_t* pitch) {
  if (strip == nullptr || !strip->solver) return 0;
  const urb::Geometry& g = strip->solver->geometry();
  put(rows, static_cast<uint64_t>(g.rows));
  put(columns, static_cast<uint64_t>(g.columns));
  put(pitch, static_cast<uint64_t>(g.pitch));
  const int bound = most > 64 ? 64 : static_cast<int>(most);
  return static_cast<uint64_t>(strip->solver->state_planes(planes, planes == nullptr ? 0 : bound));
}

unround_status unround_b200_strip_finish(unround_b200_strip* strip, unround_result** result, char* message,
                                         size_t message_size) {
  return guarded(message, message_size, [&](urb::Failure& failure) {
    if (strip == nullptr || result == nullptr) {
      failure = {urb::kArgument, "the strip and the result are not null pointers"};
      return false;
    }
    if (!strip->solver) {
      failure = {urb::kArgument, "the strip is finished"};
      return false;
    }
    const urb::Plan& plan = strip->plan;
    if (plan.record_every != 0 || plan.tolerance > 0.0 || plan.relative_tolerance > 0.0 ||
        plan.partial_tolerance > 0.0) {
      failure = {urb::kOptions, "a strip whose plan records before its last iteration or stops at a tolerance is "
                                "recorded across the ranks (unround_b200_strip_record) and finished by "
                                "unround_b200_strip_result"};
      return false;
    }
    urb::Outcome outcome;
    if (!strip->solver->finish_batch(strip->done, outcome, failure)) return false;
    strip->solver.reset();
    *result = result_of(std::move(strip->frame), std::move(outcome));
    return true;
  });
}

uint64_t unround_b200_strip_plan(const unround_b200_strip* strip, double* values, uint64_t most) {
  if (strip == nullptr) return 0;
  const urb::Plan& p = strip->plan;
  const double nan = std::numeric_limits<double>::quiet_NaN();
  const double all[11] = {static_cast<double>(p.iterations), static_cast<double>(p.record_every), p.tolerance,
                          p.relative_tolerance, p.partial_tolerance, p.partial_radius ? *p.partial_radius : nan,
                          p.alpha, p.alpha1, p.alpha0, p.tgv ? 2.0 : 1.0, static_cast<double>(strip->done)};
  const uint64_t count = std::min<uint64_t>(most, 11);
  for (uint64_t k = 0; values != nullptr && k < count; ++k) values[k] = all[k];
  return 11;
}

unround_status unround_b200_strip_rows(unround_b200_strip* strip, uint64_t first, uint64_t end, char* message,
                                       size_t message_size) {
  return guarded(message, message_size, [&](urb::Failure& failure) {
    if (strip == nullptr || !strip->solver) {
      failure = {urb::kArgument, "the strip is a null pointer or finished"};
      return false;
    }
    const auto rows = static_cast<uint64_t>(strip->solver->geometry().rows);
    if (first > end || end > rows) {
      failure = {urb::kArgument, "the record rows [" + std::to_string(first) + ", " + std::to_string(end) +
                                     ") do not lie within the strip's " + std::to_string(rows) + " canvas rows"};
      return false;
    }
    strip->solver->set_record_rows(static_cast<int>(first), static_cast<int>(end));
    return true;
  });
}

unround_status unround_b200_strip_record(unround_b200_strip* strip, int32_t advance, double* first, char* message,
                                         size_t message_size) {
  return guarded(message, message_size, [&](urb::Failure& failure) {
    if (strip == nullptr || !strip->solver || first == nullptr) {
      failure = {urb::kArgument, "the strip (not finished) and the sums are not null pointers"};
      return false;
    }
    if (advance != 0 && strip->done >= strip->plan.iterations) {
      failure = {urb::kArgument, "the strip has made all of its plan's iterations"};
      return false;
    }
    double sums[5] = {};
    if (!strip->solver->record_step(advance != 0, sums, failure)) return false;
    if (advance != 0) ++strip->done;
    std::copy(sums, sums + 5, first);
    return true;
  });
}

unround_status unround_b200_strip_record_duals(unround_b200_strip* strip, double theta, double* second, char* message,
                                               size_t message_size) {
  return guarded(message, message_size, [&](urb::Failure& failure) {
    if (strip == nullptr || !strip->solver || second == nullptr) {
      failure = {urb::kArgument, "the strip (not finished) and the sums are not null pointers"};
      return false;
    }
    double sums[3] = {};
    if (!strip->solver->record_duals(theta, sums, failure)) return false;
    std::copy(sums, sums + 3, second);
    return true;
  });
}

unround_status unround_b200_strip_result(unround_b200_strip* strip, int32_t stop, unround_result** result,
                                         char* message, size_t message_size) {
  return guarded(message, message_size, [&](urb::Failure& failure) {
    if (strip == nullptr || !strip->solver || result == nullptr) {
      failure = {urb::kArgument, "the strip (not finished) and the result are not null pointers"};
      return false;
    }
    urb::Outcome outcome;
    if (!strip->solver->finish_here(strip->done, stop, outcome, failure)) return false;
    strip->solver.reset();
    *result = result_of(std::move(strip->frame), std::move(outcome));
    return true;
  });
}

void unround_b200_strip_free(unround_b200_strip* strip) { delete strip; }

extern "C++" {
namespace {

// The NCCL calls of the halo swaps, from the libnccl.so.2 the process has loaded (torch's, whose
// communicators the callers hand over), else the one the loader finds; looked up once.
struct NcclCalls {
  decltype(&ncclSend) send = nullptr;
  decltype(&ncclRecv) recv = nullptr;
  decltype(&ncclGroupStart) group_start = nullptr;
  decltype(&ncclGroupEnd) group_end = nullptr;
  decltype(&ncclGetErrorString) text = nullptr;
  bool found() const { return send && recv && group_start && group_end && text; }
};

const NcclCalls& nccl_calls() {
  static const NcclCalls calls = [] {
    NcclCalls c;
    void* library = dlopen("libnccl.so.2", RTLD_NOW | RTLD_NOLOAD);
    if (library == nullptr) library = dlopen("libnccl.so.2", RTLD_NOW);
    if (library == nullptr) return c;
    c.send = reinterpret_cast<decltype(&ncclSend)>(dlsym(library, "ncclSend"));
    c.recv = reinterpret_cast<decltype(&ncclRecv)>(dlsym(library, "ncclRecv"));
    c.group_start = reinterpret_cast<decltype(&ncclGroupStart)>(dlsym(library, "ncclGroupStart"));
    c.group_end = reinterpret_cast<decltype(&ncclGroupEnd)>(dlsym(library, "ncclGroupEnd"));
    c.text = reinterpret_cast<decltype(&ncclGetErrorString)>(dlsym(library, "ncclGetErrorString"));
    return c;
  }();
  return calls;
}

// Whether each exchange's rows lie within the canvases of the strips it names (`rows_of(strip)`
// the canvas rows of a strip, -1 for a strip that this call does not hold).
template <class RowsOf>
bool exchanges_fit(const unround_b200_strip_exchange* exchanges, uint64_t count, RowsOf rows_of,
                   urb::Failure& failure) {
  for (uint64_t e = 0; e < count; ++e) {
    const unround_b200_strip_exchange& x = exchanges[e];
    const long long sender_rows = rows_of(x.sender), receiver_rows = rows_of(x.receiver);
    const bool sender_fits = sender_rows < 0 || (x.sender_row <= static_cast<uint64_t>(sender_rows) &&
                                                 x.rows <= static_cast<uint64_t>(sender_rows) - x.sender_row);
    const bool receiver_fits = receiver_rows < 0 || (x.receiver_row <= static_cast<uint64_t>(receiver_rows) &&
                                                     x.rows <= static_cast<uint64_t>(receiver_rows) - x.receiver_row);
    if (x.sender < 0 || x.receiver < 0 || !sender_fits || !receiver_fits) {
      failure = {urb::kArgument, "exchange " + std::to_string(e) + " names a strip that does not hold its rows"};
      return false;
    }
  }
  return true;
}

// This rank's part of the exchanges, one NCCL group on the strip's stream.
bool exchange_nccl(unround_b200_strip* strip, int32_t rank, const unround_b200_strip_exchange* exchanges,
                   uint64_t count, ncclComm_t comm, urb::Failure& failure) {
  const NcclCalls& nccl = nccl_calls();
  float* planes[64];
  const int n = strip->solver->state_planes(planes, 64);
  const std::size_t pitch = static_cast<std::size_t>(strip->solver->geometry().pitch);
  const cudaStream_t on = strip->solver->stream();
  ncclResult_t result = nccl.group_start();
  for (uint64_t e = 0; e < count && result == ncclSuccess; ++e) {
    const unround_b200_strip_exchange& x = exchanges[e];
    const std::size_t floats = x.rows * pitch;  // a plane's rows are contiguous, `pitch` floats each
    for (int k = 0; k < n && result == ncclSuccess && x.sender == rank; ++k) {
      result = nccl.send(planes[k] + x.sender_row * pitch, floats, ncclFloat32, x.receiver, comm, on);
    }
    for (int k = 0; k < n && result == ncclSuccess && x.receiver == rank; ++k) {
      result = nccl.recv(planes[k] + x.receiver_row * pitch, floats, ncclFloat32, x.sender, comm, on);
    }
  }
  const ncclResult_t ended = nccl.group_end();
  if (result == ncclSuccess) result = ended;
  if (result == ncclSuccess) return true;
  failure = {urb::kInternal, std::string("the halo exchange through NCCL: ") + nccl.text(result)};
  return false;
}

bool involves(const unround_b200_strip_exchange* exchanges, uint64_t count, int32_t rank) {
  for (uint64_t e = 0; e < count; ++e) {
    if (exchanges[e].sender == rank || exchanges[e].receiver == rank) return true;
  }
  return false;
}

}  // namespace
}  // extern "C++"

unround_status unround_b200_strip_run(unround_b200_strip* strip, uint64_t iterations, int32_t rank,
                                      const unround_b200_strip_exchange* exchanges, uint64_t count, void* comm,
                                      char* message, size_t message_size) {
  return guarded(message, message_size, [&](urb::Failure& failure) {
    if (strip == nullptr || !strip->solver || (exchanges == nullptr && count > 0)) {
      failure = {urb::kArgument, "the strip (not finished) and the exchanges are not null pointers"};
      return false;
    }
    if (strip->done + iterations >= strip->plan.iterations && iterations > 0) {
      failure = {urb::kArgument, "the strip's last iteration is made by unround_b200_strip_record or _finish"};
      return false;
    }
    const long long rows = strip->solver->geometry().rows;
    // The rows on this rank's side of each exchange; the other side's are its peer's to check.
    auto rows_of = [&](int32_t who) { return who == rank ? rows : -1LL; };
    if (!exchanges_fit(exchanges, count, rows_of, failure)) return false;
    const bool swapping = involves(exchanges, count, rank);
    if (swapping && comm == nullptr) {
      failure = {urb::kArgument, "the NCCL communicator is not a null pointer"};
      return false;
    }
    if (swapping && !nccl_calls().found()) {
      failure = {urb::kInternal, "NCCL (libnccl.so.2) could not be loaded"};
      return false;
    }
    const auto communicator = static_cast<ncclComm_t>(comm);
    for (uint64_t n = 0; n < iterations; ++n) {
      if (!strip->solver->advance(1, failure)) return false;
      ++strip->done;
      if (swapping && !exchange_nccl(strip, rank, exchanges, count, communicator, failure)) return false;
    }
    if (iterations == 0 && swapping) return exchange_nccl(strip, rank, exchanges, count, communicator, failure);
    return true;
  });
}

unround_status unround_b200_strip_exchange_local(unround_b200_strip* const* strips, uint64_t count,
                                                 const unround_b200_strip_exchange* exchanges,
                                                 uint64_t exchange_count, char* message, size_t message_size) {
  return guarded(message, message_size, [&](urb::Failure& failure) {
    if (strips == nullptr || (exchanges == nullptr && exchange_count > 0)) {
      failure = {urb::kArgument, "the strips and the exchanges are not null pointers"};
      return false;
    }
    for (uint64_t s = 0; s < count; ++s) {
      if (strips[s] == nullptr || !strips[s]->solver) {
        failure = {urb::kArgument, "strip " + std::to_string(s) + " is a null pointer or finished"};
        return false;
      }
    }
    auto rows_of = [&](int32_t who) {
      return static_cast<uint64_t>(who) < count ? static_cast<long long>(strips[who]->solver->geometry().rows)
                                                : -2LL;
    };
    for (uint64_t e = 0; e < exchange_count; ++e) {
      if (rows_of(exchanges[e].sender) == -2 || rows_of(exchanges[e].receiver) == -2) {
        failure = {urb::kArgument, "exchange " + std::to_string(e) + " names a strip beyond the " +
                                       std::to_string(count) + " given"};
        return false;
      }
    }
    if (!exchanges_fit(exchanges, exchange_count, rows_of, failure)) return false;
    for (uint64_t e = 0; e < exchange_count; ++e) {
      const urb::Solver& from = *strips[exchanges[e].sender]->solver;
      const urb::Solver& to = *strips[exchanges[e].receiver]->solver;
      if (from.state_planes(nullptr, 0) != to.state_planes(nullptr, 0) ||
          from.geometry().columns != to.geometry().columns) {
        failure = {urb::kArgument, "exchange " + std::to_string(e) + " joins strips of different widths or fields"};
        return false;
      }
    }
    // Events: each strip's work so far (the senders' rows are ready), then each receiver's copies
    // (the senders' later steps overwrite nothing still being read).
    std::vector<cudaEvent_t> ready(count, nullptr), copied(count, nullptr);
    cudaError_t error = cudaSuccess;
    for (uint64_t s = 0; s < count && error == cudaSuccess; ++s) {
      error = cudaEventCreateWithFlags(&ready[s], cudaEventDisableTiming);
      if (error == cudaSuccess) error = cudaEventCreateWithFlags(&copied[s], cudaEventDisableTiming);
      if (error == cudaSuccess) error = cudaEventRecord(ready[s], strips[s]->solver->stream());
    }
    for (uint64_t e = 0; e < exchange_count && error == cudaSuccess; ++e) {
      const unround_b200_strip_exchange& x = exchanges[e];
      urb::Solver& from = *strips[x.sender]->solver;
      urb::Solver& to = *strips[x.receiver]->solver;
      float* sent[64];
      float* received[64];
      const int n = from.state_planes(sent, 64);
      to.state_planes(received, 64);
      const std::size_t from_pitch = static_cast<std::size_t>(from.geometry().pitch);
      const std::size_t to_pitch = static_cast<std::size_t>(to.geometry().pitch);
      const std::size_t width = static_cast<std::size_t>(from.geometry().columns) * sizeof(float);
      error = cudaStreamWaitEvent(to.stream(), ready[x.sender], 0);
      for (int k = 0; k < n && error == cudaSuccess; ++k) {
        error = cudaMemcpy2DAsync(received[k] + x.receiver_row * to_pitch, to_pitch * sizeof(float),
                                  sent[k] + x.sender_row * from_pitch, from_pitch * sizeof(float), width, x.rows,
                                  cudaMemcpyDeviceToDevice, to.stream());
      }
    }
    for (uint64_t s = 0; s < count && error == cudaSuccess; ++s) {
      error = cudaEventRecord(copied[s], strips[s]->solver->stream());
    }
    for (uint64_t e = 0; e < exchange_count && error == cudaSuccess; ++e) {
      error = cudaStreamWaitEvent(strips[exchanges[e].sender]->solver->stream(), copied[exchanges[e].receiver], 0);
    }
    for (uint64_t s = 0; s < count; ++s) {
      if (ready[s] != nullptr) cudaEventDestroy(ready[s]);
      if (copied[s] != nullptr) cudaEventDestroy(copied[s]);
    }
    if (error == cudaSuccess) return true;
    failure = {urb::kInternal, std::string("the halo exchange between strips: ") + cudaGetErrorString(error)};
    return false;
  });
}

// The C layer's PNG reading and writing (c/jpegio/include/unround/jpegio.h:225-256), by png_io.hpp.
unround_jpegio_status unround_jpegio_read_png(const uint8_t* data, size_t size, uint64_t max_pixels,
                                              unround_jpegio_png_image* image, char* message, size_t message_size) {
  if (image == nullptr || (message == nullptr && message_size > 0)) return urb::kPngArgument;
  *image = unround_jpegio_png_image{};
  urb::PngPicture picture;
  std::string text;
  const int status = urb::read_png(data, size, max_pixels, picture, text);
  say(message, message_size, text);
  if (status != urb::kPngOk) return status;
  image->samples = static_cast<uint16_t*>(std::malloc(std::max<std::size_t>(picture.samples.size() * 2, 1)));
  image->icc_profile = picture.icc.empty() ? nullptr : static_cast<uint8_t*>(std::malloc(picture.icc.size()));
  if (image->samples == nullptr || (!picture.icc.empty() && image->icc_profile == nullptr)) {
    unround_jpegio_png_image_free(image);
    say(message, message_size, "out of memory");
    return urb::kPngMemory;
  }
  std::memcpy(image->samples, picture.samples.data(), picture.samples.size() * 2);
  if (!picture.icc.empty()) std::memcpy(image->icc_profile, picture.icc.data(), picture.icc.size());
  image->icc_profile_size = picture.icc.size();
  image->width = picture.width;
  image->height = picture.height;
  image->channels = picture.channels;
  image->bits = picture.bits;
  return urb::kPngOk;
}

void unround_jpegio_png_image_free(unround_jpegio_png_image* image) {
  if (image == nullptr) return;
  std::free(image->samples);
  std::free(image->icc_profile);
  *image = unround_jpegio_png_image{};
}

unround_jpegio_status unround_jpegio_write_png(const unround_jpegio_png* png, unround_jpegio_bytes* file, char* message,
                                               size_t message_size) {
  if (file == nullptr || (message == nullptr && message_size > 0)) return urb::kPngArgument;
  *file = unround_jpegio_bytes{};
  if (png == nullptr) {
    say(message, message_size, "no picture is given");
    return urb::kPngArgument;
  }
  std::vector<std::uint8_t> bytes;
  std::string warning, text;
  const int status = urb::write_png(png->samples, png->width, png->height, png->channels, png->bits, png->compression,
                                    png->icc_profile, static_cast<std::size_t>(png->icc_profile_size), bytes, warning,
                                    text);
  say(message, message_size, text);
  if (status != urb::kPngOk) return status;
  file->data = static_cast<uint8_t*>(std::malloc(bytes.size()));
  if (file->data == nullptr) {
    say(message, message_size, "out of memory");
    return urb::kPngMemory;
  }
  std::memcpy(file->data, bytes.data(), bytes.size());
  file->size = bytes.size();
  return urb::kPngOk;
}

void unround_jpegio_bytes_free(unround_jpegio_bytes* bytes) {
  if (bytes == nullptr) return;
  std::free(bytes->data);
  *bytes = unround_jpegio_bytes{};
}

}  // extern "C"

extern "C" int64_t unround_b200_set_ring_wait_limit(int64_t tries) { return urb::set_ring_wait_limit(tries); }
