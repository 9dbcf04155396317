// The decoder of the centres (docs/math.md 2.3: every coefficient at the centre of its interval,
// what unround_solve computes with --method=mmse) for callers that must not allocate device memory.
// The caller owns the two output buffers on the device. The device buffers the kernels need
// besides -- the levels and flat-block flags copied in, each component's binary64 constants, the
// start kernel's per-CTA sums -- live in one file-scope device array of kScratchBytes, which the
// CUDA runtime reserves on each device when it loads this library's device code there.
//
// Who needs this: code that runs inside a fixed device-memory budget it does not own -- a server
// process that hands a framework's allocator all of the GPU's memory at start-up, a real-time loop
// whose memory is planned once -- where a cudaMalloc can fail once the pool is spoken for, or a
// cudaFree can stall the device. unround_solve takes its device buffers from the device's memory
// pool on every call; this entry point takes none.
//
// The first call on a device also looks up the array's device address there (cudaGetSymbolAddress,
// with that device current; kept for later calls once it succeeds), which loads this library's
// device code on that device if it is not loaded yet. Every call uses the one array, which keeps
// what the last call left there: calls whose work overlaps on the same GPU (two streams, two host
// threads at once) race on it, so the caller serializes them. Every call waits for its own work
// on the stream before it returns, whether it succeeds or fails.
#include <algorithm>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include <cuda_runtime.h>

#include "kernels.hpp"
#include "model.hpp"
#include "settings.hpp"
#include "unround.h"
#include "unround_b200.h"

namespace {

// 64 MiB: 2 bytes a coefficient for the levels, so about 33 million coefficients -- a grey image
// of 33 megapixels, a 4:2:0 colour image of 22.
constexpr std::size_t kScratchBytes = std::size_t{64} << 20;
constexpr int kDevices = 64;

}  // namespace

// The scratch of every call, on every device that uses this entry point.
static __device__ __align__(256) unsigned char scratch[kScratchBytes];

namespace {

void tell(char* buffer, std::size_t size, const std::string& text) {
  if (buffer == nullptr || size == 0) return;
  std::size_t end = std::min(text.size(), size - 1);
  while (end > 0 && end < text.size() && (static_cast<unsigned char>(text[end]) & 0xC0u) == 0x80u) --end;
  std::memcpy(buffer, text.data(), end);
  buffer[end] = 0;
}

// The device address of the scratch array on the current device, looked up on the first call
// on that device that finds it and kept for later calls. A lookup that fails is not kept: the
// next call tries again.
bool scratch_of(unsigned char*& address, std::string& why) {
  static std::mutex guard;
  static unsigned char* found[kDevices] = {};
  int device = 0;
  const cudaError_t error = cudaGetDevice(&device);
  if (error != cudaSuccess) {
    why = std::string("no CUDA device for the decoder of the centres: ") + cudaGetErrorName(error) + ": " +
          cudaGetErrorString(error);
    return false;
  }
  if (device < 0 || device >= kDevices) {
    why = "the decoder of the centres serves devices 0 to " + std::to_string(kDevices - 1) + ", not device " +
          std::to_string(device);
    return false;
  }
  std::lock_guard<std::mutex> lock(guard);
  if (found[device] == nullptr) {
    void* p = nullptr;
    const cudaError_t looked = cudaGetSymbolAddress(&p, scratch);
    if (looked != cudaSuccess || p == nullptr) {
      why = std::string("the device address of the decoder's scratch: ") + cudaGetErrorName(looked) + ": " +
            cudaGetErrorString(looked);
      return false;
    }
    found[device] = static_cast<unsigned char*>(p);
  }
  address = found[device];
  return true;
}

std::size_t aligned(std::size_t n) { return (n + 255) / 256 * 256; }

urb::ComponentDevice device_of(const urb::Component& c) {
  urb::ComponentDevice d;
  d.block_rows = static_cast<int>(c.block_rows);
  d.block_columns = static_cast<int>(c.block_columns);
  d.cell_rows = static_cast<int>(c.cell_rows);
  d.cell_columns = static_cast<int>(c.cell_columns);
  return d;
}

std::size_t partial_count(const urb::Component& c) {
  return static_cast<std::size_t>(urb::start_grid_blocks(device_of(c)));
}

}  // namespace

extern "C" unround_status unround_b200_decode_centres_noalloc(const unround_input* input,
                                                              const unround_settings* settings, double* canvas,
                                                              uint64_t canvas_capacity, double* coefficients,
                                                              uint64_t coefficient_capacity, uint64_t* sizes,
                                                              void* stream, char* message, size_t message_size) {
  try {
    if (input == nullptr || settings == nullptr) {
      tell(message, message_size, "the input and the settings are not null pointers");
      return UNROUND_ERROR_ARGUMENT;
    }
    if ((canvas == nullptr) != (coefficients == nullptr)) {
      tell(message, message_size, "the canvas and the coefficients are both given, or both null to ask for sizes");
      return UNROUND_ERROR_ARGUMENT;
    }
    if (settings->settings.method != urb::Method::mmse) {
      tell(message, message_size,
           "this entry point runs the decoder of the centres: its settings have --method=mmse");
      return UNROUND_ERROR_ARGUMENT;
    }
    if (input->components == nullptr || input->count == 0) {
      tell(message, message_size, "components are given");
      return UNROUND_ERROR_ARGUMENT;
    }
    std::vector<urb::ComponentInput> inputs;
    for (std::uint32_t c = 0; c < input->count; ++c) {
      const unround_component& given = input->components[c];
      if (given.levels == nullptr) {
        tell(message, message_size, "a component's levels are a null pointer");
        return UNROUND_ERROR_ARGUMENT;
      }
      urb::ComponentInput in;
      in.levels = given.levels;
      in.rows = given.rows;
      in.columns = given.columns;
      in.h = given.h_samp_factor;
      in.v = given.v_samp_factor;
      for (int k = 0; k < 64; ++k) in.table[k] = given.quant_table[k];
      inputs.push_back(in);
    }
    urb::Failure failure;
    auto frame = urb::make_frame(input->height, input->width, input->color_space, inputs, settings->settings, failure);
    if (!frame) {
      tell(message, message_size, failure.message);
      return static_cast<unround_status>(failure.status);
    }
    const std::size_t channels = frame->channels();
    const std::size_t plane = static_cast<std::size_t>(frame->rows) * frame->columns;
    std::size_t coefficient_total = 0, need = 0;
    for (const urb::Component& c : frame->components) {
      coefficient_total += c.coefficient_count();
      need += aligned(c.levels.size() * sizeof(std::int16_t)) + aligned(c.flat.size()) +
              aligned(sizeof(urb::Constants64)) + aligned(partial_count(c) * sizeof(double));
    }
    if (sizes != nullptr) {
      sizes[0] = channels;
      sizes[1] = frame->rows;
      sizes[2] = frame->columns;
      sizes[3] = coefficient_total;
    }
    if (canvas == nullptr) return UNROUND_OK;
    if (canvas_capacity < channels * plane || coefficient_capacity < coefficient_total) {
      tell(message, message_size,
           "the output buffers hold " + std::to_string(canvas_capacity) + " and " +
               std::to_string(coefficient_capacity) + " doubles; the input needs " + std::to_string(channels * plane) +
               " for the canvas and " + std::to_string(coefficient_total) + " for the coefficients");
      return UNROUND_ERROR_ARGUMENT;
    }
    if (need > kScratchBytes) {
      tell(message, message_size,
           "the input needs " + std::to_string(need) + " bytes of device scratch, more than the " +
               std::to_string(kScratchBytes) + " this entry point holds: use unround_solve");
      return UNROUND_ERROR_ARGUMENT;
    }
    std::string why;
    unsigned char* base = nullptr;
    if (!scratch_of(base, why)) {
      tell(message, message_size, why);
      return UNROUND_ERROR_INTERNAL;
    }
    urb::Geometry g;
    g.rows = static_cast<int>(frame->rows);
    g.columns = static_cast<int>(frame->columns);
    g.pitch = g.columns;
    g.channels = static_cast<int>(channels);
    g.plane = plane;
    const cudaStream_t on = static_cast<cudaStream_t>(stream);
    std::vector<urb::Constants64> constants(frame->components.size());
    cudaError_t error = cudaSuccess;
    std::size_t offset = 0, coefficient_offset = 0;
    for (std::size_t c = 0; c < frame->components.size() && error == cudaSuccess; ++c) {
      const urb::Component& comp = frame->components[c];
      urb::ComponentDevice d = device_of(comp);
      auto* levels = reinterpret_cast<std::int16_t*>(base + offset);
      offset += aligned(comp.levels.size() * sizeof(std::int16_t));
      auto* flat = reinterpret_cast<std::uint8_t*>(base + offset);
      offset += aligned(comp.flat.size());
      auto* device_constants = reinterpret_cast<urb::Constants64*>(base + offset);
      offset += aligned(sizeof(urb::Constants64));
      auto* partials = reinterpret_cast<double*>(base + offset);
      offset += aligned(partial_count(comp) * sizeof(double));
      urb::Constants64& k = constants[c];
      k = urb::Constants64{};
      for (int i = 0; i < 64; ++i) {
        k.step[i] = comp.steps[i];
        k.weight[i] = comp.weights[i];
        k.flat_weight[i] = comp.flat_weights[i];
        k.shrink[i] = comp.shrink[i];
        k.cost[i] = comp.costs[i];
      }
      k.slack = comp.slack;
      k.mmse = comp.mmse ? 1 : 0;
      k.costed = comp.costed ? 1 : 0;
      error = cudaMemcpyAsync(levels, comp.levels.data(), comp.levels.size() * sizeof(std::int16_t),
                              cudaMemcpyHostToDevice, on);
      if (error == cudaSuccess) error = cudaMemcpyAsync(flat, comp.flat.data(), comp.flat.size(), cudaMemcpyHostToDevice, on);
      if (error == cudaSuccess) error = cudaMemcpyAsync(device_constants, &k, sizeof(k), cudaMemcpyHostToDevice, on);
      // The start kernel's sums of the data term: cleared, as the array keeps the last call's.
      if (error == cudaSuccess) error = cudaMemsetAsync(partials, 0, partial_count(comp) * sizeof(double), on);
      d.levels = levels;
      d.flat = flat;
      d.constants = device_constants;
      urb::StartParams sp;
      sp.component = d;
      sp.coefficients = coefficients + coefficient_offset;
      sp.partials = partials;
      if (error == cudaSuccess) error = urb::launch_start_coefficients(sp, on);
      urb::CanvasParams cp;
      cp.g = g;
      cp.component = d;
      cp.coefficients = coefficients + coefficient_offset;
      cp.canvas = canvas + c * plane;
      cp.beyond = 128.0;
      cp.mode = 0;
      if (error == cudaSuccess) error = urb::launch_canvas(cp, on);
      coefficient_offset += comp.coefficient_count();
    }
    // The host copies above read `frame` and `constants`, which end with this call; and on a
    // failure part of the way, nothing queued for the components before it may still be writing
    // the caller's buffers or the scratch when the call returns.
    const cudaError_t drained = cudaStreamSynchronize(on);
    if (error == cudaSuccess) error = drained;
    if (error != cudaSuccess) {
      tell(message, message_size, std::string("the device failed in the decoder of the centres: ") +
                                      cudaGetErrorName(error) + ": " + cudaGetErrorString(error));
      return UNROUND_ERROR_INTERNAL;
    }
    return UNROUND_OK;
  } catch (const std::exception& e) {
    tell(message, message_size, std::string("an internal error of JPEG-Unround: ") + e.what());
    return UNROUND_ERROR_INTERNAL;
  } catch (...) {
    tell(message, message_size, "an internal error of JPEG-Unround");
    return UNROUND_ERROR_INTERNAL;
  }
}
