// Test infrastructure: the oracle. A C face over the reference's own C++ solver
// (cpp/src of JPEG-Unround, compiled in place by oracle/ref/Makefile into
// oracle/_ref/libunround_ref.so). Only tests, __graft_entry__.smoke() and
// bench.py's CPU-baseline leg load it, as the checker; the product never does.
//
// It follows the reference's array-level path: unround_solve (rust/capi/src/lib.rs:669)
// -> decode::solve (rust/unround/src/decode.rs:269), which the C++ implementation
// restates as parse_settings (cpp/src/settings.cpp:243) -> data_of (cpp/src/settings.cpp:506)
// -> Frame::make (cpp/src/frames.cpp:155) -> pdhg::solve (cpp/src/pdhg.cpp:235), or
// Frame::start for the MMSE decoder (cpp/src/frames.cpp:401).

#include "unround/frames.hpp"
#include "unround/model.hpp"
#include "unround/operators.hpp"
#include "unround/pdhg.hpp"
#include "unround/picture.hpp"
#include "unround/samples.hpp"
#include "unround/settings.hpp"

#include <cstdint>
#include <cstring>
#include <string>
#include <string_view>
#include <vector>

namespace {

struct Component {
  const std::int16_t* levels;
  std::uint32_t rows;
  std::uint32_t columns;
  std::int32_t h;
  std::int32_t v;
  std::uint16_t table[64];
};

struct Outcome {
  std::size_t channels = 0, rows = 0, columns = 0;
  std::vector<double> canvas;                     // C x H x W
  std::vector<std::vector<double>> coefficients;  // per component, 64 per block
  std::vector<std::vector<double>> lower, upper, centres;
  std::vector<std::vector<double>> weights, flat_weights;  // 64 each
  std::vector<std::vector<std::uint8_t>> flat;
  std::vector<std::uint64_t> record_iterations;
  std::vector<double> record_values;  // 5 per record: seconds, primal, dual, scaling, partial
  std::uint64_t iterations = 0;
  std::int32_t stop = 0;  // 1 converged, 2 iterations, 3 observer, 0 none
  double tau = 0.0, sigma = 0.0;
  std::vector<std::size_t> cell_rows, cell_columns, block_rows, block_columns;
};

void say(char* message, std::size_t size, const std::string& text) {
  if (message == nullptr || size == 0) return;
  const std::size_t n = text.size() < size - 1 ? text.size() : size - 1;
  std::memcpy(message, text.data(), n);
  message[n] = 0;
}

}  // namespace

extern "C" {

// The fields of a start, channel-major, each of the canvas's rows x columns; a null
// pointer leaves that part of the start at the reference's default. Coefficients are
// all components' blocks one after another.
struct oref_start {
  const double* coefficients;
  const double* p;  // per channel: x then y
  const double* w;  // per channel: x then y
  const double* r;  // per channel: xx, yy, xy
};

void* oref_solve(std::uint32_t height, std::uint32_t width, std::int32_t color_space, std::uint32_t count,
                 const Component* components, std::size_t option_count, const char* const* options,
                 const oref_start* start, char* message, std::size_t message_size) {
  using namespace unround;
  std::vector<std::string_view> arguments;
  for (std::size_t i = 0; i < option_count; ++i) arguments.emplace_back(options[i]);
  auto parsed = parse_settings(arguments);
  if (!parsed) {
    say(message, message_size, parsed.error().message);
    return nullptr;
  }
  const Settings settings = *parsed;
  const ColourSpace space = color_space == 1 ? ColourSpace::grayscale
                            : color_space == 2 ? ColourSpace::ycbcr
                                               : ColourSpace::rgb;
  std::vector<ComponentInput> inputs;
  for (std::uint32_t c = 0; c < count; ++c) {
    ComponentInput in;
    in.levels = Blocks<const std::int16_t>(components[c].levels, block_extents(components[c].rows, components[c].columns));
    for (int k = 0; k < 64; ++k) in.table[k] = components[c].table[k];
    in.h = static_cast<std::uint32_t>(components[c].h);
    in.v = static_cast<std::uint32_t>(components[c].v);
    inputs.push_back(in);
  }
  const std::vector<DataTerm> data = data_of(settings);
  auto frame = Frame::make(height, width, space, inputs, data);
  if (!frame) {
    say(message, message_size, frame.error().message);
    return nullptr;
  }
  auto* out = new Outcome;
  out->channels = frame->channels();
  out->rows = frame->rows();
  out->columns = frame->columns();
  const std::size_t plane = out->rows * out->columns;
  for (std::size_t c = 0; c < frame->channels(); ++c) {
    const auto& component = frame->component(c);
    const Problem& problem = component.problem;
    out->lower.emplace_back(problem.lower().data_handle(), problem.lower().data_handle() + problem.lower().size());
    out->upper.emplace_back(problem.upper().data_handle(), problem.upper().data_handle() + problem.upper().size());
    out->centres.emplace_back(problem.centres().data_handle(),
                              problem.centres().data_handle() + problem.centres().size());
    out->weights.emplace_back(problem.weights().data_handle(), problem.weights().data_handle() + 64);
    out->flat_weights.emplace_back(problem.flat_weights().data_handle(), problem.flat_weights().data_handle() + 64);
    out->flat.emplace_back(problem.flat().data_handle(), problem.flat().data_handle() + problem.flat().size());
    out->cell_rows.push_back(component.cell_rows);
    out->cell_columns.push_back(component.cell_columns);
    out->block_rows.push_back(component.block_rows());
    out->block_columns.push_back(component.block_columns());
  }
  if (settings.method == Method::mmse) {
    out->canvas.assign(out->channels * plane, 0.0);
    for (std::size_t c = 0; c < frame->channels(); ++c) {
      const auto& problem = frame->component(c).problem;
      BlocksArray<double> kept(problem.extents());
      frame->start(c, Grid<double>(out->canvas.data() + c * plane, out->rows, out->columns), kept.view());
      out->coefficients.emplace_back(kept.entries().begin(), kept.entries().end());
    }
    return out;
  }
  if (settings.method != Method::tv && settings.method != Method::tgv) {
    say(message, message_size, "the oracle runs the methods mmse, tv and tgv");
    delete out;
    return nullptr;
  }
  const pdhg::Model model = settings.method == Method::tv ? pdhg::Model::tv : pdhg::Model::tgv;
  pdhg::Start given;
  const pdhg::Start* from = nullptr;
  if (start != nullptr) {
    from = &given;
    std::size_t offset = 0;
    for (std::size_t c = 0; c < frame->channels() && start->coefficients != nullptr; ++c) {
      BlocksArray<double> coefficients(frame->component(c).problem.extents());
      std::memcpy(coefficients.entries().data(), start->coefficients + offset, coefficients.size() * sizeof(double));
      offset += coefficients.size();
      given.coefficients.push_back(std::move(coefficients));
    }
    auto vector_of = [&](const double* at) {
      operators::Vector v = operators::vector_of(out->rows, out->columns);
      std::memcpy(v.x.entries().data(), at, plane * sizeof(double));
      std::memcpy(v.y.entries().data(), at + plane, plane * sizeof(double));
      return v;
    };
    for (std::size_t c = 0; c < frame->channels(); ++c) {
      if (start->p != nullptr) given.p.push_back(vector_of(start->p + 2 * c * plane));
      if (start->w != nullptr) given.w.push_back(vector_of(start->w + 2 * c * plane));
      if (start->r != nullptr) {
        operators::Tensor t = operators::tensor_of(out->rows, out->columns);
        const double* at = start->r + 3 * c * plane;
        std::memcpy(t.xx.entries().data(), at, plane * sizeof(double));
        std::memcpy(t.yy.entries().data(), at + plane, plane * sizeof(double));
        std::memcpy(t.xy.entries().data(), at + 2 * plane, plane * sizeof(double));
        given.r.push_back(std::move(t));
      }
    }
  }
  const pdhg::Regularizer& regularizer = settings.regularizer;
  auto solved = pdhg::solve(*frame, model, regularizer, settings.pdhg, from);
  if (!solved) {
    say(message, message_size, solved.error().message);
    delete out;
    return nullptr;
  }
  for (std::size_t c = 0; c < solved->canvas.size(); ++c) {
    const auto entries = solved->canvas[c].entries();
    out->canvas.insert(out->canvas.end(), entries.begin(), entries.end());
    const auto coefficients = solved->coefficients[c].entries();
    out->coefficients.emplace_back(coefficients.begin(), coefficients.end());
  }
  for (const Record& record : solved->records) {
    out->record_iterations.push_back(record.iteration);
    out->record_values.push_back(record.seconds);
    out->record_values.push_back(record.primal);
    out->record_values.push_back(record.dual);
    out->record_values.push_back(record.scaling ? *record.scaling : __builtin_nan(""));
    out->record_values.push_back(record.partial_gap ? *record.partial_gap : __builtin_nan(""));
  }
  out->iterations = solved->iterations;
  out->stop = solved->stop == Stop::converged ? 1 : solved->stop == Stop::iterations ? 2 : 3;
  out->tau = solved->steps.tau;
  out->sigma = solved->steps.sigma;
  return out;
}

// A picture of rounded samples (rust/unround/src/samples.rs; cpp/src/samples.cpp): levels of
// `bits` bits, rows x columns x channels interleaved, reconstructed as samples::reconstruct
// does a PNG file's (cpp/src/samples.cpp:344-405) -- the same refusals of options, the colours
// by samples::solve and an alpha (channels 2 or 4) apart -- without reading a file. The canvas
// is the picture's planes, C x H x W; the records, iterations and steps the colours'.
void* oref_solve_samples(const std::uint16_t* levels, std::uint32_t rows, std::uint32_t columns,
                         std::uint32_t channels, std::int32_t bits, std::size_t option_count,
                         const char* const* options, char* message, std::size_t message_size) {
  using namespace unround;
  std::vector<std::string_view> arguments;
  for (std::size_t i = 0; i < option_count; ++i) arguments.emplace_back(options[i]);
  auto parsed = parse_settings(arguments);
  if (!parsed) {
    say(message, message_size, parsed.error().message);
    return nullptr;
  }
  const Settings settings = *parsed;
  if (settings.method != Method::tv && settings.method != Method::tgv) {
    say(message, message_size, "a PNG file is reconstructed by tv or tgv");
    return nullptr;
  }
  const DataTerm& term = settings.data.front();
  const double mu = term.mu ? *term.mu : 0.0;
  const pdhg::Model method = settings.method == Method::tv ? pdhg::Model::tv : pdhg::Model::tgv;
  const Picture<const std::uint16_t> picture(levels, PictureExtents{rows, columns, channels});
  const bool alpha = channels == 2u || channels == 4u;
  const std::size_t colours = alpha ? channels - 1u : channels;
  auto* out = new Outcome;
  out->channels = channels;
  out->rows = rows;
  out->columns = columns;
  auto run = [&](std::size_t first, std::size_t count, const pdhg::Regularizer& regularizer, bool keep) {
    auto model = samples::Model::make(picture, bits, first, count, term.slack, mu);
    if (!model) {
      say(message, message_size, model.error().message);
      return false;
    }
    auto solved = samples::solve(*model, method, regularizer, settings.pdhg);
    if (!solved) {
      say(message, message_size, solved.error().message);
      return false;
    }
    for (const auto& plane : solved->canvas) {
      const auto entries = plane.entries();
      out->canvas.insert(out->canvas.end(), entries.begin(), entries.end());
    }
    if (keep) {
      for (const Record& record : solved->records) {
        out->record_iterations.push_back(record.iteration);
        out->record_values.push_back(record.seconds);
        out->record_values.push_back(record.primal);
        out->record_values.push_back(record.dual);
        out->record_values.push_back(record.scaling ? *record.scaling : __builtin_nan(""));
        out->record_values.push_back(record.partial_gap ? *record.partial_gap : __builtin_nan(""));
      }
      out->iterations = solved->iterations;
      out->stop = solved->stop == Stop::converged ? 1 : solved->stop == Stop::iterations ? 2 : 3;
      out->tau = solved->steps.tau;
      out->sigma = solved->steps.sigma;
    }
    return true;
  };
  if (!run(0, colours, settings.regularizer, true)) {
    delete out;
    return nullptr;
  }
  if (alpha) {
    pdhg::Regularizer alone = settings.regularizer;
    alone.channel_weights.clear();
    if (!run(colours, 1, alone, false)) {
      delete out;
      return nullptr;
    }
  }
  return out;
}

void oref_free(void* handle) { delete static_cast<Outcome*>(handle); }

void oref_shape(const void* handle, std::uint64_t* channels, std::uint64_t* rows, std::uint64_t* columns) {
  const auto* out = static_cast<const Outcome*>(handle);
  *channels = out->channels;
  *rows = out->rows;
  *columns = out->columns;
}

const double* oref_canvas(const void* handle) { return static_cast<const Outcome*>(handle)->canvas.data(); }

// which: 0 coefficients, 1 lower, 2 upper, 3 centres (per coefficient); 4 weights,
// 5 flat weights (64).
const double* oref_array(const void* handle, std::uint32_t component, std::int32_t which, std::uint64_t* count) {
  const auto* out = static_cast<const Outcome*>(handle);
  const std::vector<double>* values = nullptr;
  switch (which) {
    case 0: values = &out->coefficients[component]; break;
    case 1: values = &out->lower[component]; break;
    case 2: values = &out->upper[component]; break;
    case 3: values = &out->centres[component]; break;
    case 4: values = &out->weights[component]; break;
    case 5: values = &out->flat_weights[component]; break;
    default: return nullptr;
  }
  *count = values->size();
  return values->data();
}

const std::uint8_t* oref_flat(const void* handle, std::uint32_t component, std::uint64_t* count) {
  const auto* out = static_cast<const Outcome*>(handle);
  *count = out->flat[component].size();
  return out->flat[component].data();
}

void oref_component(const void* handle, std::uint32_t component, std::uint64_t* block_rows,
                    std::uint64_t* block_columns, std::uint64_t* cell_rows, std::uint64_t* cell_columns) {
  const auto* out = static_cast<const Outcome*>(handle);
  *block_rows = out->block_rows[component];
  *block_columns = out->block_columns[component];
  *cell_rows = out->cell_rows[component];
  *cell_columns = out->cell_columns[component];
}

std::uint64_t oref_records(const void* handle, const std::uint64_t** iterations, const double** values) {
  const auto* out = static_cast<const Outcome*>(handle);
  *iterations = out->record_iterations.data();
  *values = out->record_values.data();
  return out->record_iterations.size();
}

void oref_solver(const void* handle, std::uint64_t* iterations, std::int32_t* stop, double* tau, double* sigma) {
  const auto* out = static_cast<const Outcome*>(handle);
  *iterations = out->iterations;
  *stop = out->stop;
  *tau = out->tau;
  *sigma = out->sigma;
}

// The projection of a picture onto the intervals of components given as arrays, as the
// reference's picture::project makes it (cpp/src/picture.cpp:70-148: canvas_of, excess, and
// Frame::project per channel), without the picture of the result: into `canvas` (C x rows x
// columns), `zeta` (every component's blocks, 64 a block) and `excess` (the same, in steps).
// Returns 0, or 1 with the reason in message.
int oref_project(std::uint32_t height, std::uint32_t width, std::int32_t color_space, std::uint32_t count,
                 const Component* components, std::size_t option_count, const char* const* options,
                 const double* picture, std::size_t channels, double* canvas, double* zeta, double* excess,
                 char* message, std::size_t message_size) {
  using namespace unround;
  std::vector<std::string_view> arguments;
  for (std::size_t i = 0; i < option_count; ++i) arguments.emplace_back(options[i]);
  auto parsed = parse_settings(arguments);
  if (!parsed) {
    say(message, message_size, parsed.error().message);
    return 1;
  }
  const ColourSpace space = color_space == 1 ? ColourSpace::grayscale
                            : color_space == 2 ? ColourSpace::ycbcr
                                               : ColourSpace::rgb;
  std::vector<ComponentInput> inputs;
  for (std::uint32_t c = 0; c < count; ++c) {
    ComponentInput in;
    in.levels = Blocks<const std::int16_t>(components[c].levels, block_extents(components[c].rows, components[c].columns));
    for (int k = 0; k < 64; ++k) in.table[k] = components[c].table[k];
    in.h = static_cast<std::uint32_t>(components[c].h);
    in.v = static_cast<std::uint32_t>(components[c].v);
    inputs.push_back(in);
  }
  auto frame = Frame::make(height, width, space, inputs, data_of(*parsed));
  if (!frame) {
    say(message, message_size, frame.error().message);
    return 1;
  }
  auto made = picture::canvas_of(*frame, Picture<const double>(picture, PictureExtents{height, width, channels}));
  if (!made) {
    say(message, message_size, made.error().message);
    return 1;
  }
  const std::vector<BlocksArray<double>> beyond = picture::excess(*frame, *made);
  std::size_t offset = 0;
  for (std::size_t c = 0; c < frame->channels(); ++c) {
    GridArray<double>& grid = (*made)[c];
    BlocksArray<double> kept(frame->component(c).problem.extents());
    Room room = frame->room(c);
    frame->project(c, std::as_const(grid).view(), grid.view(), kept.view(), room);
    const std::size_t plane = frame->rows() * frame->columns();
    std::memcpy(canvas + c * plane, grid.view().data_handle(), plane * sizeof(double));
    const std::size_t entries = kept.entries().size();
    std::memcpy(zeta + offset, kept.entries().data(), entries * sizeof(double));
    std::memcpy(excess + offset, beyond[c].entries().data(), entries * sizeof(double));
    offset += entries;
  }
  return 0;
}

}  // extern "C"
