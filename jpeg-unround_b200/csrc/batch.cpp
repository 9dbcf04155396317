// The batched solve (batch.hpp).
#include "batch.hpp"

#include <algorithm>
#include <cstdlib>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <tuple>

#include "kernels.hpp"

namespace urb {

namespace {

std::string describe(cudaError_t error) {
  return std::string(cudaGetErrorName(error)) + ": " + cudaGetErrorString(error);
}

// Device memory owned for the call, freed on the stream at the end.
struct Owned {
  cudaStream_t stream;
  std::vector<void*> blocks;
  explicit Owned(cudaStream_t s) : stream(s) {}
  ~Owned() {
    for (void* p : blocks) cudaFreeAsync(p, stream);
    cudaStreamSynchronize(stream);
  }
  template <typename T>
  cudaError_t upload(const std::vector<T>& host, T** device) {
    *device = nullptr;
    if (host.empty()) return cudaSuccess;
    void* p = nullptr;
    cudaError_t e = cudaMallocAsync(&p, host.size() * sizeof(T), stream);
    if (e != cudaSuccess) return e;
    blocks.push_back(p);
    *device = static_cast<T*>(p);
    return cudaMemcpyAsync(p, host.data(), host.size() * sizeof(T), cudaMemcpyHostToDevice, stream);
  }
};

struct DualClass {
  bool tgv = false;
  int channels = 1;
  bool coupled = false;
  std::vector<int> pictures;       // of the batch, in this class
  std::vector<Geometry> geometry;  // theirs
  std::vector<DualTile> tiles;
  int tile_rows = 0;
  DualTile* device = nullptr;
};

// Streams to run the classes' launches of an iteration side by side: the launches of a phase
// (the primal steps, then the dual steps) fork from `main` and join it again, so that a
// captured iteration is a graph of parallel branches, one per class, and one class's last
// wave of CTAs overlaps the next class's first.
struct Branches {
  std::vector<cudaStream_t> streams;
  std::vector<cudaEvent_t> events;  // [0] the fork, [1 + b] branch b's end
  cudaError_t error = cudaSuccess;
  explicit Branches(std::size_t count) {
    streams.resize(count, nullptr);
    events.resize(count + 1, nullptr);
    for (cudaStream_t& s : streams) {
      if (error == cudaSuccess) error = cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking);
    }
    for (cudaEvent_t& e : events) {
      if (error == cudaSuccess) error = cudaEventCreateWithFlags(&e, cudaEventDisableTiming);
    }
  }
  ~Branches() {
    for (cudaStream_t s : streams) {
      if (s != nullptr) cudaStreamDestroy(s);
    }
    for (cudaEvent_t e : events) {
      if (e != nullptr) cudaEventDestroy(e);
    }
  }
  // Runs launch(b, stream) for b < count, each on its own branch of `main`.
  template <typename Launch>
  cudaError_t fork(cudaStream_t main, std::size_t count, Launch&& launch) {
    if (count <= 1) return count == 1 ? launch(0, main) : cudaSuccess;
    cudaError_t e = cudaEventRecord(events[0], main);
    for (std::size_t b = 0; b < count && e == cudaSuccess; ++b) {
      e = cudaStreamWaitEvent(streams[b], events[0], 0);
      if (e == cudaSuccess) e = launch(b, streams[b]);
      if (e == cudaSuccess) e = cudaEventRecord(events[1 + b], streams[b]);
    }
    for (std::size_t b = 0; b < count && e == cudaSuccess; ++b) e = cudaStreamWaitEvent(main, events[1 + b], 0);
    return e;
  }
};

// A class's tiles: strips of the sweep's width (sweep_width) of each of its pictures, cut into
// tiles of `rows` rows.
std::vector<DualTile> tiles_of(const DualClass& dual, int rows) {
  std::vector<DualTile> tiles;
  const int width = sweep_width(dual.channels);
  for (std::size_t m = 0; m < dual.pictures.size(); ++m) {
    const Geometry& g = dual.geometry[m];
    for (int x0 = 0; x0 < g.columns; x0 += width) {
      for (int i0 = 0; i0 < g.rows; i0 += rows) tiles.push_back({dual.pictures[m], x0, i0, std::min(i0 + rows, g.rows)});
    }
  }
  return tiles;
}

// The autotuner's record: per device, class and the sizes of its pictures, the tile height its
// measurement chose, so that a batch of the same shapes is measured once in a process.
using TuneKey = std::tuple<int, bool, int, bool, std::vector<std::pair<int, int>>>;
std::mutex tune_mutex;
std::map<TuneKey, int>& tuned() {
  static auto* record = new std::map<TuneKey, int>();  // never destroyed: used until exit
  return *record;
}

bool autotune_enabled() {
  const char* given = std::getenv("UNROUND_B200_AUTOTUNE");
  return given != nullptr && std::string(given) == "1";
}

// Measures a class's dual sweep at candidate tile heights and returns the fastest: the wave
// model's choice (batch_tile_rows), the heights beside it, and a spread from 96 to 512. Each
// candidate's table is launched once to warm up and timed over three launches by CUDA events;
// a candidate replaces the model's choice only when it is at least 2% faster. The launches read
// the state of parity 0 and the start's tilde point and write the state of parity 1, which the
// first iteration writes again: they change nothing the solve reads.
int tune_dual(const DualClass& dual, const DualBatchImage* images_device, cudaStream_t stream, cudaError_t& error) {
  const int model = batch_tile_rows(dual.geometry, dual_batch_slots(dual.tgv, dual.channels, dual.coupled));
  std::vector<int> candidates = {model};
  for (int h : {model - 32, model + 32, 96, 128, 192, 256, 320, 384, 512}) {
    if (h >= 64 && h <= 512 && std::find(candidates.begin(), candidates.end(), h) == candidates.end()) {
      candidates.push_back(h);
    }
  }
  cudaEvent_t begin = nullptr, end = nullptr;
  if (error == cudaSuccess) error = cudaEventCreate(&begin);
  if (error == cudaSuccess) error = cudaEventCreate(&end);
  int best = model;
  float best_ms = -1.0f, model_ms = -1.0f;
  for (int rows : candidates) {
    if (error != cudaSuccess) break;
    const std::vector<DualTile> tiles = tiles_of(dual, rows);
    void* table = nullptr;
    error = cudaMallocAsync(&table, tiles.size() * sizeof(DualTile), stream);
    if (error != cudaSuccess) break;
    error = cudaMemcpyAsync(table, tiles.data(), tiles.size() * sizeof(DualTile), cudaMemcpyHostToDevice, stream);
    const int count = static_cast<int>(tiles.size());
    auto launch = [&] {
      if (error == cudaSuccess) {
        error = launch_dual_batch(static_cast<const DualTile*>(table), count, images_device, 0, dual.tgv, dual.channels,
                                  dual.coupled, stream);
      }
    };
    launch();
    if (error == cudaSuccess) error = cudaEventRecord(begin, stream);
    for (int r = 0; r < 3; ++r) launch();
    if (error == cudaSuccess) error = cudaEventRecord(end, stream);
    if (error == cudaSuccess) error = cudaEventSynchronize(end);
    float ms = 0.0f;
    if (error == cudaSuccess) error = cudaEventElapsedTime(&ms, begin, end);
    cudaFreeAsync(table, stream);
    if (error != cudaSuccess) break;
    if (rows == model) model_ms = ms;
    if (best_ms < 0.0f || ms < best_ms) {
      best_ms = ms;
      best = rows;
    }
  }
  if (begin != nullptr) cudaEventDestroy(begin);
  if (end != nullptr) cudaEventDestroy(end);
  if (error != cudaSuccess || model_ms < 0.0f) return model;
  return best_ms < 0.98f * model_ms ? best : model;
}

struct PrimalClass {
  int cell_rows = 1;
  int cell_columns = 1;
  std::vector<PrimalItem> items;
  PrimalItem* device = nullptr;
};

}  // namespace

bool check_batch(const std::vector<BatchEntry>& entries, Failure& failure) {
  if (entries.empty()) {
    failure = {kArgument, "a batch has at least one picture"};
    return false;
  }
  const std::uint64_t most = entries[0].plan.iterations;
  for (const BatchEntry& e : entries) {
    if (e.plan.iterations != most) {
      failure = {kArgument, "the pictures of a batch take the same number of iterations"};
      return false;
    }
    if (e.plan.record_every != 0) {
      failure = {kArgument, "a batch records each picture at its last iteration only: give --record-every 0"};
      return false;
    }
  }
  return true;
}

bool solve_batch(const std::vector<BatchEntry>& entries, cudaStream_t stream, std::vector<Outcome>& outcomes,
                 BatchTiming& timing, Failure& failure) {
  if (!check_batch(entries, failure)) return false;
  const std::uint64_t most = entries[0].plan.iterations;
  // Each picture's solver, started.
  std::vector<std::unique_ptr<Solver>> solvers;
  for (const BatchEntry& e : entries) {
    solvers.push_back(std::make_unique<Solver>(*e.frame, stream));
    if (!solvers.back()->begin_batch(e.plan, failure)) return false;
  }
  // The tables: each picture's entry, each component's, and per class the tiles and items.
  std::vector<DualBatchImage> images(entries.size());
  std::vector<PrimalBatchComponent> components;
  std::map<std::tuple<bool, int, bool>, DualClass> duals;
  std::map<std::pair<int, int>, PrimalClass> primals;
  timing = BatchTiming{};
  for (std::size_t n = 0; n < entries.size(); ++n) {
    std::vector<PrimalBatchComponent> own;
    if (!solvers[n]->batch_entries(images[n], own)) {
      failure = {kUnsupported, "picture " + std::to_string(n) +
                                   " has cells the batched primal step does not take (1, 2 or 4 samples each way)"};
      return false;
    }
    const Geometry& g = solvers[n]->geometry();
    const Plan& plan = entries[n].plan;
    timing.samples += static_cast<std::uint64_t>(g.channels) * g.rows * g.columns;
    timing.pixels += static_cast<std::uint64_t>(entries[n].frame->height) * entries[n].frame->width;
    DualClass& dual = duals[{plan.tgv, g.channels, plan.coupled && g.channels > 1}];
    dual.tgv = plan.tgv;
    dual.channels = g.channels;
    dual.coupled = plan.coupled && g.channels > 1;
    dual.pictures.push_back(static_cast<int>(n));
    dual.geometry.push_back(g);
    for (std::size_t c = 0; c < own.size(); ++c) {
      const ComponentDevice& comp = own[c].params[0].component;
      PrimalClass& primal = primals[{comp.cell_rows, comp.cell_columns}];
      primal.cell_rows = comp.cell_rows;
      primal.cell_columns = comp.cell_columns;
      const int z = static_cast<int>(components.size());
      const int strips = (g.columns + 31) / 32, stages = primal_batch_stages(g, comp.cell_rows);
      for (int stage = 0; stage < stages; ++stage) {
        for (int strip = 0; strip < strips; ++strip) primal.items.push_back({z, strip, stage, 0});
      }
      components.push_back(own[c]);
    }
  }
  Owned owned(stream);
  DualBatchImage* images_device = nullptr;
  PrimalBatchComponent* components_device = nullptr;
  cudaError_t error = owned.upload(images, &images_device);
  if (error == cudaSuccess) error = owned.upload(components, &components_device);
  // Each class's tiles: strips of the sweep's width cut into tiles of the height that finishes the
  // class's pictures soonest in waves of the CTAs the device holds (the wave model), or, with
  // the autotuner (UNROUND_B200_AUTOTUNE=1), the height its measurement chose.
  int device = 0;
  if (error == cudaSuccess) error = cudaGetDevice(&device);
  cudaEvent_t tune_begin = nullptr, tune_end = nullptr;
  const bool tuning = autotune_enabled();
  bool measured = false;  // a class was measured in this call (not found in the record)
  if (tuning && error == cudaSuccess) error = cudaEventCreate(&tune_begin);
  if (tuning && error == cudaSuccess) error = cudaEventCreate(&tune_end);
  if (tuning && error == cudaSuccess) error = cudaEventRecord(tune_begin, stream);
  for (auto& [key, dual] : duals) {
    int rows = batch_tile_rows(dual.geometry, dual_batch_slots(dual.tgv, dual.channels, dual.coupled));
    if (tuning && error == cudaSuccess) {
      std::vector<std::pair<int, int>> sizes;
      for (const Geometry& g : dual.geometry) sizes.emplace_back(g.rows, g.columns);
      std::sort(sizes.begin(), sizes.end());
      const TuneKey tune_key{device, dual.tgv, dual.channels, dual.coupled, sizes};
      std::unique_lock<std::mutex> lock(tune_mutex);
      const auto found = tuned().find(tune_key);
      if (found != tuned().end()) {
        rows = found->second;
      } else {
        lock.unlock();
        rows = tune_dual(dual, images_device, stream, error);
        measured = true;
        lock.lock();
        if (error == cudaSuccess) tuned()[tune_key] = rows;
      }
    }
    dual.tile_rows = rows;
    dual.tiles = tiles_of(dual, rows);
    if (error == cudaSuccess) error = owned.upload(dual.tiles, &dual.device);
  }
  if (tuning && error == cudaSuccess) error = cudaEventRecord(tune_end, stream);
  if (tuning && error == cudaSuccess) error = cudaEventSynchronize(tune_end);
  if (tuning && error == cudaSuccess) {
    float ms = 0.0f;
    error = cudaEventElapsedTime(&ms, tune_begin, tune_end);
    timing.tuning_milliseconds = measured ? ms : 0.0;
  }
  if (tune_begin != nullptr) cudaEventDestroy(tune_begin);
  if (tune_end != nullptr) cudaEventDestroy(tune_end);
  for (auto& [key, primal] : primals) {
    if (error == cudaSuccess) error = owned.upload(primal.items, &primal.device);
  }
  // Iteration k (1-based): the primal steps read the state of parity (k - 1) % 2, the dual
  // steps read it and write the other.
  std::vector<const PrimalClass*> primal_list;
  std::vector<const DualClass*> dual_list;
  for (auto& [key, primal] : primals) primal_list.push_back(&primal);
  for (auto& [key, dual] : duals) dual_list.push_back(&dual);
  Branches branches(std::max(primal_list.size(), dual_list.size()));
  if (error == cudaSuccess) error = branches.error;
  auto iteration = [&](std::uint64_t k, cudaStream_t on) {
    const int parity = static_cast<int>((k - 1) % 2);
    if (error == cudaSuccess) {
      error = branches.fork(on, primal_list.size(), [&](std::size_t b, cudaStream_t s) {
        const PrimalClass& primal = *primal_list[b];
        return launch_primal_batch(primal.device, static_cast<int>(primal.items.size()), components_device, parity,
                                   primal.cell_rows, primal.cell_columns, s);
      });
    }
    if (error == cudaSuccess) {
      error = branches.fork(on, dual_list.size(), [&](std::size_t b, cudaStream_t s) {
        const DualClass& dual = *dual_list[b];
        return launch_dual_batch(dual.device, static_cast<int>(dual.tiles.size()), images_device, parity, dual.tgv,
                                 dual.channels, dual.coupled, s);
      });
    }
  };
  // The batch makes iterations 1 .. most - 1; each picture's last (which keeps its values for
  // the record and the result) runs on its own.
  const std::uint64_t batched = most > 0 ? most - 1 : 0;
  timing.iterations = batched;
  timing.launches_per_iteration = primals.size() + duals.size();
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  cudaEvent_t began = nullptr, ended = nullptr;
  if (error == cudaSuccess) error = cudaEventCreate(&began);
  if (error == cudaSuccess) error = cudaEventCreate(&ended);
  if (batched > 2 && error == cudaSuccess) {
    // Set up every launcher (shared memory, occupancy) before the capture: a launch of no work.
    for (auto& [key, primal] : primals) {
      if (error == cudaSuccess) {
        error = launch_primal_batch(primal.device, 0, components_device, 0, primal.cell_rows, primal.cell_columns,
                                    stream);
      }
    }
    for (auto& [key, dual] : duals) {
      if (error == cudaSuccess) {
        error = launch_dual_batch(dual.device, 0, images_device, 0, dual.tgv, dual.channels, dual.coupled, stream);
      }
    }
    // Two iterations, one of each parity (an iteration's launches depend on k only through the
    // parity of the state it reads): the graph of a pair, launched for every pair of 2 .. N - 1.
    if (error == cudaSuccess) error = cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal);
    if (error == cudaSuccess) {
      iteration(2, stream);
      iteration(3, stream);
      const cudaError_t ended_capture = cudaStreamEndCapture(stream, &graph);
      if (error == cudaSuccess) error = ended_capture;
    }
    if (error == cudaSuccess) error = cudaGraphInstantiate(&exec, graph, 0);
  }
  if (error == cudaSuccess) error = cudaEventRecord(began, stream);
  if (batched > 0) iteration(1, stream);
  const std::uint64_t pairs = batched > 1 ? (batched - 1) / 2 : 0;
  for (std::uint64_t n = 0; n < pairs && exec != nullptr && error == cudaSuccess; ++n) {
    error = cudaGraphLaunch(exec, stream);
  }
  // With an even count the last iteration (k = N - 1, of the pairs' first parity) is left.
  if (batched > 1 && (batched - 1) % 2 == 1) iteration(batched, stream);
  if (error == cudaSuccess) error = cudaEventRecord(ended, stream);
  if (error == cudaSuccess) error = cudaEventSynchronize(ended);
  float milliseconds = 0.0f;
  if (error == cudaSuccess) error = cudaEventElapsedTime(&milliseconds, began, ended);
  timing.milliseconds = milliseconds;
  if (exec != nullptr) cudaGraphExecDestroy(exec);
  if (graph != nullptr) cudaGraphDestroy(graph);
  if (began != nullptr) cudaEventDestroy(began);
  if (ended != nullptr) cudaEventDestroy(ended);
  if (error != cudaSuccess) {
    failure = {kInternal, "the device failed in the batched iterations: " + describe(error)};
    return false;
  }
  outcomes.clear();
  outcomes.resize(entries.size());
  for (std::size_t n = 0; n < entries.size(); ++n) {
    if (!solvers[n]->finish_batch(batched, outcomes[n], failure)) {
      failure.message = "picture " + std::to_string(n) + ": " + failure.message;
      return false;
    }
  }
  return true;
}

}  // namespace urb
