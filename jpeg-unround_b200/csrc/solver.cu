// The device solve. See solver.hpp.
#include "solver.hpp"

#include "samples_model.hpp"

#include <chrono>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <limits>
#include <string>

namespace urb {

namespace {

constexpr double kNaN = std::numeric_limits<double>::quiet_NaN();

std::string describe(cudaError_t error) {
  return std::string(cudaGetErrorName(error)) + ": " + cudaGetErrorString(error);
}

// UNROUND_B200_KERNELS=fused runs the iterations that keep nothing as one sweep each
// (iteration.cu: the dual step and the next primal step, one pass over HBM); otherwise every
// iteration is the dual sweep and the primal kernels apart, which measure faster on B200.
bool fused_kernels() {
  const char* value = std::getenv("UNROUND_B200_KERNELS");
  return value != nullptr && std::strcmp(value, "fused") == 0;
}

// How pictures of rounded samples iterate: 0 two launches (the dual sweep, then the primal
// kernel: the default, the fastest measured); 1 the fused sweep of iteration.cu
// (UNROUND_B200_KERNELS=fused); 2 the dual sweep with the primal step in it (=sweep).
int samples_kernels() {
  const char* value = std::getenv("UNROUND_B200_KERNELS");
  if (value == nullptr) return 0;
  if (std::strcmp(value, "fused") == 0) return 1;
  if (std::strcmp(value, "sweep") == 0) return 2;
  return 0;
}

// Iterations that keep nothing are launched kGraphIterations at a time as one CUDA graph
// (Impl::group; an even count, so that a group leaves the state's parity as it found it);
// UNROUND_B200_GRAPHS=0 launches every iteration's kernels one by one.
constexpr std::uint64_t kGraphIterations = 8;

bool group_graphs() {
  const char* value = std::getenv("UNROUND_B200_GRAPHS");
  return value == nullptr || std::strcmp(value, "0") != 0;
}

}  // namespace

struct Solver::Impl {
  const Frame& frame;
  cudaStream_t stream;
  Geometry g;
  std::vector<void*> owned;
  std::size_t bytes = 0;
  cudaError_t error = cudaSuccess;

  std::vector<ComponentDevice> components;
  std::vector<double*> coefficients;  // binary64, per component
  std::vector<ProxFactors*> factors;
  Fields state[2];
  Fields tilde;
  float* xt = nullptr;
  float* v = nullptr;
  float* div2 = nullptr;
  double* canvas = nullptr;
  double* partials = nullptr;        // record reductions
  double* record_partials = nullptr;  // a record's conjugates and residuals, a region each
  double* record_sums = nullptr;      // a record's sums (2 x kMaxReductions)
  double* value_partials = nullptr;  // the data term of the last kept primal step, per component
  std::size_t partial_count = 0;
  std::vector<int> value_counts;
  std::vector<int> value_written;
  bool tgv = false;
  int current = 0;  // which state holds s_n
  // The sweep's tensor maps (of each state, and of each x~ buffer), and its error word.
  CUtensorMap state_maps[2];
  CUtensorMap tilde_maps[2];
  bool swept = false;
  // x~ in two buffers when the whole iteration is one sweep (it reads x~_n and writes
  // x~_{n+1}); `xt` is the current one, xts[xt_id]. The fused sweep's maps, of 9-row boxes.
  float* xts[2] = {nullptr, nullptr};
  int xt_id = 0;
  bool fusable = false;
  int cell_rows = 1, cell_columns = 1;
  CUtensorMap iteration_state_maps[2];
  CUtensorMap iteration_tilde_maps[2];
  CUtensorMap primal_maps[2][kMaxChannels];
  bool primal_swept[kMaxChannels] = {};
  int* error_word = nullptr;
  Plan plan;
  bool planned = false;
  std::vector<double> host_partials;
  bool host_result = true;  // false: the result stays on the device (levels)
  // A picture of rounded samples in place of a JPEG file's components (samples.cu): its
  // intervals and centres, binary32 pitched for the iterations, binary64 packed for the
  // records and the result.
  const SamplesModel* samples = nullptr;
  std::uint16_t* s_levels = nullptr;  // the channels' levels, pitched like the state
  int samples_layout = 0;              // samples_kernels() when the solve began
  SampleEnds32* s_ends = nullptr;       // per level: binary32 ends rounded inward, the centre
  SampleEnds64* s_ends64 = nullptr;     // per level: binary64 ends and centre
  int samples_written = 0;  // the CTAs of the last kept primal step's sums of G
  // kGraphIterations iterations that keep nothing (the dual step and the next primal step, each
  // time) captured as one CUDA graph from the state of parity `group_parity`; made at the first
  // group after both launches have run eagerly (which sets up their launchers), made again for
  // the other parity.
  cudaGraphExec_t group_exec = nullptr;
  int group_parity = -1;
  bool plain_dual = false, plain_primal = false;  // a dual(false) and a primal(false) have run

  Impl(const Frame& f, cudaStream_t s) : frame(f), stream(s) {}

  ~Impl() {
    if (group_exec != nullptr) cudaGraphExecDestroy(group_exec);
    for (void* p : owned) cudaFreeAsync(p, stream);
    cudaStreamSynchronize(stream);
  }

  template <typename T>
  T* allocate(std::size_t count) {
    if (error != cudaSuccess) return nullptr;
    void* p = nullptr;
    const std::size_t size = std::max<std::size_t>(count * sizeof(T), 16);
    error = cudaMallocAsync(&p, size, stream);
    if (error != cudaSuccess) return nullptr;
    owned.push_back(p);
    bytes += size;
    return static_cast<T*>(p);
  }

  template <typename T>
  T* upload(const T* from, std::size_t count) {
    T* p = allocate<T>(count);
    if (p != nullptr && count > 0) error = cudaMemcpyAsync(p, from, count * sizeof(T), cudaMemcpyHostToDevice, stream);
    return p;
  }

  // A state's fields in one allocation, each field's channels one after another, in the order
  // x, p1, p2, w1, w2, r11, r22, r12: the planes of the sweep's TMA box (sweep.cu).
  Fields fields(bool with_tgv) {
    const std::size_t n = g.plane * g.channels;
    const int count = with_tgv ? 8 : 3;
    float* block = allocate<float>(n * count);
    Fields f;
    if (block == nullptr) return f;
    f.x = block;
    f.p1 = block + n;
    f.p2 = block + 2 * n;
    if (with_tgv) {
      f.w1 = block + 3 * n;
      f.w2 = block + 4 * n;
      f.r11 = block + 5 * n;
      f.r22 = block + 6 * n;
      f.r12 = block + 7 * n;
    }
    return f;
  }

  bool check(Failure& failure, const char* where) {
    if (error == cudaSuccess) error = cudaGetLastError();
    if (error == cudaSuccess && error_word != nullptr) {
      int word = 0;
      error = cudaMemcpyAsync(&word, error_word, sizeof(int), cudaMemcpyDeviceToHost, stream);
      if (error == cudaSuccess) error = cudaStreamSynchronize(stream);
      if (error == cudaSuccess && word != 0) {
        failure.status = kInternal;
        failure.message = std::string("the device failed in ") + where + ": a bounded wait of the sweep ran out";
        return false;
      }
    }
    if (error == cudaSuccess) return true;
    failure.status = kInternal;
    failure.message = std::string("the device failed in ") + where + ": " + describe(error);
    return false;
  }

  // Device copies of the model: levels, flat blocks, binary64 constants.
  // The samples' intervals and centres on the device.
  void setup_samples() {
    const std::size_t count = samples->intervals.size();
    std::vector<SampleEnds32> ends(count);
    std::vector<SampleEnds64> ends64(count);
    for (std::size_t v = 0; v < count; ++v) {
      // Binary32 ends rounded inward (the result is clipped to the binary64 ones).
      const SampleInterval& e = samples->intervals[v];
      float a = static_cast<float>(e.lower), b = static_cast<float>(e.upper);
      if (static_cast<double>(a) < e.lower) a = std::nextafter(a, 256.0f);
      if (static_cast<double>(b) > e.upper) b = std::nextafter(b, -1.0f);
      ends[v] = SampleEnds32{a, b, static_cast<float>(e.centre), 0.0f};
      ends64[v] = SampleEnds64{e.lower, e.upper, e.centre, 0.0};
    }
    s_ends = upload(ends.data(), count);
    s_ends64 = upload(ends64.data(), count);
    SamplesLevelsParams lp;
    lp.g = g;
    lp.source = upload(samples->levels, samples->rows * samples->columns * samples->stride);
    lp.stride = static_cast<int>(samples->stride);
    lp.first = static_cast<int>(samples->first);
    lp.levels = s_levels = allocate<std::uint16_t>(g.plane * g.channels);
    if (error == cudaSuccess) error = launch_samples_levels(lp, stream);
    if (error == cudaSuccess) error = cudaStreamSynchronize(stream);  // the staged copies' sources
  }

  void setup(bool with_tgv, bool solving = true) {
    tgv = with_tgv;
    const std::size_t n = g.plane * g.channels;
    if (samples != nullptr) setup_samples();
    for (const Component& c : frame.components) {
      ComponentDevice d;
      d.block_rows = static_cast<int>(c.block_rows);
      d.block_columns = static_cast<int>(c.block_columns);
      d.cell_rows = static_cast<int>(c.cell_rows);
      d.cell_columns = static_cast<int>(c.cell_columns);
      d.levels = upload(c.levels.data(), c.levels.size());
      d.flat = upload(c.flat.data(), c.flat.size());
      Constants64 k{};
      for (int i = 0; i < 64; ++i) {
        k.step[i] = c.steps[i];
        k.weight[i] = c.weights[i];
        k.flat_weight[i] = c.flat_weights[i];
        k.shrink[i] = c.shrink[i];
        k.cost[i] = c.costs[i];
      }
      k.slack = c.slack;
      k.mmse = c.mmse ? 1 : 0;
      k.costed = c.costed ? 1 : 0;
      d.constants = upload(&k, 1);
      ProxFactors* f = allocate<ProxFactors>(1);
      factors.push_back(f);
      d.factors = f;
      d.zeta = allocate<float>(c.coefficient_count());
      coefficients.push_back(allocate<double>(c.coefficient_count()));
      components.push_back(d);
    }
    state[0] = fields(with_tgv);
    state[1] = fields(with_tgv);
    tilde = fields(with_tgv);
    xt = allocate<float>(n);
    xts[0] = xt;
    xt_id = 0;
    samples_layout = samples != nullptr ? samples_kernels() : 0;
    fusable = solving && (samples != nullptr ? samples_layout != 0 && samples_iteration_takes(g)
                                             : fused_kernels() && iteration_takes(g, components.data(),
                                                                                  static_cast<int>(components.size())));
    if (fusable) {
      xts[1] = allocate<float>(n);
      cell_rows = components.size() > 1 ? components[1].cell_rows : 1;
      cell_columns = components.size() > 1 ? components[1].cell_columns : 1;
    }
    error_word = allocate<int>(1);
    if (error == cudaSuccess) error = cudaMemsetAsync(error_word, 0, sizeof(int), stream);
    const int planes = (with_tgv ? 8 : 3) * g.channels;
    if (error == cudaSuccess) {
      swept = make_sweep_map(state_maps[0], state[0].x, g, planes) &&
              make_sweep_map(state_maps[1], state[1].x, g, planes) &&
              make_sweep_map(tilde_maps[0], xts[0], g, g.channels) &&
              (!fusable || make_sweep_map(tilde_maps[1], xts[1], g, g.channels));
      fusable = fusable && swept && make_iteration_map(iteration_state_maps[0], state[0].x, g, planes) &&
                make_iteration_map(iteration_state_maps[1], state[1].x, g, planes) &&
                make_iteration_map(iteration_tilde_maps[0], xts[0], g, g.channels) &&
                make_iteration_map(iteration_tilde_maps[1], xts[1], g, g.channels);
      // The primal step's maps: a channel's x, p1 and p2 planes, `channels` planes apart.
      for (std::size_t c = 0; c < components.size(); ++c) {
        bool made = primal_tma_takes(components[c]);
        for (int s = 0; s < 2 && made; ++s) {
          made = make_primal_map(primal_maps[s][c], state[s].x + c * g.plane, g, g.plane * g.channels);
        }
        primal_swept[c] = made;
      }
    }
    v = allocate<float>(n);
    if (with_tgv) div2 = allocate<float>(2 * n);
    canvas = allocate<double>(static_cast<std::size_t>(g.channels) * g.rows * g.columns);
    std::size_t most = std::max<std::size_t>(3u * norms_grid_blocks(g), residual_grid_blocks(g));
    if (samples != nullptr) most = std::max<std::size_t>(most, samples_grid_blocks(g, g.channels));
    for (const ComponentDevice& d : components) {
      most = std::max<std::size_t>(most, conjugate_grid_blocks(g, d));
      most = std::max<std::size_t>(most, start_grid_blocks(d));
      const int count = std::max({primal_grid_blocks(g, d), primal_tma_grid_blocks(g, d), start_grid_blocks(d)});
      value_counts.push_back(count);
      value_written.push_back(0);
    }
    partial_count = most;
    partials = allocate<double>(most);
    {
      std::size_t regions = 0;
      const std::size_t channels = samples != nullptr ? samples->channels : components.size();
      for (std::size_t c = 0; c < channels; ++c) {
        regions += 2 * static_cast<std::size_t>(conjugate_count(c)) + residual_grid_blocks(g);
      }
      record_partials = allocate<double>(std::max<std::size_t>(regions, 1));
      record_sums = allocate<double>(2 * kMaxReductions);
    }
    std::size_t values = 0;
    for (int count : value_counts) values += count;
    if (samples != nullptr) values += samples_grid_blocks(g, g.channels);
    value_partials = allocate<double>(values);
    host_partials.resize(std::max(most, values));
  }

  std::size_t value_offset(std::size_t c) const {
    std::size_t offset = 0;
    for (std::size_t k = 0; k < c; ++k) offset += value_counts[k];
    return offset;
  }

  double* value_slot(std::size_t c) { return value_partials + value_offset(c); }

  // The binary32 factors of each component's proximal map at the plan's tau.
  void set_factors(const Plan& p) {
    for (std::size_t c = 0; c < frame.components.size(); ++c) {
      const Component& comp = frame.components[c];
      ProxFactors f{};
      const double step = p.tau / static_cast<double>(comp.cells());
      for (int k = 0; k < 64; ++k) {
        const double q = static_cast<double>(comp.steps[k]);
        const double reach = (0.5 + comp.slack) * q;
        const double t = step * comp.weights[k];
        const double r = 1.0 / (1.0 + t);
        const double tf = step * comp.flat_weights[k];
        const double rf = 1.0 / (1.0 + tf);
        f.plain[prox_slot(k)] = make_float4(static_cast<float>(q), static_cast<float>(r),
                                            static_cast<float>(t * r), static_cast<float>(reach));
        f.flat[prox_slot(k)] = make_float4(static_cast<float>(q), static_cast<float>(rf),
                                           static_cast<float>(tf * rf), static_cast<float>(reach));
        f.h[k] = static_cast<float>(step * comp.costs[k] * r);
        f.h_flat[k] = static_cast<float>(step * comp.costs[k] * rf);
        f.shrink[k] = static_cast<float>(comp.shrink[k]);
      }
      f.slack = static_cast<float>(comp.slack);
      f.mmse = comp.mmse ? 1 : 0;
      f.costed = comp.costed ? 1 : 0;
      if (error == cudaSuccess) error = cudaMemcpyAsync(factors[c], &f, sizeof(f), cudaMemcpyHostToDevice, stream);
      // The pageable source must outlive the copy.
      if (error == cudaSuccess) error = cudaStreamSynchronize(stream);
    }
  }

  // The sum of n doubles of the device in index order.
  double sum_of(const double* device, std::size_t n, std::size_t offset = 0) {
    if (error != cudaSuccess || n == 0) return 0.0;
    error = cudaMemcpyAsync(host_partials.data(), device + offset, n * sizeof(double), cudaMemcpyDeviceToHost, stream);
    if (error == cudaSuccess) error = cudaStreamSynchronize(stream);
    double total = 0.0;
    for (std::size_t k = 0; k < n; ++k) total += host_partials[k];
    return total;
  }

  double max_of(const double* device, std::size_t n, std::size_t offset) {
    if (error != cudaSuccess || n == 0) return 0.0;
    error = cudaMemcpyAsync(host_partials.data(), device + offset, n * sizeof(double), cudaMemcpyDeviceToHost, stream);
    if (error == cudaSuccess) error = cudaStreamSynchronize(stream);
    double most = 0.0;
    for (std::size_t k = 0; k < n; ++k) most = std::fmax(most, host_partials[k]);
    return most;
  }

  double data_value() {
    if (samples != nullptr) return sum_of(value_partials, samples_written);
    double total = 0.0;
    for (std::size_t c = 0; c < components.size(); ++c) total += sum_of(value_slot(c), value_written[c]);
    return total;
  }

  // The start (cpp/src/primal_dual.hpp:401-432): x from the clipped centres (or the given
  // coefficients), 128 past the blocks; w = grad x; the duals 0 or given, projected. The
  // start is the first tilde point.
  void start(const Start* given, bool for_solver) {
    if (samples != nullptr) {
      // The centres: x0 and the binary64 canvas; G there is 0.
      SamplesCanvasParams sp;
      sp.g = g;
      sp.mode = 0;
      sp.x = state[0].x;
      sp.levels = s_levels;
      sp.ends64 = s_ends64;
      sp.canvas = canvas;
      if (error == cudaSuccess) error = launch_samples_canvas(sp, stream);
      samples_written = 0;
    }
    for (std::size_t c = 0; c < components.size(); ++c) {
      StartParams sp;
      sp.component = components[c];
      sp.coefficients = coefficients[c];
      sp.partials = value_slot(c);
      sp.record_first = g.record_first;
      sp.record_end = g.record_end;
      const double* given_coefficients = nullptr;
      if (given != nullptr && !given->coefficients.empty()) {
        given_coefficients = upload(given->coefficients[c].data(), given->coefficients[c].size());
      }
      sp.given = given_coefficients;
      if (error == cudaSuccess) error = launch_start_coefficients(sp, stream);
      value_written[c] = start_grid_blocks(components[c]);
      CanvasParams cp;
      cp.g = g;
      cp.component = components[c];
      cp.coefficients = coefficients[c];
      cp.canvas = canvas + static_cast<std::size_t>(c) * g.rows * g.columns;
      cp.x = for_solver ? state[0].x + c * g.plane : nullptr;
      cp.beyond = 128.0;
      cp.mode = 0;
      if (error == cudaSuccess) error = launch_canvas(cp, stream);
    }
    if (!for_solver) return;
    const std::size_t n = g.plane * g.channels;
    auto put = [&](float* to, const std::vector<double>& from, std::size_t entries, std::size_t entry) {
      // channel-major host fields of `entries` planes each -> the pitched plane `entry`.
      std::vector<float> staged(n, 0.0f);
      for (int c = 0; c < g.channels; ++c) {
        for (int i = 0; i < g.rows; ++i) {
          for (int j = 0; j < g.columns; ++j) {
            staged[c * g.plane + static_cast<std::size_t>(i) * g.pitch + j] = static_cast<float>(
                from[((c * entries + entry) * g.rows + i) * static_cast<std::size_t>(g.columns) + j]);
          }
        }
      }
      if (error == cudaSuccess) error = cudaMemcpyAsync(to, staged.data(), n * sizeof(float), cudaMemcpyHostToDevice, stream);
      if (error == cudaSuccess) error = cudaStreamSynchronize(stream);
    };
    Fields& s = state[0];
    const bool given_p = given != nullptr && !given->p.empty();
    const bool given_w = given != nullptr && !given->w.empty();
    const bool given_r = given != nullptr && !given->r.empty();
    if (given_p) {
      put(s.p1, given->p, 2, 0);
      put(s.p2, given->p, 2, 1);
    } else {
      if (error == cudaSuccess) error = cudaMemsetAsync(s.p1, 0, n * sizeof(float), stream);
      if (error == cudaSuccess) error = cudaMemsetAsync(s.p2, 0, n * sizeof(float), stream);
    }
    if (tgv) {
      if (given_w) {
        put(s.w1, given->w, 2, 0);
        put(s.w2, given->w, 2, 1);
      } else if (error == cudaSuccess) {
        error = launch_gradient(s.x, s.w1, s.w2, g, stream);
      }
      if (given_r) {
        put(s.r11, given->r, 3, 0);
        put(s.r22, given->r, 3, 1);
        put(s.r12, given->r, 3, 2);
      } else {
        for (float* f : {s.r11, s.r22, s.r12}) {
          if (error == cudaSuccess) error = cudaMemsetAsync(f, 0, n * sizeof(float), stream);
        }
      }
    }
    if ((given_p || given_r) && error == cudaSuccess) {
      error = launch_project(s, g, tgv, plan.coupled, static_cast<float>(tgv ? plan.alpha1 : plan.alpha),
                             static_cast<float>(plan.alpha0), stream);
    }
    // The start is the first tilde point.
    auto copy = [&](float* to, const float* from) {
      if (error == cudaSuccess && to != nullptr) {
        error = cudaMemcpyAsync(to, from, n * sizeof(float), cudaMemcpyDeviceToDevice, stream);
      }
    };
    copy(xt, s.x);
    copy(tilde.p1, s.p1);
    copy(tilde.p2, s.p2);
    if (tgv) {
      copy(tilde.w1, s.w1);
      copy(tilde.w2, s.w2);
      copy(tilde.r11, s.r11);
      copy(tilde.r22, s.r22);
      copy(tilde.r12, s.r12);
    }
    current = 0;
  }

  PrimalParams primal_params(std::size_t c) const {
    const Fields& s = state[current];
    PrimalParams pp;
    pp.g = g;
    pp.component = components[c];
    const std::size_t base = c * g.plane;
    pp.x = s.x + base;
    pp.p1 = s.p1 + base;
    pp.p2 = s.p2 + base;
    pp.xt = xt + base;
    pp.v = v + base;
    pp.partials = value_partials + value_offset(c);
    pp.descent = static_cast<float>(plan.tau * plan.channel_weights[c]);
    pp.error = error_word;
    return pp;
  }

  // The primal step of every component; the TMA path takes two components of the same cells
  // (Cb and Cr) in one launch.
  void primal(bool keep) {
    plain_primal = plain_primal || !keep;
    if (samples != nullptr) {
      const Fields& st = state[current];
      SamplesPrimalParams sp;
      sp.g = g;
      sp.x = st.x;
      sp.p1 = st.p1;
      sp.p2 = st.p2;
      sp.xt = xt;
      sp.levels = s_levels;
      sp.ends = s_ends;
      sp.ends64 = s_ends64;
      for (int c = 0; c < g.channels; ++c) sp.descent[c] = static_cast<float>(plan.tau * plan.channel_weights[c]);
      const double t = plan.tau * samples->mu;
      sp.t = static_cast<float>(t);
      sp.r = static_cast<float>(1.0 / (1.0 + t));
      sp.half_mu = 0.5 * samples->mu;
      sp.partials = value_partials;
      if (error == cudaSuccess) error = launch_samples_primal(sp, keep, stream);
      if (keep) samples_written = samples_primal_blocks(g);
      return;
    }
    for (std::size_t c = 0; c < components.size();) {
      if (!primal_swept[c]) {
        const PrimalParams pp = primal_params(c);
        if (error == cudaSuccess) error = launch_primal(pp, keep, stream);
        if (keep) value_written[c] = primal_grid_blocks(g, components[c]);
        ++c;
        continue;
      }
      const bool pair = c + 1 < components.size() && primal_swept[c + 1] &&
                        components[c + 1].cell_rows == components[c].cell_rows &&
                        components[c + 1].cell_columns == components[c].cell_columns;
      const int count = pair ? 2 : 1;
      const PrimalParams parts[2] = {primal_params(c), primal_params(pair ? c + 1 : c)};
      const CUtensorMap maps[2] = {primal_maps[current][c], primal_maps[current][pair ? c + 1 : c]};
      int grid = 0;
      if (error == cudaSuccess) error = launch_primal_tma(maps, parts, count, keep, stream, &grid);
      if (keep) {
        value_written[c] = grid;
        if (pair) value_written[c + 1] = grid;
      }
      c += count;
    }
  }

  DualParams dual_params() const {
    DualParams dp;
    dp.g = g;
    dp.xt = xt;
    dp.in = state[current];
    dp.out = state[1 - current];
    dp.tilde = tilde;
    if (tgv && !plan.partial_radius) {
      // TGV's records read p~ only for the partial gap: without it, the dual step keeps none.
      dp.tilde.p1 = nullptr;
      dp.tilde.p2 = nullptr;
    }
    for (int c = 0; c < g.channels; ++c) {
      dp.sigma[c] = static_cast<float>(plan.sigma * plan.channel_weights[c]);
      dp.tau[c] = static_cast<float>(plan.tau * plan.channel_weights[c]);
    }
    dp.rho = static_cast<float>(plan.relaxation);
    dp.rest = static_cast<float>(1.0 - plan.relaxation);
    dp.radius = static_cast<float>(tgv ? plan.alpha1 : plan.alpha);
    dp.radius0 = static_cast<float>(plan.alpha0);
    dp.error = error_word;
    dp.ring_wait_limit = ring_wait_limit();
    return dp;
  }

  void dual(bool keep) {
    plain_dual = plain_dual || !keep;
    const DualParams dp = dual_params();
    if (error == cudaSuccess) {
      error = swept ? launch_dual_tma(state_maps[current], tilde_maps[xt_id], dp, tgv, plan.coupled, keep, stream)
                    : launch_dual(dp, tgv, plan.coupled, keep, stream);
    }
    current = 1 - current;
  }

  // The dual step of iteration n and the primal step of iteration n + 1 as one sweep
  // (iteration.cu), keeping nothing: from x~_n and s_{n-1} to s_n and x~_{n+1}.
  // Launches kGraphIterations iterations that keep nothing -- dual(false), primal(false), each
  // time -- as one graph; false (nothing launched) where the solve does not take graphs. The
  // launches depend on the iteration only through the parity of the state, which an even count
  // of iterations leaves as it found it.
  bool group() {
    if (!plain_dual || !plain_primal || fusable || samples != nullptr || error != cudaSuccess || !group_graphs()) {
      return false;
    }
    if (group_exec == nullptr || group_parity != current) {
      if (group_exec != nullptr) {
        cudaGraphExecDestroy(group_exec);
        group_exec = nullptr;
      }
      const int parity = current;
      cudaGraph_t graph = nullptr;
      if (cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
        cudaGetLastError();
        return false;
      }
      for (std::uint64_t k = 0; k < kGraphIterations; ++k) {
        dual(false);
        primal(false);
      }
      const cudaError_t ended = cudaStreamEndCapture(stream, &graph);
      if (error == cudaSuccess) error = ended;
      if (error == cudaSuccess) error = cudaGraphInstantiate(&group_exec, graph, 0);
      if (graph != nullptr) cudaGraphDestroy(graph);
      if (error != cudaSuccess) return false;
      group_parity = parity;
    }
    error = cudaGraphLaunch(group_exec, stream);
    return error == cudaSuccess;
  }

  void fused() {
    if (samples != nullptr && samples_layout == 2) {
      SamplesStep q;
      q.levels = s_levels;
      q.ends = s_ends;
      const double t = plan.tau * samples->mu;
      q.t = static_cast<float>(t);
      q.r = static_cast<float>(1.0 / (1.0 + t));
      q.next = xts[1 - xt_id];
      if (error == cudaSuccess) {
        error = launch_dual_samples(state_maps[current], tilde_maps[xt_id], dual_params(), q, tgv, plan.coupled,
                                    stream);
      }
      current = 1 - current;
      xt_id = 1 - xt_id;
      xt = xts[xt_id];
      return;
    }
    if (samples != nullptr) {
      SamplesIterationParams sp;
      sp.dual = dual_params();
      sp.levels = s_levels;
      sp.ends = s_ends;
      const double t = plan.tau * samples->mu;
      sp.t = static_cast<float>(t);
      sp.r = static_cast<float>(1.0 / (1.0 + t));
      sp.next = xts[1 - xt_id];
      if (error == cudaSuccess) {
        error = launch_samples_iteration(iteration_state_maps[current], iteration_tilde_maps[xt_id], sp, tgv,
                                         plan.coupled, stream);
      }
      current = 1 - current;
      xt_id = 1 - xt_id;
      xt = xts[xt_id];
      return;
    }
    IterationParams ip;
    ip.dual = dual_params();
    for (std::size_t c = 0; c < components.size(); ++c) ip.component[c] = components[c];
    ip.next = xts[1 - xt_id];
    if (error == cudaSuccess) {
      error = launch_iteration(iteration_state_maps[current], iteration_tilde_maps[xt_id], ip, tgv, plan.coupled,
                               cell_rows, cell_columns, stream);
    }
    current = 1 - current;
    xt_id = 1 - xt_id;
    xt = xts[xt_id];
  }

  // G* of channel c at xi = gamma div(scale q) (cpp/src/frames.cpp:428-493).
  double conjugate(std::size_t c, const float* q1, const float* q2, double scale) {
    return sum_of(partials, conjugate_into(c, q1, q2, scale, nullptr, partials));
  }

  // The per-CTA partials of G* of channel c into `out`; returns their count. With `most_at`,
  // the scale is -theta of the largest |div_2 r~| read there (negative_theta).
  int conjugate_count(std::size_t c) const {
    if (samples != nullptr) {
      Geometry one = g;
      one.channels = 1;
      return samples_grid_blocks(one, 1);
    }
    return conjugate_grid_blocks(g, components[c]);
  }
  int conjugate_into(std::size_t c, const float* q1, const float* q2, double scale, const double* most_at,
                     double* out) {
    if (samples != nullptr) {
      SamplesConjugateParams sp;
      sp.g = g;
      sp.g.channels = 1;
      sp.q1 = q1;
      sp.q2 = q2;
      sp.scale = scale;
      sp.most_at = most_at;
      sp.alpha1 = plan.alpha1;
      sp.gamma = plan.channel_weights[c];
      sp.mu = samples->mu;
      sp.levels = s_levels + c * g.plane;
      sp.ends64 = s_ends64;
      sp.partials = out;
      if (error == cudaSuccess) error = launch_samples_conjugate(sp, stream);
      return conjugate_count(c);
    }
    ConjugateParams cp;
    cp.g = g;
    cp.component = components[c];
    cp.q1 = q1;
    cp.q2 = q2;
    cp.scale = scale;
    cp.most_at = most_at;
    cp.alpha1 = plan.alpha1;
    cp.gamma = plan.channel_weights[c];
    cp.radius = plan.free_radius;
    cp.free = frame.components[c].free ? 1 : 0;
    cp.partials = out;
    if (error == cudaSuccess) error = launch_conjugate(cp, stream);
    return conjugate_count(c);
  }

  // The channels of the data term: the components, or the samples' channels.
  std::size_t data_channels() const { return samples != nullptr ? samples->channels : components.size(); }

  // The first sums of a record, over the record rows (Geometry::record_first/end: the canvas,
  // or a strip's own bands): G at the kept coefficients, the first-order norms, and for TGV the
  // second-order norms and the largest |div2 r~| (cpp/src/primal_dual.hpp:446-501, 836-895).
  struct FirstSums {
    double data = 0.0, first = 0.0, second = 0.0, most = 0.0;
  };
  FirstSums first_sums() {
    FirstSums f;
    f.data = data_value();
    NormParams np;
    np.g = g;
    np.xt = xt;
    np.tilde = tilde;
    np.div2 = div2;
    for (int c = 0; c < g.channels; ++c) np.weight[c] = plan.channel_weights[c];
    np.partials = partials;
    if (error == cudaSuccess) error = launch_norms(np, tgv, plan.coupled, stream);
    const std::size_t count = norms_grid_blocks(g);
    f.first = sum_of(partials, count, 0);
    if (tgv) {
      f.second = sum_of(partials, count, count);
      f.most = max_of(partials, count, 2 * count);
    }
    return f;
  }

  // The second sums at the scaling theta: G*(-gamma div(theta div2 r~)) (TGV) or G*(gamma div
  // p~) (TV) summed over the channels; with a partial radius (TGV), the partial gap's
  // G*(gamma div p~) and its residual.
  struct SecondSums {
    double conjugates = 0.0, partial = 0.0, residual = 0.0;
  };
  SecondSums second_sums(double theta) {
    SecondSums s;
    if (!tgv) {
      for (std::size_t c = 0; c < data_channels(); ++c) {
        s.conjugates += conjugate(c, tilde.p1 + c * g.plane, tilde.p2 + c * g.plane, 1.0);
      }
      return s;
    }
    for (std::size_t c = 0; c < data_channels(); ++c) {
      const std::size_t base = 2 * c * g.plane;
      s.conjugates += conjugate(c, div2 + base, div2 + base + g.plane, -theta);
    }
    if (plan.partial_radius) {
      const std::size_t count = residual_grid_blocks(g);
      for (std::size_t c = 0; c < data_channels(); ++c) {
        s.partial += conjugate(c, tilde.p1 + c * g.plane, tilde.p2 + c * g.plane, 1.0);
        ResidualParams rp;
        rp.g = g;
        rp.p1 = tilde.p1 + c * g.plane;
        rp.p2 = tilde.p2 + c * g.plane;
        rp.d1 = div2 + 2 * c * g.plane;
        rp.d2 = div2 + (2 * c + 1) * g.plane;
        rp.partials = partials;
        if (error == cudaSuccess) error = launch_residual(rp, stream);
        s.residual += plan.channel_weights[c] * sum_of(partials, count);
      }
    }
    return s;
  }

  // The record of the tilde point (cpp/src/primal_dual.hpp:446-501), its kernels back to back
  // with no host round trip among them: the norms, then every sum reduced on the device (the
  // norms, the largest |div_2 r~|, the data term of each component), the conjugates at the theta
  // those give (read on the device), their sums, and one copy of the sums to the host.
  Record record(std::uint64_t iteration) {
    Record r;
    r.iteration = iteration;
    r.scaling = kNaN;
    r.partial_gap = kNaN;
    NormParams np;
    np.g = g;
    np.xt = xt;
    np.tilde = tilde;
    np.div2 = div2;
    for (int c = 0; c < g.channels; ++c) np.weight[c] = plan.channel_weights[c];
    np.partials = partials;
    if (error == cudaSuccess) error = launch_norms(np, tgv, plan.coupled, stream);
    const int count = norms_grid_blocks(g);
    Reductions first;
    first.out = record_sums;
    const int at_first = first.add(partials, count);
    const int at_second = tgv ? first.add(partials + count, count) : -1;
    const int at_most = tgv ? first.add(partials + 2 * count, count, true) : -1;
    std::vector<int> at_data;
    if (samples != nullptr) {
      at_data.push_back(first.add(value_partials, static_cast<int>(samples_written)));
    } else {
      for (std::size_t c = 0; c < components.size(); ++c) {
        at_data.push_back(first.add(value_slot(c), static_cast<int>(value_written[c])));
      }
    }
    if (error == cudaSuccess) error = launch_reductions(first, stream);
    // The conjugates of each channel into regions of their own, then their sums.
    Reductions second;
    second.out = record_sums + kMaxReductions;
    double* region = record_partials;
    std::vector<int> at_dual, at_partial, at_residual;
    const double* most_at = tgv ? record_sums + at_most : nullptr;
    for (std::size_t c = 0; c < data_channels(); ++c) {
      const float* q1 = tgv ? div2 + 2 * c * g.plane : tilde.p1 + c * g.plane;
      const float* q2 = tgv ? div2 + (2 * c + 1) * g.plane : tilde.p2 + c * g.plane;
      const int n = conjugate_into(c, q1, q2, 1.0, most_at, region);
      at_dual.push_back(second.add(region, n));
      region += n;
    }
    if (tgv && plan.partial_radius) {
      for (std::size_t c = 0; c < data_channels(); ++c) {
        const int n = conjugate_into(c, tilde.p1 + c * g.plane, tilde.p2 + c * g.plane, 1.0, nullptr, region);
        at_partial.push_back(second.add(region, n));
        region += n;
        ResidualParams rp;
        rp.g = g;
        rp.p1 = tilde.p1 + c * g.plane;
        rp.p2 = tilde.p2 + c * g.plane;
        rp.d1 = div2 + 2 * c * g.plane;
        rp.d2 = div2 + (2 * c + 1) * g.plane;
        rp.partials = region;
        if (error == cudaSuccess) error = launch_residual(rp, stream);
        const int residuals = residual_grid_blocks(g);
        at_residual.push_back(second.add(region, residuals));
        region += residuals;
      }
    }
    if (error == cudaSuccess) error = launch_reductions(second, stream);
    double sums[2 * kMaxReductions] = {};
    if (error == cudaSuccess) {
      error = cudaMemcpyAsync(sums, record_sums, sizeof(sums), cudaMemcpyDeviceToHost, stream);
    }
    if (error == cudaSuccess) error = cudaStreamSynchronize(stream);
    if (error != cudaSuccess) return r;
    const double* second_sums = sums + kMaxReductions;
    double data = 0.0;
    for (int k : at_data) data += sums[k];
    double conjugates = 0.0;
    for (int k : at_dual) conjugates += second_sums[k];
    r.dual = -conjugates;
    if (!tgv) {
      r.primal = plan.alpha * sums[at_first] + data;
      return r;
    }
    r.primal = (plan.alpha1 * sums[at_first] + plan.alpha0 * sums[at_second]) + data;
    r.scaling = -negative_theta(sums[at_most], plan.alpha1);
    if (plan.partial_radius) {
      double partial = 0.0, residual = 0.0;
      for (std::size_t c = 0; c < at_partial.size(); ++c) {
        partial += second_sums[at_partial[c]];
        residual += plan.channel_weights[c] * second_sums[at_residual[c]];
      }
      r.partial_gap = r.primal + partial + *plan.partial_radius * residual;
    }
    return r;
  }

  // The binary64 result from the last kept coefficients (docs/math.md 5: the canvas whose
  // coefficients are zeta).
  void result(Outcome& out) {
    make_canvas();
    if (host_result) fetch(out);
  }

  // The binary64 canvas of the last kept tilde point into `canvas` (channels x rows x columns),
  // as the result has it: the coefficients zeta restored to binary64 and clipped to their
  // intervals, the canvas whose coefficients they are.
  void make_canvas() {
    const std::size_t size = static_cast<std::size_t>(g.rows) * g.columns;
    if (samples != nullptr) {
      // The last tilde point in binary64, each sample clipped to its interval.
      SamplesCanvasParams sp;
      sp.g = g;
      sp.mode = 1;
      sp.xt = xt;
      sp.levels = s_levels;
      sp.ends64 = s_ends64;
      sp.canvas = canvas;
      if (error == cudaSuccess) error = launch_samples_canvas(sp, stream);
    }
    for (std::size_t c = 0; c < components.size(); ++c) {
      if (error == cudaSuccess) error = launch_restore(components[c], coefficients[c], stream);
      CanvasParams cp;
      cp.g = g;
      cp.component = components[c];
      cp.coefficients = coefficients[c];
      cp.canvas = canvas + c * size;
      cp.v = v + c * g.plane;
      cp.mode = 1;
      if (error == cudaSuccess) error = launch_canvas(cp, stream);
    }
  }

  // The picture's 8- or 16-bit levels into host memory `out` (height x width x its channels,
  // interleaved; 16 bits most significant byte first), from the binary64 canvas on the device:
  // the picture made there (JFIF RGB of YCbCr), quantized there (output.cu), and only the
  // levels copied out. False, with *not_finite set, where a sample of the picture is not finite.
  void levels(bool sixteen, int dither, std::uint8_t* out, bool& not_finite) {
    not_finite = false;
    const std::size_t pixels = static_cast<std::size_t>(frame.height) * frame.width;
    const bool rgb = frame.color_space == 2 && g.channels == 3;
    PictureParams pp;
    pp.canvas = canvas;
    pp.channels = g.channels;
    pp.rows = g.rows;
    pp.columns = g.columns;
    pp.height = static_cast<int>(frame.height);
    pp.width = static_cast<int>(frame.width);
    pp.rgb = rgb;
    pp.picture = allocate<double>(pixels * g.channels);
    if (error == cudaSuccess) error = launch_picture(pp, stream);
    LevelsParams lp;
    lp.samples = pp.picture;
    lp.count = pixels * g.channels;
    lp.width = static_cast<int>(frame.width);
    lp.channels = g.channels;
    lp.scale = sixteen ? 257.0 : 1.0;
    lp.top = sixteen ? 65535.0 : 255.0;
    lp.dither = dither;
    lp.sixteen = sixteen;
    const std::size_t bytes_out = lp.count * (sixteen ? 2 : 1);
    lp.out = allocate<std::uint8_t>(bytes_out);
    lp.not_finite = allocate<int>(1);
    if (error == cudaSuccess && !prepare_levels()) error = cudaErrorInitializationError;
    if (error == cudaSuccess) error = cudaMemsetAsync(lp.not_finite, 0, sizeof(int), stream);
    if (error == cudaSuccess) error = launch_levels(lp, stream);
    int flag = 0;
    if (error == cudaSuccess) error = cudaMemcpyAsync(&flag, lp.not_finite, sizeof(int), cudaMemcpyDeviceToHost, stream);
    if (error == cudaSuccess) error = cudaMemcpyAsync(out, lp.out, bytes_out, cudaMemcpyDeviceToHost, stream);
    if (error == cudaSuccess) error = cudaStreamSynchronize(stream);
    not_finite = flag != 0;
  }

  // The result into host memory: the binary64 canvas and coefficients, and the picture made
  // from the canvas on the device (the planes cut to the picture where the canvas is larger,
  // the channels interleaved, JFIF's RGB of YCbCr), each copied once into pinned memory.
  void fetch(Outcome& out) {
    const std::size_t size = static_cast<std::size_t>(g.rows) * g.columns;
    const std::size_t pixels = static_cast<std::size_t>(frame.height) * frame.width;
    const bool cut = frame.height != frame.rows || frame.width != frame.columns;
    const bool interleaved = g.channels > 1;
    PictureParams pp;
    pp.canvas = canvas;
    pp.channels = g.channels;
    pp.rows = g.rows;
    pp.columns = g.columns;
    pp.height = static_cast<int>(frame.height);
    pp.width = static_cast<int>(frame.width);
    pp.rgb = frame.color_space == 2 && g.channels == 3;
    if (cut) pp.planes = allocate<double>(pixels * g.channels);
    if (interleaved) pp.picture = allocate<double>(pixels * g.channels);
    if (error == cudaSuccess) error = launch_picture(pp, stream);
    auto copy = [&](HostBuffer& to, const double* from, std::size_t count) {
      to.resize(count);
      if (error == cudaSuccess && count > 0) {
        error = cudaMemcpyAsync(to.data(), from, count * sizeof(double), cudaMemcpyDeviceToHost, stream);
      }
    };
    copy(out.canvas, canvas, size * g.channels);
    copy(out.planes, pp.planes, cut ? pixels * g.channels : 0);
    copy(out.picture, pp.picture, interleaved ? pixels * g.channels : 0);
    out.coefficients.resize(components.size());
    for (std::size_t c = 0; c < components.size(); ++c) {
      copy(out.coefficients[c], coefficients[c], frame.components[c].coefficient_count());
    }
    if (error == cudaSuccess) error = cudaStreamSynchronize(stream);
  }
};

Solver::Solver(const Frame& frame, cudaStream_t stream) : impl_(std::make_unique<Impl>(frame, stream)) {
  geometry_.rows = static_cast<int>(frame.rows);
  geometry_.columns = static_cast<int>(frame.columns);
  geometry_.pitch = static_cast<int>((frame.columns + 31) / 32 * 32);
  geometry_.channels = static_cast<int>(frame.channels());
  geometry_.plane = static_cast<std::size_t>(geometry_.rows) * geometry_.pitch;
  impl_->g = geometry_;
}

Solver::Solver(const Frame& frame, const SamplesModel& samples, cudaStream_t stream)
    : impl_(std::make_unique<Impl>(frame, stream)) {
  geometry_.rows = static_cast<int>(samples.rows);
  geometry_.columns = static_cast<int>(samples.columns);
  geometry_.pitch = static_cast<int>((samples.columns + 31) / 32 * 32);
  geometry_.channels = static_cast<int>(samples.channels);
  geometry_.plane = static_cast<std::size_t>(geometry_.rows) * geometry_.pitch;
  impl_->g = geometry_;
  impl_->samples = &samples;
}

Solver::~Solver() = default;

int Solver::launches_per_iteration() const {
  if (impl_->samples != nullptr) return impl_->fusable ? 1 : 2;
  return impl_->fusable ? 1 : 1 + static_cast<int>(impl_->components.size());
}

bool Solver::solve(Method method, const Plan* plan, const Start* start, const Observer& observer, Outcome& out,
                   Failure& failure) {
  Impl& m = *impl_;
  const bool solver = method == Method::tv || method == Method::tgv;
  if (!solver) {
    // The decoder of the centres (docs/math.md 2.3).
    m.setup(false, false);
    m.start(nullptr, false);
    if (m.host_result) m.fetch(out);
    bytes_ = m.bytes;
    out.solved = false;
    out.stop = 0;
    return m.check(failure, "the decoder of the centres");
  }
  m.plan = *plan;
  m.setup(plan->tgv);
  m.set_factors(*plan);
  m.start(start, true);
  bytes_ = m.bytes;
  if (!m.check(failure, "the start")) return false;
  return run(0, observer, out, failure);
}

// The method's loop from `first` iterations made (their primal and dual steps done, the state
// of iteration `first` the current one) to the end: records, stops and the result.
bool Solver::run(std::uint64_t first, const Observer& observer, Outcome& out, Failure& failure) {
  Impl& m = *impl_;
  const Plan* plan = &m.plan;
  out.tau = plan->tau;
  out.sigma = plan->sigma;
  const double samples = static_cast<double>(m.g.channels) * m.g.rows * m.g.columns;
  const std::uint64_t most = plan->iterations;
  const std::uint64_t every = plan->record_every;
  using Clock = std::chrono::steady_clock;
  const auto began = Clock::now();
  double recording = 0.0;
  std::int32_t stop = 0;
  auto take = [&](std::uint64_t iteration) -> bool {
    const auto at = Clock::now();
    if (m.error == cudaSuccess) m.error = cudaStreamSynchronize(m.stream);
    Record r = m.record(iteration);
    const auto done = Clock::now();
    recording += std::chrono::duration<double>(done - at).count();
    r.seconds = std::chrono::duration<double>(at - began).count();
    if (m.error != cudaSuccess) return true;
    const double gap = r.primal - r.dual;
    bool met = false;
    if (plan->tolerance > 0.0 && gap / samples <= plan->tolerance) met = true;
    if (plan->relative_tolerance > 0.0 && gap <= plan->relative_tolerance * r.primal) met = true;
    if (plan->partial_tolerance > 0.0 && !std::isnan(r.partial_gap) &&
        r.partial_gap / samples <= plan->partial_tolerance) {
      met = true;
    }
    out.records.push_back(r);
    if (met) {
      stop = 1;
      return true;
    }
    if (observer && out.records.size() > 1) {
      // The record's canvas as the result would have it, were the solve to stop here.
      const Geometry whole = m.g;
      m.make_canvas();
      std::vector<double> host(static_cast<std::size_t>(whole.channels) * whole.rows * whole.columns);
      if (m.error == cudaSuccess) {
        m.error = cudaMemcpyAsync(host.data(), m.canvas, host.size() * sizeof(double), cudaMemcpyDeviceToHost, m.stream);
      }
      if (m.error == cudaSuccess) m.error = cudaStreamSynchronize(m.stream);
      if (m.error == cudaSuccess && observer(r, gap / samples, host.data())) {
        stop = 3;
        return true;
      }
    }
    return false;
  };
  auto recorded = [&](std::uint64_t n) { return (every > 0 && n % every == 0) || n == most; };
  auto none_recorded = [&](std::uint64_t from, std::uint64_t to) {
    for (std::uint64_t n = from; n <= to; ++n) {
      if (recorded(n)) return false;
    }
    return true;
  };
  bool stopped = false;
  if (first == 0 && (every > 0 || most == 0)) stopped = take(0);
  std::uint64_t iteration = first;
  if (!stopped && first < most) m.primal(recorded(first + 1));
  while (!stopped && iteration < most && m.error == cudaSuccess) {
    const std::uint64_t next = iteration + 1;
    // One sweep for D_next and P_{next+1} when neither keeps anything: no record after the
    // dual step, none of the next iterate, and a next iteration to make.
    if (m.fusable && next < most && !recorded(next) && !recorded(next + 1)) {
      m.fused();
      iteration = next;
      continue;
    }
    // D_next, P_{next+1}, ..., D_{next+G-1}, P_{next+G} (G = kGraphIterations) as one graph when
    // none of them keeps anything.
    if (next + kGraphIterations - 1 < most && none_recorded(next, next + kGraphIterations) && m.group()) {
      iteration = next + kGraphIterations - 1;
      continue;
    }
    if (m.error != cudaSuccess) break;
    m.dual(recorded(next));
    iteration = next;
    if (recorded(iteration)) stopped = take(iteration);
    if (!stopped && iteration < most) m.primal(recorded(iteration + 1));
  }
  (void)recording;
  if (!m.check(failure, "the iterations")) return false;
  out.iterations = iteration;
  out.stop = stopped ? stop : 2;
  if (out.stop == 0) out.stop = 2;
  out.solved = true;
  if (iteration == 0) {
    // No iteration: the start itself, in binary64.
    if (m.host_result) m.fetch(out);
  } else {
    m.result(out);
  }
  return m.check(failure, "the result");
}

bool Solver::begin_batch(const Plan& plan, Failure& failure) {
  Impl& m = *impl_;
  m.plan = plan;
  m.setup(plan.tgv, false);
  m.set_factors(plan);
  m.start(nullptr, true);
  bytes_ = m.bytes;
  return m.check(failure, "the start");
}

bool Solver::batch_entries(DualBatchImage& image, std::vector<PrimalBatchComponent>& components) {
  Impl& m = *impl_;
  if (!m.swept) return false;
  const int saved = m.current;
  for (int s = 0; s < 2; ++s) {
    m.current = s;
    image.state[s] = m.state_maps[s];
    image.params[s] = m.dual_params();
  }
  image.tilde = m.tilde_maps[m.xt_id];
  components.clear();
  for (std::size_t c = 0; c < m.components.size(); ++c) {
    if (!m.primal_swept[c]) {
      m.current = saved;
      return false;
    }
    PrimalBatchComponent entry;
    for (int s = 0; s < 2; ++s) {
      m.current = s;
      entry.map[s] = m.primal_maps[s][c];
      entry.params[s] = m.primal_params(c);
    }
    components.push_back(entry);
  }
  m.current = saved;
  return true;
}

bool Solver::finish_batch(std::uint64_t done, Outcome& out, Failure& failure) {
  Impl& m = *impl_;
  m.current = static_cast<int>(done % 2);
  if (!m.check(failure, "the batched iterations")) return false;
  return run(done, Observer{}, out, failure);
}

bool Solver::step(std::uint64_t iterations, Failure& failure) {
  Impl& m = *impl_;
  for (std::uint64_t n = 0; n < iterations && m.error == cudaSuccess; ++n) {
    m.primal(false);
    m.dual(false);
  }
  if (m.error == cudaSuccess) m.error = cudaStreamSynchronize(m.stream);
  return m.check(failure, "the strip's iterations");
}

bool Solver::advance(std::uint64_t iterations, Failure& failure) {
  Impl& m = *impl_;
  for (std::uint64_t n = 0; n < iterations && m.error == cudaSuccess; ++n) {
    m.primal(false);
    m.dual(false);
  }
  if (m.error == cudaSuccess) m.error = cudaGetLastError();
  if (m.error == cudaSuccess) return true;
  failure.status = kInternal;
  failure.message = std::string("the device failed in the strip's iterations: ") + describe(m.error);
  return false;
}

cudaStream_t Solver::stream() const { return impl_->stream; }

void Solver::set_record_rows(int first, int end) {
  impl_->g.record_first = first;
  impl_->g.record_end = end;
  geometry_ = impl_->g;
}

bool Solver::record_step(bool advance, double (&first)[5], Failure& failure) {
  Impl& m = *impl_;
  if (advance) {
    m.primal(true);
    m.dual(true);
  }
  if (m.error == cudaSuccess) m.error = cudaStreamSynchronize(m.stream);
  const Impl::FirstSums f = m.first_sums();
  const int counted = std::max(0, std::min(m.g.record_end, m.g.rows) - std::max(m.g.record_first, 0));
  first[0] = f.data;
  first[1] = f.first;
  first[2] = f.second;
  first[3] = f.most;
  first[4] = static_cast<double>(m.g.channels) * counted * m.g.columns;
  return m.check(failure, "the strip's record");
}

bool Solver::record_duals(double theta, double (&second)[3], Failure& failure) {
  Impl& m = *impl_;
  const Impl::SecondSums s = m.second_sums(theta);
  second[0] = s.conjugates;
  second[1] = s.partial;
  second[2] = s.residual;
  return m.check(failure, "the strip's record");
}

bool Solver::finish_here(std::uint64_t done, std::int32_t stop, Outcome& out, Failure& failure) {
  Impl& m = *impl_;
  if (!m.check(failure, "the strip's iterations")) return false;
  out.tau = m.plan.tau;
  out.sigma = m.plan.sigma;
  out.iterations = done;
  out.stop = stop;
  out.solved = true;
  if (done == 0) {
    if (m.host_result) m.fetch(out);
  } else {
    m.result(out);
  }
  return m.check(failure, "the result");
}

int Solver::state_planes(float** planes, int most) const {
  const Impl& m = *impl_;
  const Fields& f = m.state[m.current];
  const float* fields[8] = {f.x, f.p1, f.p2, f.w1, f.w2, f.r11, f.r22, f.r12};
  const int channels = m.g.channels;
  const int count = (m.tgv ? 8 : 3) * channels;
  for (int k = 0; k < count && k < most; ++k) {
    planes[k] = const_cast<float*>(fields[k / channels]) + static_cast<std::size_t>(k % channels) * m.g.plane;
  }
  return count;
}

bool Solver::prepare(const Plan& plan, Failure& failure) {
  Impl& m = *impl_;
  m.plan = plan;
  m.setup(plan.tgv);
  m.set_factors(plan);
  m.start(nullptr, true);
  bytes_ = m.bytes;
  m.planned = true;
  if (!m.check(failure, "the start")) return false;
  m.primal(true);
  return m.check(failure, "the first primal step");
}

bool Solver::iterate(std::uint64_t iterations, Failure& failure) {
  Impl& m = *impl_;
  std::uint64_t n = 0;
  while (n < iterations && m.error == cudaSuccess) {
    const bool last = n + 1 == iterations;
    if (m.fusable && !last) {
      m.fused();
      ++n;
      continue;
    }
    // kGraphIterations iterations as one graph while at least one more (the last, which keeps)
    // follows.
    if (iterations - n > kGraphIterations && m.group()) {
      n += kGraphIterations;
      continue;
    }
    if (m.error != cudaSuccess) break;
    m.dual(false);
    m.primal(last);
    ++n;
  }
  return m.check(failure, "the iterations");
}

bool Solver::breakdown(std::uint64_t iterations, double& dual_ms, double& primal_ms, Failure& failure) {
  Impl& m = *impl_;
  std::vector<cudaEvent_t> events(3 * iterations);
  for (cudaEvent_t& e : events) cudaEventCreate(&e);
  // With the fused sweep, every iteration but the last is one launch, timed as the dual
  // group; the last (split, keeping its iterate) is not timed.
  const std::uint64_t timed = m.fusable && iterations > 1 ? iterations - 1 : iterations;
  for (std::uint64_t n = 0; n < iterations && m.error == cudaSuccess; ++n) {
    if (m.fusable && n < timed) {
      cudaEventRecord(events[3 * n], m.stream);
      m.fused();
      cudaEventRecord(events[3 * n + 1], m.stream);
      cudaEventRecord(events[3 * n + 2], m.stream);
      continue;
    }
    cudaEventRecord(events[3 * n], m.stream);
    m.dual(false);
    cudaEventRecord(events[3 * n + 1], m.stream);
    m.primal(n + 1 == iterations);
    cudaEventRecord(events[3 * n + 2], m.stream);
  }
  if (m.error == cudaSuccess) m.error = cudaStreamSynchronize(m.stream);
  double dual = 0.0, primal = 0.0;
  for (std::uint64_t n = 0; n < timed && m.error == cudaSuccess; ++n) {
    float a = 0.0f, b = 0.0f;
    cudaEventElapsedTime(&a, events[3 * n], events[3 * n + 1]);
    cudaEventElapsedTime(&b, events[3 * n + 1], events[3 * n + 2]);
    dual += a;
    primal += b;
  }
  for (cudaEvent_t& e : events) cudaEventDestroy(e);
  dual_ms = timed > 0 ? dual / static_cast<double>(timed) : 0.0;
  primal_ms = timed > 0 ? primal / static_cast<double>(timed) : 0.0;
  return m.check(failure, "the timed iterations");
}

void Solver::keep_result_on_device() { impl_->host_result = false; }

bool Solver::levels(bool sixteen, int dither, std::uint8_t* out, Failure& failure) {
  Impl& m = *impl_;
  bool not_finite = false;
  m.levels(sixteen, dither, out, not_finite);
  if (!m.check(failure, "the levels")) return false;
  if (not_finite) {
    failure = {kOptions, "a sample to quantize is not finite"};
    return false;
  }
  return true;
}

bool Solver::finish(Outcome& out, Failure& failure) {
  Impl& m = *impl_;
  m.result(out);
  return m.check(failure, "the result");
}

}  // namespace urb
