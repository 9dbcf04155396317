// The driver of the device solve: the reference's method loop (cpp/src/primal_dual.hpp:957-1013,
// rust/unround/src/pdhg.rs:641-686) over the kernels of kernels.hpp. Each iteration is two
// launches on the call's own stream: the dual step of iteration n with the relaxation, then
// the primal step and proximal map of iteration n+1 (the canvas x~ is the one field carried
// between them). Records take the tilde point in binary64 sums; the result is computed in
// binary64 from the last coefficients.
#pragma once

#include <cstdint>
#include <functional>
#include <memory>
#include <vector>

#include <cuda_runtime.h>

#include "kernels.hpp"
#include "host_buffer.hpp"
#include "model.hpp"

namespace urb {

// A record (cpp/include/unround/results.hpp:17-24): the iteration, the solver's seconds,
// the primal and dual values, TGV's scaling and partial gap (NaN where not taken).
struct Record {
  std::uint64_t iteration = 0;
  double seconds = 0.0;
  double primal = 0.0;
  double dual = 0.0;
  double scaling = 0.0;
  double partial_gap = 0.0;
};

// A start (cpp/include/unround/pdhg.hpp:124-133): every component's coefficients, clipped to
// their intervals, and each channel's duals, projected onto their balls, and TGV's w
// (channel-major, canvas rows x columns each); an empty part takes the default.
struct Start {
  std::vector<std::vector<double>> coefficients;
  std::vector<double> p;  // C x 2 x rows x columns
  std::vector<double> w;  // C x 2 x rows x columns
  std::vector<double> r;  // C x 3 x rows x columns
};

// What a solve made (rust/unround/src/decode.rs:70-110): the canvas C x rows x columns and
// each component's coefficients in binary64, the records, the iterations, and why it stopped
// (0 no solver, 1 converged, 2 iterations, 3 observer).
// The result on the host. `planes` is the canvas cut to the picture (empty where they are the
// same); `picture` its pixels with the channels interleaved, for YCbCr in JFIF RGB (empty where
// it is the planes: one channel).
struct Outcome {
  HostBuffer canvas;
  std::vector<HostBuffer> coefficients;
  HostBuffer planes;
  HostBuffer picture;
  std::vector<Record> records;
  std::uint64_t iterations = 0;
  std::int32_t stop = 0;
  bool solved = false;
  double tau = 0.0;
  double sigma = 0.0;
};

// Called with each record after the first, the gap per sample and the record's canvas
// (C x rows x columns binary64, valid for the call); true stops the solver.
using Observer = std::function<bool(const Record&, double gap, const double* canvas)>;

struct SamplesModel;

class Solver {
 public:
  Solver(const Frame& frame, cudaStream_t stream);
  // A picture of rounded samples (samples_model.hpp): `frame` gives only its size and colour
  // space (no components); the model outlives the solver.
  Solver(const Frame& frame, const SamplesModel& samples, cudaStream_t stream);
  ~Solver();
  Solver(const Solver&) = delete;
  Solver& operator=(const Solver&) = delete;

  // The MMSE decoder (no plan) or TV/TGV by the primal-dual method, into `out`.
  bool solve(Method method, const Plan* plan, const Start* start, const Observer& observer, Outcome& out,
             Failure& failure);

  // For measurement: `iterations` iterations of the method from the current state, no
  // records, launched on the stream and not waited for (the caller times them).
  bool prepare(const Plan& plan, Failure& failure);
  bool iterate(std::uint64_t iterations, Failure& failure);
  // The same with CUDA events around each kernel group: the average device milliseconds of
  // an iteration's dual step and of its primal steps.
  bool breakdown(std::uint64_t iterations, double& dual_ms, double& primal_ms, Failure& failure);
  // The binary64 canvas of the last tilde point, after prepare/iterate.
  bool finish(Outcome& out, Failure& failure);

  // For a batched loop (batch.cpp runs the iterations of many solvers in one graph): the start
  // and no iteration; the entries of this solver's state that the batched kernels read (false
  // where a kernel of this state has no batched form); and, after `done` iterations made by the
  // batch (the state of iteration `done` current), the rest as solve() makes it: the remaining
  // iterations, the records and the result. The batch's plans record at the last iteration only.
  bool begin_batch(const Plan& plan, Failure& failure);
  bool batch_entries(DualBatchImage& image, std::vector<PrimalBatchComponent>& components);
  bool finish_batch(std::uint64_t done, Outcome& out, Failure& failure);

  // For a strip of a picture solved in row strips (strips.py; begin_batch first, finish_batch
  // last): `iterations` iterations keeping nothing -- the primal step P_k, then the dual step
  // D_k -- waited for; and the device planes of the current state s_k, field by field (x, p1,
  // p2, and for TGV w1, w2, r11, r22, r12), each channel after channel, rows `pitch` floats apart.
  // Returns how many planes there are (up to `most` written).
  bool step(std::uint64_t iterations, Failure& failure);
  // The same iterations launched on the stream and not waited for (the next record or result
  // checks the device).
  bool advance(std::uint64_t iterations, Failure& failure);
  cudaStream_t stream() const;
  int state_planes(float** planes, int most) const;
  // A strip's records, which the ranks add up (strips.py): the canvas rows [first, end) whose
  // terms its records count (its own bands); one iteration keeping its tilde point (none with
  // `advance` false: the start's) and the record's first sums over those rows -- G at the kept
  // coefficients, the first-order norms, the second-order norms and the largest |div2 r~| (TGV),
  // the samples counted -- waited for; the second sums at the scaling theta -- the dual's G*
  // over the channels, and with a partial radius the partial gap's G* and residual; and after
  // the last iteration (made by record_step), the result with no more iterations.
  void set_record_rows(int first, int end);
  bool record_step(bool advance, double (&first)[5], Failure& failure);
  bool record_duals(double theta, double (&second)[3], Failure& failure);
  bool finish_here(std::uint64_t done, std::int32_t stop, Outcome& out, Failure& failure);

  // Before solve(): keep the result on the device (the Outcome gets the records and counts,
  // not the arrays); after it, the picture's 8- or 16-bit levels into host memory `out`
  // (height x width x channels, interleaved; dither 0 rounds, 1 and 2 take the blue-noise
  // matrix with the channels apart or together).
  void keep_result_on_device();
  bool levels(bool sixteen, int dither, std::uint8_t* out, Failure& failure);

  [[nodiscard]] std::size_t device_bytes() const { return bytes_; }
  [[nodiscard]] const Geometry& geometry() const { return geometry_; }
  [[nodiscard]] int launches_per_iteration() const;

 private:
  bool run(std::uint64_t first, const Observer& observer, Outcome& out, Failure& failure);
  struct Impl;
  std::unique_ptr<Impl> impl_;
  Geometry geometry_;
  std::size_t bytes_ = 0;
};

}  // namespace urb
