// The batched solve: many pictures of different sizes, channels, qualities and methods (TV, TGV)
// solved together. Each picture keeps its own device state and its own start, last iteration,
// record and result (Solver); the iterations between run for all pictures at once, one launch
// per kernel class an iteration -- the dual sweep of each (method, channels) class over a table
// of tiles of all its pictures, the primal step of each cell layout over a table of items of
// all its components -- two iterations (one of each parity of the state) captured in one CUDA
// graph, launched once for every pair of iterations. The kernels make each pixel and block by
// the single-picture kernels' device functions, so each result is the one unround_solve gives
// the picture alone to binary32 rounding (the compiler may fuse a multiply-add differently in
// the two kernels).
#pragma once

#include <cstdint>
#include <vector>

#include <cuda_runtime.h>

#include "model.hpp"
#include "solver.hpp"

namespace urb {

struct BatchEntry {
  const Frame* frame = nullptr;
  Plan plan;
};

// The batched part's device time (CUDA events around it on the batch's stream), the
// iterations it made, the launches it made an iteration, and the samples and pixels of all
// pictures.
struct BatchTiming {
  double milliseconds = 0.0;
  std::uint64_t iterations = 0;
  std::uint64_t launches_per_iteration = 0;
  std::uint64_t samples = 0;
  std::uint64_t pixels = 0;
  double tuning_milliseconds = 0.0;  // the autotuner's measurements, before the timed part
};

// All entries' plans have the same number of iterations and record at the last only
// (record_every 0); every component takes the TMA-fed primal step (cells of 1, 2 or 4 each way).
// check_batch refuses, without a device, a batch whose plans break the first two.
bool check_batch(const std::vector<BatchEntry>& entries, Failure& failure);
bool solve_batch(const std::vector<BatchEntry>& entries, cudaStream_t stream, std::vector<Outcome>& outcomes,
                 BatchTiming& timing, Failure& failure);

}  // namespace urb
