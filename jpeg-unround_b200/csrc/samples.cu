// Pictures of rounded samples (docs/math.md 11; rust/unround/src/samples.rs,
// cpp/src/samples.cpp): the unknown is the picture itself, each sample k held in its closed
// interval [a_k, b_k] of the values that round to its level, with a data term mu/2 (x - c)^2
// toward the level's centre. The dual step is the JPEG path's sweep (TV or TGV of the
// channels); these kernels are the rest:
//
//   samples_primal_kernel     v = x + tau gamma div p and its proximal map, sample by sample:
//                             x~ = clip((v + t c) r, a, b), t = tau mu, r = 1 / (1 + t)
//                             (cpp/src/samples.cpp:158-176); with KEEP, the CTA's sum of
//                             mu/2 (x~ - c)^2 in binary64 (samples.cpp:184-197)
//   samples_conjugate_kernel  G* at xi = gamma div q, q = scale (q1, q2): the CTA's sum of
//                             g*(xi) = xi b* - mu/2 (b* - c)^2, b* = clip(c + xi / mu, a, b), or
//                             max(xi a, xi b) at mu = 0 (samples.cpp:205-227), in binary64
//   samples_canvas_kernel     the start (x = c in binary32 and the binary64 canvas of the
//                             centres), or the result: x~ in binary64, clipped to its interval
//   samples_levels_kernel     the levels of the picture's channels, interleaved as given, into
//                             planes pitched like the state
//
// A thread per sample, CTAs of 32 x 8 samples of one channel; binary32 iterations, binary64
// records and result, as the JPEG path. A sample's ends and centre come from a table indexed
// by its level (2^bits entries: 4 KB at 8 bits, read through L1), so the primal step moves
// 18 bytes a sample: x, p1, p2 and the level read, x~ written.
#include "kernels.hpp"

namespace urb {

namespace {

constexpr unsigned kAll = 0xffffffffu;

// The sum of one double per thread of a CTA of 256, warp by warp and then the warps in order,
// into out[the CTA's index].
__device__ __forceinline__ void block_sum(double value, double* out) {
  __shared__ double partial[8];
  const int lane = threadIdx.x, warp = threadIdx.y;
#pragma unroll
  for (int offset = 16; offset > 0; offset >>= 1) value += __shfl_down_sync(kAll, value, offset);
  if (lane == 0) partial[warp] = value;
  __syncthreads();
  if (warp == 0) {
    double total = lane < 8 ? partial[lane] : 0.0;
#pragma unroll
    for (int offset = 4; offset > 0; offset >>= 1) total += __shfl_down_sync(kAll, total, offset);
    if (lane == 0) out[blockIdx.x + gridDim.x * (blockIdx.y + gridDim.y * blockIdx.z)] = total;
  }
}

// descent[c] by a chain of selects: indexing the parameter array with a register would copy
// the whole parameter block to local memory, thread by thread.
__device__ __forceinline__ float descent_of(const SamplesPrimalParams& P, int c) {
  float d = P.descent[0];
#pragma unroll
  for (int k = 1; k < kMaxChannels; ++k) d = c == k ? P.descent[k] : d;
  return d;
}

template <bool KEEP>
__global__ void __launch_bounds__(256) samples_primal_kernel(const SamplesPrimalParams P) {
  const int j = blockIdx.x * 32 + threadIdx.x, i = blockIdx.y * 8 + threadIdx.y, c = blockIdx.z;
  const int rows = P.g.rows, columns = P.g.columns, pitch = P.g.pitch;
  const float descent = descent_of(P, c);
  double term = 0.0;
  if (i < rows && j < columns) {
    const std::size_t at = c * P.g.plane + static_cast<std::size_t>(i) * pitch + j;
    const float p1 = P.p1[at], p2 = P.p2[at];
    const float above = i > 0 ? P.p2[at - pitch] : 0.0f;
    const float before = j > 0 ? P.p1[at - 1] : 0.0f;
    // div p = dy' p2 + dx' p1, backward differences with Neumann ends.
    const float dy = (i + 1 < rows ? p2 : 0.0f) - (i > 0 ? above : 0.0f);
    const float dx = (j + 1 < columns ? p1 : 0.0f) - (j > 0 ? before : 0.0f);
    const float v = P.x[at] + descent * (dy + dx);
    const unsigned level = P.levels[at];
    const float4 ends = __ldg(reinterpret_cast<const float4*>(P.ends) + level);  // lower, upper, centre
    const float z = fminf(fmaxf((v + P.t * ends.z) * P.r, ends.x), ends.y);
    P.xt[at] = z;
    if constexpr (KEEP) {
      const double away = static_cast<double>(z) - P.ends64[level].centre;
      term = P.half_mu * (away * away);
    }
  }
  if constexpr (KEEP) block_sum(term, P.partials);
}

__global__ void __launch_bounds__(256) samples_conjugate_kernel(const SamplesConjugateParams P) {
  const int j = blockIdx.x * 32 + threadIdx.x, i = blockIdx.y * 8 + threadIdx.y;
  const int rows = P.g.rows, columns = P.g.columns, pitch = P.g.pitch;
  double term = 0.0;
  if (i < rows && j < columns) {
    auto q_at = [&](const float* f, int ii, int jj) -> double {
      return P.scale * static_cast<double>(f[static_cast<std::size_t>(ii) * pitch + jj]);
    };
    const double dy = (i + 1 < rows ? q_at(P.q2, i, j) : 0.0) - (i > 0 ? q_at(P.q2, i - 1, j) : 0.0);
    const double dx = (j + 1 < columns ? q_at(P.q1, i, j) : 0.0) - (j > 0 ? q_at(P.q1, i, j - 1) : 0.0);
    const double s = P.gamma * (dy + dx);
    const SampleEnds64& ends = P.ends64[P.levels[static_cast<std::size_t>(i) * pitch + j]];
    const double low = ends.lower, high = ends.upper, centre = ends.centre, m = P.mu;
    if (m > 0.0) {
      const double best = fmin(fmax(centre + s / m, low), high);
      const double away = best - centre;
      term = s * best - 0.5 * m * (away * away);
    } else {
      term = fmax(s * low, s * high);
    }
  }
  block_sum(term, P.partials);
}

__global__ void __launch_bounds__(256) samples_canvas_kernel(const SamplesCanvasParams P) {
  const int j = blockIdx.x * 32 + threadIdx.x, i = blockIdx.y * 8 + threadIdx.y, c = blockIdx.z;
  if (i >= P.g.rows || j >= P.g.columns) return;
  const std::size_t at = c * P.g.plane + static_cast<std::size_t>(i) * P.g.pitch + j;
  const std::size_t k = (static_cast<std::size_t>(c) * P.g.rows + i) * P.g.columns + j;
  const SampleEnds64& ends = P.ends64[P.levels[at]];
  if (P.mode == 0) {
    P.x[at] = static_cast<float>(ends.centre);
    P.canvas[k] = ends.centre;
  } else {
    P.canvas[k] = fmin(fmax(static_cast<double>(P.xt[at]), ends.lower), ends.upper);
  }
}

__global__ void __launch_bounds__(256) samples_levels_kernel(const SamplesLevelsParams P) {
  const int j = blockIdx.x * 32 + threadIdx.x, i = blockIdx.y * 8 + threadIdx.y, c = blockIdx.z;
  if (i >= P.g.rows || j >= P.g.columns) return;
  const std::size_t from = (static_cast<std::size_t>(i) * P.g.columns + j) * P.stride + P.first + c;
  P.levels[c * P.g.plane + static_cast<std::size_t>(i) * P.g.pitch + j] = P.source[from];
}

dim3 sample_grid(const Geometry& g, int channels) {
  return dim3((g.columns + 31) / 32, (g.rows + 7) / 8, channels);
}

}  // namespace

int samples_grid_blocks(const Geometry& g, int channels) {
  const dim3 grid = sample_grid(g, channels);
  return static_cast<int>(grid.x * grid.y * grid.z);
}

cudaError_t launch_samples_primal(const SamplesPrimalParams& p, bool keep, cudaStream_t stream) {
  const dim3 grid = sample_grid(p.g, p.g.channels);
  if (keep) {
    samples_primal_kernel<true><<<grid, dim3(32, 8), 0, stream>>>(p);
  } else {
    samples_primal_kernel<false><<<grid, dim3(32, 8), 0, stream>>>(p);
  }
  return cudaGetLastError();
}

cudaError_t launch_samples_conjugate(const SamplesConjugateParams& p, cudaStream_t stream) {
  samples_conjugate_kernel<<<sample_grid(p.g, 1), dim3(32, 8), 0, stream>>>(p);
  return cudaGetLastError();
}

cudaError_t launch_samples_canvas(const SamplesCanvasParams& p, cudaStream_t stream) {
  samples_canvas_kernel<<<sample_grid(p.g, p.g.channels), dim3(32, 8), 0, stream>>>(p);
  return cudaGetLastError();
}

cudaError_t launch_samples_levels(const SamplesLevelsParams& p, cudaStream_t stream) {
  samples_levels_kernel<<<sample_grid(p.g, p.g.channels), dim3(32, 8), 0, stream>>>(p);
  return cudaGetLastError();
}

}  // namespace urb
