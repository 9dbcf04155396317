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

// Four consecutive samples of a row per thread (16-byte loads of x, p1, p2 and x~ stores, an
// 8-byte load of the levels; the pitch is a multiple of 32 samples), a warp per 128 columns of
// a row, CTAs of 128 columns x 8 rows. p1 at the column before comes from the lane before by
// a shuffle (lane 0 loads it); p2 at the row above by a 16-byte load, mostly from L1.
template <bool KEEP>
__global__ void __launch_bounds__(256) samples_primal_kernel(const SamplesPrimalParams P) {
  const int lane = threadIdx.x;
  const int j = blockIdx.x * 128 + 4 * lane, i = blockIdx.y * 8 + threadIdx.y, c = blockIdx.z;
  const int rows = P.g.rows, columns = P.g.columns, pitch = P.g.pitch;
  const float descent = descent_of(P, c);
  const bool row_in = i < rows;
  double term = 0.0;
  const std::size_t at = c * P.g.plane + static_cast<std::size_t>(row_in ? i : 0) * pitch + (j < pitch ? j : 0);
  float4 p1 = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
  if (row_in && j < columns) p1 = *reinterpret_cast<const float4*>(P.p1 + at);
  // The p1 of the column before this thread's first: the lane before's last, or a load.
  float before = __shfl_up_sync(kAll, p1.w, 1);
  if (lane == 0) before = row_in && j > 0 && j < columns ? P.p1[at - 1] : 0.0f;
  if (row_in && j < columns) {
    const float4 p2 = *reinterpret_cast<const float4*>(P.p2 + at);
    const float4 above = i > 0 ? *reinterpret_cast<const float4*>(P.p2 + at - pitch) : make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    const float4 x = *reinterpret_cast<const float4*>(P.x + at);
    const ushort4 level = *reinterpret_cast<const ushort4*>(P.levels + at);
    const bool last_row = i + 1 == rows;
    const float pv[4] = {p1.x, p1.y, p1.z, p1.w}, qv[4] = {p2.x, p2.y, p2.z, p2.w};
    const float av[4] = {above.x, above.y, above.z, above.w}, xv[4] = {x.x, x.y, x.z, x.w};
    const unsigned lv[4] = {level.x, level.y, level.z, level.w};
    float zv[4];
    float left = before;
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      // div p = dy' p2 + dx' p1, backward differences with Neumann ends.
      const int jj = j + u;
      const float dy = (last_row ? 0.0f : qv[u]) - (i > 0 ? av[u] : 0.0f);
      const float dx = (jj + 1 < columns ? pv[u] : 0.0f) - (jj > 0 ? left : 0.0f);
      left = pv[u];
      const float v = xv[u] + descent * (dy + dx);
      const float4 ends = __ldg(reinterpret_cast<const float4*>(P.ends) + (jj < columns ? lv[u] : 0u));
      zv[u] = fminf(fmaxf((v + P.t * ends.z) * P.r, ends.x), ends.y);
      if constexpr (KEEP) {
        if (jj < columns) {
          const double away = static_cast<double>(zv[u]) - P.ends64[lv[u]].centre;
          term += P.half_mu * (away * away);
        }
      }
    }
    if (j + 4 <= columns) {
      *reinterpret_cast<float4*>(P.xt + at) = make_float4(zv[0], zv[1], zv[2], zv[3]);
    } else {
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        if (j + u < columns) P.xt[at + u] = zv[u];
      }
    }
  }
  if constexpr (KEEP) block_sum(term, P.partials);
}

__global__ void __launch_bounds__(256) samples_conjugate_kernel(const SamplesConjugateParams P) {
  const int j = blockIdx.x * 32 + threadIdx.x, i = blockIdx.y * 8 + threadIdx.y;
  const int rows = P.g.rows, columns = P.g.columns, pitch = P.g.pitch;
  double term = 0.0;
  if (i < rows && j < columns) {
    const double scale = P.most_at != nullptr ? negative_theta(*P.most_at, P.alpha1) : P.scale;
    auto q_at = [&](const float* f, int ii, int jj) -> double {
      return scale * static_cast<double>(f[static_cast<std::size_t>(ii) * pitch + jj]);
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

dim3 primal_grid(const Geometry& g) {
  return dim3((g.columns + 127) / 128, (g.rows + 7) / 8, g.channels);
}

}  // namespace

int samples_grid_blocks(const Geometry& g, int channels) {
  const dim3 grid = sample_grid(g, channels);
  return static_cast<int>(grid.x * grid.y * grid.z);
}

int samples_primal_blocks(const Geometry& g) {
  const dim3 grid = primal_grid(g);
  return static_cast<int>(grid.x * grid.y * grid.z);
}

cudaError_t launch_samples_primal(const SamplesPrimalParams& p, bool keep, cudaStream_t stream) {
  const dim3 grid = primal_grid(p.g);
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
