// The kernels of the solver, sm_100a, binary32 iterations with binary64 records, start and
// result. See kernels.hpp for the layout. The formulas and their order of operations follow
// the reference's iteration (cpp/src/primal_dual.hpp:525-735; rust/unround/src/kernels.rs),
// a pixel or a block at a time instead of a row at a time:
//
//   dual_kernel    x- = 2x~ - x, w~ = w + tau g (p + div2 r), w- = 2w~ - w,
//                  p~ = proj_a1(p + sigma g (grad x- - w-)), r~ = proj_a0(r + sigma g E w-),
//                  and every field relaxed, x <- rho x~ + (1 - rho) x   (docs/math.md 5)
//   primal_kernel  v = x + tau g div p, then per block of the component: the means of the
//                  cells, the DCT, the clip of the proximal map, the inverse DCT, and the
//                  change spread back over the cells (docs/math.md 4.1, 4.4)
//
// The finite differences are those of docs/math.md 3.1-3.2 with Neumann ends: forward
// differences are 0 in the last column/row, backward differences drop the sample of the last
// column/row and the neighbour before the first.
#include "kernels.hpp"

#include <algorithm>
#include <atomic>
#include <cfloat>
#include <cstdint>

#include "colour.hpp"
#include "dct.cuh"
#include "prox.cuh"
#include "tma.cuh"

namespace urb {

namespace {

constexpr int kWarps = 8;

__device__ __forceinline__ float ld(const float* base, std::size_t at) { return __ldg(base + at); }

// radius / |p| beyond the ball, 1 within it (cpp/include/unround/operators.hpp:112-116).
template <typename T>
__device__ __forceinline__ T ball_scale(T square, T radius) {
  const T norm = sqrt(square);
  return norm > radius ? radius / norm : T(1);
}

// The sum (or the largest) over the CTA of one double per thread, in a fixed order: warp
// by warp with shuffles, then the warps' in order. Thread 0 holds the result.
template <bool MAX>
__device__ double cta_reduce(double value) {
  __shared__ double partial[32];
  const int tid = threadIdx.x + blockDim.x * (threadIdx.y + blockDim.y * threadIdx.z);
  const int warps = (blockDim.x * blockDim.y * blockDim.z + 31) / 32;
  for (int offset = 16; offset > 0; offset >>= 1) {
    const double other = __shfl_down_sync(0xffffffffu, value, offset);
    value = MAX ? fmax(value, other) : value + other;
  }
  if ((tid & 31) == 0) partial[tid >> 5] = value;
  __syncthreads();
  double total = 0.0;
  if (tid < 32) {
    total = tid < warps ? partial[tid] : 0.0;
    for (int offset = 16; offset > 0; offset >>= 1) {
      const double other = __shfl_down_sync(0xffffffffu, total, offset);
      total = MAX ? fmax(total, other) : total + other;
    }
  }
  __syncthreads();
  return total;
}

__device__ __forceinline__ int cta_index() { return blockIdx.x + gridDim.x * (blockIdx.y + gridDim.y * blockIdx.z); }

__device__ __forceinline__ bool cta_leader() { return threadIdx.x == 0 && threadIdx.y == 0 && threadIdx.z == 0; }

// One double per CTA into out[cta].
__device__ __forceinline__ void cta_sum(double value, double* out) {
  const double total = cta_reduce<false>(value);
  if (cta_leader()) out[cta_index()] = total;
}

// ---------------------------------------------------------------------------------------
// The dual step as a sweep: a warp owns 32 columns and walks down a segment of kSegment rows,
// so that every field of every channel is read once. Row i needs x- of row i + 1 (read one row
// ahead) and w- of row i - 1 (kept from the row before); the neighbours across come from the
// lanes beside (shuffles), and the warp's two edge lanes read the one column beyond it (lane 0
// computes w- of column j - 1, lane 31 reads x- and r of column j + 1). Each value is computed
// from the same operands by the same operations as in dual_kernel.
constexpr int kSegment = 64;

template <bool TGV, int C, bool COUPLED, bool KEEP>
__global__ void __launch_bounds__(256) dual_stream_kernel(const DualParams P) {
  constexpr unsigned kAll = 0xffffffffu;
  const int lane = threadIdx.x;
  const int j = blockIdx.x * 32 + lane;
  const int rows = P.g.rows, columns = P.g.columns, pitch = P.g.pitch;
  const int i0 = (blockIdx.y * blockDim.y + threadIdx.y) * kSegment;
  if (i0 >= rows) return;  // the whole warp
  const int i1 = min(i0 + kSegment, rows);
  const bool valid = j < columns;
  const int jc = valid ? j : columns - 1;
  const bool has_left = j > 0, has_right = j + 1 < columns;
  const bool edge_left = lane == 0 && has_left;
  const bool edge_right = lane == 31 && has_right;
  const float rho = P.rho, rest = P.rest;
  const std::size_t plane = P.g.plane;
  auto at = [pitch](int i, int jj) { return static_cast<std::size_t>(i) * pitch + jj; };

  float xt_c[C], x_c[C], xb_c[C], r11_c[C], r12_c[C], r22_c[C], wb1_p[C], wb2_p[C];
#pragma unroll
  for (int c = 0; c < C; ++c) {
    const std::size_t base = c * plane;
    xt_c[c] = ld(P.xt + base, at(i0, jc));
    x_c[c] = ld(P.in.x + base, at(i0, jc));
    xb_c[c] = 2.0f * xt_c[c] - x_c[c];
    r11_c[c] = r12_c[c] = r22_c[c] = wb1_p[c] = wb2_p[c] = 0.0f;
    if constexpr (TGV) {
      r11_c[c] = ld(P.in.r11 + base, at(i0, jc));
      r12_c[c] = ld(P.in.r12 + base, at(i0, jc));
      r22_c[c] = ld(P.in.r22 + base, at(i0, jc));
      if (i0 > 0) {
        // w- of the row above the segment, own column.
        const int u = i0 - 1;
        const float a11 = ld(P.in.r11 + base, at(u, jc)), a12 = ld(P.in.r12 + base, at(u, jc));
        const float a22 = ld(P.in.r22 + base, at(u, jc));
        float right11 = __shfl_down_sync(kAll, a11, 1), right12 = __shfl_down_sync(kAll, a12, 1);
        if (edge_right) {
          right11 = ld(P.in.r11 + base, at(u, j + 1));
          right12 = ld(P.in.r12 + base, at(u, j + 1));
        }
        float d1 = has_right ? right11 - a11 : 0.0f;
        float d2 = has_right ? right12 - a12 : 0.0f;
        d1 = d1 + (r12_c[c] - a12);
        d2 = d2 + (r22_c[c] - a22);
        const float w1 = ld(P.in.w1 + base, at(u, jc)), w2 = ld(P.in.w2 + base, at(u, jc));
        const float tau = P.tau[c];
        const float t1 = w1 + tau * (ld(P.in.p1 + base, at(u, jc)) + d1);
        const float t2 = w2 + tau * (ld(P.in.p2 + base, at(u, jc)) + d2);
        wb1_p[c] = 2.0f * t1 - w1;
        wb2_p[c] = 2.0f * t2 - w2;
      }
    }
  }

  for (int i = i0; i < i1; ++i) {
    const bool has_down = i + 1 < rows, has_up = i > 0;
    const std::size_t here = at(i, jc);
    float step_p1[C], step_p2[C], old_p1[C], old_p2[C];
    float step_r11[C], step_r22[C], step_r12[C], old_r11[C], old_r22[C], old_r12[C];
    float square_p = 0.0f, square_r = 0.0f;
#pragma unroll
    for (int c = 0; c < C; ++c) {
      const std::size_t base = c * plane;
      // Row i + 1, read ahead.
      float xt_n = 0.0f, x_n = 0.0f, r11_n = 0.0f, r12_n = 0.0f, r22_n = 0.0f;
      if (has_down) {
        xt_n = ld(P.xt + base, here + pitch);
        x_n = ld(P.in.x + base, here + pitch);
        if constexpr (TGV) {
          r11_n = ld(P.in.r11 + base, here + pitch);
          r12_n = ld(P.in.r12 + base, here + pitch);
          r22_n = ld(P.in.r22 + base, here + pitch);
        }
      }
      const float xb_n = 2.0f * xt_n - x_n;
      float xb_right = __shfl_down_sync(kAll, xb_c[c], 1);
      if (edge_right) xb_right = 2.0f * ld(P.xt + base, at(i, j + 1)) - ld(P.in.x + base, at(i, j + 1));
      const float gx = has_right ? xb_right - xb_c[c] : 0.0f;
      const float gy = has_down ? xb_n - xb_c[c] : 0.0f;
      if (valid) P.out.x[base + here] = rho * xt_c[c] + rest * x_c[c];
      const float p1 = ld(P.in.p1 + base, here), p2 = ld(P.in.p2 + base, here);
      old_p1[c] = p1;
      old_p2[c] = p2;
      const float sigma = P.sigma[c];
      if constexpr (!TGV) {
        step_p1[c] = p1 + sigma * gx;
        step_p2[c] = p2 + sigma * gy;
      } else {
        const float tau = P.tau[c];
        float right11 = __shfl_down_sync(kAll, r11_c[c], 1), right12 = __shfl_down_sync(kAll, r12_c[c], 1);
        if (edge_right) {
          right11 = ld(P.in.r11 + base, at(i, j + 1));
          right12 = ld(P.in.r12 + base, at(i, j + 1));
        }
        float d1 = has_right ? right11 - r11_c[c] : 0.0f;
        float d2 = has_right ? right12 - r12_c[c] : 0.0f;
        d1 = d1 + (has_down ? r12_n - r12_c[c] : 0.0f);
        d2 = d2 + (has_down ? r22_n - r22_c[c] : 0.0f);
        const float w1 = ld(P.in.w1 + base, here), w2 = ld(P.in.w2 + base, here);
        const float t1 = w1 + tau * (p1 + d1), t2 = w2 + tau * (p2 + d2);
        const float wb1 = 2.0f * t1 - w1, wb2 = 2.0f * t2 - w2;
        if (valid) {
          P.out.w1[base + here] = rho * t1 + rest * w1;
          P.out.w2[base + here] = rho * t2 + rest * w2;
          if constexpr (KEEP) {
            P.tilde.w1[base + here] = t1;
            P.tilde.w2[base + here] = t2;
          }
        }
        // w- of column j - 1.
        float wl1 = __shfl_up_sync(kAll, wb1, 1), wl2 = __shfl_up_sync(kAll, wb2, 1);
        if (edge_left) {
          const std::size_t left = at(i, j - 1);
          const float l11 = ld(P.in.r11 + base, left), l12 = ld(P.in.r12 + base, left);
          const float l22 = ld(P.in.r22 + base, left);
          float e1 = r11_c[c] - l11, e2 = r12_c[c] - l12;
          e1 = e1 + (has_down ? ld(P.in.r12 + base, left + pitch) - l12 : 0.0f);
          e2 = e2 + (has_down ? ld(P.in.r22 + base, left + pitch) - l22 : 0.0f);
          const float lw1 = ld(P.in.w1 + base, left), lw2 = ld(P.in.w2 + base, left);
          const float lt1 = lw1 + tau * (ld(P.in.p1 + base, left) + e1);
          const float lt2 = lw2 + tau * (ld(P.in.p2 + base, left) + e2);
          wl1 = 2.0f * lt1 - lw1;
          wl2 = 2.0f * lt2 - lw2;
        }
        if (!has_left) wl1 = wl2 = 0.0f;
        const float wu1 = has_up ? wb1_p[c] : 0.0f, wu2 = has_up ? wb2_p[c] : 0.0f;
        step_p1[c] = p1 + sigma * (gx - wb1);
        step_p2[c] = p2 + sigma * (gy - wb2);
        const float own1x = has_right ? wb1 : 0.0f, own2x = has_right ? wb2 : 0.0f;
        const float own1y = has_down ? wb1 : 0.0f, own2y = has_down ? wb2 : 0.0f;
        const float exx = own1x - wl1;
        const float eyy = own2y - wu2;
        const float exy = 0.5f * ((own1y - wu1) + (own2x - wl2));
        old_r11[c] = r11_c[c];
        old_r22[c] = r22_c[c];
        old_r12[c] = r12_c[c];
        step_r11[c] = r11_c[c] + sigma * exx;
        step_r22[c] = r22_c[c] + sigma * eyy;
        step_r12[c] = r12_c[c] + sigma * exy;
        wb1_p[c] = wb1;
        wb2_p[c] = wb2;
      }
      if constexpr (COUPLED) {
        square_p += step_p1[c] * step_p1[c] + step_p2[c] * step_p2[c];
        if constexpr (TGV) {
          square_r += step_r11[c] * step_r11[c] + step_r22[c] * step_r22[c] + 2.0f * (step_r12[c] * step_r12[c]);
        }
      }
      xt_c[c] = xt_n;
      x_c[c] = x_n;
      xb_c[c] = xb_n;
      if constexpr (TGV) {
        r11_c[c] = r11_n;
        r12_c[c] = r12_n;
        r22_c[c] = r22_n;
      }
    }
    float scale_p = 1.0f, scale_r = 1.0f;
    if constexpr (COUPLED) {
      scale_p = ball_scale(square_p, P.radius);
      if constexpr (TGV) scale_r = ball_scale(square_r, P.radius0);
    }
    if (!valid) continue;
#pragma unroll
    for (int c = 0; c < C; ++c) {
      const std::size_t base = c * plane;
      float sp = scale_p;
      if constexpr (!COUPLED) sp = ball_scale(step_p1[c] * step_p1[c] + step_p2[c] * step_p2[c], P.radius);
      const float q1 = step_p1[c] * sp, q2 = step_p2[c] * sp;
      P.out.p1[base + here] = rho * q1 + rest * old_p1[c];
      P.out.p2[base + here] = rho * q2 + rest * old_p2[c];
      if (KEEP && P.tilde.p1 != nullptr) {  // p~: TV's records and the partial gap's
        P.tilde.p1[base + here] = q1;
        P.tilde.p2[base + here] = q2;
      }
      if constexpr (TGV) {
        float sr = scale_r;
        if constexpr (!COUPLED) {
          sr = ball_scale(
              step_r11[c] * step_r11[c] + step_r22[c] * step_r22[c] + 2.0f * (step_r12[c] * step_r12[c]), P.radius0);
        }
        const float t11 = step_r11[c] * sr, t22 = step_r22[c] * sr, t12 = step_r12[c] * sr;
        P.out.r11[base + here] = rho * t11 + rest * old_r11[c];
        P.out.r22[base + here] = rho * t22 + rest * old_r22[c];
        P.out.r12[base + here] = rho * t12 + rest * old_r12[c];
        if constexpr (KEEP) {
          P.tilde.r11[base + here] = t11;
          P.tilde.r22[base + here] = t22;
          P.tilde.r12[base + here] = t12;
        }
      }
    }
  }
}

// ---------------------------------------------------------------------------------------
// The primal step and the proximal map. A CTA is 8 warps; a warp takes 4 of the component's
// blocks side by side, a lane one column of the block's 8 x 8 (cell) means: the lane computes
// v for the CR x CC samples of each of its cells, the column DCT in registers, and a
// transpose through shared memory gives each lane one row of coefficients (v = lane, u = 0..7)
// for the row DCT, the clip, and the inverse row DCT; a second transpose returns the columns.
// The interval, the centre and the proximal map of a coefficient are prox.cuh's.

// G's terms at a coefficient in binary64 (cpp/src/model.cpp:384-392): m/2 (c - centre)^2, and
// the cost of lying beyond the file's own interval.
__device__ __forceinline__ double value_term(double zeta, int q, int k, bool flat, const Constants64& K) {
  const double level = static_cast<double>(q);
  const double step = K.step[k];
  const double shift = k == 0 ? 1024.0 : 0.0;
  double centre;
  if (K.mmse && k != 0) {
    const double size = (fabs(level) - K.shrink[k]) * step;
    centre = q == 0 ? 0.0 : (q < 0 ? -size : size);
  } else {
    centre = level * step + shift;
  }
  const double m = flat ? K.flat_weight[k] : K.weight[k];
  const double away = zeta - centre;
  double term = 0.5 * m * (away * away);
  if (K.costed) {
    const double own_low = (level - 0.5) * step + shift;
    const double own_high = (level + 0.5) * step + shift;
    term = term + K.cost[k] * fmax(fmax(zeta - own_high, own_low - zeta), 0.0);
  }
  return term;
}

// A lane per canvas column: a component block covers 8 CC columns, so a warp takes 32 / (8 CC)
// blocks side by side (one for CC = 3, its last 8 lanes idle), and walks down kPrimalRows block
// rows. The CC lanes of a cell's columns sum their columns and exchange the sums (in the
// reference's order: down each column, then across), so every lane of the cell holds the
// cell means of its mean column; the transposes go through shared memory.
constexpr int kPrimalRows = 4;

template <int CR, int CC, bool KEEP>
__global__ void __launch_bounds__(256, 2) primal_kernel(const PrimalParams P) {
  constexpr unsigned kAll = 0xffffffffu;
  constexpr int L = 8 * CC;                  // lanes of a block
  constexpr int B = L <= 32 ? 32 / L : 1;    // blocks of a warp
  constexpr int BH = 8 * CR;                 // canvas rows of a block
  __shared__ ProxFactors F;
  __shared__ float tile[kWarps][4][72];
  {
    const int tid = threadIdx.x + 32 * threadIdx.y;
    const float* from = reinterpret_cast<const float*>(P.component.factors);
    float* to = reinterpret_cast<float*>(&F);
    for (int k = tid; k < static_cast<int>(sizeof(ProxFactors) / 4); k += 256) to[k] = from[k];
  }
  __syncthreads();
  const int lane = threadIdx.x;
  const int blk = lane / L, in_block = lane % L, m = in_block / CC, cell = in_block % CC;
  const bool used = blk < B;
  const int leader = lane - cell;
  const int rows = P.g.rows, columns = P.g.columns, pitch = P.g.pitch;
  const int vbx = blockIdx.x * B + blk;
  const int j = vbx * L + in_block;
  const bool column_in = used && j < columns;
  const int jc = column_in ? j : 0;
  const int first = (blockIdx.y * kWarps + threadIdx.y) * kPrimalRows;
  const int vbr = rows / BH;
  const float descent = P.descent;
  float* t = tile[threadIdx.y][used ? blk : 0];
  float p2_above = (column_in && first > 0 && first < vbr) ? ld(P.p2, static_cast<std::size_t>(first * BH - 1) * pitch + jc) : 0.0f;
  double sum = 0.0;
  for (int vby = first; vby < min(first + kPrimalRows, vbr); ++vby) {
    const int i0 = vby * BH;
    const bool in_blocks = column_in && vby < P.component.block_rows && vbx < P.component.block_columns;
    // v = x + tau g div p down the lane's column.
    float v[BH];
#pragma unroll
    for (int r = 0; r < BH; ++r) {
      const int i = i0 + r;
      const std::size_t at = static_cast<std::size_t>(i) * pitch + jc;
      const float p1 = column_in ? ld(P.p1, at) : 0.0f;
      const float p2 = column_in ? ld(P.p2, at) : 0.0f;
      const float x = column_in ? ld(P.x, at) : 0.0f;
      float before = __shfl_up_sync(kAll, p1, 1);
      if (lane == 0) before = (column_in && j > 0) ? ld(P.p1, at - 1) : 0.0f;
      // div p = dy' p2 + dx' p1, backward differences.
      const float dy = (i + 1 < rows ? p2 : 0.0f) - (i > 0 ? p2_above : 0.0f);
      const float dx = (j + 1 < columns ? p1 : 0.0f) - (j > 0 ? before : 0.0f);
      v[r] = x + descent * (dy + dx);
      p2_above = p2;
    }
    const std::size_t block =
        static_cast<std::size_t>(in_blocks ? vby : 0) * P.component.block_columns + (in_blocks ? vbx : 0);
    // The middle of the block's DC interval over 8 (exact): the block is taken centred on it.
    const float dc_level = in_blocks ? static_cast<float>(P.component.levels[block * 64]) : 0.0f;
    const float middle = (dc_level * F.plain[0].x + 1024.0f) * 0.125f;
    float mean[8];
#pragma unroll
    for (int r = 0; r < 8; ++r) {
      if constexpr (CR == 1 && CC == 1) {
        mean[r] = v[r] - middle;
      } else {
        float column = v[CR * r];
#pragma unroll
        for (int a = 1; a < CR; ++a) column += v[CR * r + a];
        float total = 0.0f;
#pragma unroll
        for (int c = 0; c < CC; ++c) {
          const float part = __shfl_sync(kAll, column, leader + c);
          total = c == 0 ? part : total + part;
        }
        mean[r] = total / static_cast<float>(CR * CC) - middle;
      }
    }
    float col[8], row[8], coef[8], zeta[8];
    forward8(mean, col);
    __syncwarp();
    if (cell == 0 && used) {
#pragma unroll
      for (int k = 0; k < 8; ++k) t[k * 9 + m] = col[k];
    }
    __syncwarp();
#pragma unroll
    for (int u = 0; u < 8; ++u) row[u] = t[m * 9 + u];
    forward8(row, coef);
    int levels[8];
    const int4 packed = in_blocks ? __ldg(reinterpret_cast<const int4*>(P.component.levels + block * 64 + m * 8))
                                  : make_int4(0, 0, 0, 0);
    const int words[4] = {packed.x, packed.y, packed.z, packed.w};
#pragma unroll
    for (int u = 0; u < 8; ++u) {
      const unsigned word = static_cast<unsigned>(words[u >> 1]);
      levels[u] = static_cast<int>(static_cast<std::int16_t>((u & 1) ? (word >> 16) : (word & 0xffffu)));
    }
    const bool flat = in_blocks && P.component.flat[block] != 0;
#pragma unroll
    for (int u = 0; u < 8; ++u) zeta[u] = prox_at(coef[u], levels[u], m * 8 + u, flat, F);
    if constexpr (KEEP) {
      // Kept coefficients as the map gives them: DC centred (less q Q + 1024).
      if (in_blocks && cell == 0) {
        float4* to = reinterpret_cast<float4*>(P.component.zeta + block * 64 + m * 8);
        to[0] = make_float4(zeta[0], zeta[1], zeta[2], zeta[3]);
        to[1] = make_float4(zeta[4], zeta[5], zeta[6], zeta[7]);
#pragma unroll
        for (int u = 0; u < 8; ++u) {
          const int k = m * 8 + u;
          const double absolute = k == 0 ? static_cast<double>(zeta[u]) +
                                               (static_cast<double>(levels[0]) * P.component.constants->step[0] + 1024.0)
                                         : static_cast<double>(zeta[u]);
          if (P.g.recorded_row(i0)) sum += value_term(absolute, levels[u], k, flat, *P.component.constants);
        }
      }
    }
    inverse8(zeta, row);
    __syncwarp();
    if (cell == 0 && used) {
#pragma unroll
      for (int c = 0; c < 8; ++c) t[m * 9 + c] = row[c];
    }
    __syncwarp();
#pragma unroll
    for (int k = 0; k < 8; ++k) col[k] = t[k * 9 + m];
    float back[8];
    inverse8(col, back);
    if (column_in) {
#pragma unroll
      for (int r = 0; r < 8; ++r) {
#pragma unroll
        for (int a = 0; a < CR; ++a) {
          const int rr = CR * r + a;
          float out;
          if constexpr (CR == 1 && CC == 1) {
            out = in_blocks ? back[r] + middle : v[rr];
          } else {
            out = in_blocks ? v[rr] + (back[r] - mean[r]) : v[rr];
          }
          const std::size_t at = static_cast<std::size_t>(i0 + rr) * pitch + jc;
          P.xt[at] = out;
          if constexpr (KEEP) P.v[at] = v[rr];
        }
      }
    }
  }
  if constexpr (KEEP) cta_sum(sum, P.partials);
}

// The primal step fed by TMA works on items, each a stage of 64 canvas rows (8 / CR block rows,
// a compute warp each) of a strip of 32 canvas columns of a component. An item is one 3D box of
// the channel's x, p1 and p2 planes (36 columns: the strip and 4 to its left; the stage's rows
// and the row above) and the levels of its blocks, loaded into a slot of a ring while the
// items before it are computed. The computation of a block row is primal_kernel's, from shared
// memory.
constexpr int kStageRows = 64;
constexpr int kPrimalSpan = 36;  // box columns: 4 + 32 (x at 16-byte boundaries; p1 from j - 1)

template <int CR>
constexpr int primal_warps() {
  return kStageRows / (8 * CR);
}

// Slots of the ring: two, which leave room for three CTAs on an SM (the loader warp fills one
// slot while the compute warps work on the other).
template <int CR>
constexpr int primal_slots() {
  return 2;
}

// A compute warp's transpose tiles (4 blocks x 72 floats) inside its slot: the warp's own rows
// of the x plane, which no other warp reads and which it has read into registers (v) before its
// first transpose.
template <int CR>
__device__ __forceinline__ float* primal_tiles(float* slot, int warp) {
  return slot + (1 + warp * 8 * CR) * kPrimalSpan;
}

// The dynamic shared memory of a primal CTA: the slots' boxes (x, p1, p2), then their levels.
template <int CR, int CC>
constexpr std::size_t primal_shared_bytes() {
  return primal_slots<CR>() * (((3 * (kStageRows + 1) * kPrimalSpan + 31) / 32 * 32) * sizeof(float) +
                               primal_warps<CR>() * (32 / (8 * CC)) * 64 * sizeof(std::int16_t));
}

// One warp's block row of a stage, from shared memory: `slot` the stage's box (x, p1, p2: the
// row above and 64 rows of 36 columns each), `stage_levels` the levels of the lane's block.
// v = x + tau gamma div p, the cell means less the middle of the DC interval, the DCT, the
// clip, the inverse DCT, x~ written (and with KEEP zeta and v, and the data term's terms added
// to `sum`). `t` is the warp's transpose tile.
template <int CR, int CC, bool KEEP>
__device__ __forceinline__ void primal_block_row(const float* slot, const std::int16_t* stage_levels,
                                                 const PrimalParams& P, const ProxFactors& F, float* t, int warp,
                                                 int lane, int vby, int j, bool column_in, bool in_blocks, bool flat,
                                                 std::size_t block, double& sum) {
  constexpr unsigned kAll = 0xffffffffu;
  constexpr int L = 8 * CC, BH = 8 * CR;
  constexpr int SPAN = kPrimalSpan, HALO = 4, PLANE = (kStageRows + 1) * SPAN;
  const int in_block = lane % L, m = in_block / CC, cell = in_block % CC;
  const int leader = lane - cell;
  const int col = HALO + lane;
  const int rows = P.g.rows, columns = P.g.columns, pitch = P.g.pitch;
  const float descent = P.descent;
  const int i0 = vby * BH;
  const int base_row = 1 + warp * BH;  // shared-memory row of canvas row i0
  float v[BH];
#pragma unroll
  for (int r = 0; r < BH; ++r) {
    const int i = i0 + r, sr = base_row + r;
    const float x = slot[0 * PLANE + sr * SPAN + col];
    const float p1 = slot[1 * PLANE + sr * SPAN + col];
    const float p2 = slot[2 * PLANE + sr * SPAN + col];
    // Row -1 and column -1 lie outside the planes: the box holds zeros there.
    const float before = slot[1 * PLANE + sr * SPAN + col - 1];
    const float above = slot[2 * PLANE + (sr - 1) * SPAN + col];
    const float dy = (i + 1 < rows ? p2 : 0.0f) - above;
    const float dx = (j + 1 < columns ? p1 : 0.0f) - before;
    v[r] = x + descent * (dy + dx);
  }
  const float dc_level = in_blocks ? static_cast<float>(stage_levels[0]) : 0.0f;
  const float middle = (dc_level * F.plain[0].x + 1024.0f) * 0.125f;
  float mean[8];
#pragma unroll
  for (int r = 0; r < 8; ++r) {
    if constexpr (CR == 1 && CC == 1) {
      mean[r] = v[r] - middle;
    } else {
      float column = v[CR * r];
#pragma unroll
      for (int a = 1; a < CR; ++a) column += v[CR * r + a];
      float total = 0.0f;
#pragma unroll
      for (int c = 0; c < CC; ++c) {
        const float part = __shfl_sync(kAll, column, leader + c);
        total = c == 0 ? part : total + part;
      }
      mean[r] = total / static_cast<float>(CR * CC) - middle;
    }
  }
  float colv[8], row[8], coef[8], zeta[8];
  forward8(mean, colv);
  __syncwarp();
  if (cell == 0) {
#pragma unroll
    for (int k = 0; k < 8; ++k) t[k * 9 + m] = colv[k];
  }
  __syncwarp();
#pragma unroll
  for (int u = 0; u < 8; ++u) row[u] = t[m * 9 + u];
  forward8(row, coef);
  int levels[8];
  const int4 packed = in_blocks ? *reinterpret_cast<const int4*>(stage_levels + m * 8) : make_int4(0, 0, 0, 0);
  const int words[4] = {packed.x, packed.y, packed.z, packed.w};
#pragma unroll
  for (int u = 0; u < 8; ++u) {
    const unsigned word = static_cast<unsigned>(words[u >> 1]);
    levels[u] = static_cast<int>(static_cast<std::int16_t>((u & 1) ? (word >> 16) : (word & 0xffffu)));
  }
#pragma unroll
  for (int u = 0; u < 8; ++u) zeta[u] = prox_at(coef[u], levels[u], m * 8 + u, flat, F);
  if constexpr (KEEP) {
    if (in_blocks && cell == 0) {
      float4* to = reinterpret_cast<float4*>(P.component.zeta + block * 64 + m * 8);
      to[0] = make_float4(zeta[0], zeta[1], zeta[2], zeta[3]);
      to[1] = make_float4(zeta[4], zeta[5], zeta[6], zeta[7]);
#pragma unroll
      for (int u = 0; u < 8; ++u) {
        const int k = m * 8 + u;
        const double absolute =
            k == 0 ? static_cast<double>(zeta[u]) +
                         (static_cast<double>(levels[0]) * P.component.constants->step[0] + 1024.0)
                   : static_cast<double>(zeta[u]);
        if (P.g.recorded_row(i0)) sum += value_term(absolute, levels[u], k, flat, *P.component.constants);
      }
    }
  }
  inverse8(zeta, row);
  __syncwarp();
  if (cell == 0) {
#pragma unroll
    for (int c = 0; c < 8; ++c) t[m * 9 + c] = row[c];
  }
  __syncwarp();
#pragma unroll
  for (int k = 0; k < 8; ++k) colv[k] = t[k * 9 + m];
  float back[8];
  inverse8(colv, back);
  if (column_in) {
#pragma unroll
    for (int r = 0; r < 8; ++r) {
#pragma unroll
      for (int a = 0; a < CR; ++a) {
        const int rr = CR * r + a;
        float out;
        if constexpr (CR == 1 && CC == 1) {
          out = in_blocks ? back[r] + middle : v[rr];
        } else {
          out = in_blocks ? v[rr] + (back[r] - mean[r]) : v[rr];
        }
        const std::size_t at = static_cast<std::size_t>(i0 + rr) * pitch + j;
        P.xt[at] = out;
        if constexpr (KEEP) P.v[at] = v[rr];
      }
    }
  }
}

// The CTA's items t = blockIdx.x + n gridDim.x, n = 0, 1, ..., as (component, stage, strip):
// one division at the start, then additions.
struct ItemWalk {
  int z, stage, strip;
  int strips, stages, step_stages, step_strips;
  __device__ ItemWalk(int first, int step, int strips_, int stages_) : strips(strips_), stages(stages_) {
    const int per_component = strips * stages;
    z = first / per_component;
    const int rest = first - z * per_component;
    stage = rest / strips;
    strip = rest - stage * strips;
    step_stages = step / strips;
    step_strips = step - step_stages * strips;
  }
  __device__ void next() {
    strip += step_strips;
    stage += step_stages;
    if (strip >= strips) {
      strip -= strips;
      ++stage;
    }
    while (stage >= stages && stages > 0) {
      stage -= stages;
      ++z;
    }
  }
};

// The loads of an item (a stage of a strip) into a slot: the box of x, p1, p2 and the levels
// of its blocks, block row by block row (a bulk copy each), on the slot's barrier.
template <int CR, int CC>
__device__ __forceinline__ void primal_issue(float* box, std::int16_t* levels, const CUtensorMap* map,
                                             std::uint64_t* bar, const PrimalParams& P, int strip, int stage) {
  constexpr int NB = primal_warps<CR>();
  constexpr int B = 32 / (8 * CC), BH = 8 * CR;
  constexpr int SLOT = 3 * (kStageRows + 1) * kPrimalSpan;
  const int vbr = P.g.rows / BH;
  const int first = stage * NB;
  const int vbx0 = strip * B;
  const int blocks = min(B, P.component.block_columns - vbx0);
  int rows_copied = 0;
  for (int w = 0; w < NB; ++w) {
    const int vby = first + w;
    if (vby < vbr && vby < P.component.block_rows && blocks > 0) ++rows_copied;
  }
  barrier_expect(bar, SLOT * 4 + rows_copied * blocks * 128);
  load_box(box, map, bar, strip * 32 - 4, first * BH - 1, 0);
  for (int w = 0; w < NB; ++w) {
    const int vby = first + w;
    if (vby < vbr && vby < P.component.block_rows && blocks > 0) {
      load_bulk(levels + w * B * 64,
                P.component.levels + (static_cast<std::size_t>(vby) * P.component.block_columns + vbx0) * 64,
                blocks * 128, bar);
    }
  }
}

// The primal step fed by TMA, persistent and warp-specialized: NB warps compute (a block row
// of every item each) and one more issues the loads. The items are a list of (component, strip,
// stage) -- a stage is 64 canvas rows, 8 / CR block rows, of a strip of 32 canvas columns of
// one of the launch's components (1 or 2 of the same cells, e.g. Cb and Cr); the CTAs the
// device holds at once take items t = blockIdx.x + n gridDim.x, neighbouring CTAs
// neighbouring strips, so that the columns two boxes share come from L2. An item's loads fill
// a slot of a ring of S: its `full` barrier ends when the bytes are in, its `empty` barrier
// when every compute warp is done with it, and only then is the slot loaded again, so the
// compute warps never wait for one another.
template <int CR, int CC, bool KEEP>
__global__ void __launch_bounds__(32 * (primal_warps<CR>() + 1), 3)
    primal_tma_kernel(const __grid_constant__ CUtensorMap map0, const __grid_constant__ CUtensorMap map1,
                      const __grid_constant__ PrimalBatch Q) {
  constexpr unsigned kAll = 0xffffffffu;
  constexpr int NB = primal_warps<CR>();
  constexpr int L = 8 * CC, B = 32 / L, BH = 8 * CR;
  constexpr int SLOT = 3 * (kStageRows + 1) * kPrimalSpan;
  // Slots 128-byte aligned, as a bulk-tensor copy's shared-memory destination is.
  constexpr int STRIDE = (SLOT + 31) / 32 * 32;
  constexpr int S = primal_slots<CR>();
  constexpr int kStageLevels = NB * B * 64;
  extern __shared__ __align__(128) float ring[];
  __shared__ __align__(8) std::uint64_t full[S], empty[S];
  __shared__ ProxFactors factors[2];
  __shared__ PrimalParams parts[2];  // the components' parameters, read per item
  __shared__ int failures;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  for (int z = 0; z < Q.count; ++z) {
    const float* from = reinterpret_cast<const float*>(Q.part[z].component.factors);
    float* to = reinterpret_cast<float*>(&factors[z]);
    for (int k = tid; k < static_cast<int>(sizeof(ProxFactors) / 4); k += 32 * (NB + 1)) to[k] = from[k];
    if (tid == 0) parts[z] = Q.part[z];
  }
  if (tid == 0) {
    for (int s = 0; s < S; ++s) {
      barrier_init(&full[s], 1);
      barrier_init(&empty[s], NB);
    }
    failures = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
  const int items = (Q.items - static_cast<int>(blockIdx.x) + static_cast<int>(gridDim.x) - 1) /
                    static_cast<int>(gridDim.x);  // this CTA's
  // The levels of an item's blocks (NB block rows of B blocks), after the slots.
  std::int16_t* const levels_ring = reinterpret_cast<std::int16_t*>(ring + S * STRIDE);
  ItemWalk walk(static_cast<int>(blockIdx.x), static_cast<int>(gridDim.x), Q.strips, Q.stages);
  double sum0 = 0.0, sum1 = 0.0;  // the data term's terms of each component
  int issued = 0;
  if (warp == NB) {
    if (lane == 0) {
      for (int n = 0; n < items; ++n, walk.next()) {
        const int slot = n % S;
        if (n >= S && !barrier_wait(&empty[slot], (n / S - 1) & 1)) {
          atomicAdd(&failures, 1);
          break;
        }
        primal_issue<CR, CC>(ring + slot * STRIDE, levels_ring + slot * kStageLevels, walk.z == 0 ? &map0 : &map1,
                             &full[slot], parts[walk.z], walk.strip, walk.stage);
        issued = n + 1;
      }
    }
  } else {
    const int blk = lane / L, in_block = lane % L;
    // The flat flag of the lane's block in an item, read an item ahead of its use.
    auto flag_of = [&](const ItemWalk& w) -> std::uint8_t {
      const PrimalParams& P = parts[w.z];
      const int vbx = w.strip * B + blk, vby = w.stage * NB + warp;
      const bool in = vby < P.g.rows / BH && vbx * L + in_block < P.g.columns && vby < P.component.block_rows &&
                      vbx < P.component.block_columns;
      return in ? P.component.flat[static_cast<std::size_t>(vby) * P.component.block_columns + vbx] : 0;
    };
    ItemWalk ahead = walk;
    std::uint8_t flat_next = items > 0 ? flag_of(ahead) : 0;
    for (int s = 0; s < items; ++s, walk.next()) {
      const int z = walk.z;
      const PrimalParams& P = parts[z];
      const ProxFactors& F = factors[z];
      double sum = 0.0;
      const int vbr = P.g.rows / BH;
      const int vbx = walk.strip * B + blk;
      const int j = vbx * L + in_block;
      const bool column_in = j < P.g.columns;
      const int vby = walk.stage * NB + warp;
      const bool in_blocks =
          vby < vbr && column_in && vby < P.component.block_rows && vbx < P.component.block_columns;
      const std::size_t block =
          static_cast<std::size_t>(in_blocks ? vby : 0) * P.component.block_columns + (in_blocks ? vbx : 0);
      const bool flat = in_blocks && flat_next != 0;
      ahead.next();
      flat_next = s + 1 < items ? flag_of(ahead) : 0;
      const bool ready = barrier_wait(&full[s % S], (s / S) & 1);
      if (__any_sync(kAll, !ready)) {
        if (lane == 0) atomicAdd(&failures, 1);
        break;
      }
      float* const slot = ring + (s % S) * STRIDE;
      const std::int16_t* stage_levels = levels_ring + (s % S) * kStageLevels + (warp * B + blk) * 64;
      float* const t = primal_tiles<CR>(slot, warp) + blk * 72;
      if (vby < vbr) {
        primal_block_row<CR, CC, KEEP>(slot, stage_levels, P, F, t, warp, lane, vby, j, column_in, in_blocks, flat,
                                       block, sum);
      }
      if (z == 0) {
        sum0 += sum;
      } else {
        sum1 += sum;
      }
      // The warp's tile writes into the slot ordered before the next load's (async proxy) writes.
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      __syncwarp();
      if (lane == 0) barrier_arrive(&empty[s % S]);  // the warp is done with the slot
    }
  }
  __syncthreads();
  if (failures != 0) {
    if (tid == 0 && parts[0].error != nullptr) atomicExch(parts[0].error, 1);
    // No load may still write into shared memory when the CTA leaves: the last one issued into
    // each slot is waited for.
    if (warp == NB && lane == 0) {
      for (int n = max(issued - S, 0); n < issued; ++n) barrier_wait(&full[n % S], (n / S) & 1);
    }
  }
  if constexpr (KEEP) {
    cta_sum(sum0, parts[0].partials);
    if (Q.count > 1) cta_sum(sum1, parts[1].partials);
  }
}

// The primal step of a batch (many components of one cell layout, of many images, of different
// sizes): a table of items (component, strip, stage); each CTA takes a contiguous range of it,
// warp-specialized as primal_tma_kernel is. Each item's parameters and box map are the
// component's entry of `components` in global memory (the map read through the tensor-map
// proxy after an acquire fence), its parameters copied into the slot's with its loads; its
// factors are read from global memory. Nothing is kept (the batch's last primal step, which
// keeps, runs per image).
template <int CR, int CC>
__global__ void __launch_bounds__(32 * (primal_warps<CR>() + 1), 3)
    primal_batch_kernel(const PrimalItem* __restrict__ list, int count, const PrimalBatchComponent* components,
                        int parity) {
  constexpr unsigned kAll = 0xffffffffu;
  constexpr int NB = primal_warps<CR>();
  constexpr int L = 8 * CC, B = 32 / L, BH = 8 * CR;
  constexpr int SLOT = 3 * (kStageRows + 1) * kPrimalSpan;
  constexpr int STRIDE = (SLOT + 31) / 32 * 32;
  constexpr int S = primal_slots<CR>();
  constexpr int kStageLevels = NB * B * 64;
  extern __shared__ __align__(128) float ring[];
  __shared__ __align__(8) std::uint64_t full[S], empty[S];
  __shared__ PrimalParams parts[S];  // of the items in the slots
  __shared__ int failures;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int first = static_cast<int>(static_cast<long long>(blockIdx.x) * count / gridDim.x);
  const int items = static_cast<int>(static_cast<long long>(blockIdx.x + 1) * count / gridDim.x) - first;
  if (tid == 0) {
    for (int s = 0; s < S; ++s) {
      barrier_init(&full[s], 1);
      barrier_init(&empty[s], NB);
    }
    failures = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
  std::int16_t* const levels_ring = reinterpret_cast<std::int16_t*>(ring + S * STRIDE);
  int issued = 0;
  if (warp == NB) {
    if (lane == 0) {
      for (int n = 0; n < items; ++n) {
        const int slot = n % S;
        if (n >= S && !barrier_wait(&empty[slot], (n / S - 1) & 1)) {
          atomicAdd(&failures, 1);
          break;
        }
        const PrimalItem item = list[first + n];
        const PrimalBatchComponent& entry = components[item.component];
        parts[slot] = entry.params[parity];  // seen by the compute warps with the slot's bytes
        const CUtensorMap* map = &entry.map[parity];
        asm volatile("fence.proxy.tensormap::generic.acquire.gpu [%0], 128;" ::"l"(map) : "memory");
        primal_issue<CR, CC>(ring + slot * STRIDE, levels_ring + slot * kStageLevels, map, &full[slot], parts[slot],
                             item.strip, item.stage);
        issued = n + 1;
      }
    }
  } else {
    const int blk = lane / L, in_block = lane % L;
    double sum = 0.0;  // unused: nothing is kept
    for (int s = 0; s < items; ++s) {
      const PrimalItem item = list[first + s];
      const bool ready = barrier_wait(&full[s % S], (s / S) & 1);
      if (__any_sync(kAll, !ready)) {
        if (lane == 0) atomicAdd(&failures, 1);
        break;
      }
      const PrimalParams& P = parts[s % S];
      const ProxFactors& F = *P.component.factors;
      const int vbr = P.g.rows / BH;
      const int vbx = item.strip * B + blk;
      const int j = vbx * L + in_block;
      const bool column_in = j < P.g.columns;
      const int vby = item.stage * NB + warp;
      const bool in_blocks =
          vby < vbr && column_in && vby < P.component.block_rows && vbx < P.component.block_columns;
      const std::size_t block =
          static_cast<std::size_t>(in_blocks ? vby : 0) * P.component.block_columns + (in_blocks ? vbx : 0);
      const bool flat = in_blocks && P.component.flat[block] != 0;
      float* const slot = ring + (s % S) * STRIDE;
      const std::int16_t* stage_levels = levels_ring + (s % S) * kStageLevels + (warp * B + blk) * 64;
      float* const t = primal_tiles<CR>(slot, warp) + blk * 72;
      if (vby < vbr) {
        primal_block_row<CR, CC, false>(slot, stage_levels, P, F, t, warp, lane, vby, j, column_in, in_blocks, flat,
                                        block, sum);
      }
      // The warp's tile writes into the slot ordered before the next load's (async proxy) writes.
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      __syncwarp();
      if (lane == 0) barrier_arrive(&empty[s % S]);  // the warp is done with the slot and its parameters
    }
  }
  __syncthreads();
  if (failures != 0) {
    if (tid == 0 && items > 0) {
      int* error = components[list[first].component].params[parity].error;
      if (error != nullptr) atomicExch(error, 1);
    }
    if (warp == NB && lane == 0) {
      for (int n = max(issued - S, 0); n < issued; ++n) barrier_wait(&full[n % S], (n / S) & 1);
    }
  }
}

// The result's picture (capi.cpp's to_rgb, rust/unround/src/decode.rs:306-364): a thread per
// pixel of the picture; JFIF's RGB by the same binary64 operations in the same order, each
// rounded on its own (no contraction into fused multiply-adds), so that it equals the host's.
__global__ void __launch_bounds__(256) picture_kernel(const PictureParams P) {
  const std::size_t k = static_cast<std::size_t>(blockIdx.x) * 256 + threadIdx.x;
  const std::size_t pixels = static_cast<std::size_t>(P.height) * P.width;
  if (k >= pixels) return;
  const std::size_t i = k / static_cast<std::size_t>(P.width), j = k % static_cast<std::size_t>(P.width);
  const std::size_t plane = static_cast<std::size_t>(P.rows) * P.columns, at = i * P.columns + j;
  if (P.picture != nullptr) {
    if (P.rgb) {
      const double y = P.canvas[at];
      const double cb = __dsub_rn(P.canvas[plane + at], 128.0), cr = __dsub_rn(P.canvas[2 * plane + at], 128.0);
      P.picture[3 * k] = __dadd_rn(y, __dmul_rn(kCr, cr));
      P.picture[3 * k + 1] = __dsub_rn(__dsub_rn(y, __dmul_rn(kGb, cb)), __dmul_rn(kGr, cr));
      P.picture[3 * k + 2] = __dadd_rn(y, __dmul_rn(kCb, cb));
    } else {
      for (int c = 0; c < P.channels; ++c) P.picture[k * P.channels + c] = P.canvas[c * plane + at];
    }
  }
  if (P.planes != nullptr) {
    for (int c = 0; c < P.channels; ++c) P.planes[c * pixels + k] = P.canvas[c * plane + at];
  }
}

// ---------------------------------------------------------------------------------------
// Binary64: the start's coefficients, and canvases of coefficients.

__global__ void __launch_bounds__(256) start_kernel(const StartParams P) {
  const int thread = blockIdx.x * 256 + threadIdx.x;
  const int blocks = P.component.block_rows * P.component.block_columns;
  const int block = thread >> 3, m = thread & 7;
  double sum = 0.0;
  if (block < blocks) {
    const Constants64& K = *P.component.constants;
    const bool flat = P.component.flat[block] != 0;
    const int canvas_row = (block / P.component.block_columns) * 8 * P.component.cell_rows;
    const bool counted = canvas_row >= P.record_first && canvas_row < P.record_end;
    for (int u = 0; u < 8; ++u) {
      const int k = m * 8 + u;
      const std::size_t at = static_cast<std::size_t>(block) * 64 + k;
      const int q = P.component.levels[at];
      const double level = static_cast<double>(q);
      const double step = K.step[k];
      const double shift = k == 0 ? 1024.0 : 0.0;
      const double low = ((level - 0.5) - K.slack) * step + shift;
      const double high = ((level + 0.5) + K.slack) * step + shift;
      double centre;
      if (K.mmse && k != 0) {
        const double size = (fabs(level) - K.shrink[k]) * step;
        centre = q == 0 ? 0.0 : (q < 0 ? -size : size);
      } else {
        centre = level * step + shift;
      }
      const double from = P.given != nullptr ? P.given[at] : centre;
      const double zeta = clamp_to(from, low, high);
      P.coefficients[at] = zeta;
      if (counted) sum += value_term(zeta, q, k, flat, K);
    }
  }
  cta_sum(sum, P.partials);
}

// The kept binary32 coefficients made binary64 and absolute: DC, kept centred, plus q Q + 1024
// (exact in binary64), every coefficient clipped to its binary64 interval.
__global__ void __launch_bounds__(256) restore_kernel(const ComponentDevice C, double* out) {
  const std::size_t at = static_cast<std::size_t>(blockIdx.x) * 256 + threadIdx.x;
  const std::size_t count = static_cast<std::size_t>(C.block_rows) * C.block_columns * 64;
  if (at >= count) return;
  const int k = static_cast<int>(at & 63);
  const Constants64& K = *C.constants;
  const double level = static_cast<double>(C.levels[at]);
  const double shift = k == 0 ? 1024.0 : 0.0;
  double value = static_cast<double>(C.zeta[at]);
  if (k == 0) value += level * K.step[0] + 1024.0;
  const double low = ((level - 0.5) - K.slack) * K.step[k] + shift;
  const double high = ((level + 0.5) + K.slack) * K.step[k] + shift;
  out[at] = clamp_to(value, low, high);
}

template <int CR, int CC>
__global__ void __launch_bounds__(256) canvas_kernel(const CanvasParams P) {
  __shared__ double tile[kWarps][4][72];
  constexpr int BH = 8 * CR, BW = 8 * CC;
  const int lane = threadIdx.x, b = lane >> 3, m = lane & 7;
  const int rows = P.g.rows, columns = P.g.columns, pitch = P.g.pitch;
  const int vbx = blockIdx.x * 4 + b;
  const int vby = blockIdx.y * kWarps + threadIdx.y;
  const bool active = vbx * BW < columns && vby * BH < rows;
  const bool in_blocks = active && vby < P.component.block_rows && vbx < P.component.block_columns;
  const int j0 = vbx * BW + m * CC, i0 = vby * BH;
  const std::size_t block =
      static_cast<std::size_t>(in_blocks ? vby : 0) * P.component.block_columns + (in_blocks ? vbx : 0);
  // The lane's row of coefficients, the inverse row DCT, transpose, inverse column DCT.
  double zeta[8], row[8], col[8], back[8];
#pragma unroll
  for (int u = 0; u < 8; ++u) zeta[u] = in_blocks ? P.coefficients[block * 64 + m * 8 + u] : 0.0;
  inverse8(zeta, row);
  double* t = tile[threadIdx.y][b];
#pragma unroll
  for (int c = 0; c < 8; ++c) t[m * 9 + c] = row[c];
  __syncwarp();
#pragma unroll
  for (int k = 0; k < 8; ++k) col[k] = t[k * 9 + m];
  inverse8(col, back);
  if (!active) return;
  double* canvas = P.canvas;
#pragma unroll
  for (int r = 0; r < 8; ++r) {
    double vs[CR][CC];
    double mean = 0.0;
    if (P.mode == 1) {
      double sum = 0.0;
#pragma unroll
      for (int c = 0; c < CC; ++c) {
        double column = 0.0;
#pragma unroll
        for (int a = 0; a < CR; ++a) {
          vs[a][c] = static_cast<double>(P.v[static_cast<std::size_t>(i0 + CR * r + a) * pitch + j0 + c]);
          column = a == 0 ? vs[a][c] : column + vs[a][c];
        }
        sum = c == 0 ? column : sum + column;
      }
      mean = sum / static_cast<double>(CR * CC);
    }
#pragma unroll
    for (int a = 0; a < CR; ++a) {
#pragma unroll
      for (int c = 0; c < CC; ++c) {
        const int i = i0 + CR * r + a, j = j0 + c;
        double value;
        if (P.mode == 0) {
          value = in_blocks ? back[r] : P.beyond;
        } else if (CR * CC == 1) {
          value = in_blocks ? back[r] : vs[a][c];
        } else {
          value = in_blocks ? vs[a][c] + (back[r] - mean) : vs[a][c];
        }
        canvas[static_cast<std::size_t>(i) * columns + j] = value;
        if (P.mode == 0 && P.x != nullptr) P.x[static_cast<std::size_t>(i) * pitch + j] = static_cast<float>(value);
      }
    }
  }
}

__global__ void gradient_kernel(const float* x, float* w1, float* w2, Geometry g) {
  const int j = blockIdx.x * 32 + threadIdx.x, i = blockIdx.y * 8 + threadIdx.y;
  if (i >= g.rows || j >= g.columns) return;
  for (int c = 0; c < g.channels; ++c) {
    const std::size_t base = c * g.plane, at = static_cast<std::size_t>(i) * g.pitch + j;
    const float here = x[base + at];
    w1[base + at] = j + 1 < g.columns ? x[base + at + 1] - here : 0.0f;
    w2[base + at] = i + 1 < g.rows ? x[base + at + g.pitch] - here : 0.0f;
  }
}

// Projects a start's duals onto their balls (cpp/src/operators.cpp project; 4.4, 5).
__global__ void project_kernel(Fields f, Geometry g, int tgv, int coupled, float radius, float radius0) {
  const int j = blockIdx.x * 32 + threadIdx.x, i = blockIdx.y * 8 + threadIdx.y;
  if (i >= g.rows || j >= g.columns) return;
  const std::size_t at = static_cast<std::size_t>(i) * g.pitch + j;
  if (coupled) {
    float sp = 0.0f, sr = 0.0f;
    for (int c = 0; c < g.channels; ++c) {
      const std::size_t k = c * g.plane + at;
      sp += f.p1[k] * f.p1[k] + f.p2[k] * f.p2[k];
      if (tgv) sr += f.r11[k] * f.r11[k] + f.r22[k] * f.r22[k] + 2.0f * (f.r12[k] * f.r12[k]);
    }
    const float ap = ball_scale(sp, radius), ar = ball_scale(sr, radius0);
    for (int c = 0; c < g.channels; ++c) {
      const std::size_t k = c * g.plane + at;
      f.p1[k] *= ap;
      f.p2[k] *= ap;
      if (tgv) {
        f.r11[k] *= ar;
        f.r22[k] *= ar;
        f.r12[k] *= ar;
      }
    }
  } else {
    for (int c = 0; c < g.channels; ++c) {
      const std::size_t k = c * g.plane + at;
      const float ap = ball_scale(f.p1[k] * f.p1[k] + f.p2[k] * f.p2[k], radius);
      f.p1[k] *= ap;
      f.p2[k] *= ap;
      if (tgv) {
        const float ar =
            ball_scale(f.r11[k] * f.r11[k] + f.r22[k] * f.r22[k] + 2.0f * (f.r12[k] * f.r12[k]), radius0);
        f.r11[k] *= ar;
        f.r22[k] *= ar;
        f.r12[k] *= ar;
      }
    }
  }
}

// ---------------------------------------------------------------------------------------
// Records, binary64 sums from the binary32 tilde point (cpp/src/primal_dual.hpp:446-501,
// 791-895): the norms of the pixels, TGV's div2 r~ and its largest norm; G* of a field
// (cpp/src/frames.cpp:428-487, model.cpp:74-111); the residual of the partial gap.

// The records' norms, a thread per pixel: every value the pixel needs, of every channel, is
// loaded first (the neighbours' from L1 and L2), before any arithmetic or store, so that a pixel
// waits for memory once; then, in binary64 from the binary32 tilde point, |grad x~ - w~| (the
// first-order term), |E w~|_F (the second-order term) and div2 r~ (written, binary32) and its
// norm, each operation as cpp/src/primal_dual.hpp:836-895 orders it. Pixels outside the record
// rows add nothing (div2 is still made for them).
template <bool TGV, int C, bool COUPLED>
__global__ void __launch_bounds__(256, 3) norms_kernel(const NormParams P) {
  const int j = blockIdx.x * 32 + threadIdx.x, i = blockIdx.y * 8 + threadIdx.y;
  const int rows = P.g.rows, columns = P.g.columns, pitch = P.g.pitch;
  double first = 0.0, second = 0.0, most = 0.0;
  if (i < rows && j < columns) {
    const std::size_t at = static_cast<std::size_t>(i) * pitch + j;
    const bool right = j + 1 < columns, down = i + 1 < rows, left = j > 0, up = i > 0;
    const std::size_t ar = right ? at + 1 : at, ad = down ? at + pitch : at;
    const std::size_t al = left ? at - 1 : at, au = up ? at - pitch : at;
    // The loads.
    float xt[C], xt_r[C], xt_d[C];
    float w1[C], w2[C], w1_l[C], w2_l[C], w1_u[C], w2_u[C];
    float r11[C], r22[C], r12[C], r11_r[C], r12_r[C], r12_d[C], r22_d[C];
#pragma unroll
    for (int c = 0; c < C; ++c) {
      const std::size_t base = c * P.g.plane;
      xt[c] = P.xt[base + at];
      xt_r[c] = P.xt[base + ar];
      xt_d[c] = P.xt[base + ad];
      if constexpr (TGV) {
        w1[c] = P.tilde.w1[base + at];
        w2[c] = P.tilde.w2[base + at];
        w1_l[c] = P.tilde.w1[base + al];
        w2_l[c] = P.tilde.w2[base + al];
        w1_u[c] = P.tilde.w1[base + au];
        w2_u[c] = P.tilde.w2[base + au];
        r11[c] = P.tilde.r11[base + at];
        r22[c] = P.tilde.r22[base + at];
        r12[c] = P.tilde.r12[base + at];
        r11_r[c] = P.tilde.r11[base + ar];
        r12_r[c] = P.tilde.r12[base + ar];
        r12_d[c] = P.tilde.r12[base + ad];
        r22_d[c] = P.tilde.r22[base + ad];
      }
    }
    // The arithmetic.
    double square = 0.0;
#pragma unroll
    for (int c = 0; c < C; ++c) {
      const double gamma = P.weight[c];
      const double here = xt[c];
      double gx = right ? static_cast<double>(xt_r[c]) - here : 0.0;
      double gy = down ? static_cast<double>(xt_d[c]) - here : 0.0;
      if constexpr (TGV) {
        gx = gx - static_cast<double>(w1[c]);
        gy = gy - static_cast<double>(w2[c]);
      }
      square += (COUPLED ? gamma * gamma : 1.0) * (gx * gx + gy * gy);
      if constexpr (!COUPLED) {
        first += gamma * sqrt(square);
        square = 0.0;
      }
    }
    if constexpr (COUPLED) first = sqrt(square);
    if constexpr (TGV) {
      square = 0.0;
#pragma unroll
      for (int c = 0; c < C; ++c) {
        const double gamma = P.weight[c];
        const double a1 = right ? w1[c] : 0.0, a2 = down ? w2[c] : 0.0;
        const double b1 = down ? w1[c] : 0.0, b2 = right ? w2[c] : 0.0;
        const double l1 = left ? w1_l[c] : 0.0, l2 = left ? w2_l[c] : 0.0;
        const double u1 = up ? w1_u[c] : 0.0, u2 = up ? w2_u[c] : 0.0;
        const double exx = a1 - l1, eyy = a2 - u2, exy = 0.5 * ((b1 - u1) + (b2 - l2));
        square += (COUPLED ? gamma * gamma : 1.0) * (exx * exx + eyy * eyy + 2.0 * (exy * exy));
        if constexpr (!COUPLED) {
          second += gamma * sqrt(square);
          square = 0.0;
        }
      }
      if constexpr (COUPLED) second = sqrt(square);
      square = 0.0;
      double d1[C], d2[C];
#pragma unroll
      for (int c = 0; c < C; ++c) {
        d1[c] = right ? static_cast<double>(r11_r[c]) - r11[c] : 0.0;
        d2[c] = right ? static_cast<double>(r12_r[c]) - r12[c] : 0.0;
        if (down) {
          d1[c] += static_cast<double>(r12_d[c]) - r12[c];
          d2[c] += static_cast<double>(r22_d[c]) - r22[c];
        }
        square += d1[c] * d1[c] + d2[c] * d2[c];
        if constexpr (!COUPLED) {
          most = fmax(most, sqrt(square));
          square = 0.0;
        }
      }
      if constexpr (COUPLED) most = fmax(most, sqrt(square));
      // The stores, last.
#pragma unroll
      for (int c = 0; c < C; ++c) {
        P.div2[(2 * c) * P.g.plane + at] = static_cast<float>(d1[c]);
        P.div2[(2 * c + 1) * P.g.plane + at] = static_cast<float>(d2[c]);
      }
    }
  }
  if (!P.g.recorded_row(i)) first = second = most = 0.0;  // div2 is still made for every row
  const double sum_first = cta_reduce<false>(first);
  const double sum_second = cta_reduce<false>(second);
  const double largest = cta_reduce<true>(most);
  if (cta_leader()) {
    const int count = gridDim.x * gridDim.y;
    const int cta = cta_index();
    P.partials[cta] = sum_first;
    P.partials[count + cta] = sum_second;
    P.partials[2 * count + cta] = largest;
  }
}

// g*(s) of a coefficient (cpp/src/model.cpp:74-111, docs/math.md 4.1).
__device__ __forceinline__ double conjugate_term(double s, int q, int k, bool flat, const Constants64& K) {
  const double level = static_cast<double>(q);
  const double step = K.step[k];
  const double shift = k == 0 ? 1024.0 : 0.0;
  const double low = ((level - 0.5) - K.slack) * step + shift;
  const double high = ((level + 0.5) + K.slack) * step + shift;
  double centre;
  if (K.mmse && k != 0) {
    const double size = (fabs(level) - K.shrink[k]) * step;
    centre = q == 0 ? 0.0 : (q < 0 ? -size : size);
  } else {
    centre = level * step + shift;
  }
  const double m = flat ? K.flat_weight[k] : K.weight[k];
  if (!K.costed) {
    const double best = clamp_to(centre + s / m, low, high);
    const double away = best - centre;
    const double weighted = s * best - 0.5 * m * (away * away);
    const double support = fmax(s * low, s * high);
    return m > 0.0 ? weighted : support;
  }
  const double lambda = K.cost[k];
  const double own_low = (level - 0.5) * step + shift;
  const double own_high = (level + 0.5) * step + shift;
  const double free = centre + s / m;
  const double upward = clamp_to(centre + (s - lambda) / m, own_high, high);
  const double downward = clamp_to(centre + (s + lambda) / m, low, own_low);
  const double within = free < own_low ? downward : free;
  const double weighted = free > own_high ? upward : within;
  const double lower_end = s < -lambda ? low : own_low;
  const double upper_end = s > lambda ? high : own_high;
  const double flat_best = s > 0.0 ? upper_end : lower_end;
  const double best = m > 0.0 ? weighted : flat_best;
  const double away = best - centre;
  const double beyond = fmax(fmax(best - own_high, own_low - best), 0.0);
  return s * best - 0.5 * m * (away * away) - lambda * beyond;
}

template <int CR, int CC>
__global__ void __launch_bounds__(256) conjugate_kernel(const ConjugateParams P) {
  __shared__ double tile[kWarps][4][72];
  constexpr int BH = 8 * CR, BW = 8 * CC;
  const int lane = threadIdx.x, b = lane >> 3, m = lane & 7;
  const int rows = P.g.rows, columns = P.g.columns, pitch = P.g.pitch;
  const int vbx = blockIdx.x * 4 + b;
  const int vby = blockIdx.y * kWarps + threadIdx.y;
  const bool active = vbx * BW < columns && vby * BH < rows;
  const bool in_blocks = active && vby < P.component.block_rows && vbx < P.component.block_columns;
  const int j0 = vbx * BW + m * CC, i0 = vby * BH;
  const bool counted = P.g.recorded_row(i0);
  // xi = gamma div q at the lane's samples, q = scale (q1, q2).
  const double scale = P.most_at != nullptr ? negative_theta(*P.most_at, P.alpha1) : P.scale;
  auto q_at = [&](const float* f, int i, int j) -> double { return scale * static_cast<double>(f[static_cast<std::size_t>(i) * pitch + j]); };
  double xi[BH][CC];
  double sums[8], means[8];
  double total = 0.0;
#pragma unroll
  for (int r = 0; r < BH; ++r) {
#pragma unroll
    for (int c = 0; c < CC; ++c) {
      const int i = i0 + r, j = j0 + c;
      double value = 0.0;
      if (active) {
        const double dy = (i + 1 < rows ? q_at(P.q2, i, j) : 0.0) - (i > 0 ? q_at(P.q2, i - 1, j) : 0.0);
        const double dx = (j + 1 < columns ? q_at(P.q1, i, j) : 0.0) - (j > 0 ? q_at(P.q1, i, j - 1) : 0.0);
        value = P.gamma * (dy + dx);
      }
      xi[r][c] = value;
    }
  }
#pragma unroll
  for (int r = 0; r < 8; ++r) {
    double sum = 0.0;
#pragma unroll
    for (int c = 0; c < CC; ++c) {
      double column = xi[CR * r][c];
#pragma unroll
      for (int a = 1; a < CR; ++a) column += xi[CR * r + a][c];
      sum = c == 0 ? column : sum + column;
    }
    sums[r] = sum;
    means[r] = sum / static_cast<double>(CR * CC);
  }
  if (P.free && active) {
#pragma unroll
    for (int r = 0; r < 8; ++r) {
#pragma unroll
      for (int a = 0; a < CR; ++a) {
#pragma unroll
        for (int c = 0; c < CC; ++c) {
          const double s = xi[CR * r + a][c];
          total += in_blocks ? P.radius * fabs(s - means[r]) : 128.0 * s + P.radius * fabs(s);
        }
      }
    }
  }
  // The DCT of the cell sums, and g* of each coefficient of the lane's row.
  double col[8], row[8], coef[8];
  forward8(sums, col);
  double* t = tile[threadIdx.y][b];
#pragma unroll
  for (int k = 0; k < 8; ++k) t[k * 9 + m] = col[k];
  __syncwarp();
#pragma unroll
  for (int u = 0; u < 8; ++u) row[u] = t[m * 9 + u];
  forward8(row, coef);
  if (in_blocks) {
    const std::size_t block = static_cast<std::size_t>(vby) * P.component.block_columns + vbx;
    const bool flat = P.component.flat[block] != 0;
#pragma unroll
    for (int u = 0; u < 8; ++u) {
      const int k = m * 8 + u;
      total += conjugate_term(coef[u], P.component.levels[block * 64 + k], k, flat, *P.component.constants);
    }
  }
  cta_sum(counted ? total : 0.0, P.partials);
}

__global__ void __launch_bounds__(256) residual_kernel(const ResidualParams P) {
  const int j = blockIdx.x * 32 + threadIdx.x, i = blockIdx.y * 8 + threadIdx.y;
  double value = 0.0;
  if (i < P.g.rows && j < P.g.columns && P.g.recorded_row(i)) {
    const std::size_t at = static_cast<std::size_t>(i) * P.g.pitch + j;
    const double a = static_cast<double>(P.p1[at]) + 1.0 * P.d1[at];
    const double b = static_cast<double>(P.p2[at]) + 1.0 * P.d2[at];
    value = sqrt(a * a + b * b);
  }
  cta_sum(value, P.partials);
}

// One array of partials a CTA: the sum (or the largest) of its entries, each thread's strided
// share in index order, then the CTA's fixed-order reduction.
__global__ void __launch_bounds__(1024) reduce_kernel(const __grid_constant__ Reductions R) {
  const int k = blockIdx.x;
  const double* in = R.in[k];
  const int n = R.count[k];
  const bool most = R.largest[k] != 0;
  // Four accumulators a thread (entries i, i + T, i + 2T, i + 3T of each stretch of 4T), so that
  // four loads are in flight; combined in a fixed order.
  double acc[4] = {0.0, 0.0, 0.0, 0.0};
  const int step = blockDim.x;
  for (int i = threadIdx.x; i < n; i += 4 * step) {
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      const int at = i + u * step;
      if (at < n) acc[u] = most ? fmax(acc[u], in[at]) : acc[u] + in[at];
    }
  }
  const double value = most ? fmax(fmax(acc[0], acc[1]), fmax(acc[2], acc[3])) : (acc[0] + acc[1]) + (acc[2] + acc[3]);
  const double total = most ? cta_reduce<true>(value) : cta_reduce<false>(value);
  if (threadIdx.x == 0) R.out[k] = total;
}

__global__ void narrow_kernel(const double* from, float* to, Geometry g) {
  const std::size_t n = static_cast<std::size_t>(g.rows) * g.columns * g.channels;
  for (std::size_t k = blockIdx.x * 256ull + threadIdx.x; k < n; k += static_cast<std::size_t>(gridDim.x) * 256) {
    const std::size_t c = k / (static_cast<std::size_t>(g.rows) * g.columns);
    const std::size_t rest = k % (static_cast<std::size_t>(g.rows) * g.columns);
    const std::size_t i = rest / g.columns, j = rest % g.columns;
    to[c * g.plane + i * g.pitch + j] = static_cast<float>(from[k]);
  }
}

dim3 pixel_grid(const Geometry& g) { return dim3((g.columns + 31) / 32, (g.rows + 7) / 8, 1); }

dim3 block_grid(const Geometry& g, const ComponentDevice& c) {
  const int vbc = (g.columns + 8 * c.cell_columns - 1) / (8 * c.cell_columns);
  const int vbr = (g.rows + 8 * c.cell_rows - 1) / (8 * c.cell_rows);
  return dim3((vbc + 3) / 4, (vbr + kWarps - 1) / kWarps, 1);
}

template <template <int, int> class Launch, typename... A>
cudaError_t by_cells(int cr, int cc, A&&... args) {
#define URB_CELL(R, C) \
  if (cr == R && cc == C) return Launch<R, C>::run(args...);
  URB_CELL(1, 1) URB_CELL(1, 2) URB_CELL(2, 1) URB_CELL(2, 2) URB_CELL(1, 3) URB_CELL(3, 1) URB_CELL(3, 3)
  URB_CELL(1, 4) URB_CELL(4, 1) URB_CELL(2, 4) URB_CELL(4, 2) URB_CELL(4, 4) URB_CELL(2, 3) URB_CELL(3, 2)
  URB_CELL(3, 4) URB_CELL(4, 3)
#undef URB_CELL
  return cudaErrorInvalidValue;
}

// The primal kernel's grid: 32 / (8 CC) blocks across a warp, kPrimalRows block rows down it,
// 8 warps down a CTA.
dim3 primal_grid(const Geometry& g, int cr, int cc) {
  const int per_warp = 8 * cc <= 32 ? 32 / (8 * cc) : 1;
  const int vbc = (g.columns + 8 * cc - 1) / (8 * cc);
  const int vbr = (g.rows + 8 * cr - 1) / (8 * cr);
  const int segments = (vbr + kPrimalRows - 1) / kPrimalRows;
  return dim3((vbc + per_warp - 1) / per_warp, (segments + kWarps - 1) / kWarps, 1);
}

template <int CR, int CC>
struct PrimalLaunch {
  static cudaError_t run(const PrimalParams& p, bool keep, cudaStream_t s) {
    const dim3 grid = primal_grid(p.g, CR, CC);
    if (keep) {
      primal_kernel<CR, CC, true><<<grid, dim3(32, kWarps), 0, s>>>(p);
    } else {
      primal_kernel<CR, CC, false><<<grid, dim3(32, kWarps), 0, s>>>(p);
    }
    return cudaGetLastError();
  }
};

template <int CR, int CC>
struct CanvasLaunch {
  static cudaError_t run(const CanvasParams& p, cudaStream_t s) {
    canvas_kernel<CR, CC><<<block_grid(p.g, p.component), dim3(32, kWarps), 0, s>>>(p);
    return cudaGetLastError();
  }
};

template <int CR, int CC>
struct ConjugateLaunch {
  static cudaError_t run(const ConjugateParams& p, cudaStream_t s) {
    conjugate_kernel<CR, CC><<<block_grid(p.g, p.component), dim3(32, kWarps), 0, s>>>(p);
    return cudaGetLastError();
  }
};

// The sweep's grid: a warp per 32 columns and kSegment rows, 8 warps (segments) to a CTA.
dim3 sweep_grid(const Geometry& g) {
  const int segments = (g.rows + kSegment - 1) / kSegment;
  return dim3((g.columns + 31) / 32, (segments + 7) / 8, 1);
}

template <bool TGV, int C, bool COUPLED>
cudaError_t dual_keep(const DualParams& p, bool keep, cudaStream_t s) {
  if (keep) {
    dual_stream_kernel<TGV, C, COUPLED, true><<<sweep_grid(p.g), dim3(32, 8), 0, s>>>(p);
  } else {
    dual_stream_kernel<TGV, C, COUPLED, false><<<sweep_grid(p.g), dim3(32, 8), 0, s>>>(p);
  }
  return cudaGetLastError();
}

template <bool TGV>
cudaError_t dual_channels(const DualParams& p, bool coupled, bool keep, cudaStream_t s) {
  switch (p.g.channels) {
    case 1: return dual_keep<TGV, 1, false>(p, keep, s);
    case 2: return coupled ? dual_keep<TGV, 2, true>(p, keep, s) : dual_keep<TGV, 2, false>(p, keep, s);
    case 3: return coupled ? dual_keep<TGV, 3, true>(p, keep, s) : dual_keep<TGV, 3, false>(p, keep, s);
    default: return cudaErrorInvalidValue;
  }
}

dim3 norms_grid(const Geometry& g) { return pixel_grid(g); }

template <bool TGV>
cudaError_t norms_channels(const NormParams& p, bool coupled, cudaStream_t s) {
  const dim3 grid = norms_grid(p.g);
  switch (p.g.channels) {
    case 1: norms_kernel<TGV, 1, false><<<grid, dim3(32, 8), 0, s>>>(p); break;
    case 2:
      if (coupled) norms_kernel<TGV, 2, true><<<grid, dim3(32, 8), 0, s>>>(p);
      else norms_kernel<TGV, 2, false><<<grid, dim3(32, 8), 0, s>>>(p);
      break;
    case 3:
      if (coupled) norms_kernel<TGV, 3, true><<<grid, dim3(32, 8), 0, s>>>(p);
      else norms_kernel<TGV, 3, false><<<grid, dim3(32, 8), 0, s>>>(p);
      break;
    default: return cudaErrorInvalidValue;
  }
  return cudaGetLastError();
}

}  // namespace

int dual_grid_blocks(const Geometry& g) {
  const dim3 d = pixel_grid(g);
  return static_cast<int>(d.x * d.y);
}
int norms_grid_blocks(const Geometry& g) {
  const dim3 d = norms_grid(g);
  return static_cast<int>(d.x * d.y);
}
int residual_grid_blocks(const Geometry& g) { return dual_grid_blocks(g); }
int primal_grid_blocks(const Geometry& g, const ComponentDevice& c) {
  const dim3 d = primal_grid(g, c.cell_rows, c.cell_columns);
  return static_cast<int>(d.x * d.y);
}
// The conjugate kernel's CTAs (one per block_grid cell: 4 block columns by kWarps block rows),
// each of which writes one partial sum.
int conjugate_grid_blocks(const Geometry& g, const ComponentDevice& c) {
  const dim3 d = block_grid(g, c);
  return static_cast<int>(d.x * d.y);
}
int start_grid_blocks(const ComponentDevice& c) { return (c.block_rows * c.block_columns * 8 + 255) / 256; }

cudaError_t launch_dual(const DualParams& p, bool tgv, bool coupled, bool keep, cudaStream_t stream) {
  return tgv ? dual_channels<true>(p, coupled, keep, stream) : dual_channels<false>(p, coupled, keep, stream);
}

namespace {

// A component's items: strips of 32 columns times stages of 64 rows.
int primal_tma_items_of(const Geometry& g, int cr) {
  const int nb = kStageRows / (8 * cr);
  const int vbr = g.rows / (8 * cr);
  return (g.columns + 31) / 32 * ((vbr + nb - 1) / nb);
}

template <int CR, int CC, bool KEEP>
cudaError_t primal_tma_one(const CUtensorMap* maps, const PrimalParams* parts, int count, cudaStream_t s,
                           int* grid) {
  auto kernel = primal_tma_kernel<CR, CC, KEEP>;
  constexpr int threads = 32 * (primal_warps<CR>() + 1);  // the compute warps and the loader
  constexpr std::size_t bytes = primal_shared_bytes<CR, CC>();
  // Once per device: the shared-memory size above 48 KB, and how many CTAs the device holds.
  static std::atomic<int> resident[64] = {};
  int device = 0;
  cudaGetDevice(&device);
  int slots = resident[device & 63].load();
  if (slots == 0) {
    cudaError_t e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(bytes));
    int per_sm = 0, sms = 0;
    if (e == cudaSuccess) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, threads, bytes);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    if (e != cudaSuccess) return e;
    slots = std::max(1, per_sm * sms);
    resident[device & 63].store(slots);
  }
  PrimalBatch batch;
  batch.count = count;
  for (int z = 0; z < count; ++z) batch.part[z] = parts[z];
  batch.strips = (parts[0].g.columns + 31) / 32;
  batch.stages = primal_tma_items_of(parts[0].g, CR) / batch.strips;
  batch.items = count * batch.strips * batch.stages;
  *grid = std::min(batch.items, slots);
  if (*grid <= 0) return cudaSuccess;  // no block row
  kernel<<<*grid, threads, bytes, s>>>(maps[0], maps[count > 1 ? 1 : 0], batch);
  return cudaGetLastError();
}

template <int CR, int CC>
cudaError_t primal_tma_keep(const CUtensorMap* maps, const PrimalParams* parts, int count, bool keep, cudaStream_t s,
                            int* grid) {
  return keep ? primal_tma_one<CR, CC, true>(maps, parts, count, s, grid)
              : primal_tma_one<CR, CC, false>(maps, parts, count, s, grid);
}

template <int CR, int CC>
cudaError_t primal_batch_one(const PrimalItem* list, int count, const PrimalBatchComponent* components, int parity,
                             cudaStream_t s) {
  auto kernel = primal_batch_kernel<CR, CC>;
  constexpr int threads = 32 * (primal_warps<CR>() + 1);  // the compute warps and the loader
  constexpr std::size_t bytes = primal_shared_bytes<CR, CC>();
  static std::atomic<int> resident[64] = {};
  int device = 0;
  cudaGetDevice(&device);
  int slots = resident[device & 63].load();
  if (slots == 0) {
    cudaError_t e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(bytes));
    int per_sm = 0, sms = 0;
    if (e == cudaSuccess) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, threads, bytes);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    if (e != cudaSuccess) return e;
    slots = std::max(1, per_sm * sms);
    resident[device & 63].store(slots);
  }
  if (count <= 0) return cudaSuccess;
  kernel<<<std::min(count, slots), threads, bytes, s>>>(list, count, components, parity);
  return cudaGetLastError();
}

}  // namespace

cudaError_t launch_primal_batch(const PrimalItem* list, int count, const PrimalBatchComponent* components, int parity,
                                int cell_rows, int cell_columns, cudaStream_t stream) {
#define URB_BATCH_CELL(R, C) \
  if (cell_rows == R && cell_columns == C) return primal_batch_one<R, C>(list, count, components, parity, stream);
  URB_BATCH_CELL(1, 1) URB_BATCH_CELL(1, 2) URB_BATCH_CELL(2, 1) URB_BATCH_CELL(2, 2) URB_BATCH_CELL(1, 4)
  URB_BATCH_CELL(4, 1) URB_BATCH_CELL(2, 4) URB_BATCH_CELL(4, 2) URB_BATCH_CELL(4, 4)
#undef URB_BATCH_CELL
  return cudaErrorInvalidValue;
}

int primal_batch_stages(const Geometry& g, int cell_rows) {
  const int nb = kStageRows / (8 * cell_rows);
  const int vbr = g.rows / (8 * cell_rows);
  return (vbr + nb - 1) / nb;
}

bool primal_tma_takes(const ComponentDevice& c) {
  auto fits = [](int n) { return n == 1 || n == 2 || n == 4; };
  return fits(c.cell_rows) && fits(c.cell_columns);
}

int primal_tma_grid_blocks(const Geometry& g, const ComponentDevice& c) {
  // At most one CTA an item of either component of a launch.
  return 2 * primal_tma_items_of(g, c.cell_rows);
}

cudaError_t launch_primal_tma(const CUtensorMap* maps, const PrimalParams* parts, int count, bool keep,
                              cudaStream_t stream, int* grid) {
  if (count < 1 || count > 2) return cudaErrorInvalidValue;
  const int cr = parts[0].component.cell_rows, cc = parts[0].component.cell_columns;
#define URB_TMA_CELL(R, C) \
  if (cr == R && cc == C) return primal_tma_keep<R, C>(maps, parts, count, keep, stream, grid);
  URB_TMA_CELL(1, 1) URB_TMA_CELL(1, 2) URB_TMA_CELL(2, 1) URB_TMA_CELL(2, 2) URB_TMA_CELL(1, 4) URB_TMA_CELL(4, 1)
  URB_TMA_CELL(2, 4) URB_TMA_CELL(4, 2) URB_TMA_CELL(4, 4)
#undef URB_TMA_CELL
  return cudaErrorInvalidValue;
}

cudaError_t launch_primal(const PrimalParams& p, bool keep, cudaStream_t stream) {
  return by_cells<PrimalLaunch>(p.component.cell_rows, p.component.cell_columns, p, keep, stream);
}

cudaError_t launch_start_coefficients(const StartParams& p, cudaStream_t stream) {
  const int blocks = start_grid_blocks(p.component);
  if (blocks == 0) return cudaSuccess;
  start_kernel<<<blocks, 256, 0, stream>>>(p);
  return cudaGetLastError();
}

cudaError_t launch_restore(const ComponentDevice& c, double* out, cudaStream_t stream) {
  const std::size_t count = static_cast<std::size_t>(c.block_rows) * c.block_columns * 64;
  if (count == 0) return cudaSuccess;
  restore_kernel<<<static_cast<unsigned>((count + 255) / 256), 256, 0, stream>>>(c, out);
  return cudaGetLastError();
}

cudaError_t launch_canvas(const CanvasParams& p, cudaStream_t stream) {
  return by_cells<CanvasLaunch>(p.component.cell_rows, p.component.cell_columns, p, stream);
}

cudaError_t launch_picture(const PictureParams& p, cudaStream_t stream) {
  const std::size_t pixels = static_cast<std::size_t>(p.height) * p.width;
  if (pixels == 0 || (p.picture == nullptr && p.planes == nullptr)) return cudaSuccess;
  picture_kernel<<<static_cast<unsigned>((pixels + 255) / 256), 256, 0, stream>>>(p);
  return cudaGetLastError();
}

cudaError_t launch_gradient(const float* x, float* w1, float* w2, const Geometry& g, cudaStream_t stream) {
  gradient_kernel<<<pixel_grid(g), dim3(32, 8), 0, stream>>>(x, w1, w2, g);
  return cudaGetLastError();
}

cudaError_t launch_project(Fields f, const Geometry& g, bool tgv, bool coupled, float radius, float radius0,
                           cudaStream_t stream) {
  project_kernel<<<pixel_grid(g), dim3(32, 8), 0, stream>>>(f, g, tgv ? 1 : 0, coupled ? 1 : 0, radius, radius0);
  return cudaGetLastError();
}

cudaError_t launch_norms(const NormParams& p, bool tgv, bool coupled, cudaStream_t stream) {
  return tgv ? norms_channels<true>(p, coupled, stream) : norms_channels<false>(p, coupled, stream);
}

cudaError_t launch_conjugate(const ConjugateParams& p, cudaStream_t stream) {
  return by_cells<ConjugateLaunch>(p.component.cell_rows, p.component.cell_columns, p, stream);
}

cudaError_t launch_reductions(const Reductions& r, cudaStream_t stream) {
  if (r.n == 0) return cudaSuccess;
  reduce_kernel<<<r.n, 1024, 0, stream>>>(r);
  return cudaGetLastError();
}

cudaError_t launch_residual(const ResidualParams& p, cudaStream_t stream) {
  residual_kernel<<<pixel_grid(p.g), dim3(32, 8), 0, stream>>>(p);
  return cudaGetLastError();
}

cudaError_t launch_narrow(const double* from, float* to, const Geometry& g, cudaStream_t stream) {
  narrow_kernel<<<1184, 256, 0, stream>>>(from, to, g);
  return cudaGetLastError();
}

}  // namespace urb
