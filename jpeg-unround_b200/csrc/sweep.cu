// The dual step of an iteration as a TMA-fed sweep (sm_100a).
//
// A CTA owns a strip of 32 canvas columns (64 with one channel: a lane takes two columns, 32
// apart) and walks down strip_rows rows of it in chunks of 8 rows, one row per warp. Each chunk
// of every field of every channel -- the state s_{n-1} (x, p, and for TGV w and r) and the
// carried canvas x~ -- comes into shared memory by two cp.async.bulk.tensor loads of a 3D box
// (the strip and 4 columns on each side, 8 rows, every plane) into a ring of three slots, so that
// the loads of chunks k + 2 and k + 3 run while chunk k is computed; each value of HBM is read
// once (the 8 columns beside the strip come from L2). The strip height is chosen per launch so that the CTAs fill the device's SMs in whole
// waves as nearly as possible.
//
// w~ = w + tau (p + div2 r) is evaluated once per pixel: a chunk's row warps make x_n, w~, w-
// and p_n at their pixels and leave w- in shared memory; after a barrier each pixel's r step
// takes w- of its left neighbour by a shuffle (of the strip's first column, from a ninth, side
// warp that makes w- at column x0 - 1) and of its upper neighbour from shared memory (of the
// chunk's first row, kept from the chunk before). The arithmetic of each value is the dual step
// of docs/math.md 5, operation for operation as cpp/src/primal_dual.hpp:572-735 orders it (see
// kernels.cu).
//
// The waits on the ring's mbarriers are bounded: a wait that runs out sets the error word,
// and the CTA leaves without computing further (the host reports an internal error).
#include <algorithm>
#include <atomic>

#include <cuda.h>
#include <cudaTypedefs.h>

#include "kernels.hpp"
#include "tma.cuh"

namespace urb {

namespace {

constexpr int kChunk = 8;    // rows of a chunk, one per warp
constexpr int kHalo = 4;     // columns loaded left of the strip (16-byte aligned start)
constexpr int kSlots = 3;    // the ring
constexpr int kStrip = 256;  // rows a CTA sweeps unless the launcher finds better
constexpr int kThreads = 32 * (kChunk + 1);  // the row warps and the side warp
constexpr unsigned kAll = 0xffffffffu;

// CTAs an SM holds: two of the colour sweeps (shared memory), three of the one-channel sweep's
// wider strips (registers, at most 75 a thread).
constexpr int resident_ctas(int channels) { return channels == 1 ? 3 : 2; }

template <typename T>
__device__ __forceinline__ T ball(T square, T radius) {
  const T norm = sqrt(square);
  return norm > radius ? radius / norm : T(1);
}

// One CTA's strip: columns x0 .. x0 + 32 L - 1 (L = lane_columns(C): a lane takes columns
// x0 + lane and, with one channel, x0 + 32 + lane too), rows i0 .. i1 - 1 (a whole number of
// chunks, or the canvas's last rows), of the image whose maps and parameters these are.
template <bool TGV, int C, bool COUPLED, bool KEEP, bool SAMPLES = false>
__device__ __forceinline__ void dual_strip(const CUtensorMap* state_map, const CUtensorMap* tilde_map,
                                           const DualParams& P, int x0, int i0, int i1,
                                           const SamplesStep* Q = nullptr) {
  constexpr int F = TGV ? 8 : 3;  // state planes per channel: x, p1, p2 (+ w1, w2, r11, r22, r12)
  constexpr int L = lane_columns(C);
  constexpr int WIDTH = 32 * L;                // the strip's columns
  constexpr int SPAN = WIDTH + 2 * kHalo;      // columns of a box
  constexpr int PLANE = kChunk * SPAN;
  constexpr int SLOT = (F + 1) * C * PLANE;  // floats: the state planes, then x~'s
  constexpr int W = TGV ? C : 1;
  extern __shared__ __align__(128) float ring[];
  __shared__ __align__(8) std::uint64_t bars[kSlots];
  __shared__ float carry[2][W][2][WIDTH];      // w- of the row above a chunk, own columns
  __shared__ float wbar[W][2][kChunk][WIDTH];  // w- of each row of the chunk
  __shared__ float wleft[W][2][kChunk];        // w- at column x0 - 1
  // With SAMPLES: p2_n of each row of the chunk, of the row above it, and p1_n at column x0 - 1.
  constexpr int PS = SAMPLES ? C : 1;
  __shared__ float p2rows[PS][kChunk][WIDTH];
  __shared__ float p2carry[2][PS][WIDTH];
  __shared__ float pleft[PS][kChunk];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int rows = P.g.rows, columns = P.g.columns, pitch = P.g.pitch;
  const std::size_t plane = P.g.plane;
  const int chunks = (i1 - i0 + kChunk - 1) / kChunk;
  // The lane's columns: h = 0 .. L - 1 at x0 + 32 h + lane, column own[h] of the box.
  int jc[L], own[L];
  bool valid[L], has_left[L], has_right[L];
#pragma unroll
  for (int h = 0; h < L; ++h) {
    const int j = x0 + 32 * h + lane;
    valid[h] = j < columns;
    jc[h] = valid[h] ? j : columns - 1;
    has_left[h] = j > 0;
    has_right[h] = j + 1 < columns;
    own[h] = kHalo + 32 * h + lane;
  }
  const float rho = P.rho, rest = P.rest;

  if (threadIdx.x == 0) {
    for (int s = 0; s < kSlots; ++s) barrier_init(&bars[s], 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
  auto issue = [&](int k) {
    if (threadIdx.x == 0 && k <= chunks) {
      const int slot = k % kSlots;
      float* to = ring + slot * SLOT;
      barrier_expect(&bars[slot], SLOT * 4);
      load_box(to, state_map, &bars[slot], x0 - kHalo, i0 + k * kChunk, 0);
      load_box(to + F * C * PLANE, tilde_map, &bars[slot], x0 - kHalo, i0 + k * kChunk, 0);
    }
  };
  for (int k = 0; k < kSlots; ++k) issue(k);

  // w- of the row above the strip (own columns), from global memory.
  if (TGV && warp == 0) {
#pragma unroll
    for (int h = 0; h < L; ++h) {
#pragma unroll
      for (int c = 0; c < C; ++c) {
        float wb1 = 0.0f, wb2 = 0.0f;
        if (i0 > 0) {
          const std::size_t base = c * plane;
          const int u = i0 - 1;
          const std::size_t a = static_cast<std::size_t>(u) * pitch + jc[h];
          const float a11 = __ldg(P.in.r11 + base + a), a12 = __ldg(P.in.r12 + base + a);
          const float a22 = __ldg(P.in.r22 + base + a);
          float d1 = has_right[h] ? __ldg(P.in.r11 + base + a + 1) - a11 : 0.0f;
          float d2 = has_right[h] ? __ldg(P.in.r12 + base + a + 1) - a12 : 0.0f;
          d1 = d1 + (__ldg(P.in.r12 + base + a + pitch) - a12);
          d2 = d2 + (__ldg(P.in.r22 + base + a + pitch) - a22);
          const float w1 = __ldg(P.in.w1 + base + a), w2 = __ldg(P.in.w2 + base + a);
          const float t1 = w1 + P.tau[c] * (__ldg(P.in.p1 + base + a) + d1);
          const float t2 = w2 + P.tau[c] * (__ldg(P.in.p2 + base + a) + d2);
          wb1 = 2.0f * t1 - w1;
          wb2 = 2.0f * t2 - w2;
        }
        carry[0][c][0][32 * h + lane] = wb1;
        carry[0][c][1][32 * h + lane] = wb2;
      }
    }
  }
  if (SAMPLES && warp == 0) {
    // p2_n of the row above the strip: the dual step at (i0 - 1, j), from global memory.
#pragma unroll
    for (int h = 0; h < L; ++h) {
      float step1[C], step2[C], old2[C];
      float square = 0.0f;
#pragma unroll
      for (int c = 0; c < C; ++c) {
        step1[c] = step2[c] = old2[c] = 0.0f;
        if (i0 > 0) {
          const std::size_t base = c * plane;
          const std::size_t a = static_cast<std::size_t>(i0 - 1) * pitch + jc[h];
          auto bar_at = [&](std::size_t at) { return 2.0f * __ldg(P.xt + base + at) - __ldg(P.in.x + base + at); };
          const float bar = bar_at(a);
          const float gx = has_right[h] ? bar_at(a + 1) - bar : 0.0f;
          const float gy = bar_at(a + pitch) - bar;
          const float p1 = __ldg(P.in.p1 + base + a), p2 = __ldg(P.in.p2 + base + a);
          float wb1 = 0.0f, wb2 = 0.0f;
          if constexpr (TGV) {
            wb1 = carry[0][c][0][32 * h + lane];  // written above by this warp
            wb2 = carry[0][c][1][32 * h + lane];
          }
          step1[c] = p1 + P.sigma[c] * (gx - wb1);
          step2[c] = p2 + P.sigma[c] * (gy - wb2);
          old2[c] = p2;
          if constexpr (COUPLED) square += step1[c] * step1[c] + step2[c] * step2[c];
        }
      }
      const float coupled_scale = COUPLED ? ball(square, P.radius) : 1.0f;
#pragma unroll
      for (int c = 0; c < C; ++c) {
        float sp = coupled_scale;
        if constexpr (!COUPLED) sp = ball(step1[c] * step1[c] + step2[c] * step2[c], P.radius);
        p2carry[0][c][32 * h + lane] = i0 > 0 ? rho * (step2[c] * sp) + rest * old2[c] : 0.0f;
      }
    }
  }
  __syncthreads();

  // With SAMPLES: the levels of the first chunk's pixels (then each chunk loads the next's).
  unsigned level[L][SAMPLES ? C : 1] = {};
  if constexpr (SAMPLES) {
    const int first = i0 + warp;
#pragma unroll
    for (int h = 0; h < L; ++h) {
      if (warp < kChunk && first < i1 && valid[h]) {
#pragma unroll
        for (int c = 0; c < C; ++c) {
          level[h][c] = __ldg(Q->levels + c * plane + static_cast<std::size_t>(first) * pitch + jc[h]);
        }
      }
    }
  }
  bool failed = false;
  int stopped = chunks;
  for (int k = 0; k < chunks; ++k) {
    const bool ready = barrier_wait(&bars[k % kSlots], (k / kSlots) & 1, P.ring_wait_limit) &&
                       barrier_wait(&bars[(k + 1) % kSlots], ((k + 1) / kSlots) & 1, P.ring_wait_limit);
    if (__syncthreads_or(!ready)) {
      failed = true;
      stopped = k;
      break;
    }
    const float* slot = ring + (k % kSlots) * SLOT;
    const float* next = ring + ((k + 1) % kSlots) * SLOT;
    // A field's value in shared memory: plane (field, channel), row r of the chunk (8: the next
    // chunk's first row), column col of the box.
    auto S = [&](int field, int c, int r, int col) -> float {
      const float* s = r < kChunk ? slot : next;
      return s[((field * C + c) * kChunk + (r < kChunk ? r : 0)) * SPAN + col];
    };
    auto XT = [&](int c, int r, int col) -> float {
      const float* s = r < kChunk ? slot : next;
      return s[((F * C + c) * kChunk + (r < kChunk ? r : 0)) * SPAN + col];
    };
    // w~ at (row rr of the chunk, column col of the box): w + tau g (p + div2 r), div2 r by
    // forward differences; (ii, jj) the pixel on the canvas.
    auto w_tilde = [&](int c, int rr, int col, int ii, int jj, float& t1, float& t2, float& w1, float& w2) {
      const float tau = P.tau[c];
      const float r11 = S(5, c, rr, col), r22 = S(6, c, rr, col), r12 = S(7, c, rr, col);
      float d1 = jj + 1 < columns ? S(5, c, rr, col + 1) - r11 : 0.0f;
      float d2 = jj + 1 < columns ? S(7, c, rr, col + 1) - r12 : 0.0f;
      d1 = d1 + (ii + 1 < rows ? S(7, c, rr + 1, col) - r12 : 0.0f);
      d2 = d2 + (ii + 1 < rows ? S(6, c, rr + 1, col) - r22 : 0.0f);
      w1 = S(3, c, rr, col);
      w2 = S(4, c, rr, col);
      t1 = w1 + tau * (S(1, c, rr, col) + d1);
      t2 = w2 + tau * (S(2, c, rr, col) + d2);
    };
    const int r = warp;
    const int i = i0 + k * kChunk + r;
    const bool row = warp < kChunk && i < i1;
    std::size_t here[L];
#pragma unroll
    for (int h = 0; h < L; ++h) here[h] = static_cast<std::size_t>(row ? i : 0) * pitch + jc[h];
    float wb1[L][C], wb2[L][C];
    float xn[L][C], pn1[L][C], pn2[L][C];  // with SAMPLES: x_n and p_n at the pixel
    // With SAMPLES: the pixel's ends (by the level loaded a chunk ago), looked up now so that the
    // dual step hides the lookup, and the level of the pixel a chunk below, for the next chunk.
    float4 ends[L][SAMPLES ? C : 1];
    if constexpr (SAMPLES) {
      const int below = i + kChunk;
#pragma unroll
      for (int h = 0; h < L; ++h) {
        const bool ahead = warp < kChunk && below < i1 && valid[h];
        const std::size_t there = static_cast<std::size_t>(ahead ? below : 0) * pitch + jc[h];
#pragma unroll
        for (int c = 0; c < C; ++c) {
          ends[h][c] = __ldg(reinterpret_cast<const float4*>(Q->ends) + level[h][c]);  // a, b, centre
          level[h][c] = ahead ? __ldg(Q->levels + c * plane + there) : 0u;
        }
      }
    }
    // ---- The row warps: x, w and p at the pixel; w- left in shared memory.
    if (row) {
      const bool has_down = i + 1 < rows;
#pragma unroll
      for (int h = 0; h < L; ++h) {
        float step_p1[C], step_p2[C], old_p1[C], old_p2[C];
        float square_p = 0.0f;
        const int o = own[h];
#pragma unroll
        for (int c = 0; c < C; ++c) {
          const std::size_t base = c * plane;
          const float xt0 = XT(c, r, o), x0v = S(0, c, r, o);
          const float bar = 2.0f * xt0 - x0v;
          const float gx = has_right[h] ? (2.0f * XT(c, r, o + 1) - S(0, c, r, o + 1)) - bar : 0.0f;
          const float gy = has_down ? (2.0f * XT(c, r + 1, o) - S(0, c, r + 1, o)) - bar : 0.0f;
          if constexpr (SAMPLES) xn[h][c] = rho * xt0 + rest * x0v;
          if (valid[h]) P.out.x[base + here[h]] = rho * xt0 + rest * x0v;
          const float p1 = S(1, c, r, o), p2 = S(2, c, r, o);
          old_p1[c] = p1;
          old_p2[c] = p2;
          const float sigma = P.sigma[c];
          if constexpr (!TGV) {
            wb1[h][c] = wb2[h][c] = 0.0f;
            step_p1[c] = p1 + sigma * gx;
            step_p2[c] = p2 + sigma * gy;
          } else {
            float t1, t2, w1, w2;
            w_tilde(c, r, o, i, x0 + 32 * h + lane, t1, t2, w1, w2);
            wb1[h][c] = 2.0f * t1 - w1;
            wb2[h][c] = 2.0f * t2 - w2;
            if (valid[h]) {
              P.out.w1[base + here[h]] = rho * t1 + rest * w1;
              P.out.w2[base + here[h]] = rho * t2 + rest * w2;
              if constexpr (KEEP) {
                P.tilde.w1[base + here[h]] = t1;
                P.tilde.w2[base + here[h]] = t2;
              }
            }
            wbar[c][0][r][32 * h + lane] = wb1[h][c];
            wbar[c][1][r][32 * h + lane] = wb2[h][c];
            if (r == kChunk - 1) {
              carry[(k + 1) & 1][c][0][32 * h + lane] = wb1[h][c];
              carry[(k + 1) & 1][c][1][32 * h + lane] = wb2[h][c];
            }
            step_p1[c] = p1 + sigma * (gx - wb1[h][c]);
            step_p2[c] = p2 + sigma * (gy - wb2[h][c]);
          }
          if constexpr (COUPLED) square_p += step_p1[c] * step_p1[c] + step_p2[c] * step_p2[c];
        }
        float scale_p = 1.0f;
        if constexpr (COUPLED) scale_p = ball(square_p, P.radius);
        if constexpr (SAMPLES) {
          // p_n at every lane (the divergence of the primal step reads the neighbours'), kept.
#pragma unroll
          for (int c = 0; c < C; ++c) {
            const std::size_t base = c * plane;
            float sp = scale_p;
            if constexpr (!COUPLED) sp = ball(step_p1[c] * step_p1[c] + step_p2[c] * step_p2[c], P.radius);
            pn1[h][c] = rho * (step_p1[c] * sp) + rest * old_p1[c];
            pn2[h][c] = rho * (step_p2[c] * sp) + rest * old_p2[c];
            if (valid[h]) {
              P.out.p1[base + here[h]] = pn1[h][c];
              P.out.p2[base + here[h]] = pn2[h][c];
            }
            p2rows[c][r][32 * h + lane] = pn2[h][c];
            if (r == kChunk - 1) p2carry[(k + 1) & 1][c][32 * h + lane] = pn2[h][c];
          }
        } else if (valid[h]) {
#pragma unroll
          for (int c = 0; c < C; ++c) {
            const std::size_t base = c * plane;
            float sp = scale_p;
            if constexpr (!COUPLED) sp = ball(step_p1[c] * step_p1[c] + step_p2[c] * step_p2[c], P.radius);
            const float q1 = step_p1[c] * sp, q2 = step_p2[c] * sp;
            P.out.p1[base + here[h]] = rho * q1 + rest * old_p1[c];
            P.out.p2[base + here[h]] = rho * q2 + rest * old_p2[c];
            if (KEEP && P.tilde.p1 != nullptr) {  // p~: TV's records and the partial gap's
              P.tilde.p1[base + here[h]] = q1;
              P.tilde.p2[base + here[h]] = q2;
            }
          }
        }
      }
    } else if ((TGV || SAMPLES) && warp == kChunk && lane < kChunk && x0 > 0 && i0 + k * kChunk + lane < i1) {
      // ---- The side warp: w- at column x0 - 1 of the chunk's rows (a lane each); with SAMPLES
      // p1_n there too (the divergence's left neighbour of the strip's first column).
      const int rr = lane, ii = i0 + k * kChunk + rr;
      float lb1[C], lb2[C];
#pragma unroll
      for (int c = 0; c < C; ++c) {
        lb1[c] = lb2[c] = 0.0f;
        if constexpr (TGV) {
          float t1, t2, w1, w2;
          w_tilde(c, rr, kHalo - 1, ii, x0 - 1, t1, t2, w1, w2);
          lb1[c] = 2.0f * t1 - w1;
          lb2[c] = 2.0f * t2 - w2;
          wleft[c][0][rr] = lb1[c];
          wleft[c][1][rr] = lb2[c];
        }
      }
      if constexpr (SAMPLES) {
        constexpr int B = kHalo - 1;  // column x0 - 1 in the box
        float step1[C], step2[C], old1[C];
        float square = 0.0f;
#pragma unroll
        for (int c = 0; c < C; ++c) {
          const float bar = 2.0f * XT(c, rr, B) - S(0, c, rr, B);
          const float gx = (2.0f * XT(c, rr, B + 1) - S(0, c, rr, B + 1)) - bar;  // x0 < columns
          const float gy = ii + 1 < rows ? (2.0f * XT(c, rr + 1, B) - S(0, c, rr + 1, B)) - bar : 0.0f;
          old1[c] = S(1, c, rr, B);
          step1[c] = old1[c] + P.sigma[c] * (gx - lb1[c]);
          step2[c] = S(2, c, rr, B) + P.sigma[c] * (gy - lb2[c]);
          if constexpr (COUPLED) square += step1[c] * step1[c] + step2[c] * step2[c];
        }
        const float coupled_scale = COUPLED ? ball(square, P.radius) : 1.0f;
#pragma unroll
        for (int c = 0; c < C; ++c) {
          float sp = coupled_scale;
          if constexpr (!COUPLED) sp = ball(step1[c] * step1[c] + step2[c] * step2[c], P.radius);
          pleft[c][rr] = rho * (step1[c] * sp) + rest * old1[c];
        }
      }
    }
    if constexpr (!TGV && SAMPLES) __syncthreads();
    if constexpr (TGV) {
      __syncthreads();
      // ---- The r step from w- of the pixel and of its left and upper neighbours.
      if (row) {
        const bool has_down = i + 1 < rows, has_up = i > 0;
#pragma unroll
        for (int h = 0; h < L; ++h) {
          float step_r11[C], step_r22[C], step_r12[C], old_r11[C], old_r22[C], old_r12[C];
          float square_r = 0.0f;
#pragma unroll
          for (int c = 0; c < C; ++c) {
            // The left neighbour: lane - 1's column of the same half; lane 0's is the side warp's
            // (h = 0) or lane 31's of the half before.
            float wl1 = __shfl_up_sync(kAll, wb1[h][c], 1), wl2 = __shfl_up_sync(kAll, wb2[h][c], 1);
            if (h > 0) {
              const float last1 = __shfl_sync(kAll, wb1[h > 0 ? h - 1 : 0][c], 31);
              const float last2 = __shfl_sync(kAll, wb2[h > 0 ? h - 1 : 0][c], 31);
              if (lane == 0) {
                wl1 = last1;
                wl2 = last2;
              }
            } else if (lane == 0) {
              wl1 = wleft[c][0][r];
              wl2 = wleft[c][1][r];
            }
            if (!has_left[h]) wl1 = wl2 = 0.0f;
            float wu1 = r > 0 ? wbar[c][0][r - 1][32 * h + lane] : carry[k & 1][c][0][32 * h + lane];
            float wu2 = r > 0 ? wbar[c][1][r - 1][32 * h + lane] : carry[k & 1][c][1][32 * h + lane];
            if (!has_up) wu1 = wu2 = 0.0f;
            const float own1x = has_right[h] ? wb1[h][c] : 0.0f, own2x = has_right[h] ? wb2[h][c] : 0.0f;
            const float own1y = has_down ? wb1[h][c] : 0.0f, own2y = has_down ? wb2[h][c] : 0.0f;
            const float exx = own1x - wl1;
            const float eyy = own2y - wu2;
            const float exy = 0.5f * ((own1y - wu1) + (own2x - wl2));
            const float r11 = S(5, c, r, own[h]), r22 = S(6, c, r, own[h]), r12 = S(7, c, r, own[h]);
            old_r11[c] = r11;
            old_r22[c] = r22;
            old_r12[c] = r12;
            const float sigma = P.sigma[c];
            step_r11[c] = r11 + sigma * exx;
            step_r22[c] = r22 + sigma * eyy;
            step_r12[c] = r12 + sigma * exy;
            if constexpr (COUPLED) {
              square_r += step_r11[c] * step_r11[c] + step_r22[c] * step_r22[c] + 2.0f * (step_r12[c] * step_r12[c]);
            }
          }
          float scale_r = 1.0f;
          if constexpr (COUPLED) scale_r = ball(square_r, P.radius0);
          if (valid[h]) {
#pragma unroll
            for (int c = 0; c < C; ++c) {
              const std::size_t base = c * plane;
              float sr = scale_r;
              if constexpr (!COUPLED) {
                sr = ball(step_r11[c] * step_r11[c] + step_r22[c] * step_r22[c] + 2.0f * (step_r12[c] * step_r12[c]),
                          P.radius0);
              }
              const float t11 = step_r11[c] * sr, t22 = step_r22[c] * sr, t12 = step_r12[c] * sr;
              P.out.r11[base + here[h]] = rho * t11 + rest * old_r11[c];
              P.out.r22[base + here[h]] = rho * t22 + rest * old_r22[c];
              P.out.r12[base + here[h]] = rho * t12 + rest * old_r12[c];
              if constexpr (KEEP) {
                P.tilde.r11[base + here[h]] = t11;
                P.tilde.r22[base + here[h]] = t22;
                P.tilde.r12[base + here[h]] = t12;
              }
            }
          }
        }
      }
    }
    if constexpr (SAMPLES) {
      // ---- The primal step of the next iteration at the pixel: v = x_n + tau gamma div p_n
      // (backward differences, Neumann ends) and its proximal map, the box of the sample's level.
      if (row) {
        const bool has_down = i + 1 < rows, has_up = i > 0;
#pragma unroll
        for (int h = 0; h < L; ++h) {
#pragma unroll
          for (int c = 0; c < C; ++c) {
            float before = __shfl_up_sync(kAll, pn1[h][c], 1);
            if (h > 0) {
              const float last = __shfl_sync(kAll, pn1[h > 0 ? h - 1 : 0][c], 31);
              if (lane == 0) before = last;
            } else if (lane == 0) {
              before = x0 > 0 ? pleft[c][r] : 0.0f;
            }
            const float above = r > 0 ? p2rows[c][r - 1][32 * h + lane] : p2carry[k & 1][c][32 * h + lane];
            const float dy = (has_down ? pn2[h][c] : 0.0f) - (has_up ? above : 0.0f);
            const float dx = (has_right[h] ? pn1[h][c] : 0.0f) - (has_left[h] ? before : 0.0f);
            const float v = xn[h][c] + P.tau[c] * (dy + dx);
            if (valid[h]) {
              Q->next[c * plane + here[h]] =
                  fminf(fmaxf((v + Q->t * ends[h][c].z) * Q->r, ends[h][c].x), ends[h][c].y);
            }
          }
        }
      }
    }
    __syncthreads();  // every warp is done with slot k
    issue(k + kSlots);
  }
  if (failed && threadIdx.x == 0 && P.error != nullptr) atomicExch(P.error, 1);
  // No load may still write into shared memory when the CTA leaves: wait (bounded) for every
  // chunk issued and not consumed.
  if (failed) {
    for (int k = stopped; k <= min(stopped + kSlots - 1, chunks); ++k) barrier_wait(&bars[k % kSlots], (k / kSlots) & 1);
  }
}

template <bool TGV, int C, bool COUPLED, bool KEEP>
__global__ void __launch_bounds__(kThreads, resident_ctas(C)) dual_tma_kernel(const __grid_constant__ CUtensorMap state_map,
                                                                const __grid_constant__ CUtensorMap tilde_map,
                                                                const DualParams P) {
  const int i0 = blockIdx.y * P.strip_rows;
  dual_strip<TGV, C, COUPLED, KEEP>(&state_map, &tilde_map, P, blockIdx.x * sweep_width(C), i0,
                                    min(i0 + P.strip_rows, P.g.rows));
}

// The dual step and the next primal step of a picture of rounded samples (SamplesStep).
template <bool TGV, int C, bool COUPLED>
__global__ void __launch_bounds__(kThreads, resident_ctas(C)) dual_samples_kernel(const __grid_constant__ CUtensorMap state_map,
                                                                    const __grid_constant__ CUtensorMap tilde_map,
                                                                    const DualParams P, const SamplesStep Q) {
  const int i0 = blockIdx.y * P.strip_rows;
  dual_strip<TGV, C, COUPLED, false, true>(&state_map, &tilde_map, P, blockIdx.x * sweep_width(C), i0,
                                           min(i0 + P.strip_rows, P.g.rows), &Q);
}

// The dual step of a batch: a CTA a tile of the table, of the image whose entry (maps and
// parameters, in global memory) the tile names; the maps are read through the tensor-map proxy
// after an acquire fence.
template <bool TGV, int C, bool COUPLED>
__global__ void __launch_bounds__(kThreads, resident_ctas(C)) dual_batch_kernel(const DualTile* __restrict__ tiles,
                                                                  const DualBatchImage* images, int parity) {
  __shared__ DualParams P;
  const DualTile tile = tiles[blockIdx.x];
  const DualBatchImage& image = images[tile.image];
  if (threadIdx.x == 0) {
    P = image.params[parity];
    asm volatile("fence.proxy.tensormap::generic.acquire.gpu [%0], 128;" ::"l"(&image.state[parity]) : "memory");
    asm volatile("fence.proxy.tensormap::generic.acquire.gpu [%0], 128;" ::"l"(&image.tilde) : "memory");
  }
  __syncthreads();
  dual_strip<TGV, C, COUPLED, false>(&image.state[parity], &image.tilde, P, tile.x0, tile.i0, tile.i1);
}

}  // namespace

std::size_t dual_tma_shared_bytes(bool tgv, int channels) {
  const int fields = tgv ? 8 : 3;
  const int span = sweep_width(channels) + 2 * kHalo;
  return static_cast<std::size_t>(kSlots) * (fields + 1) * channels * kChunk * span * sizeof(float);
}

// The strip height that finishes a sweep soonest: its CTAs in waves of `slots`, each wave as long
// as a strip and the pipeline's start (about two chunks).
int strip_rows_for(const Geometry& g, int slots, int width) {
  const int strips = (g.columns + width - 1) / width;
  int best = kStrip;
  long long best_cost = -1;
  for (int height = 64; height <= 512; height += 16) {
    const long long ctas = static_cast<long long>(strips) * ((g.rows + height - 1) / height);
    const long long cost = (ctas + slots - 1) / slots * (height + 2 * kChunk);
    if (best_cost < 0 || cost < best_cost) {
      best_cost = cost;
      best = height;
    }
  }
  return best;
}

namespace {

template <bool TGV, int C, bool COUPLED, bool KEEP>
cudaError_t launch_one(const CUtensorMap& state, const CUtensorMap& tilde, const DualParams& p, cudaStream_t s) {
  auto kernel = dual_tma_kernel<TGV, C, COUPLED, KEEP>;
  const std::size_t bytes = dual_tma_shared_bytes(TGV, C);
  // Once per device: the shared-memory size above 48 KB, and how many CTAs the device holds at
  // once (its SMs times the CTAs an SM holds).
  static std::atomic<int> resident[64] = {};
  int device = 0;
  cudaGetDevice(&device);
  int slots = resident[device & 63].load();
  if (slots == 0) {
    cudaError_t e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(bytes));
    int per_sm = 0, sms = 0;
    if (e == cudaSuccess) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, kThreads, bytes);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    if (e != cudaSuccess) return e;
    slots = std::max(1, per_sm * sms);
    resident[device & 63].store(slots);
  }
  DualParams q = p;
  q.strip_rows = strip_rows_for(p.g, slots, sweep_width(C));
  const dim3 grid((p.g.columns + sweep_width(C) - 1) / sweep_width(C), (p.g.rows + q.strip_rows - 1) / q.strip_rows, 1);
  kernel<<<grid, kThreads, bytes, s>>>(state, tilde, q);
  return cudaGetLastError();
}

template <bool TGV, int C, bool COUPLED>
cudaError_t launch_keep(const CUtensorMap& state, const CUtensorMap& tilde, const DualParams& p, bool keep,
                        cudaStream_t s) {
  return keep ? launch_one<TGV, C, COUPLED, true>(state, tilde, p, s)
              : launch_one<TGV, C, COUPLED, false>(state, tilde, p, s);
}

template <bool TGV>
cudaError_t launch_channels(const CUtensorMap& state, const CUtensorMap& tilde, const DualParams& p, bool coupled,
                            bool keep, cudaStream_t s) {
  switch (p.g.channels) {
    case 1: return launch_keep<TGV, 1, false>(state, tilde, p, keep, s);
    case 2: return coupled ? launch_keep<TGV, 2, true>(state, tilde, p, keep, s)
                           : launch_keep<TGV, 2, false>(state, tilde, p, keep, s);
    case 3: return coupled ? launch_keep<TGV, 3, true>(state, tilde, p, keep, s)
                           : launch_keep<TGV, 3, false>(state, tilde, p, keep, s);
    default: return cudaErrorInvalidValue;
  }
}

PFN_cuTensorMapEncodeTiled_v12000 encoder() {
  static PFN_cuTensorMapEncodeTiled_v12000 function = [] {
    void* found = nullptr;
    cudaDriverEntryPointQueryResult status;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &found, cudaEnableDefault, &status) != cudaSuccess ||
        status != cudaDriverEntryPointSuccess) {
      return static_cast<PFN_cuTensorMapEncodeTiled_v12000>(nullptr);
    }
    return reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(found);
  }();
  return function;
}

}  // namespace

// A 3D tiled map of `count` float planes `stride` floats apart, each the canvas's rows x columns
// (rows `pitch` apart), boxes of `box_columns` columns x `box_rows` rows x every plane.
bool make_box_map(CUtensorMap& map, const float* planes, const Geometry& g, int count, std::size_t stride,
                  unsigned box_rows, unsigned box_columns) {
  PFN_cuTensorMapEncodeTiled_v12000 encode = encoder();
  if (encode == nullptr) return false;
  const cuuint64_t dims[3] = {static_cast<cuuint64_t>(g.columns), static_cast<cuuint64_t>(g.rows),
                              static_cast<cuuint64_t>(count)};
  const cuuint64_t strides[2] = {static_cast<cuuint64_t>(g.pitch) * sizeof(float), stride * sizeof(float)};
  const cuuint32_t box[3] = {box_columns, box_rows, static_cast<cuuint32_t>(count)};
  const cuuint32_t steps[3] = {1, 1, 1};
  const CUresult result = encode(&map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, const_cast<float*>(planes), dims, strides,
                                 box, steps, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                                 CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return result == CUDA_SUCCESS;
}

bool make_fields_map(CUtensorMap& map, const float* base, int columns, int rows, int images, int fields,
                     std::size_t plane, unsigned box_columns, unsigned box_rows) {
  PFN_cuTensorMapEncodeTiled_v12000 encode = encoder();
  if (encode == nullptr) return false;
  const cuuint64_t dims[4] = {static_cast<cuuint64_t>(columns), static_cast<cuuint64_t>(rows),
                              static_cast<cuuint64_t>(images), static_cast<cuuint64_t>(fields)};
  const cuuint64_t strides[3] = {static_cast<cuuint64_t>(columns) * sizeof(float),
                                 static_cast<cuuint64_t>(rows) * columns * sizeof(float), plane * sizeof(float)};
  const cuuint32_t box[4] = {box_columns, box_rows, 1, static_cast<cuuint32_t>(fields)};
  const cuuint32_t steps[4] = {1, 1, 1, 1};
  const CUresult result = encode(&map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4, const_cast<float*>(base), dims, strides,
                                 box, steps, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                                 CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return result == CUDA_SUCCESS;
}

bool make_sweep_map(CUtensorMap& map, const float* planes, const Geometry& g, int count) {
  return make_box_map(map, planes, g, count, g.plane, kChunk, sweep_width(g.channels) + 2 * kHalo);
}

bool make_primal_map(CUtensorMap& map, const float* x, const Geometry& g, std::size_t stride) {
  return make_box_map(map, x, g, 3, stride, 65, 36);
}

namespace {

template <bool TGV, int C, bool COUPLED>
cudaError_t launch_samples_one(const CUtensorMap& state, const CUtensorMap& tilde, const DualParams& p,
                               const SamplesStep& q, cudaStream_t s) {
  auto kernel = dual_samples_kernel<TGV, C, COUPLED>;
  const std::size_t bytes = dual_tma_shared_bytes(TGV, C);
  static std::atomic<int> resident[64] = {};
  int device = 0;
  cudaGetDevice(&device);
  int slots = resident[device & 63].load();
  if (slots == 0) {
    cudaError_t e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(bytes));
    int per_sm = 0, sms = 0;
    if (e == cudaSuccess) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, kThreads, bytes);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    if (e != cudaSuccess) return e;
    slots = std::max(1, per_sm * sms);
    resident[device & 63].store(slots);
  }
  DualParams d = p;
  d.strip_rows = strip_rows_for(p.g, slots, sweep_width(C));
  const dim3 grid((p.g.columns + sweep_width(C) - 1) / sweep_width(C), (p.g.rows + d.strip_rows - 1) / d.strip_rows, 1);
  kernel<<<grid, kThreads, bytes, s>>>(state, tilde, d, q);
  return cudaGetLastError();
}

}  // namespace

cudaError_t launch_dual_samples(const CUtensorMap& state, const CUtensorMap& tilde, const DualParams& p,
                                const SamplesStep& q, bool tgv, bool coupled, cudaStream_t stream) {
  switch (p.g.channels) {
    case 1:
      return tgv ? launch_samples_one<true, 1, false>(state, tilde, p, q, stream)
                 : launch_samples_one<false, 1, false>(state, tilde, p, q, stream);
    case 3:
      if (tgv) {
        return coupled ? launch_samples_one<true, 3, true>(state, tilde, p, q, stream)
                       : launch_samples_one<true, 3, false>(state, tilde, p, q, stream);
      }
      return coupled ? launch_samples_one<false, 3, true>(state, tilde, p, q, stream)
                     : launch_samples_one<false, 3, false>(state, tilde, p, q, stream);
    default:
      return cudaErrorInvalidValue;
  }
}

cudaError_t launch_dual_tma(const CUtensorMap& state, const CUtensorMap& tilde, const DualParams& p, bool tgv,
                            bool coupled, bool keep, cudaStream_t stream) {
  return tgv ? launch_channels<true>(state, tilde, p, coupled, keep, stream)
             : launch_channels<false>(state, tilde, p, coupled, keep, stream);
}

namespace {

template <bool TGV, int C, bool COUPLED>
cudaError_t dual_batch_one(const DualTile* tiles, int count, const DualBatchImage* images, int parity, cudaStream_t s) {
  auto kernel = dual_batch_kernel<TGV, C, COUPLED>;
  const std::size_t bytes = dual_tma_shared_bytes(TGV, C);
  // The shared-memory size above 48 KB is set once per device.
  static std::atomic<unsigned long long> configured{0};
  int device = 0;
  cudaGetDevice(&device);
  const unsigned long long bit = 1ull << (device & 63);
  if ((configured.load() & bit) == 0) {
    const cudaError_t e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                               static_cast<int>(bytes));
    if (e != cudaSuccess) return e;
    configured.fetch_or(bit);
  }
  if (count <= 0) return cudaSuccess;
  kernel<<<count, kThreads, bytes, s>>>(tiles, images, parity);
  return cudaGetLastError();
}

// The CTAs of the batched dual sweep the device holds at once (its SMs times an SM's).
template <bool TGV, int C, bool COUPLED>
int dual_batch_resident() {
  auto kernel = dual_batch_kernel<TGV, C, COUPLED>;
  const std::size_t bytes = dual_tma_shared_bytes(TGV, C);
  int device = 0, per_sm = 0, sms = 0;
  cudaGetDevice(&device);
  if (cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(bytes)) !=
          cudaSuccess ||
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, kThreads, bytes) != cudaSuccess ||
      cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device) != cudaSuccess) {
    cudaGetLastError();
    return 0;
  }
  return per_sm * sms;
}

template <bool TGV>
int dual_batch_resident_channels(int channels, bool coupled) {
  switch (channels) {
    case 1: return dual_batch_resident<TGV, 1, false>();
    case 2: return coupled ? dual_batch_resident<TGV, 2, true>() : dual_batch_resident<TGV, 2, false>();
    case 3: return coupled ? dual_batch_resident<TGV, 3, true>() : dual_batch_resident<TGV, 3, false>();
    default: return 0;
  }
}

template <bool TGV>
cudaError_t dual_batch_channels(const DualTile* tiles, int count, const DualBatchImage* images, int parity,
                                int channels, bool coupled, cudaStream_t s) {
  switch (channels) {
    case 1: return dual_batch_one<TGV, 1, false>(tiles, count, images, parity, s);
    case 2: return coupled ? dual_batch_one<TGV, 2, true>(tiles, count, images, parity, s)
                           : dual_batch_one<TGV, 2, false>(tiles, count, images, parity, s);
    case 3: return coupled ? dual_batch_one<TGV, 3, true>(tiles, count, images, parity, s)
                           : dual_batch_one<TGV, 3, false>(tiles, count, images, parity, s);
    default: return cudaErrorInvalidValue;
  }
}

}  // namespace

cudaError_t launch_dual_batch(const DualTile* tiles, int count, const DualBatchImage* images, int parity, bool tgv,
                              int channels, bool coupled, cudaStream_t stream) {
  return tgv ? dual_batch_channels<true>(tiles, count, images, parity, channels, coupled, stream)
             : dual_batch_channels<false>(tiles, count, images, parity, channels, coupled, stream);
}

int dual_batch_slots(bool tgv, int channels, bool coupled) {
  return tgv ? dual_batch_resident_channels<true>(channels, coupled)
             : dual_batch_resident_channels<false>(channels, coupled);
}

int batch_tile_rows(const std::vector<Geometry>& pictures, int slots) {
  int best = 128;
  long long best_cost = -1;
  for (int height = 64; height <= 512; height += 16) {
    long long ctas = 0;
    for (const Geometry& g : pictures) {
      const int width = sweep_width(g.channels);
      ctas += static_cast<long long>((g.columns + width - 1) / width) * ((g.rows + height - 1) / height);
    }
    const long long waves = slots > 0 ? (ctas + slots - 1) / slots : ctas;
    const long long cost = waves * (height + 2 * kChunk);
    if (best_cost < 0 || cost < best_cost) {
      best_cost = cost;
      best = height;
    }
  }
  return best;
}

namespace {
constexpr long long kFullRingLimit = 1LL << 22;
std::atomic<long long> ring_limit{kFullRingLimit};
}  // namespace

long long set_ring_wait_limit(long long tries) {
  return ring_limit.exchange(tries < 0 ? kFullRingLimit : tries);
}

long long ring_wait_limit() { return ring_limit.load(); }

}  // namespace urb
