// One whole iteration as a single TMA-fed sweep (sm_100a): the dual step D_n with the
// relaxation, and the primal step P_{n+1} of the next iteration on what D_n has just made, so
// that the relaxed state s_n goes from registers straight into the proximal map of G and is
// not read back from HBM.
//
// A CTA owns a strip of 32 canvas columns and walks down strip_rows rows of it in chunks of 8
// rows. Each chunk's rows and the row below them (9 rows, 40 columns: the strip and 4 on each
// side), of every plane of the state s_{n-1} and of x~_n, come into shared memory by two
// cp.async.bulk.tensor loads into a ring of two slots; the load of chunk k + 1 runs while chunk
// k is computed. Per chunk:
//
//   A  eight row warps (a row each, a lane per column) make x_n, w~, w- and p_n at their pixel
//      (the dual step of docs/math.md 5, as cpp/src/primal_dual.hpp:572-735 orders it) and
//      write them; the side warp makes w- and p1_n at column x0 - 1 of the chunk's 8 rows (the
//      left neighbour the divergence and the symmetrised gradient read);
//   B  the r step from w- of the neighbours (left by a shuffle, above from shared memory), then
//      v = x_n + tau gamma div p_n (cpp/src/primal_dual.hpp:536-545) and the row transform of
//      each 8x8 block of v (or of its cell means, for subsampled chroma, once a band of
//      8 CR rows is complete) by shuffles within 8 lanes;
//   C  the column transform through shared memory, the clip of every coefficient to its
//      interval (cpp/src/model.cpp:57-72, 544-597), the inverse column transform;
//   D  the inverse row transform by shuffles, x~_{n+1} written.
//
// Channel 0 has cells of 1 x 1 samples; the other channels (colour) have cells of CR x CC with
// CR, CC in {1, 2}; other layouts take the split kernels. The waits on the ring's mbarriers are
// bounded: one that runs out sets the error word and the CTA leaves after its loads in flight.
#include <algorithm>
#include <atomic>

#include <cuda.h>
#include <cudaTypedefs.h>

#include "dct.cuh"
#include "kernels.hpp"
#include "prox.cuh"
#include "tma.cuh"

namespace urb {

namespace {

constexpr int kRows = 8;         // rows of a chunk, a warp each
constexpr int kBox = 9;          // rows of a chunk's box: the chunk and the row below
constexpr int kSpan = 40;        // columns of a box: 4 + 32 + 4
constexpr int kHalo = 4;         // columns left of the strip (16-byte aligned start)
constexpr int kWarps = 9;        // the row warps and the side warp
constexpr unsigned kAll = 0xffffffffu;

__device__ __forceinline__ float ball_of(float square, float radius) {
  const float norm = sqrtf(square);
  return norm > radius ? radius / norm : 1.0f;
}

// w~ = w + tau (p + div2 r) at a pixel, div2 r by forward differences (cpp/src/primal_dual.hpp
// :86-95, 547-557); `at(field, dr, dc)` reads the channel's field (0 x, 1 p1, 2 p2, 3 w1, 4 w2,
// 5 r11, 6 r22, 7 r12) at the pixel moved by (dr, dc).
template <class At>
__device__ __forceinline__ void w_tilde(const At& at, bool right, bool down, float tau, float& t1, float& t2,
                                        float& w1, float& w2) {
  const float r11 = at(5, 0, 0), r22 = at(6, 0, 0), r12 = at(7, 0, 0);
  float d1 = right ? at(5, 0, 1) - r11 : 0.0f;
  float d2 = right ? at(7, 0, 1) - r12 : 0.0f;
  d1 = d1 + (down ? at(7, 1, 0) - r12 : 0.0f);
  d2 = d2 + (down ? at(6, 1, 0) - r22 : 0.0f);
  w1 = at(3, 0, 0);
  w2 = at(4, 0, 0);
  t1 = w1 + tau * (at(1, 0, 0) + d1);
  t2 = w2 + tau * (at(2, 0, 0) + d2);
}

// A channel's part of the dual step at a pixel before the projection: x~ and x there, w~ and
// w- (TGV), and the point p + sigma (grad x- - w-) that is projected. `xt(dr, dc)` reads x~.
struct PixelDual {
  float xt, x, p1, p2, t1, t2, w1, w2, wb1, wb2, s1, s2;
};

template <bool TGV, class At, class Xt>
__device__ __forceinline__ PixelDual pixel_dual(const At& at, const Xt& xt, bool right, bool down, float sigma,
                                                float tau) {
  PixelDual d;
  d.xt = xt(0, 0);
  d.x = at(0, 0, 0);
  const float bar = 2.0f * d.xt - d.x;
  const float gx = right ? (2.0f * xt(0, 1) - at(0, 0, 1)) - bar : 0.0f;
  const float gy = down ? (2.0f * xt(1, 0) - at(0, 1, 0)) - bar : 0.0f;
  d.p1 = at(1, 0, 0);
  d.p2 = at(2, 0, 0);
  if constexpr (TGV) {
    w_tilde(at, right, down, tau, d.t1, d.t2, d.w1, d.w2);
    d.wb1 = 2.0f * d.t1 - d.w1;
    d.wb2 = 2.0f * d.t2 - d.w2;
    d.s1 = d.p1 + sigma * (gx - d.wb1);
    d.s2 = d.p2 + sigma * (gy - d.wb2);
  } else {
    d.t1 = d.t2 = d.w1 = d.w2 = d.wb1 = d.wb2 = 0.0f;
    d.s1 = d.p1 + sigma * gx;
    d.s2 = d.p2 + sigma * gy;
  }
  return d;
}

// The projections' scales of p over the channels (coupled: one ball for all; apart: one each).
template <int C, bool COUPLED>
__device__ __forceinline__ void p_scales(const PixelDual (&d)[C], float radius, float (&scale)[C]) {
  if constexpr (COUPLED) {
    float square = 0.0f;
#pragma unroll
    for (int c = 0; c < C; ++c) square += d[c].s1 * d[c].s1 + d[c].s2 * d[c].s2;
    const float s = ball_of(square, radius);
#pragma unroll
    for (int c = 0; c < C; ++c) scale[c] = s;
  } else {
#pragma unroll
    for (int c = 0; c < C; ++c) scale[c] = ball_of(d[c].s1 * d[c].s1 + d[c].s2 * d[c].s2, radius);
  }
}

// The forward column transform of one output frequency V: sum over i of C[V][i] t[i][lane].
template <int V>
__device__ __forceinline__ float column_forward(const float* t) {
  float acc = basis_as<float>(V, 0) * t[0];
#pragma unroll
  for (int i = 1; i < 8; ++i) acc = fmaf(basis_as<float>(V, i), t[i * 32], acc);
  return acc;
}

// The inverse column transform at row N: sum over v of C[v][N] z[v][lane].
template <int N>
__device__ __forceinline__ float column_inverse(const float* z) {
  float acc = basis_as<float>(0, N) * z[0];
#pragma unroll
  for (int v = 1; v < 8; ++v) acc = fmaf(basis_as<float>(v, N), z[v * 32], acc);
  return acc;
}

__device__ __forceinline__ float forward_column(int w, const float* t) {
  switch (w) {
    case 0: return column_forward<0>(t);
    case 1: return column_forward<1>(t);
    case 2: return column_forward<2>(t);
    case 3: return column_forward<3>(t);
    case 4: return column_forward<4>(t);
    case 5: return column_forward<5>(t);
    case 6: return column_forward<6>(t);
    default: return column_forward<7>(t);
  }
}

__device__ __forceinline__ float inverse_column(int w, const float* z) {
  switch (w) {
    case 0: return column_inverse<0>(z);
    case 1: return column_inverse<1>(z);
    case 2: return column_inverse<2>(z);
    case 3: return column_inverse<3>(z);
    case 4: return column_inverse<4>(z);
    case 5: return column_inverse<5>(z);
    case 6: return column_inverse<6>(z);
    default: return column_inverse<7>(z);
  }
}

// The row transforms within each group of 8 lanes (a block's 8 columns): forward, the lane of
// frequency u gets sum over n of C[u][n] x(n); inverse, the lane of column n gets sum over u
// of C[u][n] z(u). `basis` holds the lane's 8 factors.
__device__ __forceinline__ float row_transform(float value, const float (&basis)[8]) {
  float acc = basis[0] * __shfl_sync(kAll, value, 0, 8);
#pragma unroll
  for (int n = 1; n < 8; ++n) acc = fmaf(basis[n], __shfl_sync(kAll, value, n, 8), acc);
  return acc;
}

template <int C, int CR, int CC>
struct Layout {
  static constexpr bool kChroma = C > 1 && CR * CC > 1;  // channels 1.. have cells of CR x CC
  static constexpr int kPlain = kChroma ? 1 : C;          // channels of 1 x 1 cells
  static constexpr int kChromaItems = kChroma ? 2 / CC : 0;
  static constexpr int kItems = kPlain + kChromaItems;    // blocks of 8 x 8 a thread takes a value of
};

template <bool TGV, int C, bool COUPLED, int CR, int CC>
__global__ void __launch_bounds__(32 * kWarps, 2)
    iteration_kernel(const __grid_constant__ CUtensorMap state_map, const __grid_constant__ CUtensorMap tilde_map,
                     const IterationParams P) {
  using L = Layout<C, CR, CC>;
  constexpr int F = TGV ? 8 : 3;
  constexpr int PLANE = kBox * kSpan;
  constexpr int TOFF = (F * C * PLANE + 31) / 32 * 32;          // x~'s planes, 128-byte aligned
  constexpr int STRIDE = (TOFF + C * PLANE + 31) / 32 * 32;    // a slot, 128-byte aligned
  constexpr int CH = L::kChroma ? C - 1 : 1;                    // chroma channels (buffers)
  extern __shared__ __align__(128) float ring[];
  __shared__ __align__(8) std::uint64_t bars[2];
  __shared__ ProxFactors factors[C];
  __shared__ float wbar[TGV ? C : 1][2][kRows][32];   // w- of each row warp's row
  __shared__ float wcarry[TGV ? C : 1][2][32];        // w- of the row above the chunk
  __shared__ float p2rows[C][kRows][32];               // p2_n of each row warp's row
  __shared__ float p2carry[C][32];                     // p2_n of the row above the chunk
  __shared__ float wleft[TGV ? C : 1][2][kRows];      // w- at column x0 - 1
  __shared__ float pleft[C][kRows];                    // p1_n at column x0 - 1
  __shared__ float tbuf[L::kItems][kRows][32];         // after the row transform
  __shared__ float zbuf[L::kItems][kRows][32];         // the clipped coefficients
  __shared__ float vbuf[CH][L::kChroma ? 8 * CR : 1][32];  // v of the chroma channels, a band
  // The levels of the blocks a chunk clips (of each item: up to 4 blocks of the strip), copied
  // with the chunk's loads into a ring of three: a chunk's are read until its last phase, when
  // the loads of the chunk two ahead are already under way.
  __shared__ __align__(128) std::int16_t lvbuf[3][L::kItems][4][64];

  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const Geometry& g = P.dual.g;
  const int rows = g.rows, columns = g.columns, pitch = g.pitch;
  const std::size_t plane = g.plane;
  const int x0 = blockIdx.x * 32;
  const int i0 = blockIdx.y * P.strip_rows;
  const int i1 = min(i0 + P.strip_rows, rows);
  const int chunks = (i1 - i0) / kRows;
  const float rho = P.dual.rho, rest = P.dual.rest;

  {
    constexpr int words = static_cast<int>(sizeof(ProxFactors) / 4);
#pragma unroll
    for (int c = 0; c < C; ++c) {
      const float* from = reinterpret_cast<const float*>(P.component[c].factors);
      float* to = reinterpret_cast<float*>(&factors[c]);
      for (int k = tid; k < words; k += 32 * kWarps) to[k] = from[k];
    }
  }
  if (tid == 0) {
    barrier_init(&bars[0], 1);
    barrier_init(&bars[1], 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
  // Chunk k's loads: its box of every state plane and of x~, and the levels of the blocks it
  // clips -- of the channels of 1 x 1 cells the block row of its rows, and where it ends a band
  // of the chroma channels that band's block row -- on the slot's barrier.
  auto issue = [&](int k) {
    if (tid == 0 && k < chunks) {
      float* to = ring + (k & 1) * STRIDE;
      const int chunk_row = i0 + k * kRows;
      // Each copy of levels, counted (pass 0) and then issued (pass 1).
      unsigned bytes = (F * C + C) * PLANE * 4;
      auto copies = [&](bool go) {
        auto copy = [&](const ComponentDevice& comp, int vby, int vbx, int most, int q, int b0) {
          const int n = min(most, comp.block_columns - vbx);
          if (vby < comp.block_rows && n > 0) {
            if (go) {
              load_bulk(&lvbuf[k % 3][q][b0][0],
                        comp.levels + (static_cast<std::size_t>(vby) * comp.block_columns + vbx) * 64, n * 128u,
                        &bars[k & 1]);
            } else {
              bytes += n * 128u;
            }
          }
        };
#pragma unroll
        for (int c = 0; c < L::kPlain; ++c) copy(P.component[c], chunk_row / 8, x0 / 8, 4, c, 0);
        if constexpr (L::kChroma) {
          if (k % CR == CR - 1) {
            const int band_row = chunk_row - (CR - 1) * kRows;
#pragma unroll
            for (int cc = 0; cc < C - 1; ++cc) {
              copy(P.component[1 + cc], band_row / (8 * CR), x0 / (8 * CC), 4 / CC, L::kPlain + (CC == 2 ? 0 : cc),
                   CC == 2 ? 2 * cc : 0);
            }
          }
        }
      };
      copies(false);
      barrier_expect(&bars[k & 1], bytes);
      load_box(to, &state_map, &bars[k & 1], x0 - kHalo, chunk_row, 0);
      load_box(to + TOFF, &tilde_map, &bars[k & 1], x0 - kHalo, chunk_row, 0);
      copies(true);
    }
  };
  issue(0);
  issue(1);

  // The lane's factors of the row transforms: forward C[u][n] (u = lane % 8), inverse C[n][u]
  // read as C[u'][lane % 8] over u'.
  float forward_basis[8], inverse_basis[8];
  {
    const int u = lane & 7;
#pragma unroll
    for (int n = 0; n < 8; ++n) {
      float f = 0.0f, b = 0.0f;
#pragma unroll
      for (int k = 0; k < 8; ++k) {
        f = u == k ? basis_as<float>(k, n) : f;
        b = u == k ? basis_as<float>(n, k) : b;
      }
      forward_basis[n] = f;
      inverse_basis[n] = b;
    }
  }

  const int j = x0 + lane;
  const bool valid = j < columns;
  const int jc = valid ? j : columns - 1;
  const bool has_left = j > 0, has_right = j + 1 < columns;

  // The row above the strip, made from global memory by the first row warp: w- (for the r step
  // of the strip's first row) and p2_n (for the divergence of its primal step).
  if (warp == 0) {
    if (i0 > 0) {
      const int u = i0 - 1;
      PixelDual d[C];
#pragma unroll
      for (int c = 0; c < C; ++c) {
        const std::size_t base = c * plane;
        const Fields& in = P.dual.in;
        const float* planes[8] = {in.x, in.p1, in.p2, in.w1, in.w2, in.r11, in.r22, in.r12};
        auto at = [&](int field, int dr, int dc) -> float {
          return __ldg(planes[field] + base + static_cast<std::size_t>(u + dr) * pitch + jc + dc);
        };
        auto xt = [&](int dr, int dc) -> float {
          return __ldg(P.dual.xt + base + static_cast<std::size_t>(u + dr) * pitch + jc + dc);
        };
        d[c] = pixel_dual<TGV>(at, xt, has_right, true, P.dual.sigma[c], P.dual.tau[c]);
      }
      float scale[C];
      p_scales<C, COUPLED>(d, P.dual.radius, scale);
#pragma unroll
      for (int c = 0; c < C; ++c) {
        if constexpr (TGV) {
          wcarry[c][0][lane] = d[c].wb1;
          wcarry[c][1][lane] = d[c].wb2;
        }
        p2carry[c][lane] = rho * (d[c].s2 * scale[c]) + rest * d[c].p2;
      }
    } else {
#pragma unroll
      for (int c = 0; c < C; ++c) {
        if constexpr (TGV) {
          wcarry[c][0][lane] = 0.0f;
          wcarry[c][1][lane] = 0.0f;
        }
        p2carry[c][lane] = 0.0f;
      }
    }
  }
  __syncthreads();

  bool failed = false;
  int stopped = chunks;
  for (int k = 0; k < chunks; ++k) {
    const bool ready = barrier_wait(&bars[k & 1], (k >> 1) & 1);
    if (__syncthreads_or(!ready)) {
      failed = true;
      stopped = k;
      break;
    }
    const float* slot = ring + (k & 1) * STRIDE;
    const int chunk_row = i0 + k * kRows;
    const std::int16_t(*lv)[4][64] = lvbuf[k % 3];
    // The blocks the lane's coefficients belong to, and whether they are flat (read now, used
    // in C): of the channels of 1 x 1 cells the chunk's block row; of the chroma channels, where
    // the chunk ends a band, the band's.
    const bool band = L::kChroma && (k % CR) == CR - 1;
    bool plain_in[L::kPlain], plain_flat[L::kPlain];
#pragma unroll
    for (int c = 0; c < L::kPlain; ++c) {
      const ComponentDevice& comp = P.component[c];
      const int vby = chunk_row / 8, vbx = j / 8;
      plain_in[c] = warp < kRows && valid && vby < comp.block_rows && vbx < comp.block_columns;
      plain_flat[c] = plain_in[c] && comp.flat[static_cast<std::size_t>(vby) * comp.block_columns + vbx] != 0;
    }
    constexpr int NQ = L::kChromaItems > 0 ? L::kChromaItems : 1;
    bool chroma_in[NQ], chroma_flat[NQ];
    int chroma_block[NQ];
#pragma unroll
    for (int q = 0; q < NQ; ++q) {
      chroma_in[q] = chroma_flat[q] = false;
      chroma_block[q] = 0;
    }
    if constexpr (L::kChroma) {
      if (band && warp < kRows) {
        const int band_row = chunk_row - (CR - 1) * kRows;
#pragma unroll
        for (int q = 0; q < L::kChromaItems; ++q) {
          constexpr int per = 32 / CC;
          const int s = q * 32 + lane, cc = s / per, mcol = s % per, unit = mcol >> 3;
          const ComponentDevice& comp = P.component[1 + cc];
          const int vby = band_row / (8 * CR), vbx = x0 / (8 * CC) + unit;
          chroma_in[q] = x0 + mcol * CC < columns && vby < comp.block_rows && vbx < comp.block_columns;
          chroma_flat[q] =
              chroma_in[q] && comp.flat[static_cast<std::size_t>(vby) * comp.block_columns + vbx] != 0;
          chroma_block[q] = CC == 2 ? 2 * cc + unit : unit;
        }
      }
    }
    // ---- A: the dual step at the warp's pixel (row warps), at column x0 - 1 (side warp).
    float xn[C], pn1[C], pn2[C], wb1[C], wb2[C];
    PixelDual d[C];
    const int r = warp;
    const int i = chunk_row + r;
    if (warp < kRows) {
      const bool has_down = i + 1 < rows;
      const int own = kHalo + lane;
#pragma unroll
      for (int c = 0; c < C; ++c) {
        auto at = [&](int field, int dr, int dc) -> float {
          return slot[((field * C + c) * kBox + r + dr) * kSpan + own + dc];
        };
        auto xt = [&](int dr, int dc) -> float { return slot[TOFF + (c * kBox + r + dr) * kSpan + own + dc]; };
        d[c] = pixel_dual<TGV>(at, xt, has_right, has_down, P.dual.sigma[c], P.dual.tau[c]);
      }
      float scale[C];
      p_scales<C, COUPLED>(d, P.dual.radius, scale);
      const std::size_t here = static_cast<std::size_t>(i) * pitch + jc;
#pragma unroll
      for (int c = 0; c < C; ++c) {
        const std::size_t at = c * plane + here;
        xn[c] = rho * d[c].xt + rest * d[c].x;
        pn1[c] = rho * (d[c].s1 * scale[c]) + rest * d[c].p1;
        pn2[c] = rho * (d[c].s2 * scale[c]) + rest * d[c].p2;
        wb1[c] = d[c].wb1;
        wb2[c] = d[c].wb2;
        if (valid) {
          P.dual.out.x[at] = xn[c];
          P.dual.out.p1[at] = pn1[c];
          P.dual.out.p2[at] = pn2[c];
          if constexpr (TGV) {
            P.dual.out.w1[at] = rho * d[c].t1 + rest * d[c].w1;
            P.dual.out.w2[at] = rho * d[c].t2 + rest * d[c].w2;
          }
        }
        if constexpr (TGV) {
          wbar[c][0][r][lane] = wb1[c];
          wbar[c][1][r][lane] = wb2[c];
        }
        p2rows[c][r][lane] = pn2[c];
      }
    } else if (lane < kRows && x0 > 0) {
      const int rr = lane, ii = chunk_row + rr;
      const int col = kHalo - 1;
      PixelDual e[C];
#pragma unroll
      for (int c = 0; c < C; ++c) {
        auto at = [&](int field, int dr, int dc) -> float {
          return slot[((field * C + c) * kBox + rr + dr) * kSpan + col + dc];
        };
        auto xt = [&](int dr, int dc) -> float { return slot[TOFF + (c * kBox + rr + dr) * kSpan + col + dc]; };
        e[c] = pixel_dual<TGV>(at, xt, true, ii + 1 < rows, P.dual.sigma[c], P.dual.tau[c]);
      }
      float scale[C];
      p_scales<C, COUPLED>(e, P.dual.radius, scale);
#pragma unroll
      for (int c = 0; c < C; ++c) {
        if constexpr (TGV) {
          wleft[c][0][rr] = e[c].wb1;
          wleft[c][1][rr] = e[c].wb2;
        }
        pleft[c][rr] = rho * (e[c].s1 * scale[c]) + rest * e[c].p1;
      }
    }
    __syncthreads();

    // ---- B: the r step; v; the row transforms.
    float v[C];
    float middle[L::kPlain];
    if (warp < kRows) {
      const bool has_down = i + 1 < rows, has_up = i > 0;
      const std::size_t here = static_cast<std::size_t>(i) * pitch + jc;
      if constexpr (TGV) {
        float s11[C], s22[C], s12[C], o11[C], o22[C], o12[C];
        float square = 0.0f;
        const int own = kHalo + lane;
#pragma unroll
        for (int c = 0; c < C; ++c) {
          float wl1 = __shfl_up_sync(kAll, wb1[c], 1), wl2 = __shfl_up_sync(kAll, wb2[c], 1);
          if (lane == 0) {
            wl1 = wleft[c][0][r];
            wl2 = wleft[c][1][r];
          }
          if (!has_left) wl1 = wl2 = 0.0f;
          float wu1 = r > 0 ? wbar[c][0][r - 1][lane] : wcarry[c][0][lane];
          float wu2 = r > 0 ? wbar[c][1][r - 1][lane] : wcarry[c][1][lane];
          if (!has_up) wu1 = wu2 = 0.0f;
          const float own1x = has_right ? wb1[c] : 0.0f, own2x = has_right ? wb2[c] : 0.0f;
          const float own1y = has_down ? wb1[c] : 0.0f, own2y = has_down ? wb2[c] : 0.0f;
          const float exx = own1x - wl1;
          const float eyy = own2y - wu2;
          const float exy = 0.5f * ((own1y - wu1) + (own2x - wl2));
          o11[c] = slot[((5 * C + c) * kBox + r) * kSpan + own];
          o22[c] = slot[((6 * C + c) * kBox + r) * kSpan + own];
          o12[c] = slot[((7 * C + c) * kBox + r) * kSpan + own];
          const float sigma = P.dual.sigma[c];
          s11[c] = o11[c] + sigma * exx;
          s22[c] = o22[c] + sigma * eyy;
          s12[c] = o12[c] + sigma * exy;
          if constexpr (COUPLED) square += s11[c] * s11[c] + s22[c] * s22[c] + 2.0f * (s12[c] * s12[c]);
        }
        const float coupled_scale = COUPLED ? ball_of(square, P.dual.radius0) : 1.0f;
#pragma unroll
        for (int c = 0; c < C; ++c) {
          float sr = coupled_scale;
          if constexpr (!COUPLED) {
            sr = ball_of(s11[c] * s11[c] + s22[c] * s22[c] + 2.0f * (s12[c] * s12[c]), P.dual.radius0);
          }
          if (valid) {
            const std::size_t at = c * plane + here;
            P.dual.out.r11[at] = rho * (s11[c] * sr) + rest * o11[c];
            P.dual.out.r22[at] = rho * (s22[c] * sr) + rest * o22[c];
            P.dual.out.r12[at] = rho * (s12[c] * sr) + rest * o12[c];
          }
        }
      }
      // v = x_n + tau gamma div p_n, div by backward differences (Neumann ends).
#pragma unroll
      for (int c = 0; c < C; ++c) {
        float before = __shfl_up_sync(kAll, pn1[c], 1);
        if (lane == 0) before = pleft[c][r];
        const float above = r > 0 ? p2rows[c][r - 1][lane] : p2carry[c][lane];
        const float dy = (has_down ? pn2[c] : 0.0f) - (has_up ? above : 0.0f);
        const float dx = (has_right ? pn1[c] : 0.0f) - (has_left ? before : 0.0f);
        v[c] = xn[c] + P.dual.tau[c] * (dy + dx);
      }
      // Channels of 1 x 1 cells: the block's samples less the middle of its DC interval, then
      // the row transform.
#pragma unroll
      for (int c = 0; c < L::kPlain; ++c) {
        const float dc = plain_in[c] ? static_cast<float>(lv[c][lane >> 3][0]) : 0.0f;
        middle[c] = (dc * factors[c].plain[0].x + 1024.0f) * 0.125f;
        tbuf[c][r][lane] = row_transform(v[c] - middle[c], forward_basis);
      }
      if constexpr (L::kChroma) {
#pragma unroll
        for (int c = 1; c < C; ++c) vbuf[c - 1][(k % CR) * kRows + r][lane] = v[c];
      }
    }
    // The chroma channels once their band of 8 CR rows is complete: cell means (down each
    // column, then across), less the middle of the DC interval, then the row transform.
    float mean[NQ];
    if constexpr (L::kChroma) {
      if (band) {
        if constexpr (CR > 1) {
          __syncthreads();
        } else {
          __syncwarp();
        }
        if (warp < kRows) {
#pragma unroll
          for (int q = 0; q < L::kChromaItems; ++q) {
            constexpr int per = 32 / CC;
            const int s = q * 32 + lane, cc = s / per, mcol = s % per;
            const float dc =
                chroma_in[q] ? static_cast<float>(lv[L::kPlain + q][chroma_block[q]][0]) : 0.0f;
            const float chroma_middle = (dc * factors[1 + cc].plain[0].x + 1024.0f) * 0.125f;
            float total = 0.0f;
#pragma unroll
            for (int b = 0; b < CC; ++b) {
              float column = vbuf[cc][r * CR][mcol * CC + b];
#pragma unroll
              for (int a = 1; a < CR; ++a) column += vbuf[cc][r * CR + a][mcol * CC + b];
              total = b == 0 ? column : total + column;
            }
            mean[q] = total / static_cast<float>(CR * CC) - chroma_middle;
            tbuf[L::kPlain + q][r][lane] = row_transform(mean[q], forward_basis);
          }
        }
      }
    }
    __syncthreads();
    issue(k + 2);  // every read of the slot is done

    // ---- C: the column transform, the clip, the inverse column transform.
    const int items = L::kPlain + (band ? L::kChromaItems : 0);
    if (warp < kRows) {
      const int u = lane & 7;
      const int kk = r * 8 + u;  // natural order: vertical frequency r, horizontal u
      if (r == kRows - 1) {
        // The last row's w- and p2_n: the row above the next chunk.
#pragma unroll
        for (int c = 0; c < C; ++c) {
          if constexpr (TGV) {
            wcarry[c][0][lane] = wb1[c];
            wcarry[c][1][lane] = wb2[c];
          }
          p2carry[c][lane] = pn2[c];
        }
      }
#pragma unroll
      for (int q = 0; q < L::kItems; ++q) {
        if (q >= items) break;
        int c, blk;
        bool in, flat;
        if (q < L::kPlain) {
          c = q;
          blk = lane >> 3;
          in = plain_in[q];
          flat = plain_flat[q];
        } else {
          constexpr int per = 32 / CC;
          const int s = (q - L::kPlain) * 32 + lane;
          c = 1 + s / per;
          blk = chroma_block[q - L::kPlain];
          in = chroma_in[q - L::kPlain];
          flat = chroma_flat[q - L::kPlain];
        }
        const ProxFactors& fc = factors[c];
        const float e = forward_column(r, &tbuf[q][0][lane]);
        float zeta = 0.0f;
        if (in) {
          const int level = lv[q][blk][kk];
          zeta = prox_at(e, level, kk, flat, fc);
        }
        zbuf[q][r][lane] = zeta;
      }
    }
    __syncthreads();

    // ---- D: the inverse transforms; x~_{n+1}.
    if (warp < kRows) {
#pragma unroll
      for (int q = 0; q < L::kPlain; ++q) {
        const float back = row_transform(inverse_column(r, &zbuf[q][0][lane]), inverse_basis);
        if (valid) {
          P.next[q * plane + static_cast<std::size_t>(i) * pitch + j] = plain_in[q] ? back + middle[q] : v[q];
        }
      }
      if constexpr (L::kChroma) {
        if (band) {
          const int band_row = chunk_row - (CR - 1) * kRows;
#pragma unroll
          for (int q = 0; q < L::kChromaItems; ++q) {
            constexpr int per = 32 / CC;
            const int s = q * 32 + lane, cc = s / per, mcol = s % per;
            const float back = row_transform(inverse_column(r, &zbuf[L::kPlain + q][0][lane]), inverse_basis);
            const int col0 = x0 + mcol * CC;
            if (col0 < columns) {
              float* out = P.next + (1 + cc) * plane;
#pragma unroll
              for (int a = 0; a < CR; ++a) {
#pragma unroll
                for (int b = 0; b < CC; ++b) {
                  const float sample = vbuf[cc][r * CR + a][mcol * CC + b];
                  out[static_cast<std::size_t>(band_row + r * CR + a) * pitch + col0 + b] =
                      chroma_in[q] ? sample + (back - mean[q]) : sample;
                }
              }
            }
          }
        }
      }
    }
  }
  if (failed && tid == 0 && P.dual.error != nullptr) atomicExch(P.dual.error, 1);
  // No load may still write into shared memory when the CTA leaves: wait (bounded) for the
  // chunks issued and not consumed.
  if (failed) {
    for (int k = stopped; k < min(stopped + 2, chunks); ++k) barrier_wait(&bars[k & 1], (k >> 1) & 1);
  }
}

// Pictures of rounded samples in one sweep (samples.cu has the split kernels): the dual step D_n
// as iteration_kernel's phase A makes it, then in phase B the r step and the primal step
// P_{n+1} sample by sample -- v = x_n + tau gamma div p_n and x~ = clip((v + t c) r, a, b), the
// ends and centre by the sample's level from the binary32 table -- so that x_n and p_n go from
// registers into the proximal map and x~ is written once: 68 bytes a sample of the dual sweep
// plus the level read and x~ written, against 86 for the two launches. Ragged last chunks are
// taken (rows past the picture write nothing).
template <bool TGV, int C, bool COUPLED>
__global__ void __launch_bounds__(32 * kWarps, 2)
    samples_iteration_kernel(const __grid_constant__ CUtensorMap state_map,
                             const __grid_constant__ CUtensorMap tilde_map, const SamplesIterationParams P) {
  constexpr int F = TGV ? 8 : 3;
  constexpr int PLANE = kBox * kSpan;
  constexpr int TOFF = (F * C * PLANE + 31) / 32 * 32;
  constexpr int STRIDE = (TOFF + C * PLANE + 31) / 32 * 32;
  extern __shared__ __align__(128) float ring[];
  __shared__ __align__(8) std::uint64_t bars[2];
  __shared__ float wbar[TGV ? C : 1][2][kRows][32];
  __shared__ float wcarry[TGV ? C : 1][2][32];
  __shared__ float p2rows[C][kRows][32];
  __shared__ float p2carry[C][32];
  __shared__ float wleft[TGV ? C : 1][2][kRows];
  __shared__ float pleft[C][kRows];

  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const Geometry& g = P.dual.g;
  const int rows = g.rows, columns = g.columns, pitch = g.pitch;
  const std::size_t plane = g.plane;
  const int x0 = blockIdx.x * 32;
  const int i0 = blockIdx.y * P.strip_rows;
  const int i1 = min(i0 + P.strip_rows, rows);
  const int chunks = (i1 - i0 + kRows - 1) / kRows;
  const float rho = P.dual.rho, rest = P.dual.rest;

  if (tid == 0) {
    barrier_init(&bars[0], 1);
    barrier_init(&bars[1], 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
  auto issue = [&](int k) {
    if (tid == 0 && k < chunks) {
      float* to = ring + (k & 1) * STRIDE;
      const int chunk_row = i0 + k * kRows;
      barrier_expect(&bars[k & 1], (F * C + C) * PLANE * 4);
      load_box(to, &state_map, &bars[k & 1], x0 - kHalo, chunk_row, 0);
      load_box(to + TOFF, &tilde_map, &bars[k & 1], x0 - kHalo, chunk_row, 0);
    }
  };
  issue(0);
  issue(1);

  const int j = x0 + lane;
  const bool valid = j < columns;
  const int jc = valid ? j : columns - 1;
  const bool has_left = j > 0, has_right = j + 1 < columns;

  // The row above the strip, made from global memory by the first row warp.
  if (warp == 0) {
    if (i0 > 0) {
      const int u = i0 - 1;
      PixelDual d[C];
#pragma unroll
      for (int c = 0; c < C; ++c) {
        const std::size_t base = c * plane;
        const Fields& in = P.dual.in;
        const float* planes[8] = {in.x, in.p1, in.p2, in.w1, in.w2, in.r11, in.r22, in.r12};
        auto at = [&](int field, int dr, int dc) -> float {
          return __ldg(planes[field] + base + static_cast<std::size_t>(u + dr) * pitch + jc + dc);
        };
        auto xt = [&](int dr, int dc) -> float {
          return __ldg(P.dual.xt + base + static_cast<std::size_t>(u + dr) * pitch + jc + dc);
        };
        d[c] = pixel_dual<TGV>(at, xt, has_right, true, P.dual.sigma[c], P.dual.tau[c]);
      }
      float scale[C];
      p_scales<C, COUPLED>(d, P.dual.radius, scale);
#pragma unroll
      for (int c = 0; c < C; ++c) {
        if constexpr (TGV) {
          wcarry[c][0][lane] = d[c].wb1;
          wcarry[c][1][lane] = d[c].wb2;
        }
        p2carry[c][lane] = rho * (d[c].s2 * scale[c]) + rest * d[c].p2;
      }
    } else {
#pragma unroll
      for (int c = 0; c < C; ++c) {
        if constexpr (TGV) {
          wcarry[c][0][lane] = 0.0f;
          wcarry[c][1][lane] = 0.0f;
        }
        p2carry[c][lane] = 0.0f;
      }
    }
  }
  __syncthreads();

  // The levels of the first chunk's pixels (then each chunk loads the next's).
  unsigned level[C] = {};
  if (warp < kRows && i0 + warp < i1 && valid) {
#pragma unroll
    for (int c = 0; c < C; ++c) level[c] = __ldg(P.levels + c * plane + static_cast<std::size_t>(i0 + warp) * pitch + jc);
  }
  bool failed = false;
  int stopped = chunks;
  for (int k = 0; k < chunks; ++k) {
    const bool ready = barrier_wait(&bars[k & 1], (k >> 1) & 1);
    if (__syncthreads_or(!ready)) {
      failed = true;
      stopped = k;
      break;
    }
    const float* slot = ring + (k & 1) * STRIDE;
    const int chunk_row = i0 + k * kRows;
    const int r = warp;
    const int i = chunk_row + r;
    const bool row_in = i < i1;  // warp-uniform
    // The pixel's ends (by the level loaded a chunk ago), looked up now so that the dual step
    // hides the lookup, and the level of the pixel a chunk below, for the next chunk.
    float4 ends[C];
    {
      const int below = i + kRows;
      const bool ahead = warp < kRows && below < i1 && valid;
      const std::size_t there = static_cast<std::size_t>(ahead ? below : 0) * pitch + jc;
#pragma unroll
      for (int c = 0; c < C; ++c) {
        ends[c] = __ldg(reinterpret_cast<const float4*>(P.ends) + level[c]);  // lower, upper, centre
        level[c] = ahead ? __ldg(P.levels + c * plane + there) : 0u;
      }
    }
    // ---- A: the dual step at the warp's pixel (row warps), at column x0 - 1 (side warp).
    float xn[C], pn1[C], pn2[C], wb1[C], wb2[C];
    if (warp < kRows) {
      const bool has_down = i + 1 < rows;
      const int own = kHalo + lane;
      PixelDual d[C];
#pragma unroll
      for (int c = 0; c < C; ++c) {
        auto at = [&](int field, int dr, int dc) -> float {
          return slot[((field * C + c) * kBox + r + dr) * kSpan + own + dc];
        };
        auto xt = [&](int dr, int dc) -> float { return slot[TOFF + (c * kBox + r + dr) * kSpan + own + dc]; };
        d[c] = pixel_dual<TGV>(at, xt, has_right, has_down, P.dual.sigma[c], P.dual.tau[c]);
      }
      float scale[C];
      p_scales<C, COUPLED>(d, P.dual.radius, scale);
      const std::size_t here = static_cast<std::size_t>(row_in ? i : i0) * pitch + jc;
#pragma unroll
      for (int c = 0; c < C; ++c) {
        const std::size_t at = c * plane + here;
        xn[c] = rho * d[c].xt + rest * d[c].x;
        pn1[c] = rho * (d[c].s1 * scale[c]) + rest * d[c].p1;
        pn2[c] = rho * (d[c].s2 * scale[c]) + rest * d[c].p2;
        wb1[c] = d[c].wb1;
        wb2[c] = d[c].wb2;
        if (valid && row_in) {
          P.dual.out.x[at] = xn[c];
          P.dual.out.p1[at] = pn1[c];
          P.dual.out.p2[at] = pn2[c];
          if constexpr (TGV) {
            P.dual.out.w1[at] = rho * d[c].t1 + rest * d[c].w1;
            P.dual.out.w2[at] = rho * d[c].t2 + rest * d[c].w2;
          }
        }
        if constexpr (TGV) {
          wbar[c][0][r][lane] = wb1[c];
          wbar[c][1][r][lane] = wb2[c];
        }
        p2rows[c][r][lane] = pn2[c];
      }
    } else if (lane < kRows && x0 > 0) {
      const int rr = lane, ii = chunk_row + rr;
      const int col = kHalo - 1;
      PixelDual e[C];
#pragma unroll
      for (int c = 0; c < C; ++c) {
        auto at = [&](int field, int dr, int dc) -> float {
          return slot[((field * C + c) * kBox + rr + dr) * kSpan + col + dc];
        };
        auto xt = [&](int dr, int dc) -> float { return slot[TOFF + (c * kBox + rr + dr) * kSpan + col + dc]; };
        e[c] = pixel_dual<TGV>(at, xt, true, ii + 1 < rows, P.dual.sigma[c], P.dual.tau[c]);
      }
      float scale[C];
      p_scales<C, COUPLED>(e, P.dual.radius, scale);
#pragma unroll
      for (int c = 0; c < C; ++c) {
        if constexpr (TGV) {
          wleft[c][0][rr] = e[c].wb1;
          wleft[c][1][rr] = e[c].wb2;
        }
        pleft[c][rr] = rho * (e[c].s1 * scale[c]) + rest * e[c].p1;
      }
    }
    __syncthreads();

    // ---- B: the r step; v; the proximal map of the samples' boxes; x~_{n+1}.
    if (warp < kRows && row_in) {
      const bool has_down = i + 1 < rows, has_up = i > 0;
      const std::size_t here = static_cast<std::size_t>(i) * pitch + jc;
      if constexpr (TGV) {
        float s11[C], s22[C], s12[C], o11[C], o22[C], o12[C];
        float square = 0.0f;
        const int own = kHalo + lane;
#pragma unroll
        for (int c = 0; c < C; ++c) {
          float wl1 = __shfl_up_sync(kAll, wb1[c], 1), wl2 = __shfl_up_sync(kAll, wb2[c], 1);
          if (lane == 0) {
            wl1 = wleft[c][0][r];
            wl2 = wleft[c][1][r];
          }
          if (!has_left) wl1 = wl2 = 0.0f;
          float wu1 = r > 0 ? wbar[c][0][r - 1][lane] : wcarry[c][0][lane];
          float wu2 = r > 0 ? wbar[c][1][r - 1][lane] : wcarry[c][1][lane];
          if (!has_up) wu1 = wu2 = 0.0f;
          const float own1x = has_right ? wb1[c] : 0.0f, own2x = has_right ? wb2[c] : 0.0f;
          const float own1y = has_down ? wb1[c] : 0.0f, own2y = has_down ? wb2[c] : 0.0f;
          const float exx = own1x - wl1;
          const float eyy = own2y - wu2;
          const float exy = 0.5f * ((own1y - wu1) + (own2x - wl2));
          o11[c] = slot[((5 * C + c) * kBox + r) * kSpan + own];
          o22[c] = slot[((6 * C + c) * kBox + r) * kSpan + own];
          o12[c] = slot[((7 * C + c) * kBox + r) * kSpan + own];
          const float sigma = P.dual.sigma[c];
          s11[c] = o11[c] + sigma * exx;
          s22[c] = o22[c] + sigma * eyy;
          s12[c] = o12[c] + sigma * exy;
          if constexpr (COUPLED) square += s11[c] * s11[c] + s22[c] * s22[c] + 2.0f * (s12[c] * s12[c]);
        }
        const float coupled_scale = COUPLED ? ball_of(square, P.dual.radius0) : 1.0f;
#pragma unroll
        for (int c = 0; c < C; ++c) {
          float sr = coupled_scale;
          if constexpr (!COUPLED) {
            sr = ball_of(s11[c] * s11[c] + s22[c] * s22[c] + 2.0f * (s12[c] * s12[c]), P.dual.radius0);
          }
          if (valid) {
            const std::size_t at = c * plane + here;
            P.dual.out.r11[at] = rho * (s11[c] * sr) + rest * o11[c];
            P.dual.out.r22[at] = rho * (s22[c] * sr) + rest * o22[c];
            P.dual.out.r12[at] = rho * (s12[c] * sr) + rest * o12[c];
          }
        }
      }
#pragma unroll
      for (int c = 0; c < C; ++c) {
        float before = __shfl_up_sync(kAll, pn1[c], 1);
        if (lane == 0) before = pleft[c][r];
        const float above = r > 0 ? p2rows[c][r - 1][lane] : p2carry[c][lane];
        const float dy = (has_down ? pn2[c] : 0.0f) - (has_up ? above : 0.0f);
        const float dx = (has_right ? pn1[c] : 0.0f) - (has_left ? before : 0.0f);
        const float v = xn[c] + P.dual.tau[c] * (dy + dx);
        if (valid) P.next[c * plane + here] = fminf(fmaxf((v + P.t * ends[c].z) * P.r, ends[c].x), ends[c].y);
      }
    }
    __syncthreads();
    issue(k + 2);  // every read of the slot is done
    if (warp == kRows - 1) {
      // The last row's w- and p2_n: the row above the next chunk.
#pragma unroll
      for (int c = 0; c < C; ++c) {
        if constexpr (TGV) {
          wcarry[c][0][lane] = wb1[c];
          wcarry[c][1][lane] = wb2[c];
        }
        p2carry[c][lane] = pn2[c];
      }
    }
  }
  if (failed && tid == 0 && P.dual.error != nullptr) atomicExch(P.dual.error, 1);
  if (failed) {
    for (int k = stopped; k < min(stopped + 2, chunks); ++k) barrier_wait(&bars[k & 1], (k >> 1) & 1);
  }
}

template <bool TGV, int C>
constexpr std::size_t shared_bytes() {
  constexpr int F = TGV ? 8 : 3;
  constexpr int PLANE = kBox * kSpan;
  constexpr int TOFF = (F * C * PLANE + 31) / 32 * 32;
  constexpr int STRIDE = (TOFF + C * PLANE + 31) / 32 * 32;
  return 2u * STRIDE * sizeof(float);
}

template <bool TGV, int C, bool COUPLED, int CR, int CC>
cudaError_t launch_one(const CUtensorMap& state, const CUtensorMap& tilde, const IterationParams& p, cudaStream_t s) {
  auto kernel = iteration_kernel<TGV, C, COUPLED, CR, CC>;
  constexpr std::size_t bytes = shared_bytes<TGV, C>();
  // Once per device: the shared-memory size above 48 KB, and how many CTAs the device holds at
  // once (its SMs times the CTAs an SM holds).
  static std::atomic<int> resident[64] = {};
  int device = 0;
  cudaGetDevice(&device);
  int slots = resident[device & 63].load();
  if (slots == 0) {
    cudaError_t e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(bytes));
    int per_sm = 0, sms = 0;
    if (e == cudaSuccess) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, 32 * kWarps, bytes);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    if (e != cudaSuccess) return e;
    slots = std::max(1, per_sm * sms);
    resident[device & 63].store(slots);
  }
  const int strips = (p.dual.g.columns + 31) / 32;
  const int best = strip_rows_for(p.dual.g, slots, 32);
  IterationParams q = p;
  q.strip_rows = best;
  const dim3 grid(strips, (p.dual.g.rows + best - 1) / best, 1);
  kernel<<<grid, 32 * kWarps, bytes, s>>>(state, tilde, q);
  return cudaGetLastError();
}

template <bool TGV, int C, bool COUPLED>
cudaError_t launch_cells(const CUtensorMap& state, const CUtensorMap& tilde, const IterationParams& p, int cr, int cc,
                         cudaStream_t s) {
  if constexpr (C == 1) {
    return launch_one<TGV, 1, COUPLED, 1, 1>(state, tilde, p, s);
  } else {
    if (cr == 1 && cc == 1) return launch_one<TGV, C, COUPLED, 1, 1>(state, tilde, p, s);
    if (cr == 2 && cc == 2) return launch_one<TGV, C, COUPLED, 2, 2>(state, tilde, p, s);
    if (cr == 1 && cc == 2) return launch_one<TGV, C, COUPLED, 1, 2>(state, tilde, p, s);
    if (cr == 2 && cc == 1) return launch_one<TGV, C, COUPLED, 2, 1>(state, tilde, p, s);
    return cudaErrorInvalidValue;
  }
}

template <bool TGV>
cudaError_t launch_channels(const CUtensorMap& state, const CUtensorMap& tilde, const IterationParams& p,
                            bool coupled, int cr, int cc, cudaStream_t s) {
  switch (p.dual.g.channels) {
    case 1: return launch_cells<TGV, 1, false>(state, tilde, p, 1, 1, s);
    case 3: return coupled ? launch_cells<TGV, 3, true>(state, tilde, p, cr, cc, s)
                           : launch_cells<TGV, 3, false>(state, tilde, p, cr, cc, s);
    default: return cudaErrorInvalidValue;
  }
}

template <bool TGV, int C, bool COUPLED>
cudaError_t launch_samples_one(const CUtensorMap& state, const CUtensorMap& tilde, const SamplesIterationParams& p,
                               cudaStream_t s) {
  auto kernel = samples_iteration_kernel<TGV, C, COUPLED>;
  constexpr std::size_t bytes = shared_bytes<TGV, C>();
  static std::atomic<int> resident[64] = {};
  int device = 0;
  cudaGetDevice(&device);
  int slots = resident[device & 63].load();
  if (slots == 0) {
    cudaError_t e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(bytes));
    int per_sm = 0, sms = 0;
    if (e == cudaSuccess) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, 32 * kWarps, bytes);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    if (e != cudaSuccess) return e;
    slots = std::max(1, per_sm * sms);
    resident[device & 63].store(slots);
  }
  const int strips = (p.dual.g.columns + 31) / 32;
  const int best = strip_rows_for(p.dual.g, slots, 32);
  SamplesIterationParams q = p;
  q.strip_rows = best;
  const dim3 grid(strips, (p.dual.g.rows + best - 1) / best, 1);
  kernel<<<grid, 32 * kWarps, bytes, s>>>(state, tilde, q);
  return cudaGetLastError();
}

}  // namespace

bool iteration_takes(const Geometry& g, const ComponentDevice* components, int count) {
  if (count != g.channels || (count != 1 && count != 3)) return false;
  if (components[0].cell_rows != 1 || components[0].cell_columns != 1) return false;
  int cr = 1, cc = 1;
  if (count == 3) {
    cr = components[1].cell_rows;
    cc = components[1].cell_columns;
    if (components[2].cell_rows != cr || components[2].cell_columns != cc) return false;
    if (cr < 1 || cr > 2 || cc < 1 || cc > 2) return false;
  }
  // Whole chunks, bands and blocks: the canvas is made of whole MCUs.
  return g.rows % (8 * cr) == 0 && g.columns % (8 * cc) == 0 && g.rows >= 8 && g.columns >= 8;
}

std::size_t iteration_shared_bytes(bool tgv, int channels) {
  if (channels == 1) return tgv ? shared_bytes<true, 1>() : shared_bytes<false, 1>();
  return tgv ? shared_bytes<true, 3>() : shared_bytes<false, 3>();
}

bool make_iteration_map(CUtensorMap& map, const float* planes, const Geometry& g, int count) {
  return make_box_map(map, planes, g, count, g.plane, kBox, kSpan);
}

cudaError_t launch_iteration(const CUtensorMap& state, const CUtensorMap& tilde, const IterationParams& p, bool tgv,
                             bool coupled, int cell_rows, int cell_columns, cudaStream_t stream) {
  return tgv ? launch_channels<true>(state, tilde, p, coupled, cell_rows, cell_columns, stream)
             : launch_channels<false>(state, tilde, p, coupled, cell_rows, cell_columns, stream);
}

bool samples_iteration_takes(const Geometry& g) { return g.channels == 1 || g.channels == 3; }

cudaError_t launch_samples_iteration(const CUtensorMap& state, const CUtensorMap& tilde,
                                     const SamplesIterationParams& p, bool tgv, bool coupled, cudaStream_t stream) {
  const int channels = p.dual.g.channels;
  if (channels == 1) {
    return tgv ? launch_samples_one<true, 1, false>(state, tilde, p, stream)
               : launch_samples_one<false, 1, false>(state, tilde, p, stream);
  }
  if (channels != 3) return cudaErrorInvalidValue;
  if (tgv) {
    return coupled ? launch_samples_one<true, 3, true>(state, tilde, p, stream)
                   : launch_samples_one<true, 3, false>(state, tilde, p, stream);
  }
  return coupled ? launch_samples_one<false, 3, true>(state, tilde, p, stream)
                 : launch_samples_one<false, 3, false>(state, tilde, p, stream);
}

}  // namespace urb
