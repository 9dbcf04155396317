// The unrolled TGV solve of greyscale pictures and its adjoint (sm_100a): N iterations of the
// method (docs/math.md 5, the same steps as the solver's kernels) from the solver's start, with
// the per-picture parameters alpha0, alpha1, tau and sigma as inputs, and the gradient of a loss
// of the last iterate x~_N with respect to them by reverse mode through the iterations.
//
// The forward map, iteration k = 1 .. N: P_k makes x~_k = prox(x + tau div p) from the state
// s_{k-1} = (x, p, w, r); for k < N, D_k makes s_k from x~_k and s_{k-1}:
//   x- = 2 x~ - x,  w~ = w + tau (p + div2 r),  w- = 2 w~ - w,
//   p~ = proj_alpha1(p + sigma (grad x- - w-)),  r~ = proj_alpha0,F(r + sigma E w-),
//   and every field relaxed with rho. s_0 = (x0, 0, grad x0, 0).
// The proximal map clips each coefficient of each 8x8 block: zeta = clip((e + t c) / (1 + t),
// a, b) with t = tau m_k (m_k the data term's weight of frequency k, of a flat block where the
// block is flat) and e the DCT of the block less the middle of its DC interval.
//
// P_k is a block kernel (a warp per block row, the transforms in registers); D_k a tile kernel
// fed by a bulk-tensor copy of s_{k-1} and x~_k with halos.
//
// The adjoint runs the iterations backwards: the adjoint of D_k (one tile kernel: the
// projections' Jacobians, then the transposes of E, grad and div2 over the tile, from shared
// memory), then of P_k (a block kernel: the DCT of the adjoint, the clip's mask, the inverse DCT,
// to the adjoint of v, which the next dual step undone reads for div's transpose). The states
// s_k are kept every `checkpoint_every` iterations by the forward pass; the backward pass
// recomputes each segment's states from its checkpoint. The parameters' gradients are sums
// over pixels and iterations, reduced per CTA and added in binary64.
#include <algorithm>
#include <atomic>
#include <cstdint>
#include <cstring>
#include <string>
#include <type_traits>
#include <vector>

#include <cuda_runtime.h>

#include "dct.cuh"
#include "kernels.hpp"
#include "unround.h"
#include "unround_b200.h"

namespace urb {

namespace {

constexpr unsigned kAll = 0xffffffffu;

struct Planes {
  float* x;
  float* p1;
  float* p2;
  float* w1;
  float* w2;
  float* r11;
  float* r22;
  float* r12;
};

// The constants of the problem and the parameters, for the kernels.
struct Problem {
  int images, rows, columns, blocks_down, blocks_across;
  std::size_t plane;  // images x rows x columns
  const float* lower;   // [image][block][64], the DC interval centred on its middle
  const float* upper;
  const float* centre;
  const float* middle;  // [image][block]
  const float* weight;  // [image][64]
  const float* flat_weight;
  const std::uint8_t* flat;  // [image][block]
  const float* alpha0;  // [image]
  const float* alpha1;
  const float* tau;
  const float* sigma;
  float rho;
};

__device__ __forceinline__ std::size_t at(const Problem& q, int z, int i, int j) {
  return (static_cast<std::size_t>(z) * q.rows + i) * q.columns + j;
}

__device__ __forceinline__ float ball(float square, float radius) {
  const float norm = sqrtf(square);
  return norm > radius ? radius / norm : 1.0f;
}

// Sums of a value over a CTA of 256 threads, added to a binary64 total.
__device__ __forceinline__ void add_sum(float value, double* total) {
  __shared__ float partial[8];
  double v = value;
  float f = static_cast<float>(v);
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) f += __shfl_down_sync(kAll, f, o);
  const int lane = (threadIdx.y * blockDim.x + threadIdx.x) & 31, warp = (threadIdx.y * blockDim.x + threadIdx.x) >> 5;
  if (lane == 0) partial[warp] = f;
  __syncthreads();
  if (warp == 0) {
    double t = lane < 8 ? static_cast<double>(partial[lane]) : 0.0;
#pragma unroll
    for (int o = 4; o > 0; o >>= 1) t += __shfl_down_sync(kAll, t, o);
    if (lane == 0) atomicAdd(total, t);
  }
  __syncthreads();
}

// ---- Forward.

__global__ void __launch_bounds__(256) start_kernel(Problem q, const float* x0, Planes s) {
  const int j = blockIdx.x * 32 + threadIdx.x, i = blockIdx.y * 8 + threadIdx.y, z = blockIdx.z;
  if (i >= q.rows || j >= q.columns) return;
  const std::size_t k = at(q, z, i, j);
  const float x = x0[k];
  s.x[k] = x;
  s.p1[k] = s.p2[k] = 0.0f;
  s.r11[k] = s.r22[k] = s.r12[k] = 0.0f;
  s.w1[k] = j + 1 < q.columns ? x0[k + 1] - x : 0.0f;
  s.w2[k] = i + 1 < q.rows ? x0[k + q.columns] - x : 0.0f;
}

// ---- The block kernels: a warp per block row of a strip of 32 columns (4 blocks), a lane per
// column; a CTA of 8 warps takes 8 block rows of the strip. The 2D transforms run in registers,
// 8 values a lane, with one transpose through the block's tile of the warp: forward2 takes the
// lane's column of its block and gives row m = lane % 8 of the coefficients (frequency
// k = 8 m + u at [u]); inverse2 takes that row and gives the lane's column back.
__device__ __forceinline__ void forward2(const float (&column)[8], float (&row)[8], float* t, int m) {
  float f[8], g[8];
  forward8(column, f);
  __syncwarp();
#pragma unroll
  for (int k = 0; k < 8; ++k) t[k * 9 + m] = f[k];
  __syncwarp();
#pragma unroll
  for (int u = 0; u < 8; ++u) g[u] = t[m * 9 + u];
  forward8(g, row);
}

__device__ __forceinline__ void inverse2(const float (&row)[8], float (&column)[8], float* t, int m) {
  float f[8], g[8];
  inverse8(row, f);
  __syncwarp();
#pragma unroll
  for (int n = 0; n < 8; ++n) t[m * 9 + n] = f[n];
  __syncwarp();
#pragma unroll
  for (int k = 0; k < 8; ++k) g[k] = t[k * 9 + m];
  inverse8(g, column);
}

// v = x + tau div p down the lane's column of block row `by` (column jc), and div p itself;
// div p = dy' p2 + dx' p1 by backward differences, the neighbour to the left from the lane
// beside.
__device__ __forceinline__ void column_v(const Problem& q, const Planes& s, int z, int by, int jc, float tau,
                                         float (&v)[8], float (&div)[8]) {
  const int lane = threadIdx.x, i0 = by * 8;
  float above = i0 > 0 ? s.p2[at(q, z, i0 - 1, jc)] : 0.0f;
#pragma unroll
  for (int r = 0; r < 8; ++r) {
    const int i = i0 + r;
    const std::size_t k = at(q, z, i, jc);
    const float p1 = s.p1[k], p2 = s.p2[k];
    float before = __shfl_up_sync(kAll, p1, 1);
    if (lane == 0) before = jc > 0 ? s.p1[k - 1] : 0.0f;
    const float dy = (i + 1 < q.rows ? p2 : 0.0f) - (i > 0 ? above : 0.0f);
    const float dx = (jc + 1 < q.columns ? p1 : 0.0f) - (jc > 0 ? before : 0.0f);
    div[r] = dy + dx;
    v[r] = s.x[k] + tau * div[r];
    above = p2;
  }
}

// The clip of row m of a block's coefficients, `e` their values: zeta = clip((e + t c) r, a, b),
// t = tau m_k (of a flat block where the block is flat), r = 1 / (1 + t); `inside` where the
// unclipped value lies strictly inside (a, b), and the pieces of d zeta / d tau there.
struct ClipRow {
  float zeta[8], r[8], weight[8], centre[8];
  bool inside[8];
};

__device__ __forceinline__ void clip_row(const Problem& q, int z, std::size_t block, int m, float tau,
                                         const float (&e)[8], ClipRow& out) {
  const std::size_t blocks = static_cast<std::size_t>(q.blocks_down) * q.blocks_across;
  const bool flat = q.flat[static_cast<std::size_t>(z) * blocks + block] != 0;
  const float* weights = (flat ? q.flat_weight : q.weight) + z * 64 + m * 8;
  const std::size_t c = (static_cast<std::size_t>(z) * blocks + block) * 64 + m * 8;
  float lower[8], upper[8];
#pragma unroll
  for (int h = 0; h < 2; ++h) {
    const float4 wv = *reinterpret_cast<const float4*>(weights + 4 * h);
    const float4 cv = *reinterpret_cast<const float4*>(q.centre + c + 4 * h);
    const float4 lv = *reinterpret_cast<const float4*>(q.lower + c + 4 * h);
    const float4 uv = *reinterpret_cast<const float4*>(q.upper + c + 4 * h);
    out.weight[4 * h] = wv.x, out.weight[4 * h + 1] = wv.y, out.weight[4 * h + 2] = wv.z, out.weight[4 * h + 3] = wv.w;
    out.centre[4 * h] = cv.x, out.centre[4 * h + 1] = cv.y, out.centre[4 * h + 2] = cv.z, out.centre[4 * h + 3] = cv.w;
    lower[4 * h] = lv.x, lower[4 * h + 1] = lv.y, lower[4 * h + 2] = lv.z, lower[4 * h + 3] = lv.w;
    upper[4 * h] = uv.x, upper[4 * h + 1] = uv.y, upper[4 * h + 2] = uv.z, upper[4 * h + 3] = uv.w;
  }
#pragma unroll
  for (int u = 0; u < 8; ++u) {
    const float t = tau * out.weight[u];
    out.r[u] = 1.0f / (1.0f + t);
    const float zz = (e[u] + t * out.centre[u]) * out.r[u];
    out.inside[u] = zz > lower[u] && zz < upper[u];
    out.zeta[u] = fminf(fmaxf(zz, lower[u]), upper[u]);
  }
}

__global__ void __launch_bounds__(256) primal_kernel(Problem q, Planes s, float* xt) {
  __shared__ float tiles[8][4][72];
  const int lane = threadIdx.x, warp = threadIdx.y, z = blockIdx.z;
  const int by = blockIdx.y * 8 + warp;
  if (by >= q.blocks_down) return;  // the whole warp; no CTA barrier follows
  const int j = blockIdx.x * 32 + lane;
  const bool in = j < q.columns;
  const int jc = in ? j : q.columns - 1, m = lane & 7;
  const std::size_t blocks = static_cast<std::size_t>(q.blocks_down) * q.blocks_across;
  const std::size_t block = static_cast<std::size_t>(by) * q.blocks_across + jc / 8;
  float* t = tiles[warp][lane >> 3];
  const float tau = q.tau[z];
  float v[8], div[8];
  column_v(q, s, z, by, jc, tau, v, div);
  const float middle = q.middle[static_cast<std::size_t>(z) * blocks + block];
#pragma unroll
  for (int r = 0; r < 8; ++r) v[r] -= middle;
  float e[8];
  forward2(v, e, t, m);
  ClipRow c;
  clip_row(q, z, block, m, tau, e, c);
  float back[8];
  inverse2(c.zeta, back, t, m);
  if (in) {
#pragma unroll
    for (int r = 0; r < 8; ++r) xt[at(q, z, by * 8 + r, j)] = back[r] + middle;
  }
}

// ---- Adjoint. `a` holds the adjoint of s_k (the dual step's output) and, as its ninth plane,
// that of v of the primal step P_{k+1} after it; the kernels write the adjoint of s_{k-1} into
// `b` and the adjoint of x~_k into `xt_bar`. Gradients: [0] alpha0, [1] alpha1, [2] tau,
// [3] sigma, each [image].
//
// The dual step's adjoint is one kernel over tiles of 16 rows x 32 columns. A tile's CTA loads,
// by two 4D bulk-tensor copies, the 9 planes of s_{k-1} and x~_k and the 9 of the adjoint with
// halos (2 rows above and 2 below, 4 columns each side: whole 16-byte words), and then in shared
// memory: w~ over the tile and a ring of 2 (1), the adjoints of the projections' points q and s
// over the tile and a ring of 1 (2), the adjoint of w~ over the tile and the ring's left column
// and upper row (3), and the tile's adjoints (4). A halo's values are recomputed by each tile
// that needs them; the gradients count the tile's own pixels only.
constexpr int kAdjointRows = 16;                 // a tile's rows
constexpr int kAdjointSpan = 40;                 // columns of a box: 4 + 32 + 4
constexpr int kStateRows = kAdjointRows + 4;     // s_{k-1}, x~_k: rows i0 - 2 .. i0 + 17
constexpr int kBarRows = kAdjointRows + 3;       // the adjoint: rows i0 - 1 .. i0 + 17
constexpr int kFields = 9;
constexpr int kTildeRows = kAdjointRows + 3, kTildeColumns = 36;  // (1): rows i0 - 2 .., columns j0 - 2 ..
constexpr int kPointRows = kAdjointRows + 2, kPointColumns = 34;  // (2): rows i0 - 1 .., columns j0 - 1 ..
constexpr int kBackRows = kAdjointRows + 1, kBackColumns = 33;    // (3): rows i0 - 1 .., columns j0 - 1 ..
constexpr int kStateFloats = kFields * kStateRows * kAdjointSpan;
constexpr int kBarFloats = kFields * kBarRows * kAdjointSpan;
// (1), (2) and (3) are kept in rows of kAdjointSpan, as the boxes are, and walked as rows x
// kAdjointSpan points (the columns past each one's width idle): a warp's 32 points are 32
// consecutive words of every array it reads or writes, across row ends too.
constexpr int kTildeFloats = 2 * kTildeRows * kAdjointSpan;
constexpr int kPointFloats = 5 * kPointRows * kAdjointSpan;
static_assert(2 * kBackRows * kAdjointSpan <= kTildeFloats, "(3) reuses the space of (1)");
static_assert(kStateFloats % 32 == 0, "the adjoint's box starts 128-byte aligned");
constexpr std::size_t kAdjointShared =
    static_cast<std::size_t>(kStateFloats + kBarFloats + kTildeFloats + kPointFloats) * sizeof(float);

__device__ __forceinline__ unsigned shared_address(const void* p) {
  return static_cast<unsigned>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void load_fields(float* to, const CUtensorMap* map, std::uint64_t* bar, int x, int y,
                                            int z) {
  asm volatile(
      "cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, "
      "%5}], [%6];" ::"r"(shared_address(to)),
      "l"(map), "r"(x), "r"(y), "r"(z), "r"(0), "r"(shared_address(bar))
      : "memory");
}

__device__ __forceinline__ bool wait_phase(std::uint64_t* bar, unsigned parity) {
  for (long long n = 0; n < (1LL << 22); ++n) {
    unsigned done;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(done)
        : "r"(shared_address(bar)), "r"(parity)
        : "memory");
    if (done != 0) return true;
  }
  return false;
}

__global__ void __launch_bounds__(256) dual_adjoint_kernel(const __grid_constant__ CUtensorMap state_map,
                                                           const __grid_constant__ CUtensorMap bar_map, Problem q,
                                                           Planes b, float* xt_bar, double* grads) {
  extern __shared__ __align__(128) float shared[];
  __shared__ __align__(8) std::uint64_t loaded[2];  // [0] s_{k-1} and x~_k, [1] the adjoint
  float* const S = shared;                       // [field][row][column], row i0 - 2 + r, column j0 - 4 + c
  float* const A = S + kStateFloats;             // [field][row][column], row i0 - 1 + r, column j0 - 4 + c
  float* const T = A + kBarFloats;               // (1) w~, then (3) the adjoint of w~
  float* const L = T + kTildeFloats;             // (2) q^1, q^2, s^11, s^22, s^12
  const int tid = threadIdx.y * 32 + threadIdx.x;
  const int z = blockIdx.z, i0 = blockIdx.y * kAdjointRows, j0 = blockIdx.x * 32;
  const int H = q.rows, W = q.columns;
  const float rho = q.rho, rest = 1.0f - q.rho, tau = q.tau[z], sigma = q.sigma[z];
  const float alpha0 = q.alpha0[z], alpha1 = q.alpha1[z];
  if (tid == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(shared_address(&loaded[0])) : "memory");
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(shared_address(&loaded[1])) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
  // Two copies on two barriers: (1) needs only the first, which lands while the second is
  // still on its way.
  if (tid == 0) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(shared_address(&loaded[0])),
                 "r"(static_cast<unsigned>(kStateFloats * sizeof(float)))
                 : "memory");
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(shared_address(&loaded[1])),
                 "r"(static_cast<unsigned>(kBarFloats * sizeof(float)))
                 : "memory");
    load_fields(S, &state_map, &loaded[0], j0 - 4, i0 - 2, z);
    load_fields(A, &bar_map, &loaded[1], j0 - 4, i0 - 1, z);
  }
  // A copy that did not land: the gradients say so, and no copy may still be writing into the
  // CTA's shared memory when it leaves (each barrier waited for once more, bounded).
  auto give_up = [&]() {
    if (tid == 0) {
      atomicAdd(grads + 3 * q.images + z, static_cast<double>(__int_as_float(0x7fc00000)));
      wait_phase(&loaded[0], 0);
      wait_phase(&loaded[1], 0);
    }
  };
  const bool ready = wait_phase(&loaded[0], 0);
  if (__syncthreads_or(!ready)) {
    give_up();
    return;
  }
  auto s_at = [&](int f, int i, int j) -> float { return S[(f * kStateRows + i - i0 + 2) * kAdjointSpan + j - j0 + 4]; };
  auto a_at = [&](int f, int i, int j) -> float { return A[(f * kBarRows + i - i0 + 1) * kAdjointSpan + j - j0 + 4]; };
  auto t_at = [&](int f, int i, int j) -> float& { return T[(f * kTildeRows + i - i0 + 2) * kAdjointSpan + j - j0 + 2]; };
  auto l_at = [&](int f, int i, int j) -> float& { return L[(f * kPointRows + i - i0 + 1) * kAdjointSpan + j - j0 + 1]; };
  auto tb_at = [&](int f, int i, int j) -> float& { return T[(f * kBackRows + i - i0 + 1) * kAdjointSpan + j - j0 + 1]; };
  enum { X = 0, P1, P2, W1, W2, R11, R22, R12, EXTRA };  // EXTRA: x~ in S, v^ in A
  float g_alpha0 = 0.0f, g_alpha1 = 0.0f, g_sigma = 0.0f, g_tau = 0.0f;
  // A tile whose halos lie inside the picture (rows i0 - 2 .. i0 + 17, columns j0 - 2 .. j0 + 34)
  // passes every bounds test below: IN states that, and the tests fold away.
  const bool interior = i0 >= 2 && j0 >= 2 && i0 + 17 < H && j0 + 34 < W;
  bool failed = false;  // the same in every thread: set after a CTA-wide vote
  auto tile = [&](auto kind) {
    constexpr bool IN = decltype(kind)::value;

    // (1) w~ = w + tau (p + div2 r), div2 r by forward differences, and w- = 2 w~ - w.
    for (int n = tid; n < kTildeRows * kAdjointSpan; n += 256) {
      if (n % kAdjointSpan >= kTildeColumns) continue;
      const int i = i0 - 2 + n / kAdjointSpan, j = j0 - 2 + n % kAdjointSpan;
      const float r11 = s_at(R11, i, j), r22 = s_at(R22, i, j), r12 = s_at(R12, i, j);
      float d1 = IN || j + 1 < W ? s_at(R11, i, j + 1) - r11 : 0.0f;
      float d2 = IN || j + 1 < W ? s_at(R12, i, j + 1) - r12 : 0.0f;
      d1 = d1 + (IN || i + 1 < H ? s_at(R12, i + 1, j) - r12 : 0.0f);
      d2 = d2 + (IN || i + 1 < H ? s_at(R22, i + 1, j) - r22 : 0.0f);
      // Kept as w- = 2 w~ - w, the only form (2) reads.
      const float w1 = s_at(W1, i, j), w2 = s_at(W2, i, j);
      const float tilde1 = w1 + tau * (s_at(P1, i, j) + d1), tilde2 = w2 + tau * (s_at(P2, i, j) + d2);
      t_at(0, i, j) = 2.0f * tilde1 - w1;
      t_at(1, i, j) = 2.0f * tilde2 - w2;
    }
    const bool adjoint_ready = wait_phase(&loaded[1], 0);
    if (__syncthreads_or(!adjoint_ready)) {
      failed = true;
      return;
    }

    // (2) The points q = p + sigma (grad x- - w-) and s = r + sigma E w-, and the adjoints of q
    // and s through the projections onto the balls (d/d alpha1, d/d alpha0 and d/d sigma beside).
    for (int n = tid; n < kPointRows * kAdjointSpan; n += 256) {
      if (n % kAdjointSpan >= kPointColumns) continue;
      const int i = i0 - 1 + n / kAdjointSpan, j = j0 - 1 + n % kAdjointSpan;
      const bool right = IN || j + 1 < W, down = IN || i + 1 < H;
      const float bar = 2.0f * s_at(EXTRA, i, j) - s_at(X, i, j);
      const float g1 = right ? (2.0f * s_at(EXTRA, i, j + 1) - s_at(X, i, j + 1)) - bar : 0.0f;
      const float g2 = down ? (2.0f * s_at(EXTRA, i + 1, j) - s_at(X, i + 1, j)) - bar : 0.0f;
      const float b1 = t_at(0, i, j);
      const float b2 = t_at(1, i, j);
      const float q1 = s_at(P1, i, j) + sigma * (g1 - b1);
      const float q2 = s_at(P2, i, j) + sigma * (g2 - b2);
      float l1 = 0.0f, l2 = 0.0f, u1 = 0.0f, u2 = 0.0f;
      if (IN || j > 0) {
        l1 = t_at(0, i, j - 1);
        l2 = t_at(1, i, j - 1);
      }
      if (IN || i > 0) {
        u1 = t_at(0, i - 1, j);
        u2 = t_at(1, i - 1, j);
      }
      const float own1x = right ? b1 : 0.0f, own2x = right ? b2 : 0.0f;
      const float own1y = down ? b1 : 0.0f, own2y = down ? b2 : 0.0f;
      const float e11 = own1x - l1, e22 = own2y - u2, e12 = 0.5f * ((own1y - u1) + (own2x - l2));
      const float s11 = s_at(R11, i, j) + sigma * e11;
      const float s22 = s_at(R22, i, j) + sigma * e22;
      const float s12 = s_at(R12, i, j) + sigma * e12;
      // The adjoint of p of s_k: that of the relaxation's p and of P_{k+1}'s v = x + tau div p,
      // p^ += tau div^T v^ = -tau grad v^.
      const float v = a_at(EXTRA, i, j);
      float ap1 = a_at(P1, i, j), ap2 = a_at(P2, i, j);
      if (right) ap1 += -tau * (a_at(EXTRA, i, j + 1) - v);
      if (down) ap2 += -tau * (a_at(EXTRA, i + 1, j) - v);
      const float pb1 = rho * ap1, pb2 = rho * ap2;
      // The projections' branches compare squares: |q| > alpha where |q|^2 > alpha^2, but for
      // ties within rounding, where the map is continuous; 1 / |q| by the approximate rsqrt.
      float qb1 = pb1, qb2 = pb2, ga1 = 0.0f;
      const float sq = q1 * q1 + q2 * q2;
      if (sq > alpha1 * alpha1) {
        const float dot = q1 * pb1 + q2 * pb2, inverse = rsqrtf(sq);
        const float f = alpha1 * inverse, h = dot * inverse * inverse;
        qb1 = f * (pb1 - q1 * h);
        qb2 = f * (pb2 - q2 * h);
        ga1 = dot * inverse;
      }
      const float rb11 = rho * a_at(R11, i, j), rb22 = rho * a_at(R22, i, j), rb12 = rho * a_at(R12, i, j);
      float sb11 = rb11, sb22 = rb22, sb12 = rb12, ga0 = 0.0f;
      const float ss = s11 * s11 + s22 * s22 + 2.0f * (s12 * s12);
      if (ss > alpha0 * alpha0) {
        const float dot = s11 * rb11 + s22 * rb22 + s12 * rb12, inverse = rsqrtf(ss);
        const float f = alpha0 * inverse, h = dot * inverse * inverse;
        sb11 = f * (rb11 - s11 * h);
        sb22 = f * (rb22 - s22 * h);
        sb12 = f * (rb12 - 2.0f * s12 * h);
        ga0 = dot * inverse;
      }
      l_at(0, i, j) = qb1;
      l_at(1, i, j) = qb2;
      l_at(2, i, j) = sb11;
      l_at(3, i, j) = sb22;
      l_at(4, i, j) = sb12;
      if (i >= i0 && i < i0 + kAdjointRows && j >= j0 && j < j0 + 32 && (IN || (i < H && j < W))) {
        g_alpha0 += ga0;
        g_alpha1 += ga1;
        g_sigma += qb1 * (g1 - b1) + qb2 * (g2 - b2) + sb11 * e11 + sb22 * e22 + sb12 * e12;
      }
    }
    __syncthreads();

    // (3) The adjoint of w~: that of w- is -sigma q^ + sigma E^T s^ (E^T gathering s^ of the pixel
    // and of its right and lower ones), and w~ = (w- + w) / 2 gives it twice, beside the
    // relaxation's rho w'^. Over the tile and the column to its left and the row above it.
    auto w_minus_bar = [&](int i, int j, float& wb1, float& wb2) {
      wb1 = -sigma * l_at(0, i, j);
      wb2 = -sigma * l_at(1, i, j);
      float e1 = 0.0f, e2 = 0.0f;
      if (IN || j + 1 < W) {
        e1 += l_at(2, i, j) - l_at(2, i, j + 1);
        e2 += 0.5f * (l_at(4, i, j) - l_at(4, i, j + 1));
      }
      if (IN || i + 1 < H) {
        e2 += l_at(3, i, j) - l_at(3, i + 1, j);
        e1 += 0.5f * (l_at(4, i, j) - l_at(4, i + 1, j));
      }
      wb1 += sigma * e1;
      wb2 += sigma * e2;
    };
    for (int n = tid; n < kBackRows * kAdjointSpan; n += 256) {
      if (n % kAdjointSpan >= kBackColumns) continue;
      const int i = i0 - 1 + n / kAdjointSpan, j = j0 - 1 + n % kAdjointSpan;
      float wb1, wb2;
      w_minus_bar(i, j, wb1, wb2);
      tb_at(0, i, j) = rho * a_at(W1, i, j) + 2.0f * wb1;
      tb_at(1, i, j) = rho * a_at(W2, i, j) + 2.0f * wb2;
    }
    __syncthreads();

    // (4) The tile's adjoints of s_{k-1} and of x~_k.
    for (int n = tid; n < kAdjointRows * 32; n += 256) {
      const int i = i0 + n / 32, j = j0 + n % 32;
      if (!IN && (i >= H || j >= W)) continue;
      const std::size_t k = at(q, z, i, j);
      const bool right = IN || j + 1 < W, down = IN || i + 1 < H;
      const float tb1 = tb_at(0, i, j), tb2 = tb_at(1, i, j);
      const float v = a_at(EXTRA, i, j);
      float ap1 = a_at(P1, i, j), ap2 = a_at(P2, i, j);
      if (right) ap1 += -tau * (a_at(EXTRA, i, j + 1) - v);
      if (down) ap2 += -tau * (a_at(EXTRA, i + 1, j) - v);
      // w^ = (1 - rho) w'^ - w-^ + w~^, and w~^ = rho w'^ + 2 w-^ gives w-^ from w~^.
      b.w1[k] = fmaf(rest + 0.5f * rho, a_at(W1, i, j), 0.5f * tb1);
      b.w2[k] = fmaf(rest + 0.5f * rho, a_at(W2, i, j), 0.5f * tb2);
      b.p1[k] = rest * ap1 + l_at(0, i, j) + tau * tb1;
      b.p2[k] = rest * ap2 + l_at(1, i, j) + tau * tb2;
      // r^: the relaxation's, s^, and div2^T of d^ = tau w~^ (w~^ of the pixel and of its left
      // and upper ones).
      const float l1 = IN || j > 0 ? tb_at(0, i, j - 1) : 0.0f, l2 = IN || j > 0 ? tb_at(1, i, j - 1) : 0.0f;
      const float u1 = IN || i > 0 ? tb_at(0, i - 1, j) : 0.0f, u2 = IN || i > 0 ? tb_at(1, i - 1, j) : 0.0f;
      const float db1 = tau * tb1, db2 = tau * tb2;
      const float div11 = tau * l1 - (right ? db1 : 0.0f);
      const float div12 = tau * u1 - (down ? db1 : 0.0f) + tau * l2 - (right ? db2 : 0.0f);
      const float div22 = tau * u2 - (down ? db2 : 0.0f);
      b.r11[k] = rest * a_at(R11, i, j) + l_at(2, i, j) + div11;
      b.r22[k] = rest * a_at(R22, i, j) + l_at(3, i, j) + div22;
      b.r12[k] = rest * a_at(R12, i, j) + l_at(4, i, j) + div12;
      // d/dtau of w~ = p + div2 r.
      const float r11 = s_at(R11, i, j), r22 = s_at(R22, i, j), r12 = s_at(R12, i, j);
      float d1 = right ? s_at(R11, i, j + 1) - r11 : 0.0f;
      float d2 = right ? s_at(R12, i, j + 1) - r12 : 0.0f;
      d1 = d1 + (down ? s_at(R12, i + 1, j) - r12 : 0.0f);
      d2 = d2 + (down ? s_at(R22, i + 1, j) - r22 : 0.0f);
      g_tau += tb1 * (s_at(P1, i, j) + d1) + tb2 * (s_at(P2, i, j) + d2);
      // The adjoint of x- : grad^T (sigma q^) = -div (sigma q^).
      const float div = (right ? l_at(0, i, j) : 0.0f) - (IN || j > 0 ? l_at(0, i, j - 1) : 0.0f) +
                        (down ? l_at(1, i, j) : 0.0f) - (IN || i > 0 ? l_at(1, i - 1, j) : 0.0f);
      const float xbb = -sigma * div;
      const float ax = a_at(X, i, j) + v;
      xt_bar[k] = rho * ax + 2.0f * xbb;
      b.x[k] = rest * ax - xbb;
    }
  };
  if (interior) {
    tile(std::true_type{});
  } else {
    tile(std::false_type{});
  }
  if (failed) {
    give_up();
    return;
  }
  add_sum(g_alpha0, grads + 0 * q.images + z);
  add_sum(g_alpha1, grads + 1 * q.images + z);
  add_sum(g_tau, grads + 2 * q.images + z);
  add_sum(g_sigma, grads + 3 * q.images + z);
}

// The dual step D_k as tiles of 16 rows x 32 columns: s_{k-1} and x~_k (9 planes) with a halo
// of a row above and below and 4 columns each side by one 4D bulk-tensor copy, w~ over the tile
// and the column to its left and the row above it in shared memory, then each pixel's step:
// x- = 2 x~ - x, w- = 2 w~ - w, the points q and s and their projections, and the relaxation.
constexpr int kForwardRows = kAdjointRows + 2;  // rows i0 - 1 .. i0 + 16
constexpr int kForwardFloats = kFields * kForwardRows * kAdjointSpan;
constexpr int kForwardTildeRows = kAdjointRows + 1, kForwardTildeColumns = 33;
constexpr int kForwardTildeFloats = 2 * kForwardTildeRows * kAdjointSpan;  // rows of kAdjointSpan, as the box
constexpr std::size_t kForwardShared = static_cast<std::size_t>(kForwardFloats + kForwardTildeFloats) * sizeof(float);

__global__ void __launch_bounds__(256) dual_tile_kernel(const __grid_constant__ CUtensorMap state_map, Problem q,
                                                        Planes out) {
  extern __shared__ __align__(128) float shared[];
  __shared__ __align__(8) std::uint64_t loaded;
  float* const S = shared;                    // [field][row][column], row i0 - 1 + r, column j0 - 4 + c
  float* const T = S + kForwardFloats;        // w~, row i0 - 1 + r, column j0 - 1 + c
  const int lane = threadIdx.x, warp = threadIdx.y, tid = warp * 32 + lane;
  const int z = blockIdx.z, i0 = blockIdx.y * kAdjointRows, j0 = blockIdx.x * 32;
  const int H = q.rows, W = q.columns;
  const float rho = q.rho, rest = 1.0f - q.rho, tau = q.tau[z], sigma = q.sigma[z];
  const float alpha0 = q.alpha0[z], alpha1 = q.alpha1[z];
  if (tid == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(shared_address(&loaded)) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
  if (tid == 0) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(shared_address(&loaded)),
                 "r"(static_cast<unsigned>(kForwardFloats * sizeof(float)))
                 : "memory");
    load_fields(S, &state_map, &loaded, j0 - 4, i0 - 1, z);
  }
  const bool ready = wait_phase(&loaded, 0);
  if (__syncthreads_or(!ready)) {
    // The load did not land: the tile's x is not a number, and no copy may still be writing
    // into the CTA's shared memory when it leaves.
    for (int rr = warp; rr < kAdjointRows; rr += 8) {
      const int i = i0 + rr, j = j0 + lane;
      if (i < H && j < W) out.x[at(q, z, i, j)] = __int_as_float(0x7fc00000);
    }
    if (tid == 0) wait_phase(&loaded, 0);
    return;
  }
  auto s_at = [&](int f, int i, int j) -> float { return S[(f * kForwardRows + i - i0 + 1) * kAdjointSpan + j - j0 + 4]; };
  auto t_at = [&](int f, int i, int j) -> float& { return T[(f * kForwardTildeRows + i - i0 + 1) * kAdjointSpan + j - j0 + 1]; };
  enum { X = 0, P1, P2, W1, W2, R11, R22, R12, XT };
  // w~ = w + tau (p + div2 r), div2 r by forward differences.
  for (int n = tid; n < kForwardTildeRows * kAdjointSpan; n += 256) {
    if (n % kAdjointSpan >= kForwardTildeColumns) continue;
    const int i = i0 - 1 + n / kAdjointSpan, j = j0 - 1 + n % kAdjointSpan;
    const float r11 = s_at(R11, i, j), r22 = s_at(R22, i, j), r12 = s_at(R12, i, j);
    float d1 = j + 1 < W ? s_at(R11, i, j + 1) - r11 : 0.0f;
    float d2 = j + 1 < W ? s_at(R12, i, j + 1) - r12 : 0.0f;
    d1 = d1 + (i + 1 < H ? s_at(R12, i + 1, j) - r12 : 0.0f);
    d2 = d2 + (i + 1 < H ? s_at(R22, i + 1, j) - r22 : 0.0f);
    t_at(0, i, j) = s_at(W1, i, j) + tau * (s_at(P1, i, j) + d1);
    t_at(1, i, j) = s_at(W2, i, j) + tau * (s_at(P2, i, j) + d2);
  }
  __syncthreads();
  for (int rr = warp; rr < kAdjointRows; rr += 8) {
    const int i = i0 + rr, j = j0 + lane;
    if (i >= H || j >= W) continue;
    const bool right = j + 1 < W, down = i + 1 < H;
    const float xt = s_at(XT, i, j), x = s_at(X, i, j);
    const float bar = 2.0f * xt - x;
    const float g1 = right ? (2.0f * s_at(XT, i, j + 1) - s_at(X, i, j + 1)) - bar : 0.0f;
    const float g2 = down ? (2.0f * s_at(XT, i + 1, j) - s_at(X, i + 1, j)) - bar : 0.0f;
    const float t1 = t_at(0, i, j), t2 = t_at(1, i, j), w1 = s_at(W1, i, j), w2 = s_at(W2, i, j);
    const float b1 = 2.0f * t1 - w1, b2 = 2.0f * t2 - w2;
    const float p1 = s_at(P1, i, j), p2 = s_at(P2, i, j);
    const float q1 = p1 + sigma * (g1 - b1);
    const float q2 = p2 + sigma * (g2 - b2);
    float l1 = 0.0f, l2 = 0.0f, u1 = 0.0f, u2 = 0.0f;
    if (j > 0) {
      l1 = 2.0f * t_at(0, i, j - 1) - s_at(W1, i, j - 1);
      l2 = 2.0f * t_at(1, i, j - 1) - s_at(W2, i, j - 1);
    }
    if (i > 0) {
      u1 = 2.0f * t_at(0, i - 1, j) - s_at(W1, i - 1, j);
      u2 = 2.0f * t_at(1, i - 1, j) - s_at(W2, i - 1, j);
    }
    const float own1x = right ? b1 : 0.0f, own2x = right ? b2 : 0.0f;
    const float own1y = down ? b1 : 0.0f, own2y = down ? b2 : 0.0f;
    const float e11 = own1x - l1, e22 = own2y - u2, e12 = 0.5f * ((own1y - u1) + (own2x - l2));
    const float r11 = s_at(R11, i, j), r22 = s_at(R22, i, j), r12 = s_at(R12, i, j);
    const float s11 = r11 + sigma * e11, s22 = r22 + sigma * e22, s12 = r12 + sigma * e12;
    const float sp = ball(q1 * q1 + q2 * q2, alpha1);
    const float sr = ball(s11 * s11 + s22 * s22 + 2.0f * (s12 * s12), alpha0);
    const std::size_t k = at(q, z, i, j);
    out.x[k] = rho * xt + rest * x;
    out.p1[k] = rho * (q1 * sp) + rest * p1;
    out.p2[k] = rho * (q2 * sp) + rest * p2;
    out.w1[k] = rho * t1 + rest * w1;
    out.w2[k] = rho * t2 + rest * w2;
    out.r11[k] = rho * (s11 * sr) + rest * r11;
    out.r22[k] = rho * (s22 * sr) + rest * r22;
    out.r12[k] = rho * (s12 * sr) + rest * r12;
  }
}

// The primal step's adjoint, per block: from the adjoint of x~ (`xt_bar`) the adjoint of v.
// x~ = C^T zeta C + middle and e = C (v - middle) C^T, so zeta^ = C x~^ C^T and v^ = C^T e^ C.
__global__ void __launch_bounds__(256) primal_adjoint_block(Problem q, Planes s, const float* xt_bar, float* vbar,
                                                            double* grads) {
  __shared__ float tiles[8][4][72];
  const int lane = threadIdx.x, warp = threadIdx.y, z = blockIdx.z;
  const int by_raw = blockIdx.y * 8 + warp;
  const bool active = by_raw < q.blocks_down;  // every warp joins the CTA's sum
  const int by = active ? by_raw : 0;
  const int j = blockIdx.x * 32 + lane;
  const bool in = active && j < q.columns;
  const int jc = j < q.columns ? j : q.columns - 1, m = lane & 7;
  const std::size_t blocks = static_cast<std::size_t>(q.blocks_down) * q.blocks_across;
  const std::size_t block = static_cast<std::size_t>(by) * q.blocks_across + jc / 8;
  float* t = tiles[warp][lane >> 3];
  const float tau = q.tau[z];
  float v[8], div[8], xb[8];
  column_v(q, s, z, by, jc, tau, v, div);
  const float middle = q.middle[static_cast<std::size_t>(z) * blocks + block];
#pragma unroll
  for (int r = 0; r < 8; ++r) {
    v[r] -= middle;
    xb[r] = in ? xt_bar[at(q, z, by * 8 + r, j)] : 0.0f;
  }
  float e[8], zb[8];
  forward2(v, e, t, m);
  forward2(xb, zb, t, m);
  ClipRow c;
  clip_row(q, z, block, m, tau, e, c);
  // zeta = (e + t c) r inside the interval, t = tau m, r = 1 / (1 + t): d zeta / d e = r and
  // d zeta / d tau = m (c - e) r^2; outside it zeta is an end of the interval.
  float eb[8], g_tau = 0.0f;
#pragma unroll
  for (int u = 0; u < 8; ++u) {
    eb[u] = c.inside[u] ? c.r[u] * zb[u] : 0.0f;
    g_tau += c.inside[u] ? zb[u] * c.weight[u] * (c.centre[u] - e[u]) * (c.r[u] * c.r[u]) : 0.0f;
  }
  float vb[8];
  inverse2(eb, vb, t, m);
  // d v / d tau = div p.
  if (in) {
#pragma unroll
    for (int r = 0; r < 8; ++r) {
      vbar[at(q, z, by * 8 + r, j)] = vb[r];
      g_tau += vb[r] * div[r];
    }
  } else {
    g_tau = 0.0f;
  }
  add_sum(g_tau, grads + 2 * q.images + z);
}

// ---- Host side.

Planes planes_of(float* base, std::size_t plane) {
  return Planes{base, base + plane, base + 2 * plane, base + 3 * plane, base + 4 * plane,
                base + 5 * plane, base + 6 * plane, base + 7 * plane};
}

Problem problem_of(const unround_b200_unrolled& u, const float* alpha0, const float* alpha1, const float* tau,
                   const float* sigma) {
  Problem q;
  q.images = static_cast<int>(u.images);
  q.rows = static_cast<int>(u.rows);
  q.columns = static_cast<int>(u.columns);
  q.blocks_down = q.rows / 8;
  q.blocks_across = q.columns / 8;
  q.plane = static_cast<std::size_t>(u.images) * u.rows * u.columns;
  q.lower = u.lower;
  q.upper = u.upper;
  q.centre = u.centre;
  q.middle = u.middle;
  q.weight = u.weight;
  q.flat_weight = u.flat_weight;
  q.flat = u.flat;
  q.alpha0 = alpha0;
  q.alpha1 = alpha1;
  q.tau = tau;
  q.sigma = sigma;
  q.rho = u.relaxation;
  return q;
}

dim3 pixel_grid(const Problem& q) {
  return dim3((q.columns + 31) / 32, (q.rows + 7) / 8, q.images);
}

// The block kernels' grid: a CTA 8 block rows of a strip of 32 columns.
dim3 block_grid(const Problem& q) {
  return dim3((q.columns + 31) / 32, (q.blocks_down + 7) / 8, q.images);
}

// The tiled dual step's and its adjoint's grid: a CTA a tile of kAdjointRows x 32.
dim3 tile_grid(const Problem& q) {
  return dim3((q.columns + 31) / 32, (q.rows + kAdjointRows - 1) / kAdjointRows, q.images);
}

// The map of 9 planes (a state and the x~ after it) for the tiled dual step.
bool make_forward_map(CUtensorMap& map, const float* base, const Problem& q) {
  return make_fields_map(map, base, q.columns, q.rows, q.images, 9, q.plane, kAdjointSpan, kForwardRows);
}

std::string check(const unround_b200_unrolled* u) {
  if (u == nullptr) return "the problem is a null pointer";
  if (u->images == 0 || u->rows == 0 || u->columns == 0) return "the problem has pictures of rows and columns";
  if (u->rows % 8 != 0 || u->columns % 8 != 0) return "the canvas is whole 8x8 blocks";
  if (u->iterations == 0) return "at least one iteration";
  if (u->checkpoint_every == 0) return "checkpoints every one or more iterations";
  if (u->rows > 65535u * 8u || u->images > 65535u) return "too many rows or pictures for one launch";
  if (u->lower == nullptr || u->upper == nullptr || u->centre == nullptr || u->middle == nullptr ||
      u->weight == nullptr || u->flat_weight == nullptr || u->flat == nullptr || u->start == nullptr) {
    return "the problem's arrays are not null pointers";
  }
  return {};
}

void tell(char* buffer, std::size_t size, const std::string& text) {
  if (buffer == nullptr || size == 0) return;
  const std::size_t end = std::min(text.size(), size - 1);
  std::memcpy(buffer, text.data(), end);
  buffer[end] = 0;
}

// The dual step's adjoint takes more than 48 KB of shared memory: allowed once per device.
bool prepare_dual_adjoint() {
  static std::atomic<unsigned long long> configured{0};
  int device = 0;
  if (cudaGetDevice(&device) != cudaSuccess) return false;
  const unsigned long long bit = 1ull << (device & 63);
  if ((configured.load() & bit) != 0) return true;
  if (cudaFuncSetAttribute(dual_adjoint_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           static_cast<int>(kAdjointShared)) != cudaSuccess) {
    return false;
  }
  configured.fetch_or(bit);
  return true;
}

std::uint64_t checkpoints_of(const unround_b200_unrolled& u) {
  // s_0, s_K, s_2K, ... up to s_{N-1}.
  return (u.iterations - 1) / u.checkpoint_every + 1;
}

}  // namespace

}  // namespace urb

using urb::Planes;

// Storage. A checkpoint c holds s_{cK} and x~_{cK+1} (9 planes), both written by the forward pass
// where they are made (no copies). The forward pass's other states ping-pong through the first
// 18 planes of the workspace (a state and the x~ after it each). The backward pass recomputes a
// segment's states s_{k0+1} .. s_{k0+K-1} and their x~ into K - 1 slots of 9 planes, and keeps
// two adjoints of a state (each followed by that of v of the primal step after it) and the
// adjoint of x~: 9 (K - 1) + 19 planes, never fewer than the forward pass's 18.
extern "C" uint64_t unround_b200_unrolled_checkpoint_floats(const unround_b200_unrolled* problem) {
  if (!urb::check(problem).empty()) return 0;
  return urb::checkpoints_of(*problem) * 9 * problem->images * problem->rows * problem->columns;
}

extern "C" uint64_t unround_b200_unrolled_workspace_floats(const unround_b200_unrolled* problem) {
  if (!urb::check(problem).empty()) return 0;
  const std::uint64_t plane = problem->images * problem->rows * problem->columns;
  return (9 * (problem->checkpoint_every - 1) + 19) * plane;
}

extern "C" unround_status unround_b200_unrolled_forward(const unround_b200_unrolled* problem, const float* alpha0,
                                                        const float* alpha1, const float* tau, const float* sigma,
                                                        float* checkpoints, float* workspace, float* output,
                                                        void* stream, char* message, size_t message_size) {
  const std::string wrong = urb::check(problem);
  if (!wrong.empty()) {
    urb::tell(message, message_size, wrong);
    return UNROUND_ERROR_ARGUMENT;
  }
  if (alpha0 == nullptr || alpha1 == nullptr || tau == nullptr || sigma == nullptr || checkpoints == nullptr ||
      workspace == nullptr || output == nullptr) {
    urb::tell(message, message_size, "the parameters, checkpoints, workspace and output are not null pointers");
    return UNROUND_ERROR_ARGUMENT;
  }
  const cudaStream_t on = static_cast<cudaStream_t>(stream);
  const urb::Problem q = urb::problem_of(*problem, alpha0, alpha1, tau, sigma);
  const std::size_t plane = q.plane;
  const std::uint64_t n = problem->iterations, every = problem->checkpoint_every;
  float* const spare[2] = {workspace, workspace + 9 * plane};
  // The dual steps read the 9 planes of s_{k-1} and x~_k by bulk-tensor copies: a map of each
  // checkpoint and of each spare.
  const std::uint64_t segments = urb::checkpoints_of(*problem);
  std::vector<CUtensorMap> checkpoint_maps(segments);
  CUtensorMap spare_maps[2];
  bool mapped = true;
  for (std::uint64_t c = 0; c < segments && mapped; ++c) {
    mapped = urb::make_forward_map(checkpoint_maps[c], checkpoints + c * 9 * plane, q);
  }
  for (int c = 0; c < 2 && mapped; ++c) mapped = urb::make_forward_map(spare_maps[c], spare[c], q);
  if (!mapped) {
    urb::tell(message, message_size, "the device's bulk-tensor copies could not be set up for the dual steps");
    return UNROUND_ERROR_INTERNAL;
  }
  const dim3 grid = urb::pixel_grid(q), block(32, 8), tiles = urb::tile_grid(q);
  // s_{k-1} and then x~_k live at `current`: 9 planes.
  float* current = checkpoints;
  const CUtensorMap* current_map = &checkpoint_maps[0];
  urb::start_kernel<<<grid, block, 0, on>>>(q, problem->start, urb::planes_of(current, plane));
  for (std::uint64_t k = 1; k <= n; ++k) {
    urb::primal_kernel<<<urb::block_grid(q), block, 0, on>>>(q, urb::planes_of(current, plane),
                                                              k == n ? output : current + 8 * plane);
    if (k < n) {
      float* next;
      const CUtensorMap* next_map;
      if (k % every == 0) {
        next = checkpoints + k / every * 9 * plane;
        next_map = &checkpoint_maps[k / every];
      } else {
        const int c = current == spare[0] ? 1 : 0;
        next = spare[c];
        next_map = &spare_maps[c];
      }
      urb::dual_tile_kernel<<<tiles, block, urb::kForwardShared, on>>>(*current_map, q, urb::planes_of(next, plane));
      current = next;
      current_map = next_map;
    }
  }
  const cudaError_t error = cudaGetLastError();
  if (error != cudaSuccess) {
    urb::tell(message, message_size, std::string("the device failed in the unrolled solve: ") + cudaGetErrorString(error));
    return UNROUND_ERROR_INTERNAL;
  }
  return UNROUND_OK;
}

extern "C" unround_status unround_b200_unrolled_backward(const unround_b200_unrolled* problem, const float* alpha0,
                                                         const float* alpha1, const float* tau, const float* sigma,
                                                         const float* checkpoints, float* workspace,
                                                         const float* output_grad, double* grads, void* stream,
                                                         char* message, size_t message_size) {
  const std::string wrong = urb::check(problem);
  if (!wrong.empty()) {
    urb::tell(message, message_size, wrong);
    return UNROUND_ERROR_ARGUMENT;
  }
  if (alpha0 == nullptr || alpha1 == nullptr || tau == nullptr || sigma == nullptr || checkpoints == nullptr ||
      workspace == nullptr || output_grad == nullptr || grads == nullptr) {
    urb::tell(message, message_size, "the parameters, checkpoints, workspace, gradients are not null pointers");
    return UNROUND_ERROR_ARGUMENT;
  }
  const cudaStream_t on = static_cast<cudaStream_t>(stream);
  const urb::Problem q = urb::problem_of(*problem, alpha0, alpha1, tau, sigma);
  const std::size_t plane = q.plane;
  const std::uint64_t n = problem->iterations, every = problem->checkpoint_every;
  const std::uint64_t segments = urb::checkpoints_of(*problem);
  float* const recomputed = workspace;  // s_{k0+1} .. s_{k0+K-1}, 9 planes each
  float* const adjoint_base = workspace + (every - 1) * 9 * plane;
  float* const adjoint[2] = {adjoint_base, adjoint_base + 9 * plane};
  float* const xt_bar = adjoint_base + 18 * plane;
  // s_{k0 + step} and x~ after it: the checkpoint at step 0, the recomputed slots after.
  auto storage_of = [&](std::uint64_t seg, std::uint64_t step) -> float* {
    return step == 0 ? const_cast<float*>(checkpoints) + seg * 9 * plane : recomputed + (step - 1) * 9 * plane;
  };
  // The dual step and its adjoint read the 9 planes of each by bulk-tensor copies (boxes of
  // different heights).
  std::vector<CUtensorMap> checkpoint_maps(segments), recomputed_maps(every > 1 ? every - 1 : 0);
  std::vector<CUtensorMap> checkpoint_forward(segments), recomputed_forward(every > 1 ? every - 1 : 0);
  CUtensorMap bar_maps[2];
  bool mapped = urb::prepare_dual_adjoint();
  const int W = static_cast<int>(q.columns), H = static_cast<int>(q.rows), images = static_cast<int>(q.images);
  for (std::uint64_t c = 0; c < segments && mapped; ++c) {
    mapped = urb::make_fields_map(checkpoint_maps[c], storage_of(c, 0), W, H, images, 9, plane, 40, urb::kStateRows) &&
             urb::make_forward_map(checkpoint_forward[c], storage_of(c, 0), q);
  }
  for (std::uint64_t step = 1; step < every && mapped; ++step) {
    mapped = urb::make_fields_map(recomputed_maps[step - 1], storage_of(0, step), W, H, images, 9, plane, 40,
                                  urb::kStateRows) &&
             urb::make_forward_map(recomputed_forward[step - 1], storage_of(0, step), q);
  }
  for (int c = 0; c < 2 && mapped; ++c) {
    mapped = urb::make_fields_map(bar_maps[c], adjoint[c], W, H, images, 9, plane, 40, urb::kBarRows);
  }
  if (!mapped) {
    urb::tell(message, message_size, "the device's bulk-tensor copies could not be set up for the adjoint");
    return UNROUND_ERROR_INTERNAL;
  }
  const dim3 block(32, 8), tiles = urb::tile_grid(q);
  cudaMemsetAsync(grads, 0, 4 * problem->images * sizeof(double), on);
  // The adjoint of s_N's predecessor starts at zero; that of x~_N is the output's gradient.
  int current = 0;
  cudaMemsetAsync(adjoint[current], 0, 9 * plane * sizeof(float), on);
  cudaMemcpyAsync(xt_bar, output_grad, plane * sizeof(float), cudaMemcpyDeviceToDevice, on);
  for (std::uint64_t seg = segments; seg-- > 0;) {
    const std::uint64_t k0 = seg * every;                             // the checkpoint s_{k0}
    const std::uint64_t k1 = std::min<std::uint64_t>(k0 + every, n);  // the segment's iterations k0+1 .. k1
    // Recompute s_{k0+1} .. s_{k1-1} and x~_{k0+2} .. x~_{k1} (x~_{k0+1} is the checkpoint's;
    // x~_N is not needed: x~_bar starts there).
    for (std::uint64_t k = k0 + 1; k < k1; ++k) {
      const std::uint64_t step = k - 1 - k0;  // s_{k-1} is storage_of(seg, step)
      float* from = storage_of(seg, step);
      if (step > 0) {
        urb::primal_kernel<<<urb::block_grid(q), block, 0, on>>>(q, urb::planes_of(from, plane), from + 8 * plane);
      }
      const CUtensorMap& from_map = step == 0 ? checkpoint_forward[seg] : recomputed_forward[step - 1];
      urb::dual_tile_kernel<<<tiles, block, urb::kForwardShared, on>>>(from_map, q,
                                                                       urb::planes_of(storage_of(seg, step + 1), plane));
    }
    if (k1 - k0 > 1 && k1 < n) {
      // x~_{k1} of the segment's last state, for D_{k1}'s adjoint.
      float* last = storage_of(seg, k1 - 1 - k0);
      urb::primal_kernel<<<urb::block_grid(q), block, 0, on>>>(q, urb::planes_of(last, plane), last + 8 * plane);
    }
    // Backwards through the segment: at iteration k, D_k (k < N) then P_k.
    for (std::uint64_t k = k1; k > k0; --k) {
      const std::uint64_t step = k - 1 - k0;
      if (k < n) {
        // D_k: the adjoint of s_k and of P_{k+1}'s v are adjoint[current]; write that of s_{k-1}
        // into the other, and that of x~_k into xt_bar.
        const CUtensorMap& state_map = step == 0 ? checkpoint_maps[seg] : recomputed_maps[step - 1];
        urb::dual_adjoint_kernel<<<tiles, block, urb::kAdjointShared, on>>>(
            state_map, bar_maps[current], q, urb::planes_of(adjoint[1 - current], plane), xt_bar, grads);
        current = 1 - current;
      }
      // P_k: from the adjoint of x~_k that of its v, beside the adjoint of s_{k-1}, which the
      // next dual step undone (D_{k-1}) reads.
      urb::primal_adjoint_block<<<urb::block_grid(q), block, 0, on>>>(
          q, urb::planes_of(storage_of(seg, step), plane), xt_bar, adjoint[current] + 8 * plane, grads);
    }
  }
  const cudaError_t error = cudaGetLastError();
  if (error != cudaSuccess) {
    urb::tell(message, message_size, std::string("the device failed in the adjoint: ") + cudaGetErrorString(error));
    return UNROUND_ERROR_INTERNAL;
  }
  return UNROUND_OK;
}
