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
// The adjoint runs the iterations backwards: the adjoint of D_k (two per-pixel kernels: the
// projections' Jacobians at each pixel; then the transposes of E, grad and div2, which gather
// the first kernel's results of the neighbours and recompute w~'s adjoint of the left and upper
// ones), then of P_k (a block kernel: the DCT of the adjoint, the clip's mask, the inverse DCT,
// to the adjoint of v, which the next dual step undone reads for div's transpose). The states
// s_k are kept every `checkpoint` iterations by the forward pass; the
// backward pass recomputes each segment's states from its checkpoint. The parameters' gradients
// are sums over pixels and iterations, reduced per CTA and added in binary64.
#include <algorithm>
#include <cstdint>
#include <cstring>
#include <string>

#include <cuda_runtime.h>

#include "dct.cuh"
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

// w~ at a pixel: w + tau (p + div2 r), div2 r by forward differences.
__device__ __forceinline__ void w_tilde(const Problem& q, const Planes& s, int z, int i, int j, float tau, float& t1,
                                        float& t2, float& w1, float& w2) {
  const std::size_t k = at(q, z, i, j);
  const float r11 = s.r11[k], r22 = s.r22[k], r12 = s.r12[k];
  float d1 = j + 1 < q.columns ? s.r11[k + 1] - r11 : 0.0f;
  float d2 = j + 1 < q.columns ? s.r12[k + 1] - r12 : 0.0f;
  d1 = d1 + (i + 1 < q.rows ? s.r12[k + q.columns] - r12 : 0.0f);
  d2 = d2 + (i + 1 < q.rows ? s.r22[k + q.columns] - r22 : 0.0f);
  w1 = s.w1[k];
  w2 = s.w2[k];
  t1 = w1 + tau * (s.p1[k] + d1);
  t2 = w2 + tau * (s.p2[k] + d2);
}

__device__ __forceinline__ void w_bar(const Problem& q, const Planes& s, int z, int i, int j, float tau, float& b1,
                                      float& b2) {
  float t1, t2, w1, w2;
  w_tilde(q, s, z, i, j, tau, t1, t2, w1, w2);
  b1 = 2.0f * t1 - w1;
  b2 = 2.0f * t2 - w2;
}

// The dual step's points before the projections at a pixel: q = p + sigma (grad x- - w-) with
// g = grad x-, and s = r + sigma E w- with E; w- of the pixel and of its left and upper ones.
struct DualPoint {
  float g1, g2, b1, b2, q1, q2;
  float e11, e22, e12, s11, s22, s12;
  float t1, t2, w1, w2;
};

__device__ __forceinline__ DualPoint dual_point(const Problem& q, const Planes& s, const float* xt, int z, int i,
                                                int j) {
  const float tau = q.tau[z], sigma = q.sigma[z];
  const std::size_t k = at(q, z, i, j);
  const bool right = j + 1 < q.columns, down = i + 1 < q.rows;
  DualPoint d;
  const float bar = 2.0f * xt[k] - s.x[k];
  d.g1 = right ? (2.0f * xt[k + 1] - s.x[k + 1]) - bar : 0.0f;
  d.g2 = down ? (2.0f * xt[k + q.columns] - s.x[k + q.columns]) - bar : 0.0f;
  w_tilde(q, s, z, i, j, tau, d.t1, d.t2, d.w1, d.w2);
  d.b1 = 2.0f * d.t1 - d.w1;
  d.b2 = 2.0f * d.t2 - d.w2;
  d.q1 = s.p1[k] + sigma * (d.g1 - d.b1);
  d.q2 = s.p2[k] + sigma * (d.g2 - d.b2);
  float l1 = 0.0f, l2 = 0.0f, u1 = 0.0f, u2 = 0.0f;
  if (j > 0) w_bar(q, s, z, i, j - 1, tau, l1, l2);
  if (i > 0) w_bar(q, s, z, i - 1, j, tau, u1, u2);
  const float own1x = right ? d.b1 : 0.0f, own2x = right ? d.b2 : 0.0f;
  const float own1y = down ? d.b1 : 0.0f, own2y = down ? d.b2 : 0.0f;
  d.e11 = own1x - l1;
  d.e22 = own2y - u2;
  d.e12 = 0.5f * ((own1y - u1) + (own2x - l2));
  d.s11 = s.r11[k] + sigma * d.e11;
  d.s22 = s.r22[k] + sigma * d.e22;
  d.s12 = s.r12[k] + sigma * d.e12;
  return d;
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

// A CTA a row of 4 blocks: thread (tx, ty) the pixel (8 by + ty, 32 bx + tx).
__device__ __forceinline__ float primal_v(const Problem& q, const Planes& s, int z, int i, int j) {
  const std::size_t k = at(q, z, i, j);
  const float dy = (i + 1 < q.rows ? s.p2[k] : 0.0f) - (i > 0 ? s.p2[k - q.columns] : 0.0f);
  const float dx = (j + 1 < q.columns ? s.p1[k] : 0.0f) - (j > 0 ? s.p1[k - 1] : 0.0f);
  return s.x[k] + q.tau[z] * (dy + dx);
}

// The DCT basis C[k][n] at k * 9 + n (rows padded against bank conflicts), for a CTA's
// transforms: filled once per CTA from the compile-time values.
struct BasisTable {
  float v[8 * 9];
};

__device__ __forceinline__ void fill_basis(BasisTable& table) {
  const int t = threadIdx.y * blockDim.x + threadIdx.x;
  if (t < 64) {
    const int k = t >> 3, n = t & 7;
    float c = 0.0f;
#pragma unroll
    for (int kk = 0; kk < 8; ++kk) {
#pragma unroll
      for (int nn = 0; nn < 8; ++nn) c = (kk == k && nn == n) ? basis_as<float>(kk, nn) : c;
    }
    table.v[k * 9 + n] = c;
  }
  __syncthreads();
}

// The 2D transform of a CTA's 4 blocks in shared memory, in place: forward (C V C^T) or inverse
// (C^T V C); `t` holds the values [8][33], each thread one.
__device__ __forceinline__ float transform(float value, float (*t)[33], const BasisTable& basis, bool forward) {
  const int tx = threadIdx.x, ty = threadIdx.y, n0 = tx & ~7, u = tx & 7;
  t[ty][tx] = value;
  __syncthreads();
  // Columns: row ty of the result from the 8 rows of the column tx.
  float acc = 0.0f;
#pragma unroll
  for (int a = 0; a < 8; ++a) {
    const float c = forward ? basis.v[ty * 9 + a] : basis.v[a * 9 + ty];
    acc = fmaf(c, t[a][tx], acc);
  }
  __syncthreads();
  t[ty][tx] = acc;
  __syncthreads();
  // Rows: element u of the block's row ty from its 8 elements.
  float out = 0.0f;
#pragma unroll
  for (int b = 0; b < 8; ++b) {
    const float c = forward ? basis.v[u * 9 + b] : basis.v[b * 9 + u];
    out = fmaf(c, t[ty][n0 + b], out);
  }
  __syncthreads();
  return out;
}

struct Clip {
  float z, r, t, weight, centre, e;
  bool inside;
};

__device__ __forceinline__ Clip clip_of(const Problem& q, int z, std::size_t block, int kk, float e) {
  const float tau = q.tau[z];
  const bool flat = q.flat[static_cast<std::size_t>(z) * q.blocks_down * q.blocks_across + block] != 0;
  const float m = flat ? q.flat_weight[z * 64 + kk] : q.weight[z * 64 + kk];
  const std::size_t c = ((static_cast<std::size_t>(z) * q.blocks_down * q.blocks_across) + block) * 64 + kk;
  Clip out;
  out.weight = m;
  out.t = tau * m;
  out.r = 1.0f / (1.0f + out.t);
  out.centre = q.centre[c];
  out.e = e;
  const float zz = (e + out.t * out.centre) * out.r;
  const float a = q.lower[c], b = q.upper[c];
  out.inside = zz > a && zz < b;
  out.z = fminf(fmaxf(zz, a), b);
  return out;
}

__global__ void __launch_bounds__(256) primal_kernel(Problem q, Planes s, float* xt) {
  __shared__ float t[8][33];
  __shared__ BasisTable basis;
  fill_basis(basis);
  const int j = blockIdx.x * 32 + threadIdx.x, i = blockIdx.y * 8 + threadIdx.y, z = blockIdx.z;
  const bool in = j < q.columns;
  const int jc = in ? j : q.columns - 1;
  const int bx = jc / 8, by = blockIdx.y;
  const std::size_t block = static_cast<std::size_t>(by) * q.blocks_across + bx;
  const float middle = q.middle[static_cast<std::size_t>(z) * q.blocks_down * q.blocks_across + block];
  const float v = primal_v(q, s, z, i, jc);
  const float e = transform(v - middle, t, basis, true);
  const int kk = threadIdx.y * 8 + (threadIdx.x & 7);
  const Clip c = clip_of(q, z, block, kk, e);
  const float back = transform(c.z, t, basis, false);
  if (in) xt[at(q, z, i, j)] = back + middle;
}

__global__ void __launch_bounds__(256) dual_kernel(Problem q, Planes s, const float* xt, Planes out) {
  const int j = blockIdx.x * 32 + threadIdx.x, i = blockIdx.y * 8 + threadIdx.y, z = blockIdx.z;
  if (i >= q.rows || j >= q.columns) return;
  const std::size_t k = at(q, z, i, j);
  const float rho = q.rho, rest = 1.0f - q.rho;
  const DualPoint d = dual_point(q, s, xt, z, i, j);
  const float sp = ball(d.q1 * d.q1 + d.q2 * d.q2, q.alpha1[z]);
  const float sr = ball(d.s11 * d.s11 + d.s22 * d.s22 + 2.0f * (d.s12 * d.s12), q.alpha0[z]);
  out.x[k] = rho * xt[k] + rest * s.x[k];
  out.p1[k] = rho * (d.q1 * sp) + rest * s.p1[k];
  out.p2[k] = rho * (d.q2 * sp) + rest * s.p2[k];
  out.w1[k] = rho * d.t1 + rest * d.w1;
  out.w2[k] = rho * d.t2 + rest * d.w2;
  out.r11[k] = rho * (d.s11 * sr) + rest * s.r11[k];
  out.r22[k] = rho * (d.s22 * sr) + rest * s.r22[k];
  out.r12[k] = rho * (d.s12 * sr) + rest * s.r12[k];
}

// ---- Adjoint. `a` holds the adjoint of s_k (the dual step's output) on entry; the kernels
// write the adjoint of s_{k-1} into `b` and the adjoint of x~_k into `xt_bar`. Gradients:
// [0] alpha0, [1] alpha1, [2] tau, [3] sigma, each [image].

struct Scratch {
  float* q1;  // the adjoint of the projections' points q and s
  float* q2;
  float* s11;
  float* s22;
  float* s12;
  float* v;   // the adjoint of v of a primal step
};

// The adjoint of x and p of s_k: that of the dual step after it (`a`) and that of the primal
// step P_{k+1}, whose v = x + tau div p has the adjoint `vbar` (null where there is none):
// x^ += v^, p^ += tau div^T v^ = -tau grad v^.
__device__ __forceinline__ float adjoint_x(const Planes& a, const float* vbar, std::size_t k) {
  return vbar != nullptr ? a.x[k] + vbar[k] : a.x[k];
}

__device__ __forceinline__ void adjoint_p(const Problem& q, const Planes& a, const float* vbar, float tau, int i, int j,
                                          std::size_t k, float& p1, float& p2) {
  p1 = a.p1[k];
  p2 = a.p2[k];
  if (vbar != nullptr) {
    const float v = vbar[k];
    if (j + 1 < q.columns) p1 += -tau * (vbar[k + 1] - v);
    if (i + 1 < q.rows) p2 += -tau * (vbar[k + q.columns] - v);
  }
}

// The adjoint of w~ at a pixel from the local kernel's adjoints of q and s: that of w- is
// -sigma q^ + sigma E^T s^ (E^T gathering s^ of the pixel and of its right and lower ones), and
// w~ = (w- + w) / 2 gives it twice, beside the relaxation's rho w'^.
__device__ __forceinline__ void w_tilde_bar(const Problem& q, const Planes& a, const Scratch& w, int z, int i, int j,
                                            float& t1, float& t2, float& wb1, float& wb2) {
  const std::size_t k = at(q, z, i, j);
  const int W = q.columns;
  const float sigma = q.sigma[z], rho = q.rho;
  wb1 = -sigma * w.q1[k];
  wb2 = -sigma * w.q2[k];
  float e1 = 0.0f, e2 = 0.0f;
  if (j + 1 < W) {
    e1 += w.s11[k] - w.s11[k + 1];
    e2 += 0.5f * (w.s12[k] - w.s12[k + 1]);
  }
  if (i + 1 < q.rows) {
    e2 += w.s22[k] - w.s22[k + W];
    e1 += 0.5f * (w.s12[k] - w.s12[k + W]);
  }
  wb1 += sigma * e1;
  wb2 += sigma * e2;
  t1 = rho * a.w1[k] + 2.0f * wb1;
  t2 = rho * a.w2[k] + 2.0f * wb2;
}

__global__ void __launch_bounds__(256) dual_adjoint_local(Problem q, Planes s, const float* xt, Planes a,
                                                          const float* vbar, Scratch w, double* grads) {
  const int j = blockIdx.x * 32 + threadIdx.x, i = blockIdx.y * 8 + threadIdx.y, z = blockIdx.z;
  const bool in = i < q.rows && j < q.columns;
  float g_alpha0 = 0.0f, g_alpha1 = 0.0f, g_sigma = 0.0f;
  if (in) {
    const std::size_t k = at(q, z, i, j);
    const float rho = q.rho;
    const DualPoint d = dual_point(q, s, xt, z, i, j);
    // p~ = proj(q): the adjoint of q from that of p~.
    float ap1, ap2;
    adjoint_p(q, a, vbar, q.tau[z], i, j, k, ap1, ap2);
    const float pb1 = rho * ap1, pb2 = rho * ap2;
    float qb1 = pb1, qb2 = pb2;
    const float alpha1 = q.alpha1[z];
    const float nq = sqrtf(d.q1 * d.q1 + d.q2 * d.q2);
    if (nq > alpha1) {
      const float dot = d.q1 * pb1 + d.q2 * pb2;
      const float f = alpha1 / nq, h = dot / (nq * nq);
      qb1 = f * (pb1 - d.q1 * h);
      qb2 = f * (pb2 - d.q2 * h);
      g_alpha1 = dot / nq;
    }
    // r~ = proj_F(s), |s|^2 = s11^2 + s22^2 + 2 s12^2.
    const float rb11 = rho * a.r11[k], rb22 = rho * a.r22[k], rb12 = rho * a.r12[k];
    float sb11 = rb11, sb22 = rb22, sb12 = rb12;
    const float alpha0 = q.alpha0[z];
    const float ns = sqrtf(d.s11 * d.s11 + d.s22 * d.s22 + 2.0f * (d.s12 * d.s12));
    if (ns > alpha0) {
      const float dot = d.s11 * rb11 + d.s22 * rb22 + d.s12 * rb12;
      const float f = alpha0 / ns, h = dot / (ns * ns);
      sb11 = f * (rb11 - d.s11 * h);
      sb22 = f * (rb22 - d.s22 * h);
      sb12 = f * (rb12 - 2.0f * d.s12 * h);
      g_alpha0 = dot / ns;
    }
    g_sigma = qb1 * (d.g1 - d.b1) + qb2 * (d.g2 - d.b2) + sb11 * d.e11 + sb22 * d.e22 + sb12 * d.e12;
    w.q1[k] = qb1;
    w.q2[k] = qb2;
    w.s11[k] = sb11;
    w.s22[k] = sb22;
    w.s12[k] = sb12;
  }
  add_sum(g_alpha0, grads + 0 * q.images + z);
  add_sum(g_alpha1, grads + 1 * q.images + z);
  add_sum(g_sigma, grads + 3 * q.images + z);
}

__global__ void __launch_bounds__(256) dual_adjoint_gather(Problem q, Planes s, Planes a, const float* vbar,
                                                           Scratch w, Planes b, float* xt_bar, double* grads) {
  const int j = blockIdx.x * 32 + threadIdx.x, i = blockIdx.y * 8 + threadIdx.y, z = blockIdx.z;
  const bool in = i < q.rows && j < q.columns;
  float g_tau = 0.0f;
  if (in) {
    const std::size_t k = at(q, z, i, j);
    const int W = q.columns, H = q.rows;
    const float rho = q.rho, rest = 1.0f - q.rho, sigma = q.sigma[z], tau = q.tau[z];
    const bool right = j + 1 < W, down = i + 1 < H;
    float tb1, tb2, wb1, wb2;
    w_tilde_bar(q, a, w, z, i, j, tb1, tb2, wb1, wb2);
    float ap1, ap2;
    adjoint_p(q, a, vbar, tau, i, j, k, ap1, ap2);
    b.w1[k] = rest * a.w1[k] - wb1 + tb1;
    b.w2[k] = rest * a.w2[k] - wb2 + tb2;
    b.p1[k] = rest * ap1 + w.q1[k] + tau * tb1;
    b.p2[k] = rest * ap2 + w.q2[k] + tau * tb2;
    // r^: the relaxation's, s^, and div2^T of d^ = tau w~^ (w~^ of the pixel and of its left and
    // upper ones).
    float l1 = 0.0f, l2 = 0.0f, u1 = 0.0f, u2 = 0.0f, unused1, unused2;
    if (j > 0) w_tilde_bar(q, a, w, z, i, j - 1, l1, l2, unused1, unused2);
    if (i > 0) w_tilde_bar(q, a, w, z, i - 1, j, u1, u2, unused1, unused2);
    const float db1 = tau * tb1, db2 = tau * tb2;
    const float div11 = tau * l1 - (right ? db1 : 0.0f);
    const float div12 = tau * u1 - (down ? db1 : 0.0f) + tau * l2 - (right ? db2 : 0.0f);
    const float div22 = tau * u2 - (down ? db2 : 0.0f);
    b.r11[k] = rest * a.r11[k] + w.s11[k] + div11;
    b.r22[k] = rest * a.r22[k] + w.s22[k] + div22;
    b.r12[k] = rest * a.r12[k] + w.s12[k] + div12;
    // d/dtau of w~ = p + div2 r.
    const float r11 = s.r11[k], r22 = s.r22[k], r12 = s.r12[k];
    float d1 = right ? s.r11[k + 1] - r11 : 0.0f;
    float d2 = right ? s.r12[k + 1] - r12 : 0.0f;
    d1 = d1 + (down ? s.r12[k + W] - r12 : 0.0f);
    d2 = d2 + (down ? s.r22[k + W] - r22 : 0.0f);
    g_tau = tb1 * (s.p1[k] + d1) + tb2 * (s.p2[k] + d2);
    // The adjoint of x- : grad^T (sigma q^) = -div (sigma q^).
    float div = (right ? w.q1[k] : 0.0f) - (j > 0 ? w.q1[k - 1] : 0.0f) + (down ? w.q2[k] : 0.0f) -
                (i > 0 ? w.q2[k - W] : 0.0f);
    const float xbb = -sigma * div;
    const float ax = adjoint_x(a, vbar, k);
    xt_bar[k] = rho * ax + 2.0f * xbb;
    b.x[k] = rest * ax - xbb;
  }
  add_sum(g_tau, grads + 2 * q.images + z);
}

// The primal step's adjoint, per block: from the adjoint of x~ (`xt_bar`) the adjoint of v.
__global__ void __launch_bounds__(256) primal_adjoint_block(Problem q, Planes s, const float* xt_bar, Scratch w,
                                                            double* grads) {
  __shared__ float t[8][33];
  __shared__ BasisTable basis;
  fill_basis(basis);
  const int j = blockIdx.x * 32 + threadIdx.x, i = blockIdx.y * 8 + threadIdx.y, z = blockIdx.z;
  const bool in = j < q.columns;
  const int jc = in ? j : q.columns - 1;
  const int bx = jc / 8, by = blockIdx.y;
  const std::size_t block = static_cast<std::size_t>(by) * q.blocks_across + bx;
  const std::size_t k = at(q, z, i, jc);
  const float middle = q.middle[static_cast<std::size_t>(z) * q.blocks_down * q.blocks_across + block];
  const float v = primal_v(q, s, z, i, jc);
  const float e = transform(v - middle, t, basis, true);
  const int kk = threadIdx.y * 8 + (threadIdx.x & 7);
  const Clip c = clip_of(q, z, block, kk, e);
  const float zb = transform(in ? xt_bar[k] : 0.0f, t, basis, true);
  // zeta = (e + t c) r inside the interval, t = tau m, r = 1 / (1 + t): d zeta / d e = r and
  // d zeta / d tau = m (c - e) r^2; outside it zeta is an end of the interval.
  const float eb = c.inside ? c.r * zb : 0.0f;
  float g_tau = c.inside ? zb * c.weight * (c.centre - e) * (c.r * c.r) : 0.0f;
  const float vb = transform(eb, t, basis, false);
  // d v / d tau = div p.
  const float dy = (i + 1 < q.rows ? s.p2[k] : 0.0f) - (i > 0 ? s.p2[k - q.columns] : 0.0f);
  const float dx = (jc + 1 < q.columns ? s.p1[k] : 0.0f) - (jc > 0 ? s.p1[k - 1] : 0.0f);
  if (in) {
    w.v[k] = vb;
    g_tau += vb * (dy + dx);
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

std::uint64_t checkpoints_of(const unround_b200_unrolled& u) {
  // s_0, s_K, s_2K, ... up to s_{N-1}.
  return (u.iterations - 1) / u.checkpoint_every + 1;
}

}  // namespace

}  // namespace urb

using urb::Planes;

extern "C" uint64_t unround_b200_unrolled_checkpoint_floats(const unround_b200_unrolled* problem) {
  if (!urb::check(problem).empty()) return 0;
  return urb::checkpoints_of(*problem) * 8 * problem->images * problem->rows * problem->columns;
}

extern "C" uint64_t unround_b200_unrolled_workspace_floats(const unround_b200_unrolled* problem) {
  if (!urb::check(problem).empty()) return 0;
  const std::uint64_t plane = problem->images * problem->rows * problem->columns;
  // Two states ping-pong, x~, a segment's states and x~s, two adjoints, x~'s adjoint, scratch.
  return (2 * 8 + 1 + problem->checkpoint_every * 9 + 2 * 8 + 1 + 6) * plane;
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
  Planes state[2] = {urb::planes_of(workspace, plane), urb::planes_of(workspace + 8 * plane, plane)};
  float* xt = workspace + 16 * plane;
  const dim3 grid = urb::pixel_grid(q), block(32, 8);
  urb::start_kernel<<<grid, block, 0, on>>>(q, problem->start, state[0]);
  const std::uint64_t n = problem->iterations, every = problem->checkpoint_every;
  int current = 0;
  for (std::uint64_t k = 1; k <= n; ++k) {
    // s_{k-1} is state[current]; keep it where k - 1 is a checkpoint.
    if ((k - 1) % every == 0) {
      cudaMemcpyAsync(checkpoints + (k - 1) / every * 8 * plane, state[current].x, 8 * plane * sizeof(float),
                      cudaMemcpyDeviceToDevice, on);
    }
    urb::primal_kernel<<<grid, block, 0, on>>>(q, state[current], k == n ? output : xt);
    if (k < n) {
      urb::dual_kernel<<<grid, block, 0, on>>>(q, state[current], xt, state[1 - current]);
      current = 1 - current;
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
  // The workspace: the segment's states s_{k0} .. s_{k0+K-1} and x~_{k0+1} .. x~_{k0+K} (9 planes
  // each step), two adjoints of a state, the adjoint of x~, and the scratch.
  float* segment = workspace + 17 * plane;
  float* adjoint_base = segment + every * 9 * plane;
  Planes adjoint[2] = {urb::planes_of(adjoint_base, plane), urb::planes_of(adjoint_base + 8 * plane, plane)};
  float* xt_bar = adjoint_base + 16 * plane;
  float* scratch_base = xt_bar + plane;
  const urb::Scratch scratch{scratch_base,             scratch_base + plane,     scratch_base + 2 * plane,
                             scratch_base + 3 * plane, scratch_base + 4 * plane, scratch_base + 5 * plane};
  // The adjoint of v of the primal step after the dual step being undone (none after the last).
  const float* vbar = nullptr;
  auto state_of = [&](std::uint64_t step) { return urb::planes_of(segment + step * 9 * plane, plane); };
  auto tilde_of = [&](std::uint64_t step) { return segment + step * 9 * plane + 8 * plane; };
  const dim3 grid = urb::pixel_grid(q), block(32, 8);
  cudaMemsetAsync(grads, 0, 4 * problem->images * sizeof(double), on);
  // The adjoint of s_N's predecessor starts at zero; that of x~_N is the output's gradient.
  int current = 0;
  cudaMemsetAsync(adjoint[current].x, 0, 8 * plane * sizeof(float), on);
  cudaMemcpyAsync(xt_bar, output_grad, plane * sizeof(float), cudaMemcpyDeviceToDevice, on);
  const std::uint64_t segments = urb::checkpoints_of(*problem);
  for (std::uint64_t seg = segments; seg-- > 0;) {
    const std::uint64_t k0 = seg * every;                          // the checkpoint s_{k0}
    const std::uint64_t k1 = std::min<std::uint64_t>(k0 + every, n);  // the segment's iterations k0+1 .. k1
    // Recompute s_{k0} .. s_{k1-1} and x~_{k0+1} .. x~_{k1} (x~_N is not needed: x~_bar starts there).
    cudaMemcpyAsync(segment, checkpoints + seg * 8 * plane, 8 * plane * sizeof(float), cudaMemcpyDeviceToDevice, on);
    for (std::uint64_t k = k0 + 1; k <= k1; ++k) {
      const std::uint64_t step = k - 1 - k0;  // s_{k-1} is state_of(step)
      urb::primal_kernel<<<grid, block, 0, on>>>(q, state_of(step), tilde_of(step));
      if (k < k1) urb::dual_kernel<<<grid, block, 0, on>>>(q, state_of(step), tilde_of(step), state_of(step + 1));
    }
    // Backwards through the segment: at iteration k, D_k (k < N) then P_k.
    for (std::uint64_t k = k1; k > k0; --k) {
      const std::uint64_t step = k - 1 - k0;
      const Planes s = state_of(step);
      if (k < n) {
        // D_k: the adjoint of s_k is adjoint[current] and P_{k+1}'s (vbar); write that of
        // s_{k-1} into the other, and that of x~_k into xt_bar.
        const Planes a = adjoint[current], b = adjoint[1 - current];
        urb::dual_adjoint_local<<<grid, block, 0, on>>>(q, s, tilde_of(step), a, vbar, scratch, grads);
        urb::dual_adjoint_gather<<<grid, block, 0, on>>>(q, s, a, vbar, scratch, b, xt_bar, grads);
        current = 1 - current;
      }
      // P_k: from the adjoint of x~_k that of its v, which the next dual step undone (D_{k-1})
      // adds to the adjoints of x and p of s_{k-1}.
      urb::primal_adjoint_block<<<grid, block, 0, on>>>(q, s, xt_bar, scratch, grads);
      vbar = scratch.v;
    }
  }
  const cudaError_t error = cudaGetLastError();
  if (error != cudaSuccess) {
    urb::tell(message, message_size, std::string("the device failed in the adjoint: ") + cudaGetErrorString(error));
    return UNROUND_ERROR_INTERNAL;
  }
  return UNROUND_OK;
}
