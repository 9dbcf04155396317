// The proximal map of G at one coefficient in binary32 (docs/math.md 4.1, 4.4), shared by the
// primal-step kernels (kernels.cu) and the fused iteration (iteration.cu).
#pragma once

#include <cuda_runtime.h>

#include "kernels.hpp"

namespace urb {

template <typename T>
__device__ __forceinline__ T clamp_to(T value, T low, T high) {
  return fmin(fmax(value, low), high);
}

// The interval and the centre of a coefficient in binary32, from its level
// (cpp/src/model.cpp:41-46, 237-247; laplace.hpp:51-56).
struct Coefficient {
  float low, high, centre, own_low, own_high;
};

// DC is taken centred on the middle of its interval, c_DC = q Q + 1024: the block's samples
// less c_DC / 8 have the DC coefficient e - c_DC, whose interval is [-(1/2 + s) Q, (1/2 + s) Q]
// and whose centre is 0. The same map in exact arithmetic; in binary32 it keeps DC's values
// small, where the absolute ones (up to ~2000) would lose ~1e-4 a transform, and lose it alike
// every iteration in the slow modes of weakly pinned (flat) blocks.
__device__ __forceinline__ Coefficient coefficient_of(int q, int k, const ProxFactors& F) {
  const float level = static_cast<float>(q);
  const float step = F.step[k];
  Coefficient c;
  if (k == 0) {
    c.low = (-0.5f - F.slack) * step;
    c.high = (0.5f + F.slack) * step;
    c.centre = 0.0f;
    c.own_low = -0.5f * step;
    c.own_high = 0.5f * step;
    return c;
  }
  const float shift = 0.0f;
  c.low = ((level - 0.5f) - F.slack) * step + shift;
  c.high = ((level + 0.5f) + F.slack) * step + shift;
  if (F.mmse && k != 0) {
    const float size = (fabsf(level) - F.shrink[k]) * step;
    c.centre = q == 0 ? 0.0f : (q < 0 ? -size : size);
  } else {
    c.centre = level * step + shift;
  }
  c.own_low = (level - 0.5f) * step + shift;
  c.own_high = (level + 0.5f) * step + shift;
  return c;
}

// prox of a coefficient (cpp/src/model.cpp:57-72): z = (e + t c) r clipped, and with a
// slack's cost moved back by h beyond the file's own interval, not past its end.
__device__ __forceinline__ float prox_of(float e, float t, float r, float h, const Coefficient& c, bool costed) {
  const float z = (e + t * c.centre) * r;
  if (!costed) return clamp_to(z, c.low, c.high);
  const float above = fmaxf(c.own_high, z - h);
  const float below = fminf(c.own_low, z + h);
  const float inside = z < c.own_low ? below : z;
  return clamp_to(z > c.own_high ? above : inside, c.low, c.high);
}

}  // namespace urb
