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

// prox of coefficient k at level q of a block, e its value (cpp/src/model.cpp:41-46, 57-72,
// 237-247; laplace.hpp:51-56): z = (e + t c) r = e r + (t r) c, clipped to the interval
// q Q -+ (1/2 + s) Q; c = q Q, or with MMSE centres sign(q) (|q| - delta/Q) Q (0 at q = 0).
// With a slack's cost, z is moved back by h beyond the file's own interval q Q -+ Q/2, not past
// its end. One 16-byte load of the packed factors serves the common case.
//
// DC is taken centred on the middle of its interval, c_DC = q Q + 1024: the block's samples
// less c_DC / 8 have the DC coefficient e - c_DC, whose interval is [-(1/2 + s) Q, (1/2 + s) Q]
// and whose centre is 0, the map of level 0. The same map in exact arithmetic; in binary32 it
// keeps DC's values small, where the absolute ones (up to ~2000) would lose ~1e-4 a transform,
// and lose it alike every iteration in the slow modes of weakly pinned (flat) blocks.
__device__ __forceinline__ float prox_at(float e, int q, int k, bool flat, const ProxFactors& F) {
  const float4 f = flat ? F.flat[prox_slot(k)] : F.plain[prox_slot(k)];  // Q, r, t r, (1/2 + s) Q
  const float level = k == 0 ? 0.0f : static_cast<float>(q);
  const float middle = level * f.x;  // q Q, exact for the levels and steps of a file
  float centre = middle;
  if (F.mmse) {
    const float size = (fabsf(level) - F.shrink[k]) * f.x;
    centre = level == 0.0f ? 0.0f : (level < 0.0f ? -size : size);
  }
  const float z = fmaf(f.z, centre, e * f.y);
  const float low = middle - f.w, high = middle + f.w;
  if (!F.costed) return clamp_to(z, low, high);
  const float h = flat ? F.h_flat[k] : F.h[k];
  const float own_low = fmaf(-0.5f, f.x, middle), own_high = fmaf(0.5f, f.x, middle);
  const float above = fmaxf(own_high, z - h);
  const float below = fminf(own_low, z + h);
  const float inside = z < own_low ? below : z;
  return clamp_to(z > own_high ? above : inside, low, high);
}

}  // namespace urb
