// The orthonormal 8x8 DCT-II of JPEG (docs/math.md 1.1): C[k][n] = g_k cos(pi (2n+1) k / 16),
// g_0 = sqrt(1/8), g_k = 1/2 otherwise. The basis is built from the doubles nearest to
// cos(pi j / 16), j = 0..8 (the angle reduced modulo 32 in integers, so that no rounded
// angle enters a cosine), as the reference's basis is (docs/math.md 1.1, dct.rs COSINES);
// the binary32 kernels take each entry rounded once more. The 8-point transforms go by
// their even and odd halves: sums and differences of the ends, then each output a sum of
// four products (docs/math.md 1.1).
#pragma once

#include <cuda_runtime.h>

namespace urb {

// cos(pi j / 16), j = 0..8, each the double nearest to the exact value.
__host__ __device__ constexpr double cos16(int j) {
  return j == 0   ? 1.0
         : j == 1 ? 0x1.f6297cff75cb0p-1
         : j == 2 ? 0x1.d906bcf328d46p-1
         : j == 3 ? 0x1.a9b66290ea1a3p-1
         : j == 4 ? 0x1.6a09e667f3bcdp-1
         : j == 5 ? 0x1.1c73b39ae68c8p-1
         : j == 6 ? 0x1.87de2a6aea963p-2
         : j == 7 ? 0x1.8f8b83c69a60bp-3
                  : 0.0;
}
// sqrt(1/8), correctly rounded.
constexpr double kRootEighth = 0x1.6a09e667f3bcdp-2;

// cos(pi m / 16) for m in [0, 32): [0, 8] as it is, (8, 16] and (16, 24] negated, (24, 32)
// mirrored.
__host__ __device__ constexpr double cosine16(int m) {
  return m <= 8 ? cos16(m) : m <= 16 ? -cos16(16 - m) : m <= 24 ? -cos16(m - 16) : cos16(32 - m);
}

// C[k][n]; halving is exact.
__host__ __device__ constexpr double basis(int k, int n) {
  return k == 0 ? kRootEighth : 0.5 * cosine16(((2 * n + 1) * k) % 32);
}

template <typename T>
__host__ __device__ constexpr T basis_as(int k, int n) {
  return static_cast<T>(basis(k, n));
}

#ifdef __CUDACC__
// y = C x: the forward 8-point transform, even outputs from the sums, odd from the
// differences.
template <typename T>
__device__ __forceinline__ void forward8(const T (&x)[8], T (&y)[8]) {
  const T s0 = x[0] + x[7], s1 = x[1] + x[6], s2 = x[2] + x[5], s3 = x[3] + x[4];
  const T d0 = x[0] - x[7], d1 = x[1] - x[6], d2 = x[2] - x[5], d3 = x[3] - x[4];
#pragma unroll
  for (int k = 0; k < 8; k += 2) {
    y[k] = basis_as<T>(k, 0) * s0 + basis_as<T>(k, 1) * s1 + basis_as<T>(k, 2) * s2 + basis_as<T>(k, 3) * s3;
    y[k + 1] = basis_as<T>(k + 1, 0) * d0 + basis_as<T>(k + 1, 1) * d1 + basis_as<T>(k + 1, 2) * d2 +
               basis_as<T>(k + 1, 3) * d3;
  }
}

// x = C^T y: the even part from the even frequencies, the odd part from the odd ones, then
// their sum and difference.
template <typename T>
__device__ __forceinline__ void inverse8(const T (&y)[8], T (&x)[8]) {
#pragma unroll
  for (int n = 0; n < 4; ++n) {
    const T even = basis_as<T>(0, n) * y[0] + basis_as<T>(2, n) * y[2] + basis_as<T>(4, n) * y[4] +
                   basis_as<T>(6, n) * y[6];
    const T odd = basis_as<T>(1, n) * y[1] + basis_as<T>(3, n) * y[3] + basis_as<T>(5, n) * y[5] +
                  basis_as<T>(7, n) * y[7];
    x[n] = even + odd;
    x[7 - n] = even - odd;
  }
}
#endif  // __CUDACC__: the transforms are device code; host code takes the basis alone

}  // namespace urb
