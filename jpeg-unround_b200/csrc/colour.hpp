// JFIF's colour conversions in binary64 (docs/math.md 8; rust/unround/src/colour.rs:45-70),
// shared by the host's conversions (capi.cpp) and the result's picture on the device
// (kernels.cu), which round every operation alike.
#pragma once

namespace urb {

// RGB of Y, Cb and Cr: the doubles nearest to 701/500, 443/250, 25251/73375 and 209599/293500.
constexpr double kCr = 0x1.66e978d4fdf3bp+0;
constexpr double kCb = 0x1.c5a1cac083127p+0;
constexpr double kGb = 0x1.6065433a66b17p-2;
constexpr double kGr = 0x1.6da345743d962p-1;
// And back: the doubles nearest to 0.299, 0.587, 0.114, 250/443 and 500/701.
constexpr double kR = 0x1.322d0e5604189p-2;
constexpr double kG = 0x1.2c8b439581062p-1;
constexpr double kB = 0x1.d2f1a9fbe76c9p-4;
constexpr double kToCb = 0x1.20f065b4e0378p-1;
constexpr double kToCr = 0x1.6d314d0e3e153p-1;

}  // namespace urb
