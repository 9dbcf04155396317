// Test infrastructure of the oracle: what the reference's samples solver (cpp/src/samples.cpp)
// names of its C layer's C++ face -- the PNG reader's result and errors -- declared without the
// C layer (libpng is not in this image). The oracle calls samples::Model::make and
// samples::solve, never samples::reconstruct, the one user of these; png_stub.cpp defines them
// to refuse. Found before the reference's own header by the include order of the Makefile.
#pragma once

#include <cstdint>
#include <expected>
#include <span>
#include <string>

#include "unround/arrays.hpp"

namespace unround::jpegio {

enum class Errc { unsupported, limit, argument, decode, memory, encode };

struct Error {
  Errc code = Errc::unsupported;
  std::string message;
};

class PngImage {
 public:
  static std::expected<PngImage, Error> read(std::span<const std::uint8_t> file, std::uint64_t max_pixels);
  [[nodiscard]] Picture<const std::uint16_t> levels() const;
  [[nodiscard]] int channels() const;
  [[nodiscard]] int bits() const;
  [[nodiscard]] std::span<const std::uint8_t> icc_profile() const;
  [[nodiscard]] const std::string& warning() const;

 private:
  std::string warning_;
};

}  // namespace unround::jpegio
