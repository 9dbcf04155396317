// Test infrastructure of the oracle: the PNG reader that shim/unround/jpegio.hpp declares, which
// refuses every file (the oracle gives the samples solver levels, not files); and the picture of
// a canvas that the reference's decoder makes (cpp/src/decode.cpp, not compiled here, as it needs
// the C layer), which its projection (cpp/src/picture.cpp) names: the oracle's bridge takes the
// projection's canvas, never that picture, so it is made empty.
#include "unround/decode.hpp"
#include "unround/jpegio.hpp"

namespace unround::jpegio {

std::expected<PngImage, Error> PngImage::read(std::span<const std::uint8_t>, std::uint64_t) {
  return std::unexpected(Error{Errc::unsupported, "the oracle reads no PNG files"});
}
Picture<const std::uint16_t> PngImage::levels() const { return {}; }
int PngImage::channels() const { return 0; }
int PngImage::bits() const { return 8; }
std::span<const std::uint8_t> PngImage::icc_profile() const { return {}; }
const std::string& PngImage::warning() const { return warning_; }

}  // namespace unround::jpegio

namespace unround {

PictureArray picture_of(std::span<const GridArray<double>>, std::size_t, std::size_t, ColourSpace) {
  return PictureArray(PictureExtents{0, 0, 0});
}

}  // namespace unround
