// The coefficients of a JPEG file, read on the host (the reference's C layer over libjpeg-turbo,
// c/jpegio/src/jpegio.c:200-310, and its contract, c/jpegio/include/unround/jpegio.h:73-114).
// This build carries no libjpeg: the reader is its own, from ITU-T T.81: the markers, Huffman
// tables (Annex C), sequential DCT-based decoding (F.2.2) and progressive decoding by spectral
// selection and successive approximation (G.1.2), with restart intervals. Arithmetic coding,
// lossless, hierarchical and 12-bit files are refused as UNSUPPORTED, as are files of other than
// 1 (grey) or 3 (YCbCr or RGB) components. The colour space of 3 components follows libjpeg's
// rule: a JFIF marker means YCbCr; else an Adobe marker's transform (0 RGB, 1 YCbCr); else the
// component identifiers (R, G, B means RGB; anything else YCbCr).
//
// Corrupt data that a reader can work around (a Huffman code that is no code, data that ends
// within a scan, bytes before a marker, a missing restart marker) is counted as a warning and
// the first is kept, as libjpeg reports them: the blocks not decoded stay 0.
#pragma once

#include <cstddef>
#include <cstdint>
#include <string>
#include <vector>

namespace urb {

// Statuses as the C layer numbers them (unround_jpegio_status).
enum JpegStatus : int {
  kJpegOk = 0,
  kJpegArgument = 1,
  kJpegDecode = 2,
  kJpegUnsupported = 3,
  kJpegLimit = 4,
  kJpegMemory = 5,
};

struct JpegLimits {
  std::uint64_t max_pixels = std::uint64_t{1} << 28;  // width * height
  int max_scans = 500;                                // start-of-scan markers
  bool warnings_are_errors = false;
};

struct JpegComponent {
  int id = 0, h = 1, v = 1, slot = 0;
  std::uint32_t width = 0, height = 0;                       // samples that cover the picture
  std::uint32_t width_in_blocks = 0, height_in_blocks = 0;  // ceil(width / 8), ceil(height / 8)
  // The table of the component's slot when its first scan began, natural order.
  std::uint16_t table[64] = {};
  bool latched = false;
  // height_in_blocks x width_in_blocks blocks of 64 coefficients in natural order, block rows
  // from the top; no dummy blocks.
  std::vector<std::int16_t> coefficients;
};

struct JpegFile {
  std::uint32_t width = 0, height = 0;
  int color_space = 0;  // 1 grey, 2 YCbCr, 3 RGB
  int hmax = 1, vmax = 1;
  bool progressive = false;
  int exif_orientation = 0;  // 1 to 8 from an EXIF APP1 marker, 0 without one
  int warnings = 0;
  std::string warning;  // the first
  std::vector<JpegComponent> components;
  std::vector<std::uint8_t> icc;  // the profile of the APP2 markers, empty without one
};

// Reads a file in memory; on failure returns its status with the reason in message.
int read_jpeg(const std::uint8_t* data, std::size_t size, const JpegLimits& limits, JpegFile& file,
              std::string& message);

// The Orientation tag (0x0112) of the first IFD of an EXIF APP1 marker's data, 1 to 8, or 0.
int exif_orientation_of(const std::uint8_t* data, std::size_t size);

// The inverse DCT of one component's dequantized coefficients, level-shifted by 128, rounded
// and clamped to 0-255: (height_in_blocks * 8) x (width_in_blocks * 8) samples.
std::vector<std::uint8_t> component_plane(const JpegComponent& component);

}  // namespace urb
