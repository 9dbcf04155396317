// PNG files on the host (the reference's C layer over libpng, c/jpegio/src/png.c, and its
// contract, c/jpegio/include/unround/jpegio.h:134-253). This build carries no libpng: the
// reader and the writer are its own, from the PNG specification (ISO/IEC 15948), with zlib for
// the compressed data and the chunks' CRCs.
//
//   read_png    the levels a file stores: grey, grey and alpha, RGB, RGB and alpha, 1 to 16
//               bits, interlaced (Adam7) or not, with the profile of its iCCP chunk; a palette
//               file is refused (its colours were chosen, not rounded); a tRNS chunk is warned
//               about and not taken
//   write_png   8- or 16-bit levels as a file, not interlaced, each row's filter the one with
//               the least sum of absolute bytes, with an iCCP chunk where the profile is given
//   check_icc   what a reader checks of an ICC profile before it takes one for a picture
#pragma once

#include <cstddef>
#include <cstdint>
#include <string>
#include <vector>

namespace urb {

// Statuses as the C layer numbers them (unround_jpegio_status).
enum PngStatus : int {
  kPngOk = 0,
  kPngArgument = 1,
  kPngUnsupported = 3,
  kPngLimit = 4,
  kPngMemory = 5,
  kPngEncode = 6,
  kPngError = 7,
};

struct PngPicture {
  std::uint32_t width = 0, height = 0;
  int channels = 0;  // 1 grey, 2 grey and alpha, 3 RGB, 4 RGB and alpha
  int bits = 0;      // 1, 2, 4, 8 or 16
  std::vector<std::uint16_t> samples;  // height x width x channels levels, 0 to 2^bits - 1
  std::vector<std::uint8_t> icc;
  std::string warning;  // the first
};

// Whether data starts with the PNG signature.
bool is_png(const std::uint8_t* data, std::size_t size);

// Reads a file in memory; max_pixels bounds width * height (0 means 2^28). On failure returns
// its status with the reason in message.
int read_png(const std::uint8_t* data, std::size_t size, std::uint64_t max_pixels, PngPicture& picture,
             std::string& message);

// Writes levels (8 bits: bytes; 16 bits: uint16_t) as a file; compression is zlib's level, 0 to
// 9, or -1 for its default. The profile is written where check_icc takes it for the channels;
// otherwise it is left out and warning says why.
int write_png(const void* samples, std::uint32_t width, std::uint32_t height, int channels, int bits, int compression,
              const std::uint8_t* icc, std::size_t icc_size, std::vector<std::uint8_t>& file, std::string& warning,
              std::string& message);

// Whether an ICC profile goes with a picture of the channels (1 or 2: grey; 3 or 4: RGB): at
// least 132 bytes and the length its header gives, a multiple of 4 from version 4 on, the
// signature 'acsp', its tags within it, a rendering intent below 0xFFFF, a class that is neither
// abstract nor a device link, the picture's data colour space ('GRAY' or 'RGB '), and XYZ or Lab
// as its connection space. Where it does not, reason says why.
bool check_icc(const std::uint8_t* profile, std::uint64_t size, int channels, std::string& reason);

}  // namespace urb
