// PNG reading and writing (png_io.hpp), from the PNG specification with zlib.
#include "png_io.hpp"

#include <zlib.h>

#include <algorithm>
#include <cstdlib>
#include <cstring>
#include <new>

namespace urb {

namespace {

constexpr std::uint8_t kSignature[8] = {137, 80, 78, 71, 13, 10, 26, 10};

struct PngError {
  int status;
  std::string message;
};

[[noreturn]] void fail(int status, const std::string& message) { throw PngError{status, message}; }

std::uint32_t be32(const std::uint8_t* p) {
  return (std::uint32_t{p[0]} << 24) | (std::uint32_t{p[1]} << 16) | (std::uint32_t{p[2]} << 8) | std::uint32_t{p[3]};
}

void put32(std::vector<std::uint8_t>& out, std::uint32_t v) {
  out.push_back(static_cast<std::uint8_t>(v >> 24));
  out.push_back(static_cast<std::uint8_t>(v >> 16));
  out.push_back(static_cast<std::uint8_t>(v >> 8));
  out.push_back(static_cast<std::uint8_t>(v));
}

// Inflates a whole zlib stream into out (out_size bytes expected); returns the bytes made, and
// whether the stream ended and held more than expected.
std::size_t inflate_into(const std::uint8_t* in, std::size_t in_size, std::uint8_t* out, std::size_t out_size,
                         bool& ended, bool& extra, std::string& error) {
  z_stream z{};
  if (inflateInit(&z) != Z_OK) fail(kPngMemory, "zlib could not start");
  std::size_t given = 0, made = 0;
  std::uint8_t spill[4096];
  ended = extra = false;
  for (;;) {
    if (z.avail_in == 0 && given < in_size) {
      const std::size_t chunk = std::min<std::size_t>(in_size - given, std::size_t{1} << 30);
      z.next_in = const_cast<Bytef*>(in + given);
      z.avail_in = static_cast<uInt>(chunk);
      given += chunk;
    }
    const bool full = made >= out_size;
    const std::size_t room = full ? sizeof spill : std::min<std::size_t>(out_size - made, std::size_t{1} << 30);
    z.next_out = full ? spill : out + made;
    z.avail_out = static_cast<uInt>(room);
    const int status = inflate(&z, Z_NO_FLUSH);
    const std::size_t produced = room - z.avail_out;
    if (!full) {
      made += produced;
    } else if (produced > 0) {
      extra = true;
    }
    if (status == Z_STREAM_END) {
      ended = true;
      break;
    }
    if (status == Z_BUF_ERROR) {
      if (z.avail_in == 0 && given >= in_size) break;  // the data ends before the stream does
      continue;
    }
    if (status != Z_OK) {
      error = z.msg != nullptr ? z.msg : "the compressed data is broken";
      break;
    }
  }
  inflateEnd(&z);
  return made;
}

int paeth(int a, int b, int c) {
  const int p = a + b - c;
  const int pa = std::abs(p - a), pb = std::abs(p - b), pc = std::abs(p - c);
  if (pa <= pb && pa <= pc) return a;
  return pb <= pc ? b : c;
}

// Undoes a row's filter in place (prior: the row above after its own, or zeros).
void unfilter(int type, std::uint8_t* row, const std::uint8_t* prior, std::size_t bytes, std::size_t bpp) {
  switch (type) {
    case 0:
      break;
    case 1:
      for (std::size_t i = bpp; i < bytes; ++i) row[i] = static_cast<std::uint8_t>(row[i] + row[i - bpp]);
      break;
    case 2:
      for (std::size_t i = 0; i < bytes; ++i) row[i] = static_cast<std::uint8_t>(row[i] + prior[i]);
      break;
    case 3:
      for (std::size_t i = 0; i < bytes; ++i) {
        const int left = i >= bpp ? row[i - bpp] : 0;
        row[i] = static_cast<std::uint8_t>(row[i] + ((left + prior[i]) >> 1));
      }
      break;
    case 4:
      for (std::size_t i = 0; i < bytes; ++i) {
        const int left = i >= bpp ? row[i - bpp] : 0, corner = i >= bpp ? prior[i - bpp] : 0;
        row[i] = static_cast<std::uint8_t>(row[i] + paeth(left, prior[i], corner));
      }
      break;
    default:
      fail(kPngError, "bad adaptive filter value");
  }
}

// The seven passes of Adam7: first row, first column, row step, column step.
constexpr int kAdam7[7][4] = {{0, 0, 8, 8}, {0, 4, 8, 8}, {4, 0, 8, 4}, {0, 2, 4, 4},
                              {2, 0, 4, 2}, {0, 1, 2, 2}, {1, 0, 2, 1}};

}  // namespace

bool is_png(const std::uint8_t* data, std::size_t size) {
  return data != nullptr && size >= 8 && std::memcmp(data, kSignature, 8) == 0;
}

int read_png(const std::uint8_t* data, std::size_t size, std::uint64_t max_pixels, PngPicture& picture,
             std::string& message) {
  picture = PngPicture{};
  message.clear();
  if (data == nullptr && size > 0) {
    message = "the data is a null pointer";
    return kPngArgument;
  }
  try {
    if (!is_png(data, size)) fail(kPngError, "Not a PNG file");
    if (max_pixels == 0) max_pixels = std::uint64_t{1} << 28;
    std::size_t pos = 8;
    bool header = false, ended = false;
    int color_type = 0, interlace = 0;
    std::vector<std::uint8_t> compressed;
    auto warn = [&](const std::string& text) {
      if (picture.warning.empty()) picture.warning = text;
    };
    while (!ended) {
      if (size - pos < 12) fail(kPngError, "the file ends within a chunk");
      const std::uint32_t length = be32(data + pos);
      if (length > 0x7FFFFFFFu || size - pos - 12 < length) fail(kPngError, "the file ends within a chunk");
      const std::uint8_t* type = data + pos + 4;
      const std::uint8_t* body = data + pos + 8;
      const std::uint32_t crc = be32(body + length);
      const bool critical = (type[0] & 0x20) == 0;
      const std::string name(reinterpret_cast<const char*>(type), 4);
      if (static_cast<std::uint32_t>(crc32(crc32(0, nullptr, 0), type, length + 4)) != crc) {
        if (critical) fail(kPngError, name + ": CRC error");
        warn(name + ": CRC error");
        pos += 12 + length;
        continue;
      }
      pos += 12 + length;
      if (!header && name != "IHDR") fail(kPngError, "missing IHDR");
      if (name == "IHDR") {
        if (header || length != 13) fail(kPngError, "IHDR: invalid");
        picture.width = be32(body);
        picture.height = be32(body + 4);
        picture.bits = body[8];
        color_type = body[9];
        interlace = body[12];
        if (picture.width == 0 || picture.height == 0 || picture.width > 0x7FFFFFFFu || picture.height > 0x7FFFFFFFu) {
          fail(kPngError, "the picture is empty or too large");
        }
        if (body[10] != 0 || body[11] != 0 || interlace > 1) fail(kPngError, "IHDR: unknown compression, filter or interlace");
        const int b = picture.bits;
        const bool ok = (color_type == 0 && (b == 1 || b == 2 || b == 4 || b == 8 || b == 16)) ||
                        (color_type == 3 && (b == 1 || b == 2 || b == 4 || b == 8)) ||
                        ((color_type == 2 || color_type == 4 || color_type == 6) && (b == 8 || b == 16));
        if (!ok) fail(kPngError, "IHDR: invalid bit depth for the colour type");
        if (color_type == 3) fail(kPngUnsupported, "a palette PNG file is not taken: its colours were chosen, not rounded");
        picture.channels = color_type == 0 ? 1 : color_type == 4 ? 2 : color_type == 2 ? 3 : 4;
        const std::uint64_t pixels = std::uint64_t{picture.width} * picture.height;
        if (pixels > max_pixels) fail(kPngLimit, "the picture has more pixels than the options allow");
        header = true;
      } else if (name == "IDAT") {
        compressed.insert(compressed.end(), body, body + length);
      } else if (name == "IEND") {
        ended = true;
      } else if (name == "PLTE") {
        // A suggested palette of a true-colour file: not needed.
      } else if (name == "tRNS") {
        warn("the transparent colour of the tRNS chunk is not taken");
      } else if (name == "iCCP") {
        const std::uint8_t* end = static_cast<const std::uint8_t*>(std::memchr(body, 0, std::min<std::uint32_t>(length, 80)));
        bool taken = false;
        if (end != nullptr && end > body && static_cast<std::size_t>(end - body) + 2 <= length && end[1] == 0) {
          const std::uint8_t* z = end + 2;
          const std::size_t z_size = length - static_cast<std::size_t>(z - body);
          if (z_size >= 4) {
            // The profile's own length (its first 4 bytes), read from the first inflated bytes.
            std::uint8_t head[4];
            bool done = false, extra = false;
            std::string error;
            if (inflate_into(z, z_size, head, 4, done, extra, error) == 4) {
              const std::uint32_t declared = be32(head);
              if (declared >= 132 && declared <= (1u << 26)) {
                std::vector<std::uint8_t> profile(declared);
                const std::size_t made = inflate_into(z, z_size, profile.data(), declared, done, extra, error);
                std::string reason;
                if (made == declared && done && !extra && check_icc(profile.data(), declared, picture.channels, reason)) {
                  picture.icc = std::move(profile);
                  taken = true;
                }
              }
            }
          }
        }
        if (!taken) warn("iCCP: the profile is not taken");
      } else if (critical) {
        fail(kPngError, name + ": unknown critical chunk");
      }
    }
    if (compressed.empty()) fail(kPngError, "no image data");
    // The filtered rows of every pass, then the passes' samples.
    const std::size_t channels = picture.channels, bits = picture.bits;
    const std::size_t bpp = std::max<std::size_t>(1, channels * bits / 8);
    struct Pass {
      std::size_t rows, columns, first_row, first_column, row_step, column_step;
    };
    std::vector<Pass> passes;
    if (interlace == 0) {
      passes.push_back({picture.height, picture.width, 0, 0, 1, 1});
    } else {
      for (const auto& a : kAdam7) {
        const std::size_t rows = picture.height > static_cast<std::uint32_t>(a[0])
                                     ? (picture.height - a[0] + a[2] - 1) / a[2] : 0;
        const std::size_t columns = picture.width > static_cast<std::uint32_t>(a[1])
                                        ? (picture.width - a[1] + a[3] - 1) / a[3] : 0;
        passes.push_back({rows, columns, static_cast<std::size_t>(a[0]), static_cast<std::size_t>(a[1]),
                          static_cast<std::size_t>(a[2]), static_cast<std::size_t>(a[3])});
      }
    }
    std::size_t total = 0;
    for (const Pass& p : passes) {
      if (p.rows == 0 || p.columns == 0) continue;
      total += p.rows * (1 + (p.columns * channels * bits + 7) / 8);
    }
    std::vector<std::uint8_t> raw(total);
    bool done = false, extra = false;
    std::string error;
    const std::size_t made = inflate_into(compressed.data(), compressed.size(), raw.data(), total, done, extra, error);
    if (!error.empty()) fail(kPngError, "IDAT: " + error);
    if (made < total) fail(kPngError, "Not enough image data");
    if (extra) warn("Too much image data");
    picture.samples.assign(static_cast<std::size_t>(picture.height) * picture.width * channels, 0);
    std::size_t offset = 0;
    for (const Pass& p : passes) {
      if (p.rows == 0 || p.columns == 0) continue;
      const std::size_t row_bytes = (p.columns * channels * bits + 7) / 8;
      std::vector<std::uint8_t> zeros(row_bytes, 0);
      const std::uint8_t* prior = zeros.data();
      for (std::size_t r = 0; r < p.rows; ++r) {
        std::uint8_t* row = raw.data() + offset + 1;
        unfilter(raw[offset], row, prior, row_bytes, bpp);
        prior = row;
        offset += 1 + row_bytes;
        std::uint16_t* out = picture.samples.data();
        const std::size_t y = p.first_row + r * p.row_step;
        for (std::size_t c = 0; c < p.columns; ++c) {
          const std::size_t x = p.first_column + c * p.column_step;
          std::uint16_t* pixel = out + (y * picture.width + x) * channels;
          for (std::size_t k = 0; k < channels; ++k) {
            const std::size_t i = c * channels + k;  // the sample's index in the row
            std::uint16_t value;
            if (bits == 16) {
              value = static_cast<std::uint16_t>((row[2 * i] << 8) | row[2 * i + 1]);
            } else if (bits == 8) {
              value = row[i];
            } else {
              const std::size_t bit = i * bits;
              value = static_cast<std::uint16_t>((row[bit / 8] >> (8 - bits - bit % 8)) & ((1u << bits) - 1));
            }
            pixel[k] = value;
          }
        }
      }
    }
    message = picture.warning;
    return kPngOk;
  } catch (const PngError& e) {
    picture = PngPicture{};
    message = e.message;
    return e.status;
  } catch (const std::bad_alloc&) {
    picture = PngPicture{};
    message = "out of memory";
    return kPngMemory;
  }
}

bool check_icc(const std::uint8_t* profile, std::uint64_t size, int channels, std::string& reason) {
  auto refuse = [&](const std::string& why) {
    reason = why;
    return false;
  };
  reason.clear();
  if (profile == nullptr || size < 132) return refuse("the profile has fewer than 132 bytes");
  const std::uint32_t length = be32(profile);
  if (length != size) return refuse("the profile's header gives " + std::to_string(length) + " bytes, not " +
                                    std::to_string(size));
  if (profile[8] >= 4 && length % 4 != 0) return refuse("a profile of version 4 is a whole number of 4 bytes");
  if (std::memcmp(profile + 36, "acsp", 4) != 0) return refuse("the profile's signature is not 'acsp'");
  const std::uint32_t intent = be32(profile + 64);
  if (intent >= 0xFFFF) return refuse("the profile's rendering intent is not known");
  const std::uint8_t* kind = profile + 12;
  if (std::memcmp(kind, "abst", 4) == 0 || std::memcmp(kind, "link", 4) == 0) {
    return refuse("an abstract or device link profile does not describe a picture");
  }
  const char* space = channels <= 2 ? "GRAY" : "RGB ";
  if (std::memcmp(profile + 16, space, 4) != 0) {
    return refuse(std::string("the profile's colour space is not the picture's ('") + space + "')");
  }
  if (std::memcmp(profile + 20, "XYZ ", 4) != 0 && std::memcmp(profile + 20, "Lab ", 4) != 0) {
    return refuse("the profile's connection space is neither XYZ nor Lab");
  }
  const std::uint32_t tags = be32(profile + 128);
  if (tags > (length - 132) / 12) return refuse("the profile's tag table runs past its end");
  for (std::uint32_t t = 0; t < tags; ++t) {
    const std::uint8_t* entry = profile + 132 + 12 * t;
    const std::uint64_t offset = be32(entry + 4), bytes = be32(entry + 8);
    if (offset > length || bytes > length - offset) return refuse("a tag of the profile runs past its end");
  }
  return true;
}

int write_png(const void* samples, std::uint32_t width, std::uint32_t height, int channels, int bits, int compression,
              const std::uint8_t* icc, std::size_t icc_size, std::vector<std::uint8_t>& file, std::string& warning,
              std::string& message) {
  file.clear();
  warning.clear();
  message.clear();
  if (samples == nullptr || width == 0 || height == 0 || width > 0x7FFFFFFFu || height > 0x7FFFFFFFu ||
      channels < 1 || channels > 4 || (bits != 8 && bits != 16) || compression < -1 || compression > 9) {
    message = "a picture of 1 to 4 channels, 8 or 16 bits, not empty, and a compression of -1 to 9";
    return kPngArgument;
  }
  try {
    const std::size_t bpp = static_cast<std::size_t>(channels) * (bits / 8);
    const std::size_t row_bytes = static_cast<std::size_t>(width) * bpp;
    // The rows in the file's byte order, each after its filter byte.
    std::vector<std::uint8_t> filtered(static_cast<std::size_t>(height) * (1 + row_bytes));
    std::vector<std::uint8_t> row(row_bytes), prior(row_bytes, 0), trial(row_bytes), best(row_bytes);
    for (std::uint32_t y = 0; y < height; ++y) {
      if (bits == 8) {
        std::memcpy(row.data(), static_cast<const std::uint8_t*>(samples) + y * row_bytes, row_bytes);
      } else {
        const std::uint16_t* from = static_cast<const std::uint16_t*>(samples) + static_cast<std::size_t>(y) * width * channels;
        for (std::size_t i = 0; i < row_bytes / 2; ++i) {
          row[2 * i] = static_cast<std::uint8_t>(from[i] >> 8);
          row[2 * i + 1] = static_cast<std::uint8_t>(from[i]);
        }
      }
      // Each of the five filters; the one whose bytes, taken as signed, sum to the least.
      std::uint64_t least = ~std::uint64_t{0};
      int chosen = 0;
      for (int type = 0; type < 5; ++type) {
        std::uint64_t sum = 0;
        for (std::size_t i = 0; i < row_bytes; ++i) {
          const int left = i >= bpp ? row[i - bpp] : 0, up = prior[i], corner = i >= bpp ? prior[i - bpp] : 0;
          const int predicted = type == 0 ? 0 : type == 1 ? left : type == 2 ? up : type == 3 ? (left + up) >> 1
                                                                                               : paeth(left, up, corner);
          trial[i] = static_cast<std::uint8_t>(row[i] - predicted);
          sum += trial[i] < 128 ? trial[i] : 256 - trial[i];
        }
        if (sum < least) {
          least = sum;
          chosen = type;
          best.swap(trial);
        }
      }
      std::uint8_t* out = filtered.data() + static_cast<std::size_t>(y) * (1 + row_bytes);
      out[0] = static_cast<std::uint8_t>(chosen);
      std::memcpy(out + 1, best.data(), row_bytes);
      prior.swap(row);
    }
    auto deflate_all = [&](const std::uint8_t* in, std::size_t in_size) {
      uLongf bound = compressBound(static_cast<uLong>(in_size));
      std::vector<std::uint8_t> out(bound);
      const int level = compression < 0 ? Z_DEFAULT_COMPRESSION : compression;
      if (compress2(out.data(), &bound, in, static_cast<uLong>(in_size), level) != Z_OK) {
        fail(kPngEncode, "zlib could not compress the picture");
      }
      out.resize(bound);
      return out;
    };
    auto chunk = [&](const char* type, const std::uint8_t* body, std::size_t length) {
      put32(file, static_cast<std::uint32_t>(length));
      const std::size_t at = file.size();
      file.insert(file.end(), type, type + 4);
      if (length > 0) file.insert(file.end(), body, body + length);
      put32(file, static_cast<std::uint32_t>(crc32(crc32(0, nullptr, 0), file.data() + at, static_cast<uInt>(length + 4))));
    };
    file.insert(file.end(), kSignature, kSignature + 8);
    std::vector<std::uint8_t> ihdr;
    put32(ihdr, width);
    put32(ihdr, height);
    ihdr.push_back(static_cast<std::uint8_t>(bits));
    ihdr.push_back(static_cast<std::uint8_t>(channels == 1 ? 0 : channels == 2 ? 4 : channels == 3 ? 2 : 6));
    ihdr.push_back(0);
    ihdr.push_back(0);
    ihdr.push_back(0);
    chunk("IHDR", ihdr.data(), ihdr.size());
    if (icc != nullptr) {
      std::string reason;
      if (!check_icc(icc, icc_size, channels, reason)) {
        warning = "the ICC profile is not written: " + reason;
      } else {
        static const char name[] = "ICC profile";
        std::vector<std::uint8_t> body(name, name + sizeof name);  // the name and its NUL
        body.push_back(0);                                        // deflate
        const std::vector<std::uint8_t> packed = deflate_all(icc, icc_size);
        body.insert(body.end(), packed.begin(), packed.end());
        chunk("iCCP", body.data(), body.size());
      }
    }
    const std::vector<std::uint8_t> packed = deflate_all(filtered.data(), filtered.size());
    // IDAT chunks of at most 1 GiB each.
    for (std::size_t at = 0; at < packed.size(); at += std::size_t{1} << 30) {
      chunk("IDAT", packed.data() + at, std::min<std::size_t>(packed.size() - at, std::size_t{1} << 30));
    }
    chunk("IEND", nullptr, 0);
    message = warning;
    return kPngOk;
  } catch (const PngError& e) {
    file.clear();
    message = e.message;
    return e.status;
  } catch (const std::bad_alloc&) {
    file.clear();
    message = "out of memory";
    return kPngMemory;
  }
}

}  // namespace urb
