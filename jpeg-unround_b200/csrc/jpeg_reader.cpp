// The JPEG reader (jpeg_reader.hpp), from ITU-T T.81. One pass over the markers: tables and
// frame header as they come, each scan's entropy-coded data decoded into the components'
// coefficient arrays (padded to whole MCUs while decoding, cut to the blocks that carry the
// picture at the end).
#include "jpeg_reader.hpp"

#include <algorithm>
#include <array>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <stdexcept>

namespace urb {

namespace {

// The zig-zag sequence: natural position of the k-th coefficient of a block's scan order
// (T.81 Figure A.6). 16 extra entries absorb a corrupt run that overshoots the block.
constexpr std::array<int, 80> kNatural = {
    0,  1,  8,  16, 9,  2,  3,  10, 17, 24, 32, 25, 18, 11, 4,  5,  12, 19, 26, 33, 40, 48, 41, 34, 27, 20, 13,
    6,  7,  14, 21, 28, 35, 42, 49, 56, 57, 50, 43, 36, 29, 22, 15, 23, 30, 37, 44, 51, 58, 59, 52, 45, 38, 31,
    39, 46, 53, 60, 61, 54, 47, 55, 62, 63, 63, 63, 63, 63, 63, 63, 63, 63, 63, 63, 63, 63, 63, 63, 63, 63};

struct JpegError {
  int status;
  std::string message;
};

[[noreturn]] void fail(int status, const std::string& message) { throw JpegError{status, message}; }

std::string hex(int value) {
  char text[8];
  std::snprintf(text, sizeof text, "0x%02x", value & 0xFF);
  return text;
}

// A Huffman table (T.81 Annex C and F.2.2.3): codes of up to 9 bits by one lookup, longer ones
// by the largest code of each length.
struct Huffman {
  bool defined = false;
  std::array<std::uint16_t, 512> fast{};  // (length << 8) | symbol for 9-bit prefixes; 0: longer
  std::array<std::int32_t, 18> maxcode{};  // the largest code of each length, -1 without one
  std::array<std::int32_t, 17> offset{};   // symbol index minus code, per length
  std::array<std::uint8_t, 256> symbols{};
};

void build(Huffman& h, const std::uint8_t counts[16], const std::uint8_t* symbols, int total) {
  h = Huffman{};
  std::copy(symbols, symbols + total, h.symbols.begin());
  std::int32_t code = 0;
  int k = 0;
  for (int length = 1; length <= 16; ++length) {
    const int n = counts[length - 1];
    h.offset[length] = k - code;
    for (int i = 0; i < n; ++i, ++k, ++code) {
      if (length <= 9) {
        const int shift = 9 - length;
        for (int fill = 0; fill < (1 << shift); ++fill) {
          h.fast[(code << shift) | fill] = static_cast<std::uint16_t>((length << 8) | symbols[k]);
        }
      }
    }
    // Codes of a length must fit in that many bits (and leave room for the longer ones).
    if (code > (1 << length)) fail(kJpegDecode, "a Huffman table has more codes than its lengths hold");
    h.maxcode[length] = n > 0 ? code - 1 : -1;
    code <<= 1;
  }
  h.maxcode[17] = 0x7FFFFFFF;
  h.defined = true;
}

}  // namespace

int exif_orientation_of(const std::uint8_t* data, std::size_t size) {
  static const std::uint8_t signature[6] = {'E', 'x', 'i', 'f', 0, 0};
  if (size < 6 + 8 || std::memcmp(data, signature, 6) != 0) return 0;
  const std::uint8_t* tiff = data + 6;
  const std::size_t length = size - 6;
  bool little;
  if (tiff[0] == 'I' && tiff[1] == 'I') {
    little = true;
  } else if (tiff[0] == 'M' && tiff[1] == 'M') {
    little = false;
  } else {
    return 0;
  }
  auto u16 = [&](const std::uint8_t* p) -> std::uint32_t {
    return little ? (p[0] | (p[1] << 8)) : ((p[0] << 8) | p[1]);
  };
  auto u32 = [&](const std::uint8_t* p) -> std::uint32_t {
    return little ? (std::uint32_t{p[0]} | (std::uint32_t{p[1]} << 8) | (std::uint32_t{p[2]} << 16) |
                     (std::uint32_t{p[3]} << 24))
                  : ((std::uint32_t{p[0]} << 24) | (std::uint32_t{p[1]} << 16) | (std::uint32_t{p[2]} << 8) |
                     std::uint32_t{p[3]});
  };
  if (u16(tiff + 2) != 42) return 0;
  const std::size_t ifd = u32(tiff + 4);
  if (ifd > length || length - ifd < 2) return 0;
  const std::size_t count = u16(tiff + ifd);
  for (std::size_t i = 0; i < count; ++i) {
    const std::size_t entry = ifd + 2 + 12 * i;
    if (entry > length || length - entry < 12) return 0;
    const std::uint8_t* e = tiff + entry;
    if (u16(e) != 0x0112) continue;
    if (u16(e + 2) != 3 || u32(e + 4) != 1) return 0;  // one SHORT
    const std::uint32_t value = u16(e + 8);
    return value >= 1 && value <= 8 ? static_cast<int>(value) : 0;
  }
  return 0;
}

namespace {

// A component while the file is read: its coefficients padded to whole MCUs.
struct Working {
  JpegComponent out;
  int quant_slot = 0;
  std::uint32_t padded_columns = 0, padded_rows = 0;  // blocks
  std::vector<std::int16_t> blocks;
  std::int32_t predictor = 0;  // the last DC value, in a scan
  std::int16_t* block(std::uint32_t row, std::uint32_t column) {
    return blocks.data() + (static_cast<std::size_t>(row) * padded_columns + column) * 64;
  }
};

class Reader {
 public:
  Reader(const std::uint8_t* data, std::size_t size, const JpegLimits& limits, JpegFile& file)
      : data_(data), size_(size), limits_(limits), file_(file) {}

  void read() {
    if (size_ < 2 || data_[0] != 0xFF || data_[1] != 0xD8) fail(kJpegDecode, "Not a JPEG file: starts with " +
                                                                                hex(size_ > 0 ? data_[0] : 0) + " " +
                                                                                hex(size_ > 1 ? data_[1] : 0));
    pos_ = 2;
    bool scanned = false;
    for (;;) {
      const int marker = next_marker();
      if (marker < 0) {
        // The data ends without an end-of-image marker.
        if (!scanned) fail(kJpegDecode, "JPEG datastream contains no image");
        if (!eof_warned_) warn("Premature end of JPEG file");
        break;
      }
      if (marker == 0xD9) {
        if (!scanned) fail(kJpegDecode, "JPEG datastream contains no image");
        break;
      }
      switch (marker) {
        case 0xC0:
        case 0xC1:
        case 0xC2:
          frame(marker == 0xC2);
          break;
        case 0xC3:
          fail(kJpegUnsupported, "lossless JPEG is not supported");
        case 0xC5:
        case 0xC6:
        case 0xC7:
        case 0xCD:
        case 0xCE:
        case 0xCF:
          fail(kJpegUnsupported, "hierarchical JPEG is not supported");
        case 0xC9:
        case 0xCA:
        case 0xCB:
          fail(kJpegUnsupported, "arithmetic-coded JPEG is not supported by this reader");
        case 0xC4:
          huffman_tables();
          break;
        case 0xCC:
          fail(kJpegUnsupported, "arithmetic-coded JPEG is not supported by this reader");
        case 0xDB:
          quant_tables();
          break;
        case 0xDD:
          restart_interval();
          break;
        case 0xDA:
          scan();
          scanned = true;
          break;
        case 0xDC:
          fail(kJpegUnsupported, "a DNL marker (the height after the first scan) is not supported");
        case 0xD8:
          fail(kJpegDecode, "Invalid JPEG file structure: two SOI markers");
        default:
          if (marker >= 0xD0 && marker <= 0xD7) {
            warn("Corrupt JPEG data: found marker " + hex(marker) + " outside a scan");
            break;
          }
          segment(marker);
          break;
      }
    }
    finish();
  }

 private:
  const std::uint8_t* data_;
  std::size_t size_;
  std::size_t pos_ = 0;
  const JpegLimits& limits_;
  JpegFile& file_;
  std::uint16_t quant_[4][64] = {};
  bool quant_defined_[4] = {};
  Huffman dc_[4], ac_[4];
  std::uint32_t restart_ = 0;
  bool framed_ = false, jfif_ = false, adobe_ = false;
  int transform_ = -1;
  int scans_ = 0;
  std::vector<Working> comps_;
  std::vector<std::pair<int, std::vector<std::uint8_t>>> icc_parts_;
  int icc_count_ = -1;
  bool icc_bad_ = false;
  // The entropy-coded data's bits.
  std::uint64_t acc_ = 0;
  int bits_ = 0;
  int fake_ = 0;  // zero bits past the data's end or a marker, at the accumulator's end
  bool stopped_ = false;
  bool fake_used_ = false;
  bool eof_warned_ = false;
  std::uint32_t eobrun_ = 0;

  void warn(const std::string& text) {
    if (file_.warnings == 0) file_.warning = text;
    if (file_.warnings < 0x7FFFFFFF) ++file_.warnings;
    if (limits_.warnings_are_errors) fail(kJpegDecode, text);
  }

  // The next marker's code, skipping (and counting as extraneous) what is not one; -1 at the end.
  int next_marker() {
    std::size_t skipped = 0;
    for (;;) {
      while (pos_ < size_ && data_[pos_] != 0xFF) {
        ++pos_;
        ++skipped;
      }
      while (pos_ < size_ && data_[pos_] == 0xFF) ++pos_;  // fill bytes
      if (pos_ >= size_) return -1;
      const int code = data_[pos_++];
      if (code == 0x00) {
        skipped += 2;  // a stuffed byte outside a scan
        continue;
      }
      if (skipped > 0) {
        warn("Corrupt JPEG data: " + std::to_string(skipped) + " extraneous bytes before marker " + hex(code));
      }
      return code;
    }
  }

  // A marker segment's length and bounds: returns the data after the length field.
  std::pair<const std::uint8_t*, std::size_t> payload() {
    if (size_ - pos_ < 2) fail(kJpegDecode, "Premature end of JPEG file within a marker");
    const std::size_t length = (std::size_t{data_[pos_]} << 8) | data_[pos_ + 1];
    if (length < 2) fail(kJpegDecode, "Bogus marker length");
    if (size_ - pos_ < length) fail(kJpegDecode, "Premature end of JPEG file within a marker");
    const std::uint8_t* p = data_ + pos_ + 2;
    pos_ += length;
    return {p, length - 2};
  }

  void frame(bool progressive) {
    const auto [p, n] = payload();
    if (framed_) fail(kJpegDecode, "Invalid JPEG file structure: two SOF markers");
    if (n < 6) fail(kJpegDecode, "Bogus marker length");
    const int precision = p[0];
    if (precision != 8) fail(kJpegUnsupported, std::to_string(precision) + "-bit JPEG is not supported");
    file_.height = (std::uint32_t{p[1]} << 8) | p[2];
    file_.width = (std::uint32_t{p[3]} << 8) | p[4];
    const int count = p[5];
    if (n != 6 + 3 * static_cast<std::size_t>(count) || count == 0) fail(kJpegDecode, "Bogus marker length");
    if (file_.width == 0 || file_.height == 0) fail(kJpegDecode, "Empty JPEG image (DNL not supported)");
    if (count > 4) fail(kJpegUnsupported, "a JPEG of " + std::to_string(count) + " components is not supported");
    file_.progressive = progressive;
    comps_.resize(count);
    for (int c = 0; c < count; ++c) {
      Working& w = comps_[c];
      w.out.id = p[6 + 3 * c];
      w.out.h = p[7 + 3 * c] >> 4;
      w.out.v = p[7 + 3 * c] & 15;
      w.quant_slot = w.out.slot = p[8 + 3 * c];
      if (w.out.h < 1 || w.out.h > 4 || w.out.v < 1 || w.out.v > 4) fail(kJpegDecode, "Bogus sampling factors");
      if (w.quant_slot > 3) fail(kJpegDecode, "Bogus quantization table number " + std::to_string(w.quant_slot));
      file_.hmax = std::max(file_.hmax, w.out.h);
      file_.vmax = std::max(file_.vmax, w.out.v);
    }
    const std::uint64_t pixels = std::uint64_t{file_.width} * file_.height;
    if (pixels > limits_.max_pixels) {
      fail(kJpegLimit, "the image has " + std::to_string(file_.width) + " x " + std::to_string(file_.height) +
                           " pixels, more than " + std::to_string(limits_.max_pixels));
    }
    // The MCUs of an interleaved scan; a component's blocks padded to them.
    const std::uint32_t mcu_columns = (file_.width + 8 * file_.hmax - 1) / (8 * file_.hmax);
    const std::uint32_t mcu_rows = (file_.height + 8 * file_.vmax - 1) / (8 * file_.vmax);
    for (Working& w : comps_) {
      w.out.width = static_cast<std::uint32_t>((std::uint64_t{file_.width} * w.out.h + file_.hmax - 1) / file_.hmax);
      w.out.height = static_cast<std::uint32_t>((std::uint64_t{file_.height} * w.out.v + file_.vmax - 1) / file_.vmax);
      w.out.width_in_blocks = (w.out.width + 7) / 8;
      w.out.height_in_blocks = (w.out.height + 7) / 8;
      w.padded_columns = std::max(w.out.width_in_blocks, mcu_columns * w.out.h);
      w.padded_rows = std::max(w.out.height_in_blocks, mcu_rows * w.out.v);
      w.blocks.assign(static_cast<std::size_t>(w.padded_columns) * w.padded_rows * 64, 0);
    }
    framed_ = true;
  }

  void huffman_tables() {
    auto [p, n] = payload();
    while (n > 0) {
      if (n < 17) fail(kJpegDecode, "Bogus DHT marker length");
      const int kind = p[0] >> 4, slot = p[0] & 15;
      if (kind > 1 || slot > 3) fail(kJpegDecode, "Bogus DHT index " + hex(p[0]));
      std::uint8_t counts[16];
      int total = 0;
      for (int i = 0; i < 16; ++i) total += counts[i] = p[1 + i];
      if (total > 256 || n < 17 + static_cast<std::size_t>(total)) fail(kJpegDecode, "Bogus Huffman table definition");
      build(kind == 0 ? dc_[slot] : ac_[slot], counts, p + 17, total);
      p += 17 + total;
      n -= 17 + total;
    }
  }

  void quant_tables() {
    auto [p, n] = payload();
    while (n > 0) {
      const int precision = p[0] >> 4, slot = p[0] & 15;
      if (slot > 3 || precision > 1) fail(kJpegDecode, "Bogus DQT index " + std::to_string(slot));
      const std::size_t need = 1 + 64 * static_cast<std::size_t>(precision + 1);
      if (n < need) fail(kJpegDecode, "Bogus marker length");
      for (int k = 0; k < 64; ++k) {
        const std::uint16_t value = precision == 0 ? p[1 + k] : static_cast<std::uint16_t>((p[1 + 2 * k] << 8) | p[2 + 2 * k]);
        quant_[slot][kNatural[k]] = value;
      }
      quant_defined_[slot] = true;
      p += need;
      n -= need;
    }
  }

  void restart_interval() {
    const auto [p, n] = payload();
    if (n != 2) fail(kJpegDecode, "Bogus marker length");
    restart_ = (std::uint32_t{p[0]} << 8) | p[1];
  }

  // APPn, COM and the rest: JFIF (APP0), EXIF (APP1), ICC (APP2) and Adobe (APP14) are read.
  void segment(int marker) {
    const auto [p, n] = payload();
    if (marker == 0xE0 && n >= 14 && std::memcmp(p, "JFIF\0", 5) == 0) jfif_ = true;
    if (marker == 0xEE && n >= 12 && std::memcmp(p, "Adobe", 5) == 0) {
      adobe_ = true;
      transform_ = p[11];
    }
    if (marker == 0xE1 && file_.exif_orientation == 0) file_.exif_orientation = exif_orientation_of(p, n);
    if (marker == 0xE2 && n >= 14 && std::memcmp(p, "ICC_PROFILE\0", 12) == 0) {
      const int sequence = p[12], count = p[13];
      if (icc_count_ < 0) icc_count_ = count;
      if (count == 0 || count != icc_count_ || sequence == 0 || sequence > count) icc_bad_ = true;
      icc_parts_.emplace_back(sequence, std::vector<std::uint8_t>(p + 14, p + n));
    }
  }

  // --- The entropy-coded data. -------------------------------------------------------------

  void reset_bits() {
    acc_ = 0;
    bits_ = 0;
    fake_ = 0;
  }

  // Tops the accumulator up to at least 57 bits: data bytes (0xFF 0x00 is 0xFF), and zeros once
  // a marker or the end is reached.
  void fill() {
    // Four bytes at once where none of them is 0xFF (no stuffing, no marker).
    while (bits_ <= 32 && !stopped_ && size_ - pos_ >= 4) {
      const std::uint32_t word = (std::uint32_t{data_[pos_]} << 24) | (std::uint32_t{data_[pos_ + 1]} << 16) |
                                 (std::uint32_t{data_[pos_ + 2]} << 8) | std::uint32_t{data_[pos_ + 3]};
      // A byte of the word is 0xFF where its complement has a zero byte.
      const std::uint32_t inverse = ~word;
      if (((inverse - 0x01010101u) & ~inverse & 0x80808080u) != 0) break;
      acc_ |= std::uint64_t{word} << (32 - bits_);
      bits_ += 32;
      pos_ += 4;
    }
    while (bits_ <= 56) {
      std::uint64_t byte = 0;
      if (!stopped_ && pos_ < size_) {
        const std::uint8_t b = data_[pos_];
        if (b != 0xFF) {
          byte = b;
          ++pos_;
        } else if (pos_ + 1 < size_ && data_[pos_ + 1] == 0x00) {
          byte = 0xFF;
          pos_ += 2;
        } else {
          stopped_ = true;  // a marker (or 0xFF at the end): the segment ends here
        }
      } else {
        stopped_ = true;
        if (pos_ >= size_ && !eof_warned_) {
          // The data ends within a scan: as a reader whose source runs dry, before any bits are
          // found missing.
          eof_warned_ = true;
          warn("Premature end of JPEG file");
        }
      }
      if (stopped_) fake_ += 8;
      acc_ |= byte << (56 - bits_);
      bits_ += 8;
    }
  }

  void consume(int n) {
    acc_ <<= n;
    bits_ -= n;
    if (bits_ < fake_) {
      fake_used_ = true;
      fake_ = bits_;
    }
  }

  std::uint32_t get(int n) {
    if (n == 0) return 0;
    if (bits_ < n) fill();
    const std::uint32_t value = static_cast<std::uint32_t>(acc_ >> (64 - n));
    consume(n);
    return value;
  }

  // T.81 F.2.2.1: the s-bit value's two's-complement extension.
  std::int32_t extend(int s) {
    if (s == 0) return 0;
    if (s > 16) {
      warn("Corrupt JPEG data: bad Huffman code");
      s = 16;
    }
    const std::int32_t v = static_cast<std::int32_t>(get(s));
    return v < (1 << (s - 1)) ? v - (1 << s) + 1 : v;
  }

  int decode(const Huffman& h) {
    if (bits_ < 16) fill();
    const std::uint16_t hit = h.fast[acc_ >> 55];
    if (hit != 0) {
      consume(hit >> 8);
      return hit & 0xFF;
    }
    for (int length = 10; length <= 16; ++length) {
      const std::int32_t code = static_cast<std::int32_t>(acc_ >> (64 - length));
      if (code <= h.maxcode[length]) {
        consume(length);
        return h.symbols[(h.offset[length] + code) & 0xFF];
      }
    }
    consume(16);
    warn("Corrupt JPEG data: bad Huffman code");
    return 0;
  }

  // After restart_ units: the RSTn marker, the predictors and the end-of-band run reset.
  void restart(int& expected) {
    reset_bits();
    stopped_ = false;
    std::size_t skipped = 0;
    while (pos_ < size_ && data_[pos_] != 0xFF) {
      ++pos_;
      ++skipped;
    }
    std::size_t at = pos_;
    while (at < size_ && data_[at] == 0xFF) ++at;
    const int code = at < size_ ? data_[at] : -1;
    if (code == 0xD0 + expected) {
      if (skipped > 0) {
        warn("Corrupt JPEG data: " + std::to_string(skipped) + " extraneous bytes before marker " + hex(code));
      }
      pos_ = at + 1;
    } else if (code >= 0xD0 && code <= 0xD7) {
      warn("Corrupt JPEG data: found marker " + hex(code) + " instead of RST" + std::to_string(expected));
      pos_ = at + 1;
    } else {
      // Not a restart marker: the rest of the scan reads as zeros.
      warn("Corrupt JPEG data: found marker " + hex(code < 0 ? 0 : code) + " instead of RST" +
           std::to_string(expected));
      stopped_ = true;
    }
    expected = (expected + 1) & 7;
    for (Working& w : comps_) w.predictor = 0;
    eobrun_ = 0;
  }

  // --- Scans. --------------------------------------------------------------------------------

  struct ScanPart {
    Working* w;
    const Huffman* dc;
    const Huffman* ac;
  };

  void scan() {
    const auto [p, n] = payload();
    if (!framed_) fail(kJpegDecode, "Invalid JPEG file structure: SOS before SOF");
    if (++scans_ > limits_.max_scans) fail(kJpegLimit, "the file has more than " + std::to_string(limits_.max_scans) + " scans");
    if (n < 1) fail(kJpegDecode, "Bogus marker length");
    const int count = p[0];
    if (count < 1 || count > 4 || n != 4 + 2 * static_cast<std::size_t>(count)) fail(kJpegDecode, "Bogus marker length");
    const int ss = p[1 + 2 * count], se = p[2 + 2 * count], ah = p[3 + 2 * count] >> 4, al = p[3 + 2 * count] & 15;
    std::vector<ScanPart> parts;
    int blocks_per_mcu = 0;
    for (int i = 0; i < count; ++i) {
      const int id = p[1 + 2 * i], tables = p[2 + 2 * i];
      Working* w = nullptr;
      for (Working& c : comps_) {
        if (c.out.id == id) w = &c;
      }
      if (w == nullptr) fail(kJpegDecode, "Invalid component ID " + std::to_string(id) + " in SOS");
      for (const ScanPart& q : parts) {
        if (q.w == w) fail(kJpegDecode, "Invalid component ID " + std::to_string(id) + " in SOS");
      }
      const int dc = tables >> 4, ac = tables & 15;
      if (dc > 3 || ac > 3) fail(kJpegDecode, "Bogus Huffman table number");
      parts.push_back({w, &dc_[dc], &ac_[ac]});
      blocks_per_mcu += w->out.h * w->out.v;
    }
    if (count > 1 && blocks_per_mcu > 10) fail(kJpegDecode, "Sampling factors too large for interleaved scan");
    if (file_.progressive) {
      const bool valid = ss == 0 ? se == 0 : (se >= ss && se <= 63 && count == 1);
      if (!valid || ah > 13 || al > 13) {
        fail(kJpegDecode, "Invalid progressive parameters Ss=" + std::to_string(ss) + " Se=" + std::to_string(se) +
                              " Ah=" + std::to_string(ah) + " Al=" + std::to_string(al));
      }
    } else if (ss != 0 || se != 63 || ah != 0 || al != 0) {
      // libjpeg takes a sequential scan's Ss, Se, Ah and Al as 0, 63, 0, 0 with a warning.
      warn("Invalid SOS parameters for sequential JPEG");
    }
    const bool sequential = !file_.progressive;
    const int start = sequential ? 0 : ss, end = sequential ? 63 : se;
    const int high = sequential ? 0 : ah, low = sequential ? 0 : al;
    for (ScanPart& part : parts) {
      Working& w = *part.w;
      if (!w.out.latched) {
        if (!quant_defined_[w.quant_slot]) {
          fail(kJpegDecode, "Quantization table " + hex(w.quant_slot) + " was not defined");
        }
        std::copy(quant_[w.quant_slot], quant_[w.quant_slot] + 64, w.out.table);
        w.out.latched = true;
      }
      const bool needs_dc = start == 0 && high == 0, needs_ac = end > 0;
      if ((needs_dc && !part.dc->defined) || (needs_ac && !part.ac->defined)) {
        fail(kJpegDecode, "Huffman table was not defined");
      }
      w.predictor = 0;
    }
    reset_bits();
    stopped_ = false;
    fake_used_ = false;
    eobrun_ = 0;
    int expected = 0;
    std::uint32_t left = restart_;
    auto unit = [&](Working& w, const ScanPart& part, std::uint32_t row, std::uint32_t column) {
      std::int16_t* b = w.block(row, column);
      if (sequential) {
        sequential_block(b, w, part);
      } else if (start == 0) {
        if (high == 0) {
          const int s = decode(*part.dc);
          w.predictor += extend(s);
          b[0] = static_cast<std::int16_t>(w.predictor * (1 << low));
        } else if (get(1) != 0) {
          b[0] = static_cast<std::int16_t>(b[0] | (1 << low));
        }
      } else if (high == 0) {
        ac_first(b, *part.ac, start, end, low);
      } else {
        ac_refine(b, *part.ac, start, end, low);
      }
    };
    if (count == 1) {
      Working& w = *parts[0].w;
      for (std::uint32_t row = 0; row < w.out.height_in_blocks; ++row) {
        for (std::uint32_t column = 0; column < w.out.width_in_blocks; ++column) {
          if (restart_ != 0 && left == 0) {
            restart(expected);
            left = restart_;
          }
          unit(w, parts[0], row, column);
          --left;
        }
      }
    } else {
      const std::uint32_t mcu_columns = (file_.width + 8 * file_.hmax - 1) / (8 * file_.hmax);
      const std::uint32_t mcu_rows = (file_.height + 8 * file_.vmax - 1) / (8 * file_.vmax);
      for (std::uint32_t my = 0; my < mcu_rows; ++my) {
        for (std::uint32_t mx = 0; mx < mcu_columns; ++mx) {
          if (restart_ != 0 && left == 0) {
            restart(expected);
            left = restart_;
          }
          for (const ScanPart& part : parts) {
            Working& w = *part.w;
            for (int v = 0; v < w.out.v; ++v) {
              for (int h = 0; h < w.out.h; ++h) {
                unit(w, part, my * w.out.v + v, mx * w.out.h + h);
              }
            }
          }
          --left;
        }
      }
    }
    if (fake_used_) warn("Corrupt JPEG data: premature end of data segment");
    // What the bit reader fetched ahead belongs to this scan; the next marker follows.
    reset_bits();
    stopped_ = false;
  }

  // T.81 F.2.2: the DC difference and the run-length coded AC coefficients of a block.
  void sequential_block(std::int16_t* b, Working& w, const ScanPart& part) {
    const int s = decode(*part.dc);
    w.predictor += extend(s);
    b[0] = static_cast<std::int16_t>(w.predictor);
    for (int k = 1; k < 64;) {
      const int rs = decode(*part.ac);
      const int r = rs >> 4, size = rs & 15;
      if (size != 0) {
        k += r;
        const std::int32_t value = extend(size);
        if (k > 63) {
          warn("Corrupt JPEG data: a run of coefficients past the block's end");
          break;
        }
        b[kNatural[k]] = static_cast<std::int16_t>(value);
        ++k;
      } else if (r == 15) {
        k += 16;
      } else {
        break;
      }
    }
  }

  // T.81 G.1.2.2: the first pass over a band of AC coefficients, with end-of-band runs.
  void ac_first(std::int16_t* b, const Huffman& ac, int start, int end, int low) {
    if (eobrun_ > 0) {
      --eobrun_;
      return;
    }
    for (int k = start; k <= end;) {
      const int rs = decode(ac);
      const int r = rs >> 4, size = rs & 15;
      if (size != 0) {
        k += r;
        const std::int32_t value = extend(size);
        if (k > end) {
          warn("Corrupt JPEG data: a run of coefficients past the band's end");
          break;
        }
        b[kNatural[k]] = static_cast<std::int16_t>(value * (1 << low));
        ++k;
      } else if (r == 15) {
        k += 16;
      } else {
        eobrun_ = (1u << r) - 1;
        if (r != 0) eobrun_ += get(r);
        break;
      }
    }
  }

  // T.81 G.1.2.3: a refinement pass over a band: one correction bit for each coefficient that
  // is already nonzero, and new coefficients of magnitude 1 << low placed among the zeros.
  void ac_refine(std::int16_t* b, const Huffman& ac, int start, int end, int low) {
    const int plus = 1 << low, minus = -(1 << low);
    auto correct = [&](std::int16_t& c) {
      if (get(1) != 0 && (c & plus) == 0) c = static_cast<std::int16_t>(c + (c >= 0 ? plus : minus));
    };
    int k = start;
    if (eobrun_ == 0) {
      for (; k <= end; ++k) {
        const int rs = decode(ac);
        int r = rs >> 4;
        const int size = rs & 15;
        int value = 0;
        if (size != 0) {
          if (size != 1) warn("Corrupt JPEG data: a refinement coefficient of more than one bit");
          value = get(1) != 0 ? plus : minus;
        } else if (r != 15) {
          eobrun_ = 1u << r;
          if (r != 0) eobrun_ += get(r);
          break;  // the rest of the band takes its correction bits below
        }
        // Skip r zero coefficients (correcting the nonzero ones passed), then place the new one.
        while (k <= end) {
          std::int16_t& c = b[kNatural[k]];
          if (c != 0) {
            correct(c);
          } else {
            if (r == 0) break;
            --r;
          }
          ++k;
        }
        if (value != 0 && k <= end) b[kNatural[k]] = static_cast<std::int16_t>(value);
      }
    }
    if (eobrun_ > 0) {
      for (; k <= end; ++k) {
        std::int16_t& c = b[kNatural[k]];
        if (c != 0) correct(c);
      }
      --eobrun_;
    }
  }

  // The colour space, the ICC profile, and the coefficients cut to the picture's blocks.
  void finish() {
    const int count = static_cast<int>(comps_.size());
    if (count == 1) {
      file_.color_space = 1;
    } else if (count == 3) {
      if (jfif_) {
        file_.color_space = 2;
      } else if (adobe_) {
        if (transform_ == 0) {
          file_.color_space = 3;
        } else {
          if (transform_ != 1) warn("Unknown Adobe color transform code " + std::to_string(transform_));
          file_.color_space = 2;
        }
      } else {
        const int a = comps_[0].out.id, b = comps_[1].out.id, c = comps_[2].out.id;
        file_.color_space = a == 82 && b == 71 && c == 66 ? 3 : 2;
      }
    } else {
      fail(kJpegUnsupported, "a JPEG of " + std::to_string(count) + " components is not supported");
    }
    if (!icc_parts_.empty()) {
      std::vector<const std::vector<std::uint8_t>*> ordered(icc_count_ > 0 ? icc_count_ : 0, nullptr);
      for (const auto& [sequence, bytes] : icc_parts_) {
        if (icc_bad_ || sequence < 1 || sequence > static_cast<int>(ordered.size()) || ordered[sequence - 1] != nullptr) {
          icc_bad_ = true;
          break;
        }
        ordered[sequence - 1] = &bytes;
      }
      for (const auto* part : ordered) icc_bad_ = icc_bad_ || part == nullptr;
      if (icc_bad_) {
        warn("Corrupt JPEG data: bad ICC marker");
      } else {
        for (const auto* part : ordered) file_.icc.insert(file_.icc.end(), part->begin(), part->end());
      }
    }
    file_.components.clear();
    for (Working& w : comps_) {
      if (!w.out.latched) fail(kJpegDecode, "the file ends before the data of every component");
      JpegComponent out = w.out;
      if (w.padded_columns == out.width_in_blocks && w.padded_rows == out.height_in_blocks) {
        out.coefficients = std::move(w.blocks);  // no dummy blocks: the arrays are the picture's
      } else {
        const std::size_t row = static_cast<std::size_t>(out.width_in_blocks) * 64;
        out.coefficients.resize(row * out.height_in_blocks);
        for (std::uint32_t r = 0; r < out.height_in_blocks; ++r) {
          std::memcpy(out.coefficients.data() + r * row, w.block(r, 0), row * sizeof(std::int16_t));
        }
      }
      std::vector<std::int16_t>().swap(w.blocks);
      file_.components.push_back(std::move(out));
    }
  }
};

}  // namespace

int read_jpeg(const std::uint8_t* data, std::size_t size, const JpegLimits& limits, JpegFile& file,
              std::string& message) {
  file = JpegFile{};
  message.clear();
  if (data == nullptr && size > 0) {
    message = "the data is a null pointer";
    return kJpegArgument;
  }
  try {
    Reader reader(data, size, limits, file);
    reader.read();
    message = file.warning;
    return kJpegOk;
  } catch (const JpegError& e) {
    file = JpegFile{};
    message = e.message;
    return e.status;
  } catch (const std::bad_alloc&) {
    file = JpegFile{};
    message = "out of memory";
    return kJpegMemory;
  }
}

std::vector<std::uint8_t> component_plane(const JpegComponent& component) {
  // The orthonormal 8-point inverse DCT, rows then columns, in binary64.
  static const auto basis = [] {
    std::array<double, 64> t{};
    const double pi = std::acos(-1.0);
    for (int x = 0; x < 8; ++x) {
      for (int u = 0; u < 8; ++u) {
        t[x * 8 + u] = (u == 0 ? std::sqrt(0.125) : 0.5) * std::cos((2 * x + 1) * u * pi / 16.0);
      }
    }
    return t;
  }();
  const std::size_t columns = static_cast<std::size_t>(component.width_in_blocks) * 8;
  const std::size_t rows = static_cast<std::size_t>(component.height_in_blocks) * 8;
  std::vector<std::uint8_t> plane(rows * columns);
  for (std::uint32_t by = 0; by < component.height_in_blocks; ++by) {
    for (std::uint32_t bx = 0; bx < component.width_in_blocks; ++bx) {
      const std::int16_t* c =
          component.coefficients.data() + (static_cast<std::size_t>(by) * component.width_in_blocks + bx) * 64;
      double f[64], g[64];
      for (int k = 0; k < 64; ++k) f[k] = static_cast<double>(c[k]) * component.table[k];
      for (int v = 0; v < 8; ++v) {  // rows of coefficients to rows of samples across
        for (int x = 0; x < 8; ++x) {
          double s = 0.0;
          for (int u = 0; u < 8; ++u) s += basis[x * 8 + u] * f[v * 8 + u];
          g[v * 8 + x] = s;
        }
      }
      for (int y = 0; y < 8; ++y) {
        for (int x = 0; x < 8; ++x) {
          double s = 0.0;
          for (int v = 0; v < 8; ++v) s += basis[y * 8 + v] * g[v * 8 + x];
          const double level = std::nearbyint(s + 128.0);
          plane[(by * 8 + y) * columns + bx * 8 + x] =
              static_cast<std::uint8_t>(level < 0.0 ? 0.0 : (level > 255.0 ? 255.0 : level));
        }
      }
    }
  }
  return plane;
}

}  // namespace urb
