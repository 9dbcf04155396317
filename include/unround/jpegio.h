/* The types of the reference's C layer that the C interface names
 * (c/jpegio/include/unround/jpegio.h:51-175 of JPEG-Unround, ABI version 3): its statuses,
 * colour spaces and the structures of a read file, laid out field for field as the reference
 * has them so that a caller's ctypes or cgo mirror binds unchanged. This build carries no
 * libjpeg-turbo or libpng: its own JPEG reader (ITU-T T.81) and PNG reader and writer (zlib)
 * stand behind the same contracts. */
#ifndef UNROUND_JPEGIO_H
#define UNROUND_JPEGIO_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define UNROUND_JPEGIO_ABI_VERSION 3
#define UNROUND_JPEGIO_MAX_COMPONENTS 4
#define UNROUND_JPEGIO_BLOCK_SIZE 64

typedef int32_t unround_jpegio_status; /* 0 ok; 1 argument; 2 decode; 3 unsupported; 4 limit; 5 memory; 6 encode; 7 png */

enum {
  UNROUND_JPEGIO_GRAYSCALE = 1,
  UNROUND_JPEGIO_YCBCR = 2,
  UNROUND_JPEGIO_RGB = 3,
};

typedef struct unround_jpegio_options {
  uint64_t max_pixels;
  int32_t max_scans;
  int32_t warnings_are_errors;
} unround_jpegio_options;

typedef struct unround_jpegio_component {
  int32_t id;
  int32_t h_samp_factor;
  int32_t v_samp_factor;
  int32_t quant_table_slot;
  uint32_t width;
  uint32_t height;
  uint32_t width_in_blocks;
  uint32_t height_in_blocks;
  uint16_t quant_table[UNROUND_JPEGIO_BLOCK_SIZE];
  int16_t* coefficients;
} unround_jpegio_component;

typedef struct unround_jpegio_image {
  uint32_t width;
  uint32_t height;
  int32_t color_space;
  int32_t num_components;
  int32_t max_h_samp_factor;
  int32_t max_v_samp_factor;
  int32_t progressive;
  int32_t arithmetic;
  int32_t exif_orientation;
  int32_t warnings;
  unround_jpegio_component components[UNROUND_JPEGIO_MAX_COMPONENTS];
  uint8_t* icc_profile;
  uint64_t icc_profile_size;
} unround_jpegio_image;

typedef struct unround_jpegio_plane {
  uint32_t width;
  uint32_t height;
  uint32_t stride;
  uint32_t reserved;
  uint8_t* samples;
} unround_jpegio_plane;

typedef struct unround_jpegio_planes {
  int32_t num_components;
  int32_t reserved;
  unround_jpegio_plane planes[UNROUND_JPEGIO_MAX_COMPONENTS];
} unround_jpegio_planes;

/* c/jpegio/include/unround/jpegio.h:134-175: a picture to write as a PNG file, a PNG file's
 * levels as it stores them, and bytes this layer allocated. */
typedef struct unround_jpegio_png {
  uint32_t width;
  uint32_t height;
  int32_t channels;    /* 1 grey, 2 grey and alpha, 3 RGB, 4 RGB and alpha */
  int32_t bits;        /* 8 or 16 */
  int32_t compression; /* zlib's level 0 to 9, or -1 for its default */
  int32_t reserved;
  const void* samples; /* height * width * channels: uint8_t, or uint16_t in this machine's order */
  const uint8_t* icc_profile;
  uint64_t icc_profile_size;
} unround_jpegio_png;

typedef struct unround_jpegio_png_image {
  uint32_t width;
  uint32_t height;
  int32_t channels;
  int32_t bits; /* 1, 2, 4, 8 or 16 */
  uint16_t* samples;
  uint8_t* icc_profile;
  uint64_t icc_profile_size;
} unround_jpegio_png_image;

typedef struct unround_jpegio_bytes {
  uint8_t* data;
  uint64_t size;
} unround_jpegio_bytes;

/* The C layer's PNG functions (c/jpegio/include/unround/jpegio.h:225-256), under its names, by
 * this build's own reader and writer (zlib): reads a file's levels (a palette file is refused,
 * UNSUPPORTED; max_pixels 0 means 1 << 28), and writes 8- or 16-bit levels with an iCCP chunk
 * where the profile goes with the picture. Each frees what it allocated. */
unround_jpegio_status unround_jpegio_read_png(const uint8_t* data, size_t size, uint64_t max_pixels,
                                              unround_jpegio_png_image* image, char* message, size_t message_size);
void unround_jpegio_png_image_free(unround_jpegio_png_image* image);
unround_jpegio_status unround_jpegio_write_png(const unround_jpegio_png* png, unround_jpegio_bytes* file, char* message,
                                               size_t message_size);
void unround_jpegio_bytes_free(unround_jpegio_bytes* bytes);

#ifdef __cplusplus
}
#endif

#endif
