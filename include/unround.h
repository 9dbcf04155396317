/* The C interface of JPEG-Unround's reconstruction, ABI version 5, as a drop-in for the
 * reference's cdylib unround_capi (rust/capi/include/unround.h of JPEG-Unround): the same
 * functions, structures and statuses, so that the reference's Python package (ctypes,
 * python/src/unround/native.py:169-214) and any cgo/JNI/N-API binding load this library
 * unchanged. The reconstruction runs on a B200: the TV/TGV primal-dual iterations are
 * binary32 CUDA kernels, the records and the result binary64.
 *
 * Every function that computes returns a status and writes what went wrong into the caller's
 * message buffer (NUL-terminated, cut at a UTF-8 character boundary; null allowed). No error
 * crosses the interface as anything but a status: a device error (launch failure, out of
 * memory) is UNROUND_ERROR_INTERNAL with its message. Different settings and results can be
 * used on different threads at once: each call has its own CUDA stream and device buffers.
 *
 * Each declaration cites the reference declaration it replaces (rust/capi/include/unround.h,
 * line numbers of that file). Files are read and written on the host by this build's own JPEG
 * reader (ITU-T T.81: baseline, extended and progressive Huffman files) and PNG reader and writer
 * (zlib), in place of libjpeg-turbo and libpng; a picture's projection onto a file's intervals
 * (unround_project) is computed on the host in binary64, and the TIFF writer holds binary64
 * samples bit for bit; the command line is exported and refuses (unround_main returns 3). */
#ifndef UNROUND_H
#define UNROUND_H

#include <stddef.h>
#include <stdint.h>

#include "unround/jpegio.h"

#ifdef __cplusplus
extern "C" {
#endif

#define UNROUND_ABI_VERSION 5

/* unround.h:44-52 */
typedef int32_t unround_status;
enum {
  UNROUND_OK = 0,
  UNROUND_ERROR_ARGUMENT = 1,
  UNROUND_ERROR_READ = 2,
  UNROUND_ERROR_UNSUPPORTED = 3,
  UNROUND_ERROR_OPTIONS = 4,
  UNROUND_ERROR_IO = 5,
  UNROUND_ERROR_INTERNAL = 6,
};

/* unround.h:54-57 */
int32_t unround_abi_version(void);
const char* unround_version(void);

/* Settings: unround.h:62-76. Options by the reference command line's names. */
typedef struct unround_settings unround_settings;
unround_settings* unround_settings_new(size_t count, const char* const* options, char* message, size_t message_size);
void unround_settings_free(unround_settings* settings);
size_t unround_settings_options(const unround_settings* settings, char* buffer, size_t size);

/* unround.h:85-94: a record as an observer sees it. */
typedef struct unround_record {
  uint64_t iteration;
  double gap;
  double primal;
  double dual;
  uint64_t channels;
  uint64_t height;
  uint64_t width;
  const double* canvas;
} unround_record;

/* unround.h:97: called with each record after the first; nonzero stops the solver. */
typedef int32_t (*unround_observer)(void* user, const unround_record* record);

/* unround.h:101-108 */
typedef struct unround_component {
  const int16_t* levels;
  uint32_t rows;
  uint32_t columns;
  int32_t h_samp_factor;
  int32_t v_samp_factor;
  uint16_t quant_table[64];
} unround_component;

/* unround.h:112-118 */
typedef struct unround_input {
  uint32_t height;
  uint32_t width;
  int32_t color_space;
  uint32_t count;
  const unround_component* components;
} unround_input;

typedef struct unround_result unround_result;

/* unround.h:123-126 */
enum {
  UNROUND_FORMAT_JPEG = 1,
  UNROUND_FORMAT_PNG = 2,
};

/* unround.h:134-136: needs libjpeg-turbo; UNROUND_ERROR_UNSUPPORTED here. */
unround_status unround_decode(const uint8_t* data, size_t size, const unround_settings* settings,
                              unround_observer observer, void* user, unround_result** result, char* message,
                              size_t message_size);

/* unround.h:139-140: the hot path. Reconstructs components given as arrays on the GPU. */
unround_status unround_solve(const unround_input* input, const unround_settings* settings, unround_observer observer,
                             void* user, unround_result** result, char* message, size_t message_size);

/* unround.h:142-150: a picture measured against a JPEG file's intervals and projected onto them,
 * on the host in binary64; the result has no solver, and unround_result_excess gives each
 * component's excess in steps. */
unround_status unround_project(const uint8_t* data, size_t size, const unround_settings* settings,
                               const double* picture, uint64_t height, uint64_t width, uint64_t channels,
                               unround_result** result, char* message, size_t message_size);

/* Result getters: unround.h:152-253. */
void unround_result_free(unround_result* result);
const double* unround_result_picture(const unround_result* result, uint64_t* height, uint64_t* width,
                                     uint64_t* channels);
const double* unround_result_planes(const unround_result* result, uint64_t* count);
int32_t unround_result_color_space(const unround_result* result);
const double* unround_result_canvas(const unround_result* result, uint64_t* channels, uint64_t* height,
                                    uint64_t* width);
uint64_t unround_result_components(const unround_result* result);
const double* unround_result_coefficients(const unround_result* result, uint64_t component, uint64_t* count);
const double* unround_result_problem(const unround_result* result, uint64_t component, int32_t which, uint64_t* count);
unround_status unround_result_component(const unround_result* result, uint64_t component, uint64_t* rows,
                                        uint64_t* columns, uint64_t* down, uint64_t* across);
int32_t unround_result_solver(const unround_result* result, uint64_t* iterations, int32_t* stop);
const uint64_t* unround_result_record_iterations(const unround_result* result, uint64_t* count);
const double* unround_result_record_values(const unround_result* result, int32_t which, uint64_t* count);
int32_t unround_result_alpha_solver(const unround_result* result, uint64_t* iterations, int32_t* stop);
const uint64_t* unround_result_alpha_record_iterations(const unround_result* result, uint64_t* count);
const double* unround_result_alpha_record_values(const unround_result* result, int32_t which, uint64_t* count);
const uint8_t* unround_result_icc_profile(const unround_result* result, uint64_t* size);
int32_t unround_result_exif_orientation(const unround_result* result);
int32_t unround_result_format(const unround_result* result);
int32_t unround_result_bits(const unround_result* result);
const char* unround_result_warning(const unround_result* result);
const double* unround_result_excess(const unround_result* result, uint64_t component, uint64_t* count);

/* Output and conversion: unround.h:258-302. The writers need zlib/libpng and return
 * UNROUND_ERROR_UNSUPPORTED here; JFIF's conversions are computed. */
unround_status unround_tiff(const double* samples, uint64_t height, uint64_t width, uint64_t channels, int32_t ycbcr,
                            const uint8_t* icc, uint64_t icc_size, uint8_t** bytes, uint64_t* size, char* message,
                            size_t message_size);
enum {
  UNROUND_DITHER_NONE = 0,
  UNROUND_DITHER_BLUE_NOISE = 1,
  UNROUND_DITHER_BLUE_NOISE_TOGETHER = 2,
};
unround_status unround_png(const double* samples, uint64_t height, uint64_t width, uint64_t channels, int32_t sixteen,
                           int32_t dither, int32_t compression, const uint8_t* icc, uint64_t icc_size, uint8_t** bytes,
                           uint64_t* size, char* message, size_t message_size);
unround_status unround_pnm(const double* samples, uint64_t height, uint64_t width, uint64_t channels, int32_t sixteen,
                           int32_t dither, uint8_t** bytes, uint64_t* size, char* message, size_t message_size);
void unround_bytes_free(uint8_t* bytes, uint64_t size);
unround_status unround_orient(const double* samples, uint64_t height, uint64_t width, uint64_t channels,
                              int32_t orientation, double* turned, uint64_t* turned_height, uint64_t* turned_width,
                              char* message, size_t message_size);
unround_status unround_to_rgb(const double* planes, uint64_t height, uint64_t width, double* picture);
unround_status unround_to_ycbcr(const double* picture, uint64_t height, uint64_t width, double* planes);

/* unround.h:306-307: the command line is outside this library's path; returns 3. */
int32_t unround_main(size_t count, const char* const* arguments);

/* The C layer through this library: unround.h:309-320. No libjpeg here. */
int32_t unround_jpeg_abi_version(void);
const char* unround_jpeg_libjpeg_version(void);
const char* unround_jpeg_libpng_version(void);
int32_t unround_jpeg_check_icc(const uint8_t* profile, uint64_t size, int32_t channels, char* reason,
                               size_t reason_size);
unround_jpegio_status unround_jpeg_read(const uint8_t* data, size_t size, const unround_jpegio_options* options,
                                        unround_jpegio_image* image, char* message, size_t message_size);
void unround_jpeg_image_free(unround_jpegio_image* image);
unround_jpegio_status unround_jpeg_decode_planes(const uint8_t* data, size_t size,
                                                 const unround_jpegio_options* options, unround_jpegio_planes* planes,
                                                 char* message, size_t message_size);
void unround_jpeg_planes_free(unround_jpegio_planes* planes);

#ifdef __cplusplus
}
#endif

#ifdef __cplusplus
static_assert(sizeof(unround_record) == 64, "the layout of unround_record");
static_assert(sizeof(unround_component) == 152, "the layout of unround_component");
static_assert(offsetof(unround_component, quant_table) == 24, "the layout of unround_component");
static_assert(sizeof(unround_input) == 24, "the layout of unround_input");
static_assert(offsetof(unround_input, components) == 16, "the layout of unround_input");
#else
_Static_assert(sizeof(unround_record) == 64, "the layout of unround_record");
_Static_assert(sizeof(unround_component) == 152, "the layout of unround_component");
_Static_assert(sizeof(unround_input) == 24, "the layout of unround_input");
#endif

#endif
