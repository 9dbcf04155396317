/* Extensions of this build beside the reference's C interface (unround.h). They have no
 * counterpart in unround.h of the reference unless a comment names one; the reference's
 * callers need none of them.
 *
 * Plain pointers and sizes only. Host arrays are binary64 unless named otherwise. */
#ifndef UNROUND_B200_H
#define UNROUND_B200_H

#include <stddef.h>
#include <stdint.h>

#include "unround.h"

#ifdef __cplusplus
extern "C" {
#endif

/* A state to start from (the reference library's pdhg::Start, cpp/include/unround/pdhg.hpp:124-133,
 * which its C interface does not expose): every component's coefficients, all components'
 * blocks one after another, which are clipped to their intervals; and each channel's dual
 * fields p (2 planes), w (2 planes, TGV) and r (3 planes, TGV) of canvas rows x columns,
 * channel after channel, which are projected onto their balls. A null pointer leaves that
 * part at the default start (docs/math.md 5). */
typedef struct unround_b200_start {
  const double* coefficients;
  const double* p;
  const double* w;
  const double* r;
} unround_b200_start;

/* unround_solve from a given start. */
unround_status unround_b200_solve_from(const unround_input* input, const unround_settings* settings,
                                       const unround_b200_start* start, unround_observer observer, void* user,
                                       unround_result** result, char* message, size_t message_size);

/* Measurement of the iteration loop alone (no records, no host copies): the settings' method
 * on the input, `warmup` iterations untimed, then `iterations` timed with CUDA events on the
 * solve's stream. Writes the device milliseconds of the timed iterations, the kernels
 * launched per iteration, the canvas's samples and the device bytes held, and each kernel
 * group's average time from 20 further iterations with events around every launch. With `result`
 * non-null, the binary64 result of the last iterate is made as unround_solve makes it. */
typedef struct unround_b200_timing {
  double milliseconds;
  double dual_milliseconds;   /* one iteration's dual-step kernel, averaged over 20 timed apart */
  double primal_milliseconds; /* one iteration's primal-step kernels (every component), likewise */
  uint64_t iterations;
  uint64_t launches_per_iteration;
  uint64_t samples;
  uint64_t pixels;
  uint64_t device_bytes;
} unround_b200_timing;

unround_status unround_b200_measure(const unround_input* input, const unround_settings* settings, uint64_t warmup,
                                    uint64_t iterations, unround_b200_timing* timing, unround_result** result,
                                    char* message, size_t message_size);

/* Many pictures solved together (no counterpart in the reference, whose callers solve one
 * picture a call): `count` inputs, each with its settings (tv or tgv, the same number of
 * iterations, --record-every 0), into `count` results, each freed by unround_result_free and
 * each the result unround_solve gives that picture alone to binary32 rounding. The iterations
 * but the last run for all pictures at once -- one launch per kernel class an iteration (the
 * dual sweep of each method and channel count, the primal step of each cell layout) over tables
 * of tiles of all pictures, two iterations captured in one CUDA graph launched for every pair.
 * `timing` (may be null) gets that part's device milliseconds (CUDA events), its iterations and
 * launches per iteration, and the samples and pixels of all pictures. On failure no result is
 * made. */
typedef struct unround_b200_batch_timing {
  double milliseconds;
  uint64_t iterations;
  uint64_t launches_per_iteration;
  uint64_t samples;
  uint64_t pixels;
  /* The autotuner's measurements of the classes' tile heights, before the timed part: with
   * UNROUND_B200_AUTOTUNE=1 in the environment, 0 when a batch of the same shapes was measured
   * before in the process; without it the wave model chooses and this is 0. */
  double tuning_milliseconds;
} unround_b200_batch_timing;

unround_status unround_b200_solve_batch(uint64_t count, const unround_input* inputs,
                                        const unround_settings* const* settings, unround_result** results,
                                        unround_b200_batch_timing* timing, char* message, size_t message_size);

/* The unrolled TGV solve of greyscale pictures and its adjoint (no counterpart in the
 * reference, which solves and does not differentiate): `iterations` iterations of the method
 * from the solver's start, with per-picture alpha0, alpha1, tau and sigma given as device
 * arrays, to the last primal iterate x~_N; and the gradient of a loss of x~_N with respect to
 * the four parameters, by the adjoint of every step, the states recomputed between checkpoints
 * kept every `checkpoint_every` iterations. Every pointer is device memory of the current
 * device; the caller allocates `checkpoint_floats` floats for the checkpoints and
 * `workspace_floats` for the workspace; the work runs on `stream` and is not waited for.
 * The problem's constants (made by the host model, unround_b200_model): */
typedef struct unround_b200_unrolled {
  uint64_t images, rows, columns; /* canvases of whole 8x8 blocks */
  uint64_t iterations;
  uint64_t checkpoint_every;
  float relaxation;
  const float* lower;       /* [images][blocks][64]: each coefficient's interval and centre, the */
  const float* upper;       /* DC's less the middle of its interval (the block's mean times 8) */
  const float* centre;
  const float* middle;      /* [images][blocks]: the middle of the DC interval / 8 */
  const float* weight;      /* [images][64]: the data term's weights, and those of flat blocks */
  const float* flat_weight;
  const uint8_t* flat;      /* [images][blocks] */
  const float* start;       /* [images][rows][columns]: x0, the start's canvas */
} unround_b200_unrolled;

uint64_t unround_b200_unrolled_checkpoint_floats(const unround_b200_unrolled* problem);
uint64_t unround_b200_unrolled_workspace_floats(const unround_b200_unrolled* problem);
unround_status unround_b200_unrolled_forward(const unround_b200_unrolled* problem, const float* alpha0,
                                             const float* alpha1, const float* tau, const float* sigma,
                                             float* checkpoints, float* workspace, float* output, void* stream,
                                             char* message, size_t message_size);
/* `output_grad` the loss's gradient with respect to x~_N; `grads` [4][images] binary64: alpha0,
 * alpha1, tau, sigma. Needs the checkpoints of a forward pass with the same parameters. */
unround_status unround_b200_unrolled_backward(const unround_b200_unrolled* problem, const float* alpha0,
                                              const float* alpha1, const float* tau, const float* sigma,
                                              const float* checkpoints, float* workspace, const float* output_grad,
                                              double* grads, void* stream, char* message, size_t message_size);

/* unround_solve to 8- or 16-bit levels (no counterpart in the reference, whose solve returns
 * binary64 and whose writers quantize on the host, rust/unround/src/output.rs:187-218): the
 * picture (JFIF RGB of YCbCr, else its channels) is made and quantized on the device -- dither
 * as unround_pnm takes it (0 rounds, halves away from 0; 1 and 2 the blue-noise matrix with the
 * channels apart or together), 16 bits as 257 times the sample, most significant byte first --
 * and only the levels, height x width x channels interleaved, come back into `levels`
 * (`capacity` bytes, host memory). `sizes` (3, may be null) gets the height, the width and the
 * channels; with `levels` null only they are made. No records are returned. */
unround_status unround_b200_solve_levels(const unround_input* input, const unround_settings* settings, int32_t sixteen,
                                        int32_t dither, uint8_t* levels, uint64_t capacity, uint64_t* sizes,
                                        char* message, size_t message_size);

/* A picture of rounded samples reconstructed on the device -- what the reference does to a PNG
 * file in unround_decode (rust/unround/src/samples.rs, cpp/src/samples.cpp:344-405), here from
 * its levels, since this build reads no PNG files: `levels` rows x columns x channels (1 to 4:
 * grey, grey and alpha, RGB, RGB and alpha) interleaved, of `bits` bits (1 to 16). Each sample is
 * held within the values that round to its level (docs/math.md 11), TV or TGV as the settings
 * say with the defaults of PNG files (a gap per sample of 1e-4, 10000 iterations, TGV's ratio of
 * the steps 0.3); an alpha is reconstructed apart, as one channel. The result is as
 * unround_solve's: the picture, its planes and canvas, the records; no coefficients. */
unround_status unround_b200_solve_samples(const uint16_t* levels, uint64_t rows, uint64_t columns, uint64_t channels,
                                         int32_t bits, const unround_settings* settings, unround_observer observer,
                                         void* user, unround_result** result, char* message, size_t message_size);

/* unround_b200_measure for pictures of rounded samples (grey or RGB levels): the iteration loop
 * alone, `warmup` iterations and then `iterations` timed by CUDA events, and the dual and primal
 * steps timed apart. */
unround_status unround_b200_measure_samples(const uint16_t* levels, uint64_t rows, uint64_t columns, uint64_t channels,
                                           int32_t bits, const unround_settings* settings, uint64_t warmup,
                                           uint64_t iterations, unround_b200_timing* timing, char* message,
                                           size_t message_size);

/* The interval and centre of a level of `bits` bits as unround_b200_solve_samples models it
 * (cpp/src/samples.cpp:86-105): ends[0] the least value held, ends[1] the greatest, ends[2] the
 * level's centre; without a device. */
unround_status unround_b200_sample_interval(uint32_t level, int32_t bits, double slack, double* ends, char* message,
                                           size_t message_size);

/* The blue-noise matrix of the ordered dither of 8- and 16-bit output (unround_pnm): 64 x 64
 * ranks, row by row, into `ranks` (4096 values, each of 0 .. 4095 once), made by the
 * void-and-cluster method as the reference's scripts/blue_noise.py makes the table of
 * rust/unround/src/blue_noise.rs; without a device. */
unround_status unround_b200_blue_noise(uint16_t* ranks, char* message, size_t message_size);

/* What the host model makes of an input and settings, without a GPU (the reference computes the
 * same in Problem::make, cpp/src/model.cpp:134-256, and plan, cpp/src/pdhg.cpp:147-233): of
 * component `component`, `which` 0 the lower ends of the intervals, 1 the upper ends, 2 the
 * centres (one per coefficient); 3 the steps, 4 the weights, 5 the weights of flat blocks (64);
 * 6 whether each block is flat (1 or 0, one per block); 7 the plan: tau, sigma, the most
 * iterations and the tolerance (4). Writes at most `capacity` doubles into `out` and the count
 * into *count (out may be null to ask for the count). */
unround_status unround_b200_model(const unround_input* input, const unround_settings* settings, uint64_t component,
                                  int32_t which, double* out, uint64_t capacity, uint64_t* count, char* message,
                                  size_t message_size);

/* The decoder of the centres (what unround_solve computes with --method=mmse, which the settings
 * must say) into the caller's device buffers, allocating no device memory. It has no counterpart
 * in the reference's interface. It is for callers that run inside a device-memory budget they do
 * not own (a framework's allocator that holds the GPU's memory, a loop whose memory is planned
 * once), where a cudaMalloc may fail or a cudaFree stall the device.
 *
 * `canvas` (channels x canvas rows x canvas columns, binary64, the input's colour space) and
 * `coefficients` (every component's blocks one after another, binary64) are device pointers on
 * the current device holding `canvas_capacity` and `coefficient_capacity` doubles; both null asks
 * only for `sizes`, without a device. `sizes` (4, may be null) gets the channels, the canvas rows,
 * the canvas columns and the coefficient count. The work runs on `stream` (a cudaStream_t; null
 * is the legacy default stream) and is complete on return.
 *
 * Its device scratch is one fixed array of 64 MiB on each device, reserved when this library's
 * device code is loaded there: an input whose levels, flat flags and constants need more (about
 * 33 million coefficients) is refused with UNROUND_ERROR_ARGUMENT and left to unround_solve. The
 * first call on a device looks up the array's address there (cudaGetSymbolAddress, with that
 * device current), and later calls keep it once a lookup has succeeded. Calls share the array:
 * calls that run at the same time on one device race on it, and the caller serializes them.
 * Every call waits for its own work on `stream` before it returns, on failure too. */
unround_status unround_b200_decode_centres_noalloc(const unround_input* input, const unround_settings* settings,
                                                   double* canvas, uint64_t canvas_capacity, double* coefficients,
                                                   uint64_t coefficient_capacity, uint64_t* sizes, void* stream,
                                                   char* message, size_t message_size);

/* One picture solved in row strips across ranks (no counterpart in the reference; its strip
 * decomposition is the threads' of docs/math.md, here across GPUs): each rank makes the solver
 * of its strip -- the picture's MCU bands it owns and two halo bands either side, given as an
 * unround_input of those bands -- and drives it iteration by iteration, exchanging between the
 * steps the halo rows of the state with its neighbours (the python package's strips module, over
 * NCCL). A plan that records before its last iteration, or stops at a tolerance, is recorded
 * across the ranks by the functions below.
 *   _new     the strip's solver, started (the start s_0 on the device);
 *   _step    `iterations` iterations keeping nothing, waited for; the last one is _finish's
 *            (_run below makes them with the exchanges, not waited for);
 *   _state   the device planes of the current state (x, p1, p2, and for TGV w1, w2, r11, r22,
 *            r12, each channel after channel), rows x columns each, rows `pitch` floats apart:
 *            returns the count, up to `most` written;
 *   _finish  the last iteration and the result, as unround_solve makes it, of the strip's canvas;
 *   _free    frees the strip. */
typedef struct unround_b200_strip unround_b200_strip;
unround_status unround_b200_strip_new(const unround_input* input, const unround_settings* settings,
                                      unround_b200_strip** strip, char* message, size_t message_size);
unround_status unround_b200_strip_step(unround_b200_strip* strip, uint64_t iterations, char* message,
                                       size_t message_size);
uint64_t unround_b200_strip_state(const unround_b200_strip* strip, float** planes, uint64_t most, uint64_t* rows,
                                  uint64_t* columns, uint64_t* pitch);
unround_status unround_b200_strip_finish(unround_b200_strip* strip, unround_result** result, char* message,
                                         size_t message_size);
void unround_b200_strip_free(unround_b200_strip* strip);

/* The records of a picture solved in row strips, added up across the ranks (the reference's
 * records over all its strips, rust/unround/src/records.rs:154-186; here each rank's sums over
 * its own bands, added in rank order):
 *   _plan          the plan's {iterations, record_every, tolerance, relative tolerance, partial
 *                  tolerance, partial radius (NaN: none), alpha, alpha1, alpha0, method (1 TV,
 *                  2 TGV), iterations made}: returns 11, up to `most` written;
 *   _rows          the strip's canvas rows [first, end) whose terms its records count: its own
 *                  bands;
 *   _record        one iteration keeping its tilde point (`advance` 0: none, the start's) and
 *                  the record's first sums over those rows, waited for: {G at the kept
 *                  coefficients, the first-order norms, the second-order norms (TGV), the
 *                  largest |div2 r~| (TGV), the samples counted};
 *   _record_duals  the second sums at the scaling theta (TGV: min(1, alpha1 / the largest
 *                  |div2 r~| of all ranks); TV: 1): {the dual's G* over the channels (the dual
 *                  value is minus the ranks' total), and with a partial radius the partial gap's
 *                  G* and its residual};
 *   _result        after the last iteration (made by _record), the result of the strip's canvas
 *                  with the stop given (1 converged, 2 iterations, 3 observer), no more
 *                  iterations. A strip whose plan records before its last iteration is finished
 *                  by _result, not _finish. */
uint64_t unround_b200_strip_plan(const unround_b200_strip* strip, double* values, uint64_t most);
unround_status unround_b200_strip_rows(unround_b200_strip* strip, uint64_t first, uint64_t end, char* message,
                                       size_t message_size);
unround_status unround_b200_strip_record(unround_b200_strip* strip, int32_t advance, double* first, char* message,
                                         size_t message_size);
unround_status unround_b200_strip_record_duals(unround_b200_strip* strip, double theta, double* second,
                                               char* message, size_t message_size);
unround_status unround_b200_strip_result(unround_b200_strip* strip, int32_t stop, unround_result** result,
                                         char* message, size_t message_size);

/* The halo swaps inside the library. An exchange copies `rows` canvas rows of every state plane
 * (as _state lists them) from the strip `sender`, starting at its row `sender_row`, over the
 * rows of the strip `receiver` starting at `receiver_row` (the python strips module's
 * exchanges()).
 *   _run             `iterations` iterations of the strip, each followed by the exchanges in
 *                    which `rank` sends or receives (sender and receiver are ranks of the NCCL
 *                    communicator `comm`, an ncclComm_t; a rank may exchange with itself): every
 *                    plane's rows one ncclSend or ncclRecv, all of an iteration in one NCCL
 *                    group, on the strip's stream after its kernels; the call returns without
 *                    waiting for the device (the next _record or _result waits). `iterations` 0:
 *                    the exchanges only. NCCL is the libnccl.so.2 already loaded in the process
 *                    (the one torch.distributed uses), else the one the loader finds; the last
 *                    iteration is _record's or _finish's.
 *   _exchange_local  the exchanges among `count` strips of one process and device (sender and
 *                    receiver index `strips`): device copies on each receiver's stream after the
 *                    sender's work so far, and each sender's later work after the copies of its
 *                    rows; not waited for. */
typedef struct unround_b200_strip_exchange {
  int32_t sender;
  int32_t receiver;
  uint64_t sender_row;
  uint64_t receiver_row;
  uint64_t rows;
} unround_b200_strip_exchange;
unround_status unround_b200_strip_run(unround_b200_strip* strip, uint64_t iterations, int32_t rank,
                                      const unround_b200_strip_exchange* exchanges, uint64_t count, void* comm,
                                      char* message, size_t message_size);
unround_status unround_b200_strip_exchange_local(unround_b200_strip* const* strips, uint64_t count,
                                                 const unround_b200_strip_exchange* exchanges,
                                                 uint64_t exchange_count, char* message, size_t message_size);

/* The failure path of the bounded waits (no counterpart in the reference, whose solver has no
 * device): every wait of a kernel on an mbarrier is bounded, and one that runs out sets an error
 * word that the solve reports as UNROUND_ERROR_INTERNAL ("a bounded wait of the sweep ran out")
 * after draining the loads still in flight. This sets the tries that the dual sweep's compute
 * warps give a chunk of their ring, for the solves of this process from now on: `tries` >= 0
 * sets it, a negative value puts back the full limit (2^22). It returns the limit before. With
 * 0, every sweep gives up at its first chunk although its loads complete as usual: a test of
 * the failure path that neither faults nor hangs the device. */
int64_t unround_b200_set_ring_wait_limit(int64_t tries);

#ifdef __cplusplus
}
#endif

#endif
