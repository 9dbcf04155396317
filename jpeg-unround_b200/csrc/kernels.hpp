// The device side of the solver: plain structures of device pointers and constants that the
// host driver fills, and the launchers of the kernels (kernels.cu). The canvas fields are
// binary32 planes in HBM, channel after channel, each rows x pitch with the pitch a multiple
// of 32 samples (128-byte rows); the levels are int16 in block order, 64 to a block in
// natural order, as the file gives them.
#pragma once

#include <cstddef>
#include <cstdint>
#include <vector>

#include <cuda.h>
#include <cuda_runtime.h>

namespace urb {

constexpr int kMaxChannels = 3;

// The per-frequency factors of a component's proximal map in binary32, for one step tau
// (docs/math.md 4.1, 4.4; cpp/src/model.cpp:483-497), with t = (tau / n_c) m and
// r = 1 / (1 + t): z = (e + t c) r = e r + (t r) c, clipped to q Q -+ (1/2 + s) Q. They are
// packed four to a frequency, {Q, r, t r, (1/2 + s) Q}, so that one 16-byte load gives a
// coefficient's map: `plain` for a block that is not flat, `flat` for one that is, frequency k
// at prox_slot(k). With a slack's cost, h = (tau / n_c) lambda r of each; delta / Q of the MMSE
// centres.
//
// prox_slot keeps frequency k = 8 v + u in row v and puts it at column u ^ v of that row: a
// warp's eight lanes of a block read one frequency of every row (the primal step's lanes hold
// rows), or every frequency of one row (the fused iteration's hold columns), and either way
// eight different 16-byte bank groups of shared memory, one wavefront.
__host__ __device__ constexpr int prox_slot(int k) {
  return (k & ~7) | ((k ^ (k >> 3)) & 7);
}

struct ProxFactors {
  float4 plain[64];
  float4 flat[64];
  float h[64];
  float h_flat[64];
  float shrink[64];
  float slack;
  int mmse;
  int costed;
  int pad;
};

// The same constants in binary64 for the records and the start (G, G*, the centres).
struct Constants64 {
  double step[64];
  double weight[64];
  double flat_weight[64];
  double shrink[64];
  double cost[64];
  double slack;
  int mmse;
  int costed;
};

struct ComponentDevice {
  const std::int16_t* levels = nullptr;  // [by][bx][64]
  const std::uint8_t* flat = nullptr;    // [by][bx]
  int block_rows = 0;
  int block_columns = 0;
  int cell_rows = 1;
  int cell_columns = 1;
  const ProxFactors* factors = nullptr;
  const Constants64* constants = nullptr;
  float* zeta = nullptr;  // kept coefficients, [by][bx][64]
};

struct Geometry {
  int rows = 0;
  int columns = 0;
  int pitch = 0;
  int channels = 1;
  std::size_t plane = 0;  // rows * pitch
  // The rows whose terms the records add up: every row, but in a strip of a picture solved in
  // row strips its own bands (whole blocks), so that the strips' sums make the picture's.
  int record_first = 0;
  int record_end = 1 << 30;
  __host__ __device__ bool recorded_row(int i) const { return i >= record_first && i < record_end; }
};

// A state of the method (docs/math.md 5): x, p and for TGV w and r, each channels planes.
struct Fields {
  float* x = nullptr;
  float* p1 = nullptr;
  float* p2 = nullptr;
  float* w1 = nullptr;
  float* w2 = nullptr;
  float* r11 = nullptr;
  float* r22 = nullptr;
  float* r12 = nullptr;
};

// The dual step of iteration n and the relaxation (docs/math.md 5): from x~_n and the state
// s_{n-1} (in) to s_n (out); with keep, the tilde point's p~, r~ and w~ into `tilde`.
struct DualParams {
  Geometry g;
  const float* xt = nullptr;
  Fields in;
  Fields out;
  Fields tilde;
  float sigma[kMaxChannels] = {};  // sigma gamma_c
  float tau[kMaxChannels] = {};    // tau gamma_c
  float rho = 1.9f;
  float rest = -0.9f;
  float radius = 1.0f;   // alpha of TV, alpha1 of TGV
  float radius0 = 2.0f;  // alpha0
  int* error = nullptr;  // set to 1 where a bounded wait of the sweep ran out
  int strip_rows = 256;  // rows a CTA of the sweep walks, a multiple of 8 (set by its launcher)
  // Tries of the compute warps' wait for a chunk of the ring (the drain of the loads in flight
  // before a CTA leaves always has the full limit): the full limit but where a test of the
  // failure path shortens it (ring_wait_limit()).
  long long ring_wait_limit = 1LL << 22;
};

// The tries the dual sweep's compute warps give a chunk of its ring, for every solve of this
// process from now on: `tries` >= 0 sets it, and a negative value puts back the full limit.
// Returns the limit before. A test of the failure path sets 0, so that the waits give up on
// loads that complete as usual.
long long set_ring_wait_limit(long long tries);
long long ring_wait_limit();

// The primal step of iteration n+1 for one channel: v = x + tau gamma div p and its proximal
// map x~ (docs/math.md 4.4, 5); with keep, the coefficients zeta, v, and each CTA's sum of
// the data term's terms at zeta.
struct PrimalParams {
  Geometry g;
  ComponentDevice component;
  const float* x = nullptr;
  const float* p1 = nullptr;
  const float* p2 = nullptr;
  float* xt = nullptr;
  float* v = nullptr;
  double* partials = nullptr;
  float descent = 0.0f;  // tau gamma_c
  int* error = nullptr;  // set to 1 where a bounded wait of the TMA path ran out
};

// The records (docs/math.md 6): sums over the canvas in binary64 from the binary32 tilde
// point, each CTA's into `partials`.
struct NormParams {
  Geometry g;
  const float* xt = nullptr;
  Fields tilde;          // p~, w~, r~
  float* div2 = nullptr;  // div_2 r~ of each channel: 2 planes per channel
  double weight[kMaxChannels] = {};
  double* partials = nullptr;  // 3 per CTA: first-order norms, second-order norms, max |div_2 r~|
};

struct ConjugateParams {
  Geometry g;
  ComponentDevice component;
  const float* q1 = nullptr;  // the field whose divergence xi is: p~, or div_2 r~ scaled
  const float* q2 = nullptr;
  double scale = 1.0;   // q = scale * (q1, q2): 1 for p~, -theta for div_2 r~
  // Where given, the scale is -theta, theta = min(1, alpha1 / most) with `most` (the largest
  // |div_2 r~| of a record) read from the device, so that no host round trip comes between a
  // record's norms and its conjugates.
  const double* most_at = nullptr;
  double alpha1 = 1.0;
  double gamma = 1.0;   // xi = gamma div q
  double radius = 255.0;  // R of the free samples (docs/math.md 6.6)
  int free = 0;
  double* partials = nullptr;  // 1 per CTA
};

// -theta of a record from its largest |div_2 r~| (the host's formula, operation for operation).
__host__ __device__ inline double negative_theta(double most, double alpha1) {
  return -(most > alpha1 ? alpha1 / most : 1.0);
}

// Sums (or largest values) of arrays of per-CTA partials, each by one CTA in a fixed order:
// out[k] of the k-th array. A record's sums, taken on the device and copied back at once.
constexpr int kMaxReductions = 16;
struct Reductions {
  const double* in[kMaxReductions] = {};
  int count[kMaxReductions] = {};
  int largest[kMaxReductions] = {};
  int n = 0;
  double* out = nullptr;
  int add(const double* array, int entries, bool most = false) {
    in[n] = array;
    count[n] = entries;
    largest[n] = most ? 1 : 0;
    return n++;
  }
};
cudaError_t launch_reductions(const Reductions& r, cudaStream_t stream);

struct ResidualParams {
  Geometry g;
  const float* p1 = nullptr;
  const float* p2 = nullptr;
  const float* d1 = nullptr;
  const float* d2 = nullptr;
  double* partials = nullptr;
};

// The FP64 canvas of coefficients (docs/math.md 1.3): mode 0, the start, their inverse DCT
// spread over the cells and `beyond` past the blocks; mode 1, a result, v plus the change of
// each cell (its inverse DCT less the mean of v), and v past the blocks (n_c = 1: the inverse
// DCT itself).
struct CanvasParams {
  Geometry g;
  ComponentDevice component;
  const double* coefficients = nullptr;  // [by][bx][64]
  const float* v = nullptr;              // mode 1
  double* canvas = nullptr;              // rows x columns (unpadded), this channel's
  float* x = nullptr;                    // mode 0: the binary32 start, pitched
  double beyond = 128.0;
  int mode = 0;
};

// The start's coefficients: the centres, or given ones, clipped to their intervals; with
// sums of the data term's terms there into `partials`.
struct StartParams {
  ComponentDevice component;
  const double* given = nullptr;  // null: the centres
  double* coefficients = nullptr;
  double* partials = nullptr;
  int record_first = 0;  // the canvas rows whose blocks the data term adds up (Geometry's)
  int record_end = 1 << 30;
};

int dual_grid_blocks(const Geometry& g);
int primal_grid_blocks(const Geometry& g, const ComponentDevice& c);
int conjugate_grid_blocks(const Geometry& g, const ComponentDevice& c);
int norms_grid_blocks(const Geometry& g);
int residual_grid_blocks(const Geometry& g);
int start_grid_blocks(const ComponentDevice& c);

cudaError_t launch_dual(const DualParams& p, bool tgv, bool coupled, bool keep, cudaStream_t stream);
cudaError_t launch_primal(const PrimalParams& p, bool keep, cudaStream_t stream);
cudaError_t launch_start_coefficients(const StartParams& p, cudaStream_t stream);
cudaError_t launch_canvas(const CanvasParams& p, cudaStream_t stream);
// The result's picture from the binary64 canvas (C planes of rows x columns): its height x width
// pixels with the channels interleaved into `picture` (null: none), for YCbCr (`rgb`) JFIF's
// RGB; and the planes cut to height x width into `planes` (null: none).
struct PictureParams {
  const double* canvas = nullptr;
  int channels = 1;
  int rows = 0, columns = 0;
  int height = 0, width = 0;
  bool rgb = false;
  double* picture = nullptr;
  double* planes = nullptr;
};
cudaError_t launch_picture(const PictureParams& p, cudaStream_t stream);
// 8- or 16-bit levels (output.cu) of `count` binary64 samples, rows of `width` pixels of
// `channels` interleaved samples: dither 0 rounds, 1 and 2 take the blue-noise matrix with the
// channels apart or together; 16-bit levels most significant byte first. A sample that is not
// finite sets *not_finite. prepare_levels loads the matrix onto the current device (once).
struct LevelsParams {
  const double* samples = nullptr;
  std::size_t count = 0;
  int width = 1;
  int channels = 1;
  double scale = 1.0;
  double top = 255.0;
  int dither = 1;
  bool sixteen = false;
  std::uint8_t* out = nullptr;
  int* not_finite = nullptr;
};
bool prepare_levels();
cudaError_t launch_levels(const LevelsParams& p, cudaStream_t stream);

// Pictures of rounded samples (samples.cu): the primal step with its sample-by-sample proximal
// map, G* at a field, and the start or the result canvas. A sample's level (16 bits) sits in a
// plane pitched like the state (channel-major); its interval and centre are looked up by level
// in a table, in binary32 (the ends rounded inward, the centre to nearest) for the iterations
// and in binary64 for the records and the result. Binary64 canvases are packed, channel-major,
// rows x columns each.
struct alignas(16) SampleEnds32 {
  float lower, upper, centre, unused;
};
struct alignas(32) SampleEnds64 {
  double lower, upper, centre, unused;
};
struct SamplesLevelsParams {
  Geometry g;
  const std::uint16_t* source = nullptr;  // rows x columns x stride, interleaved
  int stride = 1;
  int first = 0;
  std::uint16_t* levels = nullptr;  // the channels' planes, pitched
};
struct SamplesPrimalParams {
  Geometry g;
  const float* x = nullptr;
  const float* p1 = nullptr;
  const float* p2 = nullptr;
  float* xt = nullptr;
  const std::uint16_t* levels = nullptr;
  const SampleEnds32* ends = nullptr;
  const SampleEnds64* ends64 = nullptr;
  float descent[kMaxChannels] = {};  // tau gamma_c
  float t = 0.0f;                    // tau mu
  float r = 1.0f;                    // 1 / (1 + tau mu)
  double half_mu = 0.0;
  double* partials = nullptr;  // with keep: mu/2 sum (x~ - c)^2, one per CTA
};
struct SamplesConjugateParams {
  Geometry g;  // one channel's
  const float* q1 = nullptr;
  const float* q2 = nullptr;
  double scale = 1.0;
  const double* most_at = nullptr;  // where given, the scale is negative_theta(*most_at, alpha1)
  double alpha1 = 1.0;
  double gamma = 1.0;
  double mu = 0.0;
  const std::uint16_t* levels = nullptr;  // the channel's plane
  const SampleEnds64* ends64 = nullptr;
  double* partials = nullptr;  // one per CTA
};
struct SamplesCanvasParams {
  Geometry g;
  int mode = 0;  // 0: the start from the centres; 1: the result from x~
  float* x = nullptr;
  const float* xt = nullptr;
  const std::uint16_t* levels = nullptr;
  const SampleEnds64* ends64 = nullptr;
  double* canvas = nullptr;  // C x rows x columns
};
int samples_grid_blocks(const Geometry& g, int channels);  // a sample per thread
int samples_primal_blocks(const Geometry& g);              // the primal step's CTAs
cudaError_t launch_samples_primal(const SamplesPrimalParams& p, bool keep, cudaStream_t stream);
cudaError_t launch_samples_conjugate(const SamplesConjugateParams& p, cudaStream_t stream);
cudaError_t launch_samples_canvas(const SamplesCanvasParams& p, cudaStream_t stream);
cudaError_t launch_samples_levels(const SamplesLevelsParams& p, cudaStream_t stream);
// The kept coefficients (binary32, DC centred) as binary64 absolute coefficients.
cudaError_t launch_restore(const ComponentDevice& c, double* out, cudaStream_t stream);
cudaError_t launch_gradient(const float* x, float* w1, float* w2, const Geometry& g, cudaStream_t stream);
cudaError_t launch_project(Fields f, const Geometry& g, bool tgv, bool coupled, float radius, float radius0,
                           cudaStream_t stream);
cudaError_t launch_norms(const NormParams& p, bool tgv, bool coupled, cudaStream_t stream);
cudaError_t launch_conjugate(const ConjugateParams& p, cudaStream_t stream);
cudaError_t launch_residual(const ResidualParams& p, cudaStream_t stream);
// The dual step as a TMA-fed sweep (sweep.cu): `state` maps the input state's planes (fields x,
// p1, p2 and for TGV w1, w2, r11, r22, r12, each channel after channel, one allocation), `tilde`
// the planes of x~. A CTA sweeps a strip of sweep_width(channels) columns: with one channel each
// lane takes two columns, so that a chunk's barriers and fixed work cover as many samples as
// with more channels.
__host__ __device__ constexpr int lane_columns(int channels) { return channels == 1 ? 2 : 1; }
__host__ __device__ constexpr int sweep_width(int channels) { return 32 * lane_columns(channels); }
std::size_t dual_tma_shared_bytes(bool tgv, int channels);
bool make_sweep_map(CUtensorMap& map, const float* planes, const Geometry& g, int count);
// The primal step fed by TMA, persistent CTAs over (component, strip, stage) items: `maps[z]`
// boxes component z's x, p1 and p2 planes (make_primal_map, planes `stride` floats apart); one
// launch takes 1 or 2 components of the same cells and geometry (e.g. Cb and Cr) and writes each
// CTA's sum of each component's data term into that component's partials. Cells of 1, 2 or 4
// samples each way; others take launch_primal. *grid: the CTAs launched.
struct PrimalBatch {
  PrimalParams part[2];
  int count = 1;
  int strips = 0;
  int stages = 0;
  int items = 0;
};
bool make_primal_map(CUtensorMap& map, const float* x, const Geometry& g, std::size_t stride);
bool primal_tma_takes(const ComponentDevice& c);
// An upper bound of the CTAs of a launch (the partials a component needs).
int primal_tma_grid_blocks(const Geometry& g, const ComponentDevice& c);
cudaError_t launch_primal_tma(const CUtensorMap* maps, const PrimalParams* parts, int count, bool keep,
                              cudaStream_t stream, int* grid);
// The rows a CTA of a strip sweep walks (a multiple of 16) so that the sweep's CTAs, `slots`
// of them resident at once, finish soonest (sweep.cu); strips of `width` columns.
int strip_rows_for(const Geometry& g, int slots, int width);

// The batched solve (batch.cu): one launch steps many images' states. A component's or an
// image's entry holds its tensor maps and parameters for each state parity (the state the step
// reads: 0 or 1), in device memory; the maps are read through the tensor-map proxy.
struct alignas(64) PrimalBatchComponent {
  CUtensorMap map[2];      // the component's x, p1, p2 planes of each state (make_primal_map)
  PrimalParams params[2];  // its primal step reading each state
};
// An item of a batched primal step: a stage of 64 canvas rows of a strip of 32 columns.
struct PrimalItem {
  int component = 0;
  int strip = 0;
  int stage = 0;
  int pad = 0;
};
// The stages of a strip of a component of cells `cell_rows` high.
int primal_batch_stages(const Geometry& g, int cell_rows);
// The primal step (no values kept) of every item of `list`, of components of the same cells.
cudaError_t launch_primal_batch(const PrimalItem* list, int count, const PrimalBatchComponent* components, int parity,
                                int cell_rows, int cell_columns, cudaStream_t stream);

struct alignas(64) DualBatchImage {
  CUtensorMap state[2];   // the sweep's maps of each state (make_sweep_map)
  CUtensorMap tilde;      // of x~
  DualParams params[2];   // the dual step from each state
};
// A tile of a batched dual step: columns x0 .. x0 + 31, rows i0 .. i1 - 1 of an image.
struct DualTile {
  int image = 0;
  int x0 = 0;
  int i0 = 0;
  int i1 = 0;
};
// The dual step (no values kept) of every tile of `tiles`, of images of the same method and
// channels.
cudaError_t launch_dual_batch(const DualTile* tiles, int count, const DualBatchImage* images, int parity, bool tgv,
                              int channels, bool coupled, cudaStream_t stream);
// The CTAs of that sweep the current device holds at once (0 where it cannot tell), and the
// tile height (a multiple of 16) that finishes a class's pictures soonest in waves of `slots`.
int dual_batch_slots(bool tgv, int channels, bool coupled);
int batch_tile_rows(const std::vector<Geometry>& pictures, int slots);
cudaError_t launch_dual_tma(const CUtensorMap& state, const CUtensorMap& tilde, const DualParams& p, bool tgv,
                            bool coupled, bool keep, cudaStream_t stream);
// A 3D tiled map of `count` float planes `stride` floats apart, boxes of `box_columns` columns
// (a multiple of 4) x `box_rows` rows x every plane (sweep.cu).
bool make_box_map(CUtensorMap& map, const float* planes, const Geometry& g, int count, std::size_t stride,
                  unsigned box_rows, unsigned box_columns);
// A 4D tiled map of `fields` planes `plane` floats apart, each `images` pictures of rows x
// columns (packed), boxes of `box_columns` (a multiple of 4) x `box_rows` of one picture x every
// field (sweep.cu).
bool make_fields_map(CUtensorMap& map, const float* base, int columns, int rows, int images, int fields,
                     std::size_t plane, unsigned box_columns, unsigned box_rows);

// The whole iteration as one sweep (iteration.cu): the dual step D_n with the relaxation, from
// x~_n and s_{n-1} (dual.in, dual.xt) to s_n (dual.out), and the primal step P_{n+1} on s_n,
// x~_{n+1} into `next`; no kept values (records take the split kernels).
struct IterationParams {
  DualParams dual;
  ComponentDevice component[kMaxChannels];
  float* next = nullptr;
  int strip_rows = 256;  // rows a CTA sweeps, a multiple of 16 (set by the launcher)
};

// Whether the fused sweep takes this canvas: 1 or 3 channels, channel 0 of 1 x 1 cells, the
// others of CR x CC, CR and CC 1 or 2.
bool iteration_takes(const Geometry& g, const ComponentDevice* components, int count);
std::size_t iteration_shared_bytes(bool tgv, int channels);
// The sweep's maps: boxes of 9 rows (a chunk and the row below it).
bool make_iteration_map(CUtensorMap& map, const float* planes, const Geometry& g, int count);
cudaError_t launch_iteration(const CUtensorMap& state, const CUtensorMap& tilde, const IterationParams& p, bool tgv,
                             bool coupled, int cell_rows, int cell_columns, cudaStream_t stream);

// Pictures of rounded samples in one sweep per iteration (iteration.cu): the dual step and the
// next primal step with its sample-by-sample proximal map; maps as make_iteration_map makes them.
struct SamplesIterationParams {
  DualParams dual;
  const std::uint16_t* levels = nullptr;  // the channels' levels, pitched like the state
  const SampleEnds32* ends = nullptr;      // per level
  float t = 0.0f;                          // tau mu
  float r = 1.0f;                          // 1 / (1 + tau mu)
  float* next = nullptr;                   // x~ of the next iteration
  int strip_rows = 256;                    // set by the launcher
};
bool samples_iteration_takes(const Geometry& g);  // 1 or 3 channels
// The same in the dual sweep's layout (sweep.cu: 8-row boxes in a ring of three slots, the
// sweep's maps): the primal step of pictures of rounded samples after the dual step, per chunk.
struct SamplesStep {
  const std::uint16_t* levels = nullptr;  // the channels' levels, pitched like the state
  const SampleEnds32* ends = nullptr;      // per level
  float t = 0.0f;                          // tau mu
  float r = 1.0f;                          // 1 / (1 + tau mu)
  float* next = nullptr;                   // x~ of the next iteration
};
cudaError_t launch_dual_samples(const CUtensorMap& state, const CUtensorMap& tilde, const DualParams& p,
                                const SamplesStep& q, bool tgv, bool coupled, cudaStream_t stream);
cudaError_t launch_samples_iteration(const CUtensorMap& state, const CUtensorMap& tilde,
                                     const SamplesIterationParams& p, bool tgv, bool coupled, cudaStream_t stream);

cudaError_t launch_narrow(const double* from, float* to, const Geometry& g, cudaStream_t stream);

}  // namespace urb
