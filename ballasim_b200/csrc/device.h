// Device-side data layout of the sensor models and the launch entry points of kernels.cu (host-callable).
//
// HBM layout, per model, structure of arrays so that a warp's 32 consecutive pixels load and store one
// contiguous segment per field:
//   state (double-buffered: a call reads one copy and writes the other, so a failed or overflowing call
//   leaves the model as it was): t_ref, t_search, blind_until, t_shot, t_ba (i64); s3_ref, n3_ref, dr_ref,
//   i_scale, held (f32); flags, n_shot, n_ba (u32): 72 B per pixel (the noise words are read only with noise on);
//   with the cascade photoreceptor also z, x1, s2, s3, tv (f32): 20 B more.
//   map: theta_on, theta_off, leak, dark, scale, phi0 (f32), ba_rate, shot_max (f64): 40 B per pixel.
// Sample runs follow the reference's DeviceRuns (src/sensor/sensor_model.h:81-89): pixel[i], row_start[i],
// row_count[i], t (i64), irr (f32): 12 B per sample.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "cascade.cuh"
#include "fields.cuh"
#include "lattice.cuh"
#include "learned.cuh"
#include "pixel.cuh"
#include "sampler.cuh"

namespace bs {

struct StateSoA {
  int64_t *t_ref, *t_search, *blind_until, *t_shot, *t_ba;
  float *s3_ref, *n3_ref, *dr_ref, *i_scale, *held;
  uint32_t *flags, *n_shot, *n_ba;
  float *z, *x1, *s2, *s3, *tv;  // the cascade's (null without it)
  float* lat;                    // the noise lattice's: 8 planes of n (nk 0..2, nk1 0..2, ln_a1, rho); null without it
  int64_t* cell;
  uint32_t* have_k1;
};

struct MapSoA {
  float *theta_on, *theta_off, *leak, *dark, *scale, *phi0;
  double *ba_rate, *shot_max;
};

// Device counters of one call, read back once after it.
enum CounterWord : int {
  kCntEvents = 0,     // events produced (may exceed the capacity: the call is then re-run)
  kCntErrors = 1,     // error bits (kErr*)
  kCntClamps = 2,     // samples clamped into [0, irr_max]
  kCntPieces = 3,     // linear pieces of the pixel model
  kCntLeaves = 4,     // bisection nodes tested
  kCntSamples = 5,    // pixel-samples consumed
  kCntNoise = 6,      // noise candidates
  kCntSubsteps = 7,   // accepted cascade sub-steps
  kCntWords = 8
};
enum ErrorBit : unsigned long long {
  kErrPixelRange = 1ull,
  kErrDuplicate = 2ull,
  kErrRunRange = 4ull,
  kErrOrder = 8ull,
  kErrAfterEnd = 16ull,
  kErrNonFinite = 32ull,
  kErrSearchBound = 64ull,  // a warp-cooperative crossing search or its warp loop ran past its bound
  kErrRestList = 128ull,    // the split engine's list of posted pixels overflowed (it holds every pixel: not reached)
};

struct EventBuf {
  RawEvent* data;
  unsigned long long capacity;
};

// Walk state of the learned-proposal sampler, per pixel (double-buffered with the pixel state): hx, 8 planes of
// n pixels (plane k = the k-th previous walk point's log irradiance); gaps (8 log2 gaps, byte 0 newest); pv
// (irradiance at the previous walk point); valid (a real previous walk point exists). 45 B per pixel.
struct LearnedSoA {
  float* hx;
  uint64_t* gaps;
  float* pv;
  uint8_t* valid;
};

// A device record of (time, pixel, value) rows, appended with warp-aggregated atomics (tests and diagnostics).
struct RecRow {
  int64_t t;
  uint32_t pixel;  // sensor index << 24 | pixel
  float v;         // the sample's irradiance, or the step's log2 for a proposal
};
struct RecBuf {
  RecRow* data;
  unsigned long long* count;
  unsigned long long capacity;
};

// One sensor of a fused engine launch.
struct EngineSensor {
  LearnedSoA lin, lout;  // learned-proposal walk state (unused by the plain engine)
  FieldDev field;
  SensorConsts consts;
  CascadeConsts cc;      // the cascade's constants (consts.cascade)
  NoiseTableDev tab;     // the noise lattice's tables (data null without the lattice)
  StateSoA in, out;
  MapSoA map;
  float* carried_in;   // the sampler's carried sample (irradiance at the window start), per pixel
  float* carried_out;
  uint32_t width, height;
  uint32_t tiles_x, tiles_y;
  uint32_t tile0;      // first global tile of the sensor
  EventBuf ev;         // the sensor's own event buffer and counters
  unsigned long long* counters;
};

// Launchers (stream-ordered; no synchronization inside). tab.data non-null: the cascade's noise lattice is on.
void launch_init_counted(const SensorConsts& k, const CascadeConsts& cc, const NoiseTableDev& tab, const MapSoA& map,
                         StateSoA st, uint32_t n_pixels, int64_t t0, const float* irr0, unsigned long long* counters,
                         cudaStream_t stream);
void launch_scatter_rows(const uint32_t* pixel, uint32_t n, int32_t* row_of, uint32_t n_pixels,
                         unsigned long long* counters, cudaStream_t stream);
// The CSR-runs kernel of the instantaneous response, or of the cascade when k.cascade (cc its constants).
void launch_advance_runs(const SensorConsts& k, const CascadeConsts& cc, const NoiseTableDev& tab, const MapSoA& map,
                         StateSoA in, StateSoA out, uint32_t n_pixels,
                         const uint32_t* pixel_ids, const int32_t* row_of, const int64_t* row_start,
                         const int32_t* row_count, const int64_t* t, const float* irr, uint64_t n_samples,
                         int64_t t_state, int64_t t_end, EventBuf ev, unsigned long long* counters, int block,
                         cudaStream_t stream);
// The instantaneous response on CSR runs, row-major (one warp per 32 runs; runs longer than long_row samples walked
// by the whole warp, the others one per lane); listed: a bitmap of n_pixels bits, zeroed by the caller; the pixels
// no run lists advance too.
void launch_advance_rows(const SensorConsts& k, const MapSoA& map, StateSoA in, StateSoA out, uint32_t n_pixels,
                         const uint32_t* pixel, uint32_t n_rows, const int64_t* row_start, const int32_t* row_count,
                         const int64_t* t, const float* irr, uint64_t n_samples, int64_t t_state, int64_t t_end,
                         int32_t long_row, uint32_t* listed, EventBuf ev, unsigned long long* counters,
                         const SensorConsts* k_dev, void* rest, unsigned int* rest_count, int rest_blocks,
                         bool first_call, cudaStream_t stream);
// With `rest` (room for n_rows records of row_rest_bytes(); *rest_count zero before the launch), the row-major kernel
// runs split: advance_rows_split_kernel stops a short run at its first segment that is not clean (or before its held
// stretch to t_end) and advance_rows_rest_kernel (rest_blocks x 128 threads) finishes those rows one thread each.
// first_call: the model's first call since init (its first segments are then also tested with the search armed
// after their start).
size_t row_rest_bytes();
int rows_rest_blocks_per_sm();
// sample_window in one walk: pass 0 checks the ids (< n_field) and levels (<= max_level; a bad one ORed into *err,
// 1 level, 2 id, and not walked), walks, counts, and stages each pixel's carried sample, signature and samples in
// scratch (stage_dt / stage_v, stage_cap entries, *stage_used zero before; stage_at[i] the pixel's start or
// 0xFFFFFFFF); pass 1, after the scan of the counts and only if *err is clear, writes every row at its offset from
// the list (walking again a pixel the list does not hold) and the carried samples and signatures.
void launch_sample_window_staged(const FieldDev& f, const SamplerRules& r, int64_t t_w, const uint32_t* pixel,
                                 const uint8_t* level, uint32_t n, const float* carried_in, const uint64_t* sig_in,
                                 uint32_t* counts, const int64_t* offsets, int64_t* t_out, float* irr_out,
                                 float* carried_out, uint64_t* sig_out, uint32_t* stage_dt, float* stage_v,
                                 uint32_t* stage_at, unsigned int* stage_used, uint32_t stage_cap, float* stage_carried,
                                 uint64_t* stage_sig, uint32_t n_field, int max_level, unsigned long long* err,
                                 int pass, cudaStream_t stream);
// sample_window: pass 0 counts, pass 1 writes at offsets.
void launch_sample_window(const FieldDev& f, const SamplerRules& r, int64_t t_w, const uint32_t* pixel,
                          const uint8_t* level, uint32_t n, const float* carried_in, const uint64_t* sig_in,
                          uint32_t* counts, const int64_t* offsets, int64_t* t_out, float* irr_out,
                          float* carried_out, uint64_t* sig_out, int pass, cudaStream_t stream);
// Exclusive scan of n u32 counts into n + 1 i64 offsets (scratch: scan_scratch_words(n) i64 words).
size_t scan_scratch_words(uint32_t n);
void launch_scan(const uint32_t* counts, uint32_t n, int64_t* offsets, int64_t* scratch, cudaStream_t stream);
void launch_levels(const FieldDev& f, int64_t t_w, int32_t l_min, int32_t l_max, uint32_t n_pixels, uint8_t* level,
                   cudaStream_t stream);
void launch_field_frame(const FieldDev& f, int64_t t, uint32_t n_pixels, float* out, cudaStream_t stream);
// The fused engine: windows [w0, w1) of every sensor, one warp per 8 x 4 pixel tile, tiles taken from a global
// counter (work stealing) by a persistent grid. stage 0: the sampler feeds the pixel model sample by sample;
// 16 or 32: per window the samples are staged in shared memory (that many per lane) between the two phases.
// t0: the model time in device memory; tiles of 2^tile_lw x 2^(5 - tile_lw) pixels (tile_lw in [2, 5]).
// cascade: 0 the instantaneous response; 1 every sensor runs the cascade photoreceptor, 2 with its noise lattice
// (streaming form; stage is ignored).
void launch_engine(const EngineSensor* sensors_dev, int n_sensors, uint32_t total_tiles, const int64_t* t0,
                   int32_t w0, int32_t w1, const SamplerRules& r, unsigned int* tile_counter, int blocks,
                   int warps_per_block, int stage, int tile_lw, int cascade, cudaStream_t stream);
int engine_max_blocks_per_sm(int warps_per_block, int stage, int cascade);
// The split engine (stage kStageSplit): window w as engine_window_kernel (blocks x warps_per_block warps, persistent
// over the tiles) then engine_rest_kernel (rest_blocks x 128 threads) over the pixels the first posted to `rest`
// (rest_capacity records of rest_record_bytes(); *rest_count and *tile_counter zero before the launch).
constexpr int kStageSplit = 1;
void launch_engine_split(const EngineSensor* sensors_dev, int n_sensors, uint32_t total_tiles, const int64_t* t0,
                         int32_t w, const SamplerRules& r, unsigned int* tile_counter, void* rest, unsigned int* rest_count,
                         unsigned int rest_capacity, int blocks, int warps_per_block, int tile_lw, int rest_blocks,
                         cudaStream_t stream);
size_t rest_record_bytes();
int engine_rest_blocks_per_sm();
// The fused engine with the learned step proposal (BF16 MLP operands and FP32 parameters in device memory):
// the same tiles and pixel model, each window sampled by proposed power-of-two steps judged by the plain rule.
// rec_samples / rec_steps (capacity 0: off) record every sample and every proposed step.
struct LearnedLaunch {
  const uint16_t* ops;
  const float* params;
  float margin;
  int32_t sh;  // log2 min_dt_ns
  RecBuf rec_samples, rec_steps;
};
void launch_learned_engine(const EngineSensor* sensors_dev, int n_sensors, uint32_t total_tiles, const int64_t* t0,
                           int32_t w0, int32_t w1, const SamplerRules& r, const LearnedLaunch& l,
                           unsigned int* tile_counter, int blocks, int warps_per_block, int tile_lw,
                           cudaStream_t stream);
int learned_engine_max_blocks_per_sm(int warps_per_block);
// Resets the walk state of n pixels from their initial irradiance.
void launch_learned_reset(LearnedSoA st, uint32_t n, const float* irr0, cudaStream_t stream);

// ---- event output order (events.cu) ----
// Sorts n device events by (t_cross, pixel) into out (device), using sort_events_scratch_bytes(n) bytes of scratch.
size_t sort_events_scratch_bytes(uint32_t n);
cudaError_t sort_events(const RawEvent* ev, uint32_t n, RawEvent* out, void* scratch, cudaStream_t stream);

// The readout of a crossing (Readout, src/sensor/readout.h:14-27): delayed, floored to the counter quantum from its
// phase, then on the sensor clock (offset, drift).
struct ReadoutDev {
  int64_t quantum_ns, delay_ns, phase_ns, offset_ns;
  double drift_ppm;
};
BS_HD int64_t reported_time(const ReadoutDev& r, int64_t t_cross) {
  int64_t t = t_cross + r.delay_ns;
  if (r.quantum_ns > 0) {
    const int64_t a = t - r.phase_ns;
    const int64_t fd = a / r.quantum_ns - ((a % r.quantum_ns) < 0 ? 1 : 0);
    t = r.phase_ns + r.quantum_ns * fd;
  }
  return t + r.offset_ns + llround(r.drift_ppm * 1e-6 * static_cast<double>(t));
}
// The output cut after model time t_end (output_cut, src/sensor/output_order.h:48-53): the window end on the sensor
// clock (no delay, no quantum).
BS_HD int64_t output_cut(const ReadoutDev& r, int64_t t_end) {
  ReadoutDev clock = r;
  clock.delay_ns = 0;
  clock.quantum_ns = 0;
  return reported_time(clock, t_end);
}

// One output event (OutEvent, src/engine/output.h:25-32, without the ground-truth fields): 24 bytes.
// Device event columns (any pointer null: that column is skipped).
struct EventColumnsDev {
  uint32_t* pixel;
  uint16_t *x, *y;
  uint8_t* p;
  int64_t *t_cross, *t_reported;
  uint8_t* label;
  uint16_t* flags;
  float *ds, *dn, *dl, *l_first;
};
cudaError_t event_columns(const RawEvent* ev, uint32_t n, uint32_t width, const ReadoutDev& rd,
                          const EventColumnsDev& cols, cudaStream_t stream);

struct OutRecord {
  int64_t t_reported, t_cross;
  uint16_t x, y, flags;
  uint8_t p, label;  // label: the S1 code (label_s1, src/sensor/output_order.h:23-26)
};

// The output stage (Camera::output, src/engine/engine_impl.h:1761-1847, without crop and ground truth): the held
// records (device, n_held) and the call's raw events become records, all sorted by (t_reported, x, y, t_cross) by
// three stable radix passes (t_cross, (x, y), t_reported: order_key, src/sensor/output_order.h:28-36) into out
// (device, n_held + n_raw); *n_ready gets how many lead with t_reported < limit (the released ones).
size_t output_scratch_bytes(uint32_t n);
cudaError_t output_stage(const OutRecord* held, uint32_t n_held, const RawEvent* raw, uint32_t n_raw, uint32_t width,
                         int y_bits, const ReadoutDev& rd, int64_t limit, OutRecord* all, OutRecord* out,
                         void* scratch, unsigned long long* ready_dev, cudaStream_t stream);

// ---- the MLP (learned.cu) ----
// Training pairs from one window's plain runs (all n_pixels listed in order; t absolute): every stride-th pixel
// walks its run; pairs are appended (x: 16 BF16 features, y: target, key: pixel << 32 | window << 11 | step).
struct WalkArgs {
  const int64_t* offsets;
  const int64_t* t;
  const float* irr;
  const uint8_t* level;
  uint32_t n_pixels, stride;
  int64_t t_w;
  int32_t window, reset;
  int32_t sh;
  float eps;
  uint64_t seed;
  LearnedSoA st;
  uint16_t* x;
  float* y;
  uint64_t* key;
  unsigned long long* count;
  unsigned long long capacity;
};
void launch_walk_pairs(const WalkArgs& a, cudaStream_t stream);
// One training step's gradient partials: grid = ceil(rows / 128) CTAs of 128 threads.
struct TrainArgs {
  const uint16_t* x;
  const float* y;
  uint64_t n;
  uint32_t rows;     // rows of this step
  int32_t sampled;   // 1: rows drawn with replacement from n (Philox, keyed by the step counter); 0: rows 0..n-1
  uint64_t seed;
  const int64_t* step;
  const uint16_t* ops;
  const float* params;
  float* partial;         // [grid][kMlpParamsPad]
  double* partial_loss;   // [grid]
  float inv_rows;
  // Expectile weight tau: a row's squared error counts 2 tau when the net predicts below its target and
  // 2 (1 - tau) above it (0.5: the plain mean squared error).
  float tau;
  unsigned int* err;  // set when a tensor-core chain's completion was not seen within the wait's bound
};
int train_grid(uint32_t rows);
void launch_train_partials(const TrainArgs& a, cudaStream_t stream);
// Adam over the partials of `ctas` CTAs (lr, beta 0.9 / 0.999, eps 1e-8); advances the step counter; writes the
// step's loss (sum / (2 rows)) at losses[step] when step < loss_cap.
void launch_adam(float* params, float* m, float* v, uint16_t* ops, const float* partial, const double* partial_loss,
                 int ctas, float lr, float inv_rows, int64_t* step, float* losses, int64_t loss_cap,
                 unsigned int* done, cudaStream_t stream);
// The summed gradient (FP64) and loss of the partials (the gradient check).
void launch_reduce_partials(const float* partial, const double* partial_loss, int ctas, float inv_rows,
                            double* grad, double* loss, cudaStream_t stream);
void launch_operands(const float* params, uint16_t* ops, cudaStream_t stream);
void launch_mlp_forward(const uint16_t* ops, const float* params, const uint16_t* x, uint64_t n, float* y,
                        cudaStream_t stream);
// MidpointTest.eta over n triples of g groups (rows of g floats).
void launch_midpoint_eta(float tol, float dark, int32_t g, const float* m_min, const float* m_max, const float* ea,
                         const float* em, const float* eb, uint32_t n, float* eta, uint8_t* exceeds,
                         cudaStream_t stream);

}  // namespace bs
