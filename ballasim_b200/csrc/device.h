// Device-side data layout of the sensor models and the launch entry points of kernels.cu (host-callable).
//
// HBM layout, per model, structure of arrays so that a warp's 32 consecutive pixels load and store one
// contiguous segment per field:
//   state (double-buffered: a call reads one copy and writes the other, so a failed or overflowing call
//   leaves the model as it was): t_ref, t_search, blind_until, t_shot, t_ba (i64); s3_ref, n3_ref, dr_ref,
//   i_scale, held (f32); flags, n_shot, n_ba (u32): 72 B per pixel (the noise words are read only with noise on).
//   map: theta_on, theta_off, leak, dark, scale, phi0 (f32), ba_rate, shot_max (f64): 40 B per pixel.
// Sample runs follow the reference's DeviceRuns (src/sensor/sensor_model.h:81-89): pixel[i], row_start[i],
// row_count[i], t (i64), irr (f32): 12 B per sample.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "fields.cuh"
#include "pixel.cuh"
#include "sampler.cuh"

namespace bs {

struct StateSoA {
  int64_t *t_ref, *t_search, *blind_until, *t_shot, *t_ba;
  float *s3_ref, *n3_ref, *dr_ref, *i_scale, *held;
  uint32_t *flags, *n_shot, *n_ba;
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
  kCntWords = 8
};
enum ErrorBit : unsigned long long {
  kErrPixelRange = 1ull,
  kErrDuplicate = 2ull,
  kErrRunRange = 4ull,
  kErrOrder = 8ull,
  kErrAfterEnd = 16ull,
  kErrNonFinite = 32ull,
};

struct EventBuf {
  RawEvent* data;
  unsigned long long capacity;
};

// One sensor of a fused engine launch.
struct EngineSensor {
  FieldDev field;
  SensorConsts consts;
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

// Launchers (stream-ordered; no synchronization inside).
void launch_init_counted(const SensorConsts& k, const MapSoA& map, StateSoA st, uint32_t n_pixels, int64_t t0,
                         const float* irr0, unsigned long long* counters, cudaStream_t stream);
void launch_scatter_rows(const uint32_t* pixel, uint32_t n, int32_t* row_of, uint32_t n_pixels,
                         unsigned long long* counters, cudaStream_t stream);
void launch_advance_runs(const SensorConsts& k, const MapSoA& map, StateSoA in, StateSoA out, uint32_t n_pixels,
                         const uint32_t* pixel_ids, const int32_t* row_of, const int64_t* row_start,
                         const int32_t* row_count, const int64_t* t, const float* irr, uint64_t n_samples,
                         int64_t t_state, int64_t t_end, EventBuf ev, unsigned long long* counters, int block,
                         cudaStream_t stream);
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
void launch_engine(const EngineSensor* sensors_dev, int n_sensors, uint32_t total_tiles, int64_t t0, int32_t w0,
                   int32_t w1, const SamplerRules& r, unsigned int* tile_counter, int blocks, int warps_per_block,
                   int stage, cudaStream_t stream);
int engine_max_blocks_per_sm(int warps_per_block, int stage);
// MidpointTest.eta over n triples of g groups (rows of g floats).
void launch_midpoint_eta(float tol, float dark, int32_t g, const float* m_min, const float* m_max, const float* ea,
                         const float* em, const float* eb, uint32_t n, float* eta, uint8_t* exceeds,
                         cudaStream_t stream);

}  // namespace bs
