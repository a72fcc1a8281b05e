/* ballasim_b200: the C ABI of a B200-native (sm_100a) implementation of BallaSim's per-pixel event-generation
 * path: the window sampler (src/engine) and the instantaneous continuous-time pixel model (src/sensor).
 *
 * Plain C types only: opaque handles, plain pointers and sizes, an explicit CUDA stream as void* (NULL: the
 * library's own stream). Every call returns a bs_status; bs_last_error() holds the message of the last failure
 * on the calling thread. Status codes map to the reference's Python exceptions:
 *   BS_EINVAL -> ValueError (std::invalid_argument), BS_ELOGIC -> RuntimeError (std::logic_error),
 *   BS_ENOMEM -> MemoryError (MemoryBudgetError), BS_ECUDA -> RuntimeError (a CUDA failure or no device),
 *   BS_EREFUSED -> ExportError, a ValueError (the exporters' Refused), BS_EIO -> OSError (a file that cannot be
 *   created, written or read), BS_ECANCELLED -> Cancelled (a window stopped by its cancel flag).
 * There is no CPU fallback: without a CUDA device every compute call returns BS_ECUDA.
 *
 * Citations are to the reference project's files; each entry point names the interface it replaces. */
#ifndef BALLASIM_B200_H
#define BALLASIM_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef int32_t bs_status;
#define BS_OK 0
#define BS_EINVAL 1
#define BS_ELOGIC 2
#define BS_ENOMEM 3
#define BS_ECUDA 4
#define BS_EREFUSED 5
#define BS_EIO 6
#define BS_ECANCELLED 7

typedef struct bs_model bs_model;
typedef struct bs_sampler bs_sampler;
typedef struct bs_engine bs_engine;

/* The SensorParams rows this path reads (src/sensor/params.h:65-176), resolved from a preset and overrides by
 * the caller. photoreceptor: 1 instantaneous or 0 cascade; enums as in params.h (reset_mode 0 physical / 1 ideal,
 * initial_phase 0 uniform / 1 symmetric / 2 zero, noise_diffusion 0 frozen / 1 transient). k, tau_o, tau_sf, eps_L
 * and noise (the cascade's in-path noise lattice) with sigma_o, noise_margin_z, noise_leaf_level and
 * noise_diffusion are the cascade's rows (read only with photoreceptor 0; the lattice runs frozen diffusion), and
 * initial_state (0 phase / 1 stationary), stationary_probe_pixels and stationary_burnin_ns its initial state. The
 * noise_shot_rate_hz / noise_ba_* rows are this project's shot and background-activity noise (0 = off;
 * instantaneous response only; no reference counterpart). */
typedef struct {
  int32_t photoreceptor;
  double theta_on, theta_off, sigma_theta_on, sigma_theta_off, theta_onoff_corr, theta_floor;
  int32_t reset_mode;
  double refractory_s, eps_ci;
  int32_t initial_phase;
  double leak_rate_hz, leak_sigma_log10, leak_ea_eV;
  double dark_current_fA, dark_sigma_ln, dark_ea_eV, temperature_K, reference_temperature_K;
  double illuminance_scale, label_share_cut;
  double readout_quantum_s, readout_delay_s, clock_drift_ppm;
  int64_t clock_offset_ns;
  double hot_fraction;
  double noise_shot_rate_hz, noise_ba_median_hz, noise_ba_sigma_ln;
  double k, tau_o, tau_sf, eps_L;
  int32_t noise;
  double sigma_o, noise_margin_z;
  int32_t noise_leaf_level, noise_diffusion;
  int32_t initial_state, stationary_probe_pixels;
  int64_t stationary_burnin_ns;
  /* The parameter set's fingerprint as the reference computes it (fingerprint(params, light groups),
   * src/sensor/params.cpp:246, over every SensorParams row), written into saved states and required of a state to
   * load (the reference's own refusal); this library does not see every row, so the caller's parameter layer passes
   * it (the Python shim restates the reference's function). */
  uint64_t fingerprint;
} bs_params;

/* Event columns of the caller's arrays (count entries each; any pointer may be NULL to skip a column), sorted by
 * (t_cross, pixel) as SensorModel::finish_events returns them (src/sensor/sensor_model.cpp:996-1029). */
typedef struct {
  uint32_t* pixel;
  uint16_t *x, *y;
  uint8_t* p;
  int64_t *t_cross_ns, *t_reported_ns;
  uint8_t* label;
  uint16_t* flags;
  float *ds, *dn, *dl, *l_first;
} bs_event_columns;

/* Sample runs in device memory (DeviceRuns, src/sensor/sensor_model.h:81-89): listed pixel pixel[i] takes
 * row_count[i] samples starting at row_start[i] of t (int64 ns) and irr (n_samples x 1 group). */
typedef struct {
  const uint32_t* pixel;
  const int64_t* row_start;
  const int32_t* row_count;
  size_t n;
  const int64_t* t;
  const float* irr;
  size_t n_samples;
} bs_device_runs;

/* Events left in device memory (DeviceEvents, src/sensor/sensor_model.h:91-96): RawEvent records of 32 bytes
 * (src/sensor/pixel.h:123-135), unordered; valid until the model advances again. */
typedef struct {
  const void* data;
  size_t count;
} bs_device_events;

const char* bs_last_error(void);
const char* bs_version(void);
/* sensor_cuda_available (src/sensor/sensor_model.h:53): a CUDA device of compute capability 10.x is visible. */
int32_t bs_cuda_available(void);

/* ---- the sensor model: SensorModel (src/sensor/sensor_model.h:98-320) ---- */

/* SensorModel(params, width, height, seed, light_groups, camera, precision='fp32', device='cuda')
 * (sensor_model.h:114-117, sensor_module.cpp:236-253): validates, draws the frozen maps (maps.cpp:78-156) and
 * allocates the device state. groups must be 1 (one constant light group). */
bs_status bs_model_create(const bs_params* params, uint32_t width, uint32_t height, uint64_t seed, uint32_t camera,
                          int32_t groups, bs_model** out);
bs_status bs_model_destroy(bs_model* m);
/* SensorModel::init (sensor_model.h:124-128): irr0 is a host array of width * height * groups floats. */
bs_status bs_model_init(bs_model* m, int64_t t0_ns, const float* irr0);
/* init from a device array (the engine's own frame). */
bs_status bs_model_init_device(bs_model* m, int64_t t0_ns, const float* irr0_dev, void* stream);
/* SensorModel::advance_runs (sensor_model.h:150-154) on host arrays: the runs are copied to the device, every
 * pixel advances to t_end_ns, and the events are kept (sorted) for bs_model_take_events; *n_events receives their
 * count. Refused input (ValueError) leaves the model unchanged. */
bs_status bs_model_advance_runs(bs_model* m, const uint32_t* pixel_ids, size_t n, const int64_t* t, const float* irr,
                                size_t n_samples, const int64_t* row_start, const int32_t* row_count,
                                int64_t t_end_ns, size_t* n_events);
/* SensorModel::advance_device (sensor_model.h:157-167): runs in device memory, queued on `stream`; the events stay
 * on the device (out). One synchronization reads the call's counters. */
bs_status bs_model_advance_device(bs_model* m, const bs_device_runs* runs, int64_t t_end_ns, void* stream,
                                  bs_device_events* out);
/* SensorModel::download_events (sensor_model.h:167): the device events of the last call, sorted, into host columns;
 * and the kept events of bs_model_advance_runs / an engine run (then cleared). */
bs_status bs_model_download_events(bs_model* m, const bs_device_events* ev, bs_event_columns* out);
bs_status bs_model_event_count(const bs_model* m, size_t* n);
/* The last device-event download's parts (ms; no reference counterpart): [0] the sort by (t_cross, pixel) and the
 * split into columns on the device, [1] the columns' copy to pinned host memory (CUDA events on the model's stream),
 * [2] the copies from pinned memory into the caller's arrays, [3] the whole download (host clock). */
bs_status bs_model_take_timing(const bs_model* m, double out[4]);
bs_status bs_model_take_events(bs_model* m, bs_event_columns* out);
/* SensorModel::maps (sensor_model.h:180; sensor_module.cpp sensor_maps): the fp64 maps, width * height each. */
bs_status bs_model_maps(const bs_model* m, double* theta_on, double* theta_off, double* leak, double* dark_fA,
                        double* phi0);
/* The engine's output stage (Camera::output, src/engine/engine_impl.h:1761-1847, without crop and ground truth):
 * records with the reported time (src/sensor/readout.h:22-27) and the S1 label (label_s1,
 * src/sensor/output_order.h:23-26), in output order (t_reported, x, y, t_cross) (output_order,
 * src/sensor/output_order.h:88-107). bs_model_output_prepare moves the last call's events (those not taken with
 * bs_model_take_events) and the held ones through the stage on the device and releases those reported before the
 * model time on the sensor clock (output_cut, :48-53); the rest stay held for the next call. *n_ready receives the
 * released count; bs_model_output_take copies them to host columns (any may be NULL). init() clears what is held. */
typedef struct {
  int64_t *t_reported_ns, *t_cross_ns;
  uint16_t *x, *y, *flags;
  uint8_t *p, *label;
} bs_output_columns;
bs_status bs_model_output_prepare(bs_model* m, size_t* n_ready);
bs_status bs_model_output_take(bs_model* m, bs_output_columns* out);
bs_status bs_model_output_held(const bs_model* m, size_t* n_held);
/* This build's noise maps (no reference counterpart), width * height each: the pixel's background-activity rate
 * and its shot-noise dominating rate r sqrt(100 fA / I_dk) (Hz; 0 when that noise is off). */
bs_status bs_model_noise_maps(const bs_model* m, double* ba_rate_hz, double* shot_max_hz);
/* Work counters since creation or bs_model_reset_stats (SensorModel::stats, sensor_module.cpp:112-136):
 * [pieces, leaf_intervals, input_clamps, pixel_samples, noise_candidates, gpu_launches, gpu_reruns,
 *  gpu_launch_ms_total x1000, gpu_launch_ms_max x1000]. */
bs_status bs_model_stats(const bs_model* m, uint64_t out[9]);
bs_status bs_model_reset_stats(bs_model* m);
/* SensorModel.set_photometry (sensor_module.cpp:477-486, sensor_model.cpp:350-373): the photocurrent scale (fA
 * per renderer unit) and the per-pixel gain map, width * height floats in pixel order (gain NULL, n_gain 0: 1
 * everywhere). Each gain finite and > 0; irr_max becomes 1e9 fA / (scale x the largest gain). The states take the
 * new photometry at the next init. */
bs_status bs_model_set_photometry(bs_model* m, double illuminance_scale, const float* gain, size_t n_gain);
/* SensorModel.gain_map (sensor_module.cpp:487-502): width * height gains (1 without a gain map). */
bs_status bs_model_gain_map(const bs_model* m, float* out);
/* time_ns, irr_max, initialized (sensor_model.h:212-236). */
bs_status bs_model_info(const bs_model* m, int64_t* time_ns, float* irr_max, int32_t* initialized);
/* save_state / load_state / state_bytes (sensor_model.h:175-178) in the reference's format
 * (src/sensor/sensor_model.cpp:1198-1262): its 56-byte StateHeader (magic "BSNS", version 6, shape, groups, camera,
 * seed, the state fingerprint: the parameters' fingerprint, continued over the gain map when some gain is not 1, the
 * model time, initialized, 200), then one 200-byte PixelState (src/sensor/pixel.h:105-121) per pixel. A state saved
 * by the reference's SensorModel loads here and the reverse, and each refuses a state of another shape, seed, camera
 * or fingerprint. With this project's shot and background-activity noise on, 32 bytes per pixel follow (the noise
 * chains' next candidate times and counts). */
bs_status bs_model_state_bytes(const bs_model* m, size_t* n);
bs_status bs_model_save_state(const bs_model* m, uint8_t* out, size_t n);
bs_status bs_model_load_state(bs_model* m, const uint8_t* data, size_t n);
/* Launch policy of the pixel model on CSR runs. 0 (the default): the instantaneous response runs row-major, one warp
 * per 32 runs, runs longer than the long-run threshold walked by the whole warp, split in two launches: a run stopped
 * at its first segment that is not clean (or before its held stretch to t_end) is finished by a second kernel, one
 * thread per run (the cascade runs one thread per pixel, 128 per block); 1: the same row-major kernel in one launch;
 * 32, 64, 96 or 128: one thread per pixel with that many threads per block, for every photoreceptor. */
bs_status bs_model_set_block(bs_model* m, int32_t threads);
/* The row-major kernel's threads per pixel: runs longer than `samples` are walked by all 32 lanes of a warp, 32
 * consecutive samples at a time (their logs and exclusion tests in parallel, a ballot finding the first segment that
 * can fire), the others by one lane each (0: the default, 32; -1: every run by one lane). */
bs_status bs_model_set_long_run(bs_model* m, int32_t samples);

/* ---- the window sampler: sample_window (src/engine/bindings/engine_module.cpp:311-355), MidpointTest ---- */

/* A seeded analytic field, evaluated on the device in place of the render hook (src/engine/window.h:69-84).
 * kind 1: tanh edge (base, amp, nx, ny, c, speed, width_px); kind 2: blobs (base, n_blobs rows of 10 floats:
 * a, cx0, cy0, vx, vy, 1/(2 r^2), (6 r)^2, (3 r)^2, |v|, pad), host memory, copied at create. */
typedef struct {
  int32_t kind;
  uint32_t width, height;
  float base, amp, nx, ny, c, speed, width_px;
  int32_t n_blobs;
  const float* blobs;
} bs_field;

/* SampleRules of sample_window: MidpointTest(tol, dark, [1], [1]) when midpoint != 0, refine_signature,
 * max_refine_levels (>= 0), min_dt_ns (a power of two in [1, 2^23]); l_min / l_max clamp the field's level rule
 * (the engine only). */
typedef struct {
  float tol, dark;
  int32_t midpoint, refine_signature, max_refine_levels;
  int64_t min_dt_ns;
  int32_t l_min, l_max;
} bs_sample_rules;

bs_status bs_sampler_create(const bs_field* field, bs_sampler** out);
bs_status bs_sampler_destroy(bs_sampler* s);
/* sample_window on the device field: n active pixels (ids, lattice levels) with their carried samples (host, in
 * and out: each pixel's last sample at t_w + W). The runs stay in the sampler's device memory; *n_samples gets
 * their total. Levels must lie in [0, 23 - log2(min_dt_ns)] (engine_module.cpp:317-323). */
bs_status bs_sample_window(bs_sampler* s, int64_t t_w, const uint32_t* pixel_ids, const uint8_t* levels, size_t n,
                           float* carried_irr, uint64_t* carried_sig, const bs_sample_rules* rules,
                           size_t* n_samples);
/* sample_window with the inputs in device memory, as the reference's device window engine takes them
 * (WindowEngine<Space::kDevice>::run, src/engine/window.h:133-174; its caller Camera::sample_and_sense,
 * src/engine/engine_impl.h:1253-1343): pixel_ids, levels and the carried samples (carried_irr / carried_sig in,
 * each pixel's last sample at t_w + W to carried_irr_out / carried_sig_out, arrays that must not alias the inputs)
 * are the caller's device arrays, read on `stream` (NULL: the sampler's own stream). The ids and levels are checked
 * on the device first (BS_EINVAL as bs_sample_window, nothing written). The runs stay in the sampler's memory for
 * bs_sampler_device_runs -> bs_model_advance_device on the same stream; *n_samples gets their total. The call
 * synchronizes `stream` twice (the check, the sample count) and leaves the write pass queued on it. */
bs_status bs_sample_window_device(bs_sampler* s, int64_t t_w, const uint32_t* pixel_ids, const uint8_t* levels,
                                  size_t n, const float* carried_irr, const uint64_t* carried_sig,
                                  float* carried_irr_out, uint64_t* carried_sig_out, const bs_sample_rules* rules,
                                  void* stream, size_t* n_samples);
/* bs_field_levels and bs_field_frame into device arrays (width * height), queued on `stream`. */
bs_status bs_field_levels_device(bs_sampler* s, int64_t t_w, int32_t l_min, int32_t l_max, uint8_t* out,
                                 void* stream);
bs_status bs_field_frame_device(bs_sampler* s, int64_t t_ns, float* out, void* stream);
/* The last window's runs to host arrays (WindowRuns: offsets n + 1, t_ns, irradiance), or as device runs for
 * bs_model_advance_device (valid until the sampler runs again; after bs_sample_window_device the runs' pixel ids
 * are the caller's array). */
bs_status bs_sampler_download(bs_sampler* s, int64_t* offsets, int64_t* t_ns, float* irr);
bs_status bs_sampler_device_runs(bs_sampler* s, bs_device_runs* out);
/* sample_window for callers that cannot allocate device memory: code running under an external memory manager with
 * a fixed budget, or code that must not call cudaMalloc / cudaFree because they synchronize the device. No
 * counterpart in the reference. Every array is the caller's, in device memory: the field's blob table, pixel ids,
 * levels, carried samples in and out, offsets (n + 1), and t_ns / irr with room for `capacity` samples. The
 * entry point allocates nothing: its scratch (the per-pixel sample counts and the scan's block sums) is one static
 * device array sized for at most 1,048,576 pixels (about 4 MiB, held by every GPU that loads the library until the
 * process exits); more pixels are refused (BS_EINVAL). It runs on the current device and on `stream` (NULL: the
 * default stream); its first call on a device looks up the array's device address, so make that first call before
 * any stream capture. Each call synchronizes `stream` three times: it copies the input check's result and the
 * window's sample count to the host, and returns once the runs are written. *n_samples receives the window's sample
 * count, also when it exceeds capacity (BS_EINVAL, the outputs then unwritten). All calls share the one array: calls that overlap on the GPU (other streams, other host
 * threads) race and must be serialized by the caller. */
bs_status bs_sample_window_static(const bs_field* field, int64_t t_w, const uint32_t* pixel_ids,
                                  const uint8_t* levels, size_t n, const float* carried_irr,
                                  const uint64_t* carried_sig, const bs_sample_rules* rules, int64_t* offsets,
                                  int64_t* t_ns, float* irr, size_t capacity, float* carried_irr_out,
                                  uint64_t* carried_sig_out, void* stream, size_t* n_samples);
/* ---- sample_window with a renderer behind a callback: the reference's host window engine (WindowEngine<kHost>,
 * src/engine/window_impl.h:462-714) driving a RenderHook (src/engine/window.h:69-84) ---- */

/* One pixel-sample request (render::SampleRequest, src/backend/api.h:25-34), 24 bytes: camera, flags (0: a regular
 * lattice sample), pixel id, sub-sample range [k_begin, k_begin + k_count), time offset from the window start (ns),
 * and the time slot t_off_ns >> log2(min_dt_ns) in pose_slot. */
typedef struct {
  uint16_t cam;
  uint16_t flags;
  uint32_t pixel;
  uint32_t k_begin;
  uint32_t k_count;
  int32_t t_off_ns;
  uint32_t pose_slot;
} bs_sample_request;
/* RenderHook::render as a C callback: request i's irradiance goes to row out_index[i] of irr (groups floats each) and
 * its signature to sig[out_index[i]]; every request of a call has k_count == subsamples. Returns 0, or a non-zero
 * status that stops the window (BS_EINVAL). Called on the calling thread, one call per render round. */
typedef int32_t (*bs_render_fn)(void* user, bs_sample_request* requests, size_t n, const uint32_t* out_index,
                                float* irr, uint64_t* sig, uint32_t subsamples);
/* The window's rules (SampleConfig, src/engine/window.h:98-110, with the Phase 1 sample rules): the eta_L midpoint
 * test (tol, dark) when midpoint != 0, refine_signature, max_refine_levels, min_dt_ns (a power of two in [1, 2^23]),
 * the camera and sub-samples of the requests; cancel (may be NULL): a flag another thread may set, checked before the
 * window and at every refinement round (the reference's CancelToken; BS_ECANCELLED). */
typedef struct {
  float tol, dark;
  int32_t midpoint, refine_signature, max_refine_levels;
  int64_t min_dt_ns;
  uint16_t cam;
  uint32_t subsamples;
  const volatile int32_t* cancel;
} bs_window_rules;
typedef struct bs_window bs_window;
/* groups light groups (1 to 8) with their waveform ranges m_min / m_max (NULL: 1), the midpoint test's MidpointTest
 * (tol, dark, m_min, m_max) (engine_module.cpp:1363-1411). */
bs_status bs_window_create(int32_t groups, const float* m_min, const float* m_max, bs_window** out);
bs_status bs_window_destroy(bs_window* w);
/* One window at t_w (a multiple of 2^23) of n listed pixels (ids in render order, lattice levels in [0, 23 -
 * log2(min_dt_ns)]) with their carried samples (host, n x groups irradiance and n signatures, in and out: each pixel's
 * sample at t_w + 2^23): the lattice in one render call, round 0's flags, then the refinement rounds, one render call
 * each; each round's midpoint tests run on the device (no device call without the midpoint test). *n_samples receives
 * the runs' total. */
bs_status bs_window_run(bs_window* w, int64_t t_w, const uint32_t* pixel_ids, const uint8_t* levels, size_t n,
                        float* carried_irr, uint64_t* carried_sig, const bs_window_rules* rules, bs_render_fn render,
                        void* user, size_t* n_samples);
/* The last window's runs (WindowRuns: offsets n + 1, t_ns, irradiance n_samples x groups), host arrays. */
bs_status bs_window_runs(const bs_window* w, int64_t* offsets, int64_t* t_ns, float* irr);
/* Its WindowStats (src/engine/window.h:111-131): counters [flagged_signature, flagged_midpoint, refine_cap_hits,
 * render_calls], samples_by_round (up to cap rounds) and *rounds their number. */
bs_status bs_window_stats(const bs_window* w, uint64_t counters[4], uint64_t* samples_by_round, size_t cap,
                          size_t* rounds);

/* The field's level rule per pixel at t_w, and the field itself at t (width * height, host outputs). */
bs_status bs_field_levels(bs_sampler* s, int64_t t_w, int32_t l_min, int32_t l_max, uint8_t* out);
bs_status bs_field_frame(bs_sampler* s, int64_t t_ns, float* out);
/* MidpointTest.eta / .exceeds (engine_module.cpp:1363-1411): eta_L of n triples of `groups` light groups (host
 * arrays n x groups; m_min / m_max per group, the mediant when they differ), evaluated on the device. */
bs_status bs_midpoint_eta(float tol, float dark, int32_t groups, const float* m_min, const float* m_max,
                          const float* ea, const float* em, const float* eb, size_t n, float* eta, uint8_t* exceeds);
/* level_cap (src/engine/window.cpp:25-50): the finest level keeping a window within budget samples (-1: none). */
bs_status bs_level_cap(const int64_t* levels, size_t n, int64_t budget, int32_t l_min, int32_t* cap);

/* ---- the fused engine: every window of several sensors in one launch per call (Camera::sample_and_sense,
 * src/engine/engine_impl.h:1253-1357, with the runs kept in registers) ---- */

/* models[i] is sampled from fields[i]; the engine borrows the models (they must outlive it). */
bs_status bs_engine_create(bs_model* const* models, const bs_field* fields, int32_t n, const bs_sample_rules* rules,
                           bs_engine** out);
bs_status bs_engine_destroy(bs_engine* e);
/* Renders every field at t0 and initializes every model from it (CameraEngine::start without warm-up). */
bs_status bs_engine_start(bs_engine* e, int64_t t0_ns, void* stream);
/* The same from host frames: frames[i] holds sensor i's irradiance at t0 (width * height floats), copied to the
 * device; each model starts from it and it is the window sampler's first carried sample. */
bs_status bs_engine_start_frames(bs_engine* e, int64_t t0_ns, const float* const* frames, void* stream);
/* Samples and senses `windows` whole windows of every sensor from the current model time; the events are kept in
 * each model (bs_model_take_events). *pixel_samples and *events receive the totals of the call. */
bs_status bs_engine_run(bs_engine* e, int32_t windows, void* stream, uint64_t* pixel_samples, uint64_t* events);
/* bs_model_take_events for every sensor of the engine at once (out[i]: sensor i's columns, sized by
 * bs_model_event_count): the sensors' device sorts, column splits and copies out are queued together, and each
 * sensor's copies into the caller's arrays run while the device works on the sensors after it. No counterpart in the
 * reference, whose engine takes one camera's events at a time; the columns and the order are bs_model_take_events'. */
bs_status bs_engine_take_events(bs_engine* e, bs_event_columns* out);
/* Launch shape: warps per block and blocks per SM of the persistent grid (0: the defaults, 4 and as many as fit),
 * the staging depth (0: the sampler feeds the pixel model sample by sample; 16 or 32: per window each lane's samples
 * are staged in shared memory between a sampling phase and a sensing phase; 64: staged 32 deep with the crossing
 * search taken by the whole warp; 1: the split engine, two launches per window, the first running the staged phases
 * and the pixel model's clean segments for every pixel and posting each pixel at its first other segment, the second
 * finishing the posted pixels' windows one thread per pixel; the instantaneous response only) and the tile width in
 * pixels (4, 8, 16 or 32; the tile is 32 / width pixels high, one warp per tile; 0: 8). The learned engine runs 4 warps
 * per block. */
bs_status bs_engine_set_launch(bs_engine* e, int32_t warps_per_block, int32_t blocks_per_sm, int32_t stage,
                               int32_t tile_width);
/* The current launch shape: warps per block, blocks per SM, staging depth, tile width. */
bs_status bs_engine_get_launch(const bs_engine* e, int32_t out[4]);
/* Runs each step as a CUDA graph (on, the default) or as separate stream operations (off). The graph holds the
 * counter resets, the descriptor and model-time uploads, the persistent kernel and the counter read-back; it is
 * rebuilt when the window count, launch shape or proposal changes. */
bs_status bs_engine_set_graph(bs_engine* e, int32_t on);
/* The autotuner: times trial steps of `windows` windows from the current state for each candidate launch shape
 * (tile width 4, 8, 16 x warps per block 2, 4 x stage 0, 1, 16, 64; the learned engine: tile widths) without
 * moving the models, and keeps the fastest. rows (cap x 4 doubles: tile width, warps, stage, ms) receives the
 * candidates tried, *n their number. */
bs_status bs_engine_autotune(bs_engine* e, int32_t windows, void* stream, double* rows, size_t cap, size_t* n);
/* Kernel time of the last bs_engine_run's launches (ms, CUDA events on its stream). */
bs_status bs_engine_last_ms(const bs_engine* e, double* ms);

/* ---- the learned step proposal (no reference counterpart: BallaSim samples with the plain lattice + midpoint rule
 * only, src/engine/sampling.h; the plain rule stays the judge of every proposed step and its fallback) ----
 *
 * An MLP 16 -> 64 -> 64 -> 1 (ReLU), BF16 weights and activations with FP32 accumulation on the tensor cores,
 * predicts log2(step / min_dt) of a pixel's next power-of-two sample step from its last 8 walk points. Parameters
 * (FP32, BS_MLP_PARAMS floats): W1 [16 in][64 out], b1 [64], W2 [64 in][64 out], b2 [64], W3 [64], b3. Device
 * arrays of pairs: x (n x 16 BF16 features, as uint16 bits), y (n FP32 targets). */
#define BS_MLP_PARAMS 5313
typedef struct bs_mlp bs_mlp;
/* He-uniform weights drawn from Philox(seed), zero biases, Adam state zero. */
bs_status bs_mlp_create(uint64_t seed, bs_mlp** out);
bs_status bs_mlp_destroy(bs_mlp* m);
bs_status bs_mlp_get_params(const bs_mlp* m, float* params);
/* Sets the parameters (host, BS_MLP_PARAMS floats) and resets the Adam state and step counter. */
bs_status bs_mlp_set_params(bs_mlp* m, const float* params);
/* Adam steps taken so far. */
bs_status bs_mlp_steps(const bs_mlp* m, int64_t* steps);
/* y[i] = MLP(x[i]) for n rows (device arrays). */
bs_status bs_mlp_forward(bs_mlp* m, const uint16_t* x, size_t n, float* y, void* stream);
/* The gradient (host, BS_MLP_PARAMS doubles) and the loss of L = sum_i (MLP(x_i) - y_i)^2 / (2 n) over all n rows,
 * from the training kernels' forward and backward passes. */
bs_status bs_mlp_gradient(bs_mlp* m, const uint16_t* x, const float* y, size_t n, double* grad, double* loss,
                          void* stream);
/* `steps` Adam steps (lr, beta 0.9 / 0.999, eps 1e-8) over batches of `batch` rows drawn with replacement from the
 * n pairs (Philox(seed), keyed by the step count) on the expectile loss sum_i w_i (MLP(x_i) - y_i)^2 / (2 batch),
 * w_i = 2 tau where the net predicts below y_i and 2 (1 - tau) above (tau = 0.5: the mean squared error above);
 * losses (host, may be NULL) gets every step's batch loss. Runs from a CUDA graph of 32 steps. */
bs_status bs_mlp_train(bs_mlp* m, const uint16_t* x, const float* y, size_t n, int32_t steps, int32_t batch, float lr,
                       float tau, uint64_t seed, float* losses, void* stream);
/* Training pairs from the plain sampler: windows [0, windows) of the field from t0 are sampled with the rules
 * (every pixel, levels by the field's rule) and every stride-th pixel walks its runs. At each walk point the
 * target is the longest aligned power-of-two step whose chord stays within eps of the run's log irradiance at every
 * run sample it spans (never shorter than the plain lattice step); the walk then moves by the target lowered by
 * 0-3 octaves (Philox(seed)). Pairs go to device arrays x (cap x 16 BF16), y (cap) and keys (cap, may be NULL:
 * pixel << 32 | window << 11 | step); *n_out = pairs written, *total = pairs produced. */
bs_status bs_trace_pairs(const bs_field* field, const bs_sample_rules* rules, int64_t t0_ns, int32_t windows,
                         uint32_t stride, float eps, uint64_t seed, uint16_t* x, float* y, uint64_t* keys, size_t cap,
                         size_t* n_out, size_t* total, void* stream);
/* Samples the engine's windows with the learned proposal (mlp NULL: the plain sampler again). A proposal y becomes
 * the step 2^s, s = log2 min_dt + floor(y + 0.5 - margin) clamped to [log2 min_dt, 23], raised to the plain level's
 * lattice step and lowered until aligned. The walk state restarts from the current frame (and at every start). */
bs_status bs_engine_set_proposal(bs_engine* e, const bs_mlp* mlp, float margin);
/* Records up to `capacity` rows of every sample and every proposed step of each following run (0: off). */
bs_status bs_engine_set_record(bs_engine* e, size_t capacity);
/* Copies up to cap rows of the last run's record `which` (0: samples, v = irradiance; 1: steps, v = log2 step) to
 * host columns t, pixel (sensor << 24 | pixel), v (any may be NULL); *n = rows recorded (> capacity: cut short). */
bs_status bs_engine_take_record(bs_engine* e, int32_t which, size_t cap, int64_t* t, uint32_t* pixel, float* v,
                                size_t* n);

/* ---- the event file sink: Prophesee RAW and DAT files of one camera's events ---- */

typedef struct bs_event_writer bs_event_writer;

/* What close returns (FileInfo and its one events stream, src/export/sink.h:24-36): the file's size and SHA-256
 * (lower-case hex), the events written and the first and last T1a time u (us after the origin; 0 without events). */
typedef struct {
  uint64_t bytes;
  char sha256[65];
  int64_t count, t_first, t_last;
} bs_file_info;

/* RawWriter (src/export/raw_writer.h:33-49; ballasim._export.RawWriter, export_module.cpp:331-361): format "evt2",
 * "evt21" or "evt3"; width and height in [1, 2048]; origin_us and epoch_ns of the T1a rule u = floor(t_ns / 1000) -
 * origin_us (epoch_ns a multiple of 1000, recorded in the header); evt2_time_high "openeb" or "change" (EVT 2.0
 * only); [t_ns_rem_min, t_ns_rem_max] the window's sub-us parts (-1, -1: no events); version (may be NULL) goes to
 * the header's plugin_version. The file is created and its header written here (no device needed). */
bs_status bs_raw_writer_create(const char* path, const char* format, int32_t width, int32_t height, int64_t origin_us,
                               int64_t epoch_ns, const char* evt2_time_high, int32_t t_ns_rem_min,
                               int32_t t_ns_rem_max, const char* version, bs_event_writer** out);
/* DatWriter (raw_writer.h:51-66; export_module.cpp:363-387): as RawWriter with width and height in [1, 16384]; the
 * version is not written. */
bs_status bs_dat_writer_create(const char* path, int32_t width, int32_t height, int64_t origin_us, int64_t epoch_ns,
                               int32_t t_ns_rem_min, int32_t t_ns_rem_max, const char* version,
                               bs_event_writer** out);
/* RawWriter::append / DatWriter::append (raw_writer.h:41-46): n events in output order from host columns x, y
 * (uint16), p (uint8, 0/1) and t_ns (int64, t_reported). The words are built on the device. A batch that breaks a
 * rule (order within and across calls, x < width, y < height, p <= 1, t_ns mod 1000 in the declared range, u >= 0,
 * EVT 2.0/2.1's first u < 2^34, DAT's u < 2^32) is refused whole: BS_EREFUSED, nothing written. */
bs_status bs_event_writer_append(bs_event_writer* w, const uint16_t* x, const uint16_t* y, const uint8_t* p,
                                 const int64_t* t_ns, size_t n);
/* As bs_event_writer_append with device columns (for example an output stage's), on stream (NULL: the legacy
 * default stream); returns after the batch's words are in the file. */
bs_status bs_event_writer_append_device(bs_event_writer* w, const uint16_t* x, const uint16_t* y, const uint8_t* p,
                                        const int64_t* t_ns, size_t n, void* stream);
/* RawWriter::close / DatWriter::close (raw_writer.h:47, 65): EVT 2.1's open word, then the file closed and hashed. */
bs_status bs_event_writer_close(bs_event_writer* w, bs_file_info* info);
/* This build's counters (no reference counterpart; any may be NULL): kernel launches of the appends so far; of the
 * last append the device time of its kernels (ms, CUDA events around them) and the bytes of its words; host_ms the
 * wall time (ms) of the last append, of its file writes, and of close's hash of the file. */
bs_status bs_event_writer_stats(const bs_event_writer* w, uint64_t* launches, double* kernel_ms, uint64_t* bytes_out,
                                double host_ms[3]);
bs_status bs_event_writer_destroy(bs_event_writer* w);
/* SHA-256 (FIPS 180-4) of n bytes as 64 lower-case hex digits and a NUL (config::Sha256, src/config/sha256.h). */
bs_status bs_sha256_hex(const void* data, size_t n, char out[65]);

#ifdef __cplusplus
}
#endif

#endif
