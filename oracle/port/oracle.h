/* CPU restatement of BallaSim's per-pixel event-generation path: the window sampler
 * (src/engine/sampling.h, src/engine/window_impl.h) feeding the instantaneous pixel model
 * (src/sensor/pixel.h advance_instant), with the frozen per-pixel maps (src/sensor/maps.cpp),
 * the deterministic maths (src/core/pmath/explog.h, trig.h) and Philox4x32-10
 * (src/core/rng/philox.h, purpose.h).
 *
 * TEST INFRASTRUCTURE ONLY. This is the oracle the CUDA path is checked against: only tests/,
 * __graft_entry__.smoke() and bench.py's cpu_baseline leg load it. The product never links it.
 *
 * Plain C11, compiled with -ffp-contract=off (no fused multiply-add), scalar and single-threaded.
 * Parity is pinned against the reference compiled from its own sources (oracle/_ref) and against the
 * golden vectors in tests/golden/. Shot and background-activity noise have no reference
 * counterpart: their part of this file restates the project's own noise law (see noise section). */
#ifndef BALLASIM_ORACLE_H
#define BALLASIM_ORACLE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- Philox and the purpose-tagged counter layout (src/core/rng/philox.h:45-53, purpose.h:47-53) ---- */
void orc_philox(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]);
void orc_draw(uint64_t seed, uint32_t purpose, uint32_t camera, uint32_t pixel, uint64_t index, uint32_t out[4]);

/* ---- deterministic maths (src/core/pmath/explog.h:159-225, trig.h:130-155) ---- */
float orc_logf(float x);
double orc_log(double x);
float orc_expf(float x);
double orc_exp(double x);
void orc_sincos(double x, double* s, double* c);

/* ---- analytic irradiance fields (the renderer's stand-in; this project's own definition) ---- */
enum { ORC_FIELD_TANH_EDGE = 1, ORC_FIELD_BLOBS = 2 };
/* One blob: amplitude, centre at t = 0, velocity (px/s), 1 / (2 r^2), the cut-off d^2 (36 r^2), the
 * level rule's support d^2 (9 r^2) and its speed |v|. */
enum { ORC_BLOB_WORDS = 10 };
typedef struct {
  int32_t kind;
  uint32_t width, height;
  float base, amp, nx, ny, c, speed, width_px; /* tanh edge */
  int32_t n_blobs;
  const float* blobs; /* n_blobs x ORC_BLOB_WORDS: a, cx0, cy0, vx, vy, inv2r2, cut2, cover2, vabs, pad */
} orc_field;

float orc_field_eval(const orc_field* f, uint32_t x, uint32_t y, int64_t t_ns);
/* Lattice level of pixel (x, y) at t_w: the level rule clamp(ceil(log2(v W / 0.25 px)), l_min, l_max) with v
 * the fastest blob whose 3 r support covers the pixel (l_min without one; the tanh edge: l_min). */
int32_t orc_field_level(const orc_field* f, uint32_t x, uint32_t y, int64_t t_w, int32_t l_min, int32_t l_max);

void orc_field_frame(const orc_field* f, int64_t t_ns, float* out);              /* width x height */
void orc_field_levels(const orc_field* f, int64_t t_w, int32_t l_min, int32_t l_max, uint8_t* out);
/* The field at (pixel id, t) pairs, as a renderer callback would sample it. */
void orc_field_samples(const orc_field* f, const uint32_t* pixel, const int64_t* t_ns, size_t n, float* out);

/* ---- sensor parameters (src/sensor/params.h:65-176) ---- */
typedef struct {
  double theta_on, theta_off, sigma_theta_on, sigma_theta_off, theta_onoff_corr, theta_floor;
  int32_t reset_mode; /* 0 physical, 1 ideal */
  double refractory_s, eps_ci;
  int32_t initial_phase; /* 0 uniform, 1 symmetric, 2 zero */
  double leak_rate_hz, leak_sigma_log10, leak_ea_eV;
  double dark_current_fA, dark_sigma_ln, dark_ea_eV, temperature_K, reference_temperature_K;
  double illuminance_scale, label_share_cut;
  double readout_quantum_s, readout_delay_s, clock_drift_ppm;
  int64_t clock_offset_ns;
  /* noise of the new model (no reference counterpart): shot rate at 100 fA (Hz), background activity
   * median (Hz) and its log-normal spread; off when noise == 0 */
  int32_t noise;
  double shot_rate_hz, ba_median_hz, ba_sigma_ln;
} orc_params;

typedef struct {
  uint32_t pixel;
  uint8_t polarity, label;
  uint16_t flags;
  int64_t t_cross;
  float ds, dn, dl, l_first;
} orc_event;

typedef struct orc_model orc_model;

orc_model* orc_model_create(const orc_params* p, uint32_t width, uint32_t height, uint64_t seed, uint32_t camera,
                            int32_t groups);
void orc_model_destroy(orc_model* m);
int orc_model_init(orc_model* m, int64_t t0, const float* irr0);
/* Advances every pixel to t_end; listed pixel pixel_ids[i] takes row_count[i] samples at row_start[i]. The events
 * are appended to the model's event list (orc_model_events). Returns 0, or -1 on a refused input. */
int orc_model_advance_runs(orc_model* m, const uint32_t* pixel_ids, size_t n, const int64_t* t, const float* irr,
                           size_t n_samples, const int64_t* row_start, const int32_t* row_count, int64_t t_end);
size_t orc_model_event_count(const orc_model* m);
/* Copies the events sorted by (t_cross, pixel) and clears the list. */
void orc_model_take_events(orc_model* m, orc_event* out);
/* The maps (fp64) and a few state words per pixel. */
void orc_model_maps(const orc_model* m, double* theta_on, double* theta_off, double* leak, double* dark,
                    double* phi0);
void orc_model_state(const orc_model* m, int64_t* t_ref, int64_t* t_search, float* s3_ref, float* dr_ref,
                     float* held);
uint64_t orc_model_stat(const orc_model* m, int32_t which); /* 0 pieces, 1 leaf intervals, 2 clamps */
void orc_model_noise_maps(const orc_model* m, double* ba_rate_hz); /* the background-activity rate map */
const char* orc_last_error(void);

/* ---- the window sampler (src/engine/sampling.h, window_impl.h:461-713) ---- */
typedef struct {
  float tol, dark;
  int32_t midpoint, refine_signature, max_refine_levels;
  int64_t min_dt_ns;
} orc_rules;

/* Samples one window for n active pixels (levels per pixel), with carried samples (G = 1 group). Writes the
 * runs in active-pixel order: offsets (n + 1), t and irr up to cap samples; returns the sample count (or
 * -(needed) when cap is too small), and each pixel's last sample into carried_irr / carried_sig. */
int64_t orc_sample_window(const orc_field* f, const orc_rules* r, int64_t t_w, const uint32_t* pixel,
                          const uint8_t* level, size_t n, float* carried_irr, uint64_t* carried_sig,
                          int64_t* offsets, int64_t* t_out, float* irr_out, size_t cap);

/* eta_L of triples (src/engine/sampling.h:36-53), G = 1. */
float orc_midpoint_eta(float tol, float dark, float a, float m, float b);

/* ---- the learned step proposal (this project's own method; no reference counterpart) ---- */
typedef struct {
  float hx[8];    /* log irradiance of the last 8 walk points, newest first */
  uint64_t gaps;  /* byte k: log2 of the k-th previous gap (byte 0 newest) */
  float pv;       /* irradiance at the previous walk point */
  int32_t valid;  /* a real previous walk point exists */
} orc_walk;

uint16_t orc_bf16(float f); /* round to nearest even */
void orc_step_features(const float hx[8], uint64_t gaps, float x, float out[16]);
void orc_walk_reset(orc_walk* w, float v0);
/* The training walk over one pixel's plain run of one window (t absolute, n samples, slot 0 at t_w and the last at
 * t_w + 2^23): appends up to cap pairs (16 BF16 features, target log2(step) - sh, key pixel << 32 | window << 11 |
 * step) and returns the number of walk points. */
int orc_walk_window(const int64_t* t, const float* v, int n, int64_t t_w, int level, int sh, float eps, uint64_t seed,
                    uint32_t pixel, int32_t window, orc_walk* w, uint16_t* x_out, float* y_out, uint64_t* key_out,
                    int cap);
/* The learned sampler's samples of one pixel and window for the given step sequence (log2 of each proposed step, as
 * the device used them): the judge and the plain-rule refinement. Returns the samples written after slot 0, or a
 * negative code: -1 too few steps, -2 a step below the plain lattice step, above 2^23 or unaligned, -3 steps left. */
int64_t orc_learned_window(const orc_field* f, const orc_rules* r, int64_t t_w, uint32_t x, uint32_t y, int level,
                           float carried, orc_walk* w, const int32_t* steps, int n_steps, int64_t* t_out,
                           float* v_out, size_t cap);

#ifdef __cplusplus
}
#endif

#endif
